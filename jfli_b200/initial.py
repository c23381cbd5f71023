"""Gaussian initial conditions (reference initial.py:18-199, infer/dist.py:27-113).

delta = irfft(rfft(w) * sqrt(P_lin(|k|) * N^3 / V)) with |k| in h/Mpc, the P_lin table
interpolated linearly on the GPU inside the x pass of the FFT (kspace_ops.cuh IcOp).
"""

from __future__ import annotations

import numpy as np
import torch

from . import cosmology as cj
from . import ops
from .fields import DensityField, DensityUnit, FieldStatus


def _pk_tables(cosmo, pk_fn, n_table: int, mesh_size, box_size):
    if pk_fn is None:
        if cosmo is None:
            raise ValueError("Either pk_fn or cosmo must be provided to compute the power spectrum.")
        k, pk = cj.pk_table(cosmo, n_table)
    else:
        # A user P(k) callable is tabulated on a dense log grid spanning the mesh's |k| range.
        kmax = np.sqrt(3.0) * np.pi * max(n / L for n, L in zip(mesh_size, box_size)) * 1.01
        kmin = 2 * np.pi / max(box_size) * 0.99
        k = np.concatenate([[0.0], np.logspace(np.log10(kmin), np.log10(kmax), 4096)])
        pk = np.asarray(pk_fn(k), dtype=np.float64)
    kt = ops.device_table(k)
    pt = ops.device_table(pk)
    return kt, pt


def _as_device(field, mesh_size):
    if isinstance(field, DensityField):
        field = field.array
    if isinstance(field, torch.Tensor):
        t = field.to(device="cuda", dtype=torch.float32)
    else:
        t = torch.as_tensor(np.asarray(field, dtype=np.float32), device="cuda")
    if tuple(t.shape[-3:]) != tuple(mesh_size):
        raise ValueError(f"initial field shape {tuple(t.shape)} does not match mesh_size {mesh_size}")
    return t.contiguous()


def interpolate_initial_conditions(initial_field, mesh_size, box_size, *, cosmo=None, pk_fn=None,
                                   observer_position=(0.5, 0.5, 0.5), flatsky_npix=None, nside=None, field_size=None,
                                   halo_size=(0, 0), sharding=None, n_table: int = 128,
                                   zero_mode_one: bool = False) -> DensityField:
    """White noise -> linear density field (reference initial.py:124-199). `n_table=256`
    with `zero_mode_one=True` gives infer/dist.py's PowerSpectrumTransform."""
    mesh_size = tuple(int(v) for v in mesh_size)
    box_size = tuple(float(v) for v in box_size)
    if isinstance(halo_size, int):
        halo_size = (halo_size, halo_size)
    w = _as_device(initial_field, mesh_size)
    kt, pt = _pk_tables(cosmo, pk_fn, n_table, mesh_size, box_size)
    if torch.is_grad_enabled() and w.requires_grad and not zero_mode_one:
        from .pm.adjoint import ForwardTables, ICFilter

        tables = ForwardTables(ktab=kt, ptab=pt, lpt=None, kicks=None, drifts=None)
        field = ICFilter.apply(w, None, None, tables, box_size)
    else:
        field = ops.ic_filter(w, kt, pt, box_size, zero_mode_one=zero_mode_one)
    return DensityField(array=field, mesh_size=mesh_size, box_size=box_size, observer_position=observer_position,
                        sharding=sharding, halo_size=tuple(halo_size), nside=nside, field_size=field_size,
                        flatsky_npix=flatsky_npix, scale_factors=0.0, status=FieldStatus.INITIAL_FIELD,
                        unit=DensityUnit.DENSITY)


def white_noise(seed: int, mesh_size) -> np.ndarray:
    """Seeded N(0,1) white noise (float32), the synthetic input used across the repo."""
    return np.random.default_rng(seed).standard_normal(tuple(mesh_size)).astype(np.float32)


def gaussian_initial_conditions(key, mesh_size, box_size, *, cosmo=None, pk_fn=None,
                                observer_position=(0.5, 0.5, 0.5), flatsky_npix=None, nside=None, field_size=None,
                                halo_size=(0, 0), sharding=None) -> DensityField:
    """Seeded Gaussian ICs (reference initial.py:33-106). `key` is an integer seed for
    numpy's default_rng (JAX PRNG keys are not available on this path)."""
    noise = white_noise(int(key), mesh_size)
    return interpolate_initial_conditions(noise, mesh_size, box_size, cosmo=cosmo, pk_fn=pk_fn,
                                          observer_position=observer_position, flatsky_npix=flatsky_npix,
                                          nside=nside, field_size=field_size, halo_size=halo_size,
                                          sharding=sharding)
