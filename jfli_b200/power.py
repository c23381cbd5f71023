"""Power spectrum estimator (reference power/compute.py:13-33, _src/power/_compute.py:23-119).

P(k) = <|FFT_ortho(mesh)|^2> per digitize(|k|, kedges) bin over the full Fourier grid,
with the under/overflow bins dropped and the result scaled by prod(L/N). The FFT and the
histogram run on the GPU (one fused x pass feeds the bins; nothing is written back),
the sums are FP64 and reduced in a fixed order.
"""

from __future__ import annotations

import numpy as np
import torch

from . import ops


def default_kedges(mesh_shape, box_shape) -> np.ndarray:
    """Bins used when kedges is None (reference _src/power/_compute.py:31-37)."""
    m = np.asarray(mesh_shape, dtype=np.float64)
    b = np.asarray(box_shape, dtype=np.float64)
    kmax = np.pi * np.min(m / b)
    dk = 2 * np.pi / np.min(b) * 2
    kedges = np.arange(dk, kmax, dk) + dk / 2
    if kedges.size < 2:
        kedges = np.linspace(kmax / 4, kmax * 0.9, 2)
    return kedges


def power_sums(mesh: torch.Tensor, box_shape, kedges) -> torch.Tensor:
    ke = torch.as_tensor(np.asarray(kedges, dtype=np.float32), device=mesh.device)
    return ops.power_sums(mesh.contiguous(), ke, box_shape)


def finalize(sums: torch.Tensor, mesh_shape, box_shape):
    """(k_avg, P(k)) from the (..., 3, nbins) sums, bins 1..nbins-2 kept."""
    psum, cnt, ksum = sums[..., 0, :], sums[..., 1, :], sums[..., 2, :]
    norm = torch.where(cnt > 0, cnt, torch.ones_like(cnt))
    vol = float(np.prod(np.asarray(box_shape, np.float64) / np.asarray(mesh_shape, np.float64)))
    pk = (psum / norm)[..., 1:-1] * vol
    kavg = (ksum / norm)[..., 1:-1]
    if kavg.ndim > 1:
        kavg = kavg.reshape(-1, kavg.shape[-1])[0]
    return kavg, pk


def power(mesh, mesh2=None, *, box_shape, kedges=None, multipoles=0, los=(0.0, 0.0, 1.0)):
    """Array-level 3D auto power spectrum -> (wavenumber, spectra)."""
    if mesh2 is not None:
        raise NotImplementedError("cross spectra are not on the B200 path")
    if multipoles not in (0, (0,), [0]):
        raise NotImplementedError("only the monopole is on the B200 path")
    if not isinstance(mesh, torch.Tensor):
        mesh = torch.as_tensor(np.asarray(mesh, dtype=np.float32), device="cuda")
    mesh = mesh.to(torch.float32)
    mesh_shape = tuple(int(v) for v in mesh.shape[-3:])
    box_shape = tuple(float(v) for v in box_shape)
    if kedges is None:
        kedges = default_kedges(mesh_shape, box_shape)
    if torch.is_grad_enabled() and mesh.requires_grad:
        # differentiable path: the adjoint kernel gives dL/dmesh (pm/adjoint.py)
        from .pm.adjoint import PowerSpectrum

        with torch.no_grad():
            kavg, _ = finalize(power_sums(mesh, box_shape, kedges), mesh_shape, box_shape)
        return kavg, PowerSpectrum.apply(mesh, np.asarray(kedges, np.float64), box_shape)
    sums = power_sums(mesh, box_shape, kedges)
    return finalize(sums, mesh_shape, box_shape)
