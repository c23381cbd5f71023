"""Power spectrum estimator (reference power/compute.py:13-33, _src/power/_compute.py:23-119).

P(k) = <|FFT_ortho(mesh)|^2> per digitize(|k|, kedges) bin over the full Fourier grid,
with the under/overflow bins dropped and the result scaled by prod(L/N). The FFT and the
histogram run on the GPU (one fused x pass feeds the bins; nothing is written back),
the sums are FP64 and reduced in a fixed order.
"""

from __future__ import annotations

import math

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
    ke = ops.device_table(kedges, mesh.device)
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


def poles_sums(mesh: torch.Tensor, mesh2, box_shape, kedges, poles, los):
    """The raw per-bin sums of jfli_power_poles: (batch, 2 npoles + 2, nedges + 1) FP64 --
    Re and Im of sum (2l + 1) L_l(mu) F1 conj(F2) per multipole, then the mode count and the
    sum of |k| -- and the number of multipoles."""
    mesh_shape = tuple(int(v) for v in mesh.shape[-3:])
    lead = tuple(mesh.shape[:-3])
    batch = int(np.prod(lead)) if lead else 1
    edges = ops.device_table(kedges, mesh.device)
    ells = np.ascontiguousarray(np.asarray(poles, dtype=np.int32))
    nell, nedges = int(ells.size), int(edges.numel())
    nb = ops.query("jfli_power_poles_workspace_bytes", *mesh_shape, batch, nedges, nell, int(mesh2 is not None))
    ws = ops.workspace(nb, "poles", mesh.device)
    out = torch.empty(batch, 2 * nell + 2, nedges + 1, dtype=torch.float64, device=mesh.device)
    lv = np.asarray(los, np.float64)
    lv = lv / np.linalg.norm(lv)
    import ctypes

    ops.call("jfli_power_poles", ops.stream_ptr(), ops.ptr(mesh), ops.ptr(mesh2), ops.ptr(edges), nedges,
             *(float(v) for v in box_shape), *(float(v) for v in lv), ells.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
             nell, ops.ptr(out), ops.ptr(ws), ws.numel(), *mesh_shape, batch)
    return out, nell


def power_poles(mesh: torch.Tensor, mesh2, box_shape, kedges, poles, los):
    """Cross spectra and/or multipoles (reference _src/power/_compute.py:68-119): for each
    multipole the sum over the full grid of (2l + 1) L_l(mu) F1 conj(F2) per bin, its real
    part for an auto spectrum and its modulus for a cross spectrum, over the mode count,
    bins 0 and nedges dropped, times prod(L/N). -> (kavg, pk (npoles, nbins) or (nbins,))."""
    mesh_shape = tuple(int(v) for v in mesh.shape[-3:])
    lead = tuple(mesh.shape[:-3])
    out, nell = poles_sums(mesh, mesh2, box_shape, kedges, poles, los)
    cnt = out[:, 2 * nell]
    norm = torch.where(cnt > 0, cnt, torch.ones_like(cnt))
    re, im = out[:, 0:2 * nell:2], out[:, 1:2 * nell:2]
    psum = torch.sqrt(re**2 + im**2) if mesh2 is not None else re
    vol = float(np.prod(np.asarray(box_shape, np.float64) / np.asarray(mesh_shape, np.float64)))
    pk = (psum / norm[:, None, :])[..., 1:-1] * vol
    kavg = (out[0, 2 * nell + 1] / norm[0])[1:-1]
    pk = pk.reshape(*lead, nell, -1) if lead else pk[0]
    if nell == 1:
        pk = pk[..., 0, :]
    return kavg, pk


def power(mesh, mesh2=None, *, box_shape, kedges=None, multipoles=0, los=(0.0, 0.0, 1.0)):
    """Array-level 3D power spectrum -> (wavenumber, spectra): auto or cross (mesh2), the
    monopole or Legendre multipoles along `los` (reference power/compute.py:13-33)."""
    if not isinstance(mesh, torch.Tensor):
        mesh = torch.as_tensor(np.asarray(mesh, dtype=np.float32), device="cuda")
    mesh = mesh.to(torch.float32)
    mesh_shape = tuple(int(v) for v in mesh.shape[-3:])
    box_shape = tuple(float(v) for v in box_shape)
    if kedges is None:
        kedges = default_kedges(mesh_shape, box_shape)
    poles = tuple(multipoles) if isinstance(multipoles, (list, tuple)) else (multipoles,)
    if mesh2 is not None or poles != (0,):
        grad = torch.is_grad_enabled() and (mesh.requires_grad or (isinstance(mesh2, torch.Tensor)
                                                                   and mesh2.requires_grad))
        if grad and mesh.dim() != 3:
            raise NotImplementedError("gradients of batched spectra are not on the B200 path")
        m2 = None
        if mesh2 is not None:
            m2 = mesh2 if isinstance(mesh2, torch.Tensor) else torch.as_tensor(np.asarray(mesh2, np.float32),
                                                                                device="cuda")
            m2 = m2.to(torch.float32).contiguous()
            if m2.shape != mesh.shape:
                raise ValueError("mesh2 must have the shape of mesh")
        # multipoles == 0 uses mu = 1 in the reference (no line of sight): L_0 = 1 either way
        if grad and mesh2 is None:  # multipoles of an auto spectrum
            from .pm.adjoint import PowerPoles

            with torch.no_grad():
                kavg, _ = power_poles(mesh.contiguous(), None, box_shape, kedges, poles, los)
            return kavg, PowerPoles.apply(mesh.contiguous(), np.asarray(kedges, np.float64), box_shape, poles, los)
        if grad and poles != (0,):  # cross-spectrum multipoles
            from .pm.adjoint import CrossPoles

            with torch.no_grad():
                kavg, _ = power_poles(mesh.contiguous(), m2, box_shape, kedges, poles, los)
            return kavg, CrossPoles.apply(mesh.contiguous(), m2, np.asarray(kedges, np.float64), box_shape, poles, los)
        if grad:
            from .pm.adjoint import CrossPowerSpectrum

            with torch.no_grad():
                kavg, _ = power_poles(mesh.contiguous(), m2, box_shape, kedges, poles, los)
            return kavg, CrossPowerSpectrum.apply(mesh.contiguous(), m2, np.asarray(kedges, np.float64), box_shape)
        return power_poles(mesh.contiguous(), m2, box_shape, kedges, poles, los)
    if torch.is_grad_enabled() and mesh.requires_grad:
        # differentiable path: the adjoint kernel gives dL/dmesh (pm/adjoint.py)
        from .pm.adjoint import PowerSpectrum

        with torch.no_grad():
            kavg, _ = finalize(power_sums(mesh, box_shape, kedges), mesh_shape, box_shape)
        return kavg, PowerSpectrum.apply(mesh, np.asarray(kedges, np.float64), box_shape)
    sums = power_sums(mesh, box_shape, kedges)
    return finalize(sums, mesh_shape, box_shape)


def flat_ell_grid_max(npx: int, npy: int, px: float, py: float) -> np.float32:
    """Largest |ell| of the flat-sky FFT grid, formed in FP32 as the kernel forms it."""
    def comp(n, d):
        k = np.float32(-(n // 2)) if n % 2 == 0 else np.float32((n - 1) // 2)
        return np.float32(np.float32(2.0 * np.pi) * np.float32(k / np.float32(n * d)))

    lx, ly = comp(npx, px), comp(npy, py)
    return np.float32(np.sqrt(np.float32(np.float32(lx * lx) + np.float32(ly * ly))))


def angular_cl_flat(map1, map2=None, *, pixel_size=None, field_size=None, ell_edges=None):
    """Flat-sky C_ell (reference power/compute.py:70-86 -> _src/power/_compute.py:122-172):
    (ell, cl) with cl the mean of Re(F1 conj F2) (px py) / (npx npy) over the modes of each
    ell bin (numpy.digitize on the edges; under/overflow bins dropped) and ell the mean |ell|.
    pixel_size (px, py) in radians per pixel, or field_size (fx, fy) with px = fx / npx.
    Default edges: 50 from 0 to the largest |ell| of the grid."""
    m1 = map1 if isinstance(map1, torch.Tensor) else torch.as_tensor(np.asarray(map1, np.float32), device="cuda")
    m1 = m1.to(torch.float32).contiguous()
    m2 = None
    if map2 is not None:
        m2 = map2 if isinstance(map2, torch.Tensor) else torch.as_tensor(np.asarray(map2, np.float32), device="cuda")
        m2 = m2.to(torch.float32).contiguous()
        if m2.shape != m1.shape:
            raise ValueError("map2 must have the same shape as map2d for cross Cl")
    npx, npy = m1.shape[-2:]
    if pixel_size is None:
        if field_size is None:
            raise ValueError("pixel_size or field_size must be provided for flat-sky Cl")
        fx, fy = (field_size, field_size) if np.ndim(field_size) == 0 else field_size
        px, py = float(fx) / npx, float(fy) / npy
    else:
        px, py = (pixel_size, pixel_size) if np.ndim(pixel_size) == 0 else pixel_size
        px, py = float(px), float(py)
    if ell_edges is None:
        top = flat_ell_grid_max(npx, npy, px, py)
        edges = np.linspace(0.0, float(top), 50).astype(np.float32)
        edges[-1] = top
    else:
        edges = np.asarray(ell_edges, dtype=np.float32)
    sums = ops.flat_cl_sums(m1, m2, npx * px, npy * py, torch.as_tensor(edges))
    norm = (px * py) / (npx * npy)
    cnt = torch.where(sums[:, 1] > 0, sums[:, 1], torch.ones_like(sums[:, 1]))
    cl = (sums[:, 0] / cnt * norm)[:, 1:-1]
    ell = (sums[0, 2] / cnt[0])[1:-1]
    if m1.ndim == 2:
        cl = cl[0]
    return ell, cl


def transfer(mesh0, mesh1, *, box_shape, kedges=None):
    """Monopole transfer function sqrt(P1 / P0) (reference _src/power/_compute.py:239-243)."""
    k, pk0 = power(mesh0, box_shape=box_shape, kedges=kedges)
    _, pk1 = power(mesh1, box_shape=box_shape, kedges=kedges)
    return k, (pk1 / pk0) ** 0.5


def coherence(mesh0, mesh1, *, box_shape, kedges=None):
    """Monopole coherence P01 / sqrt(P0 P1) (reference _src/power/_compute.py:246-251)."""
    k, pk01 = power(mesh0, mesh1, box_shape=box_shape, kedges=kedges)
    _, pk0 = power(mesh0, box_shape=box_shape, kedges=kedges)
    _, pk1 = power(mesh1, box_shape=box_shape, kedges=kedges)
    return k, pk01 / (pk0 * pk1) ** 0.5


def angular_cl_spherical(map_sphere, map_sphere2=None, *, lmax: int | None = None, method: str = "jax"):
    """Spherical C_l, auto or cross (reference power/compute.py:89-98 -> healpy anafast):
    (ell, cl) as device float64 tensors. Both method values run healpy's algorithm in this
    library's GPU engine; the maps, a_lm and spectra stay on the device."""
    from . import sht

    if method not in ("jax", "healpy"):
        raise ValueError(f"unknown method {method!r}")
    npix = map_sphere.numel() if isinstance(map_sphere, torch.Tensor) else np.asarray(map_sphere).size
    lmax = 3 * sht._nside_of(int(npix)) - 1 if lmax is None else int(lmax)
    a1 = sht.map2alm(map_sphere, lmax)
    a2 = None if map_sphere2 is None else sht.map2alm(map_sphere2, lmax)
    cl = sht.alm2cl(a1, lmax, a2)
    return torch.arange(lmax + 1, dtype=torch.float64, device=cl.device), cl


def cross_angular_cl_spherical(maps, *, lmax: int | None = None, method: str = "healpy"):
    """All cross C_l of B maps in healpy's order (reference power/compute.py:101-109)."""
    from . import sht

    if method != "healpy":
        raise ValueError(f"cross_angular_cl_spherical only supports method='healpy', got method='{method}'.")
    cls = sht.cross_cls(maps, lmax)
    return torch.arange(cls.shape[-1], dtype=torch.float64, device=cls.device), cls
