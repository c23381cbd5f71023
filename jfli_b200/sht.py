"""Spherical harmonic analysis of HEALPix RING maps (FP64) on the GPU, for C_ell.

The reference computes angular power spectra with healpy.anafast
(_src/power/_compute.py:175-191 -> hp.anafast / jhp.anafast). This module runs that
published algorithm with the map, the a_lm and the spectrum on the device, in the
library's FP64 kernels:

* the ring transforms along phi as direct DFTs (`jfli_sht_ring_analysis`,
  `jfli_sht_ring_synthesis`): F_r(m) = e^{-i m phi_0} sum_j f_j e^{-2 pi i m j / n_r};
* the O(lmax^2 x rings) Legendre stages (`jfli_sht_map2alm`, `jfli_sht_alm2map`) with
  uniform quadrature weights 4 pi / npix and a_lm packed by m (a[m][l - m]);
* healpy's default iterative refinement (iter=3): a += map2alm(map - alm2map(a));
* C_l = (Re a_l0 b_l0* + 2 sum_{m>0} Re a_lm b_lm*) / (2l + 1) (`jfli_sht_alm2cl`).
lambda_lm are the orthonormal associated Legendre functions with the Condon-Shortley
phase (three-term recursion in l at fixed m, lambda_mm formed in log space).
"""

from __future__ import annotations

import math

import numpy as np
import torch


def ring_geometry(nside: int):
    """(z, n_pix, phi0, start) per ring, RING ordering, north to south."""
    nr = 4 * nside - 1
    z = np.empty(nr)
    npr = np.empty(nr, np.int64)
    phi0 = np.empty(nr)
    start = np.empty(nr, np.int64)
    s = 0
    for r in range(nr):
        i = r + 1
        if i < nside:  # north cap
            npr[r] = 4 * i
            z[r] = 1.0 - i * i / (3.0 * nside * nside)
            phi0[r] = math.pi / (4.0 * i)
        elif i <= 3 * nside:  # equatorial belt
            npr[r] = 4 * nside
            z[r] = 4.0 / 3.0 - 2.0 * i / (3.0 * nside)
            shifted = (i - nside + 1) % 2
            phi0[r] = 0.0 if shifted == 1 else math.pi / (4.0 * nside)
        else:  # south cap
            j = 4 * nside - i
            npr[r] = 4 * j
            z[r] = -(1.0 - j * j / (3.0 * nside * nside))
            phi0[r] = math.pi / (4.0 * j)
        start[r] = s
        s += npr[r]
    return z, npr, phi0, start


def packed_offsets(lmax: int) -> np.ndarray:
    """Start of each m in the packed a_lm array (a[m][l - m])."""
    m = np.arange(lmax + 2, dtype=np.int64)
    return m * (lmax + 1) - m * (m - 1) // 2


class _GpuSht:
    """Device tables of one (nside, lmax) and the four device stages: ring transforms along
    phi (direct FP64 DFTs) and the Legendre stages. Maps and a_lm stay on the device."""

    def __init__(self, nside: int, lmax: int, device=None):
        self.nside, self.lmax = nside, lmax
        self.device = torch.device("cuda") if device is None else torch.device(device)
        z, _, _, _ = ring_geometry(nside)
        self.nrings = z.size
        self.z = torch.as_tensor(z, dtype=torch.float64, device=self.device)
        self.nalm = (lmax + 1) * (lmax + 2) // 2
        self.F = torch.empty(self.nrings, lmax + 1, dtype=torch.complex128, device=self.device)

    def map2alm_once(self, m: torch.Tensor) -> torch.Tensor:
        """Packed a_lm (device, complex128) of a device FP64 map."""
        from ._lib import call, stream_ptr

        call("jfli_sht_ring_analysis", stream_ptr(), m.data_ptr(), self.nside, self.lmax, self.F.data_ptr())
        alm = torch.empty(self.nalm, dtype=torch.complex128, device=self.device)
        call("jfli_sht_map2alm", stream_ptr(), self.F.data_ptr(), self.z.data_ptr(), self.nrings, self.lmax,
             4.0 * math.pi / m.numel(), alm.data_ptr())
        return alm

    def alm2map(self, alm: torch.Tensor) -> torch.Tensor:
        """Device FP64 map of packed device a_lm."""
        from ._lib import call, stream_ptr

        call("jfli_sht_alm2map", stream_ptr(), alm.data_ptr(), self.z.data_ptr(), self.nrings, self.lmax,
             self.F.data_ptr())
        out = torch.empty(12 * self.nside * self.nside, dtype=torch.float64, device=self.device)
        call("jfli_sht_ring_synthesis", stream_ptr(), self.F.data_ptr(), self.nside, self.lmax, out.data_ptr())
        return out


_ENGINES: dict = {}


def _engine(nside: int, lmax: int, device) -> _GpuSht:
    key = (nside, lmax, str(device))
    eng = _ENGINES.get(key)
    if eng is None:
        if len(_ENGINES) > 8:
            _ENGINES.clear()
        eng = _ENGINES[key] = _GpuSht(nside, lmax, device)
    return eng


def _device_map(m) -> torch.Tensor:
    """A contiguous FP64 CUDA copy (or view) of a map given as a tensor or an array."""
    if isinstance(m, torch.Tensor):
        dev = m.device if m.is_cuda else torch.device("cuda")
        return m.detach().to(device=dev, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.asarray(m, dtype=np.float64), device="cuda")


def _nside_of(npix: int) -> int:
    nside = int(round(math.sqrt(npix / 12)))
    if 12 * nside * nside != npix:
        raise ValueError("map size is not 12 nside^2")
    return nside


def map2alm(m, lmax: int | None = None, iter: int = 3) -> torch.Tensor:
    """Packed a_lm (device complex128, (lmax + 1)(lmax + 2) / 2) of a RING map (healpy
    map2alm with uniform weights and `iter` Jacobi iterations); the map may be a tensor on
    any device or an array, and is moved to the GPU once."""
    md = _device_map(m).reshape(-1)
    nside = _nside_of(md.numel())
    lmax = 3 * nside - 1 if lmax is None else int(lmax)
    eng = _engine(nside, lmax, md.device)
    alm = eng.map2alm_once(md)
    for _ in range(iter):
        alm = alm + eng.map2alm_once(md - eng.alm2map(alm))
    return alm


def alm2cl(alm1: torch.Tensor, lmax: int, alm2: torch.Tensor | None = None) -> torch.Tensor:
    """C_l (device float64, l = 0..lmax) of packed device a_lm; the cross spectrum with alm2."""
    from ._lib import call, stream_ptr

    cl = torch.empty(lmax + 1, dtype=torch.float64, device=alm1.device)
    call("jfli_sht_alm2cl", stream_ptr(), alm1.data_ptr(), None if alm2 is None else alm2.data_ptr(), lmax,
         cl.data_ptr())
    return cl


def anafast(m, lmax: int | None = None, iter: int = 3) -> torch.Tensor:
    """C_l, l = 0..lmax, of a RING-ordered HEALPix map (healpy.anafast defaults), as a
    device float64 tensor."""
    md = _device_map(m).reshape(-1)
    lmax = 3 * _nside_of(md.numel()) - 1 if lmax is None else int(lmax)
    return alm2cl(map2alm(md, lmax, iter), lmax)


def cross_cls(maps, lmax: int | None = None, iter: int = 3) -> torch.Tensor:
    """All auto and cross C_l of B maps (B, npix), each map analysed once, in healpy's
    alm2cl order: the diagonal first (11, 22, ...), then the first off-diagonal (12, 23,
    ...), and so on. -> device (B (B + 1) / 2, lmax + 1)."""
    md = _device_map(maps)
    md = md.reshape(-1, md.shape[-1])
    lmax = 3 * _nside_of(md.shape[1]) - 1 if lmax is None else int(lmax)
    alms = [map2alm(row, lmax, iter) for row in md]
    b = len(alms)
    return torch.stack([alm2cl(alms[i], lmax, alms[i + d]) for d in range(b) for i in range(b - d)])
