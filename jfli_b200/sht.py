"""Spherical harmonic analysis of HEALPix RING maps (FP64), for C_ell.

The reference computes angular power spectra with healpy.anafast
(_src/power/_compute.py:175-191 -> hp.anafast / jhp.anafast). This module restates that
published algorithm:

* map2alm with uniform quadrature weights 4 pi / npix: per ring, an FFT along phi gives
  F_r(m) = e^{-i m phi_0} sum_j f_j e^{-2 pi i m j / n_r} (m folded modulo the ring length),
  then a_lm = 4 pi / npix sum_r lambda_lm(theta_r) F_r(m);
* alm2map, the transpose synthesis;
* healpy's default iterative refinement (iter=3): a += map2alm(map - alm2map(a));
* C_l = (|a_l0|^2 + 2 sum_{m>0} |a_lm|^2) / (2l + 1).
lambda_lm are the orthonormal associated Legendre functions with the Condon-Shortley
phase, built by the standard three-term recursion in l at fixed m; the starting value
lambda_mm is formed in log space so that polar rings at large m underflow to zero
instead of to NaN.

Two engines:
* "gpu" (default): everything on the device in the library's FP64 kernels: the ring
  transforms along phi as direct DFTs (`jfli_sht_ring_analysis`, `jfli_sht_ring_synthesis`)
  and the O(lmax^2 x rings) Legendre stages (`jfli_sht_map2alm`, `jfli_sht_alm2map`; a_lm
  packed by m); the map and the a_lm stay on the device through the iterations;
* "host": numpy FFTs along the rings and the same recursion in numpy, kept as the
  restatement the GPU engine is tested against.
"""

from __future__ import annotations

import math

import numpy as np


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


_BIG = 1e100
_LN_BIG = math.log(_BIG)


def _lambda_m(m: int, lmax: int, x: np.ndarray, sint: np.ndarray) -> np.ndarray:
    """lambda_lm(theta_r) for l = m..lmax at fixed m: array (lmax - m + 1, nrings).

    lambda_mm = (-1)^m sqrt((2m+1)/(4 pi) prod_{k<=m} (2k-1)/(2k)) sin^m theta is formed in
    log space. Where it is below FP64 range the recursion runs on values scaled by e^s
    (per ring) and the scale is removed as the values grow, so that rings where the
    function becomes significant before lmax are not lost to underflow."""
    out = np.zeros((lmax - m + 1, x.size))
    k = np.arange(1, m + 1)
    logc = 0.5 * math.log((2 * m + 1) / (4 * math.pi)) + 0.5 * float(np.sum(np.log((2 * k - 1) / (2.0 * k))))
    with np.errstate(divide="ignore"):
        logv = logc + m * np.log(sint)
    logv = np.where(np.isfinite(logv), logv, -np.inf)
    scale = np.where(logv < -600.0, -300.0 - logv, 0.0)  # computed = true * e^scale
    scale = np.where(np.isfinite(scale), scale, np.inf)
    sign = -1.0 if m % 2 else 1.0
    with np.errstate(over="ignore", invalid="ignore"):
        cur = np.where(np.isfinite(scale), sign * np.exp(logv + scale), 0.0)

    def emit(vals):
        with np.errstate(under="ignore"):
            return np.where(scale < 745.0, vals * np.exp(-np.minimum(scale, 745.0)), 0.0)

    out[0] = emit(cur)
    if lmax == m:
        return out
    prev = cur
    cur = x * math.sqrt(2 * m + 3) * prev
    out[1] = emit(cur)
    for l in range(m + 2, lmax + 1):
        a = math.sqrt((4.0 * l * l - 1.0) / (l * l - m * m))
        b = math.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1.0) ** 2 - 1.0))
        nxt = a * (x * cur - b * prev)
        big = (np.abs(nxt) > _BIG) & (scale > 0)
        if big.any():
            nxt = np.where(big, nxt / _BIG, nxt)
            cur = np.where(big, cur / _BIG, cur)
            scale = np.where(big, scale - _LN_BIG, scale)
        prev, cur = cur, nxt
        out[l - m] = emit(cur)
    return out


def _ring_ffts(maps: np.ndarray, nside: int, mmax: int):
    z, npr, phi0, start = ring_geometry(nside)
    F = np.zeros((z.size, mmax + 1), dtype=np.complex128)
    m = np.arange(mmax + 1)
    for r in range(z.size):
        ring = maps[start[r]:start[r] + npr[r]]
        f = np.fft.fft(ring)
        F[r] = f[m % npr[r]] * np.exp(-1j * m * phi0[r])
    return F


def map2alm(m: np.ndarray, lmax: int | None = None, iter: int = 3):
    """a_lm as a dict m -> complex array over l = m..lmax (healpy map2alm, uniform weights)."""
    m = np.asarray(m, dtype=np.float64)
    nside = int(round(math.sqrt(m.size / 12)))
    if 12 * nside * nside != m.size:
        raise ValueError("map size is not 12 nside^2")
    lmax = 3 * nside - 1 if lmax is None else int(lmax)
    alm = _map2alm_once(m, nside, lmax)
    for _ in range(iter):
        alm_res = _map2alm_once(m - alm2map(alm, nside, lmax), nside, lmax)
        alm = {k: alm[k] + alm_res[k] for k in alm}
    return alm


def _map2alm_once(m, nside, lmax):
    z, _, _, _ = ring_geometry(nside)
    sint = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    F = _ring_ffts(m, nside, lmax)
    w = 4.0 * math.pi / m.size
    out = {}
    for mm in range(lmax + 1):
        lam = _lambda_m(mm, lmax, z, sint)  # (L, R)
        out[mm] = w * (lam @ F[:, mm])
    return out


def alm2map(alm: dict, nside: int, lmax: int) -> np.ndarray:
    z, npr, phi0, start = ring_geometry(nside)
    sint = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    G = np.zeros((z.size, lmax + 1), dtype=np.complex128)
    for mm in range(lmax + 1):
        lam = _lambda_m(mm, lmax, z, sint)
        G[:, mm] = alm[mm] @ lam
    out = np.empty(12 * nside * nside)
    mvec = np.arange(lmax + 1)
    for r in range(z.size):
        n = int(npr[r])
        c = G[r] * np.exp(1j * mvec * phi0[r])
        spec = np.zeros(n, dtype=np.complex128)
        spec[0] += c[0].real
        np.add.at(spec, mvec[1:] % n, c[1:])
        # real part of sum_m>=0 c_m e^{i m phi} with the m > 0 terms counted twice
        vals = np.fft.ifft(spec) * n
        out[start[r]:start[r] + n] = 2.0 * vals.real - c[0].real
    return out


def alm2cl(alm: dict, lmax: int) -> np.ndarray:
    cl = np.zeros(lmax + 1)
    for l in range(lmax + 1):
        s = abs(alm[0][l]) ** 2
        acc = [abs(alm[mm][l - mm]) ** 2 for mm in range(1, l + 1)]
        cl[l] = (s + 2.0 * math.fsum(acc)) / (2 * l + 1)
    return cl


# ------------------------------------------------------------------------- GPU engine
def _ring_synth(G: np.ndarray, nside: int, lmax: int) -> np.ndarray:
    """Map from per-ring coefficients G[r][m] (inverse of _ring_ffts)."""
    z, npr, phi0, start = ring_geometry(nside)
    out = np.empty(12 * nside * nside)
    mvec = np.arange(lmax + 1)
    for r in range(z.size):
        n = int(npr[r])
        c = G[r] * np.exp(1j * mvec * phi0[r])
        spec = np.zeros(n, dtype=np.complex128)
        spec[0] += c[0].real
        np.add.at(spec, mvec[1:] % n, c[1:])
        vals = np.fft.ifft(spec) * n
        out[start[r]:start[r] + n] = 2.0 * vals.real - c[0].real
    return out


class _GpuSht:
    """Device tables of one (nside, lmax) and the four device stages: ring transforms along
    phi (direct FP64 DFTs) and the Legendre stages. Maps and a_lm stay on the device."""

    def __init__(self, nside: int, lmax: int):
        import torch

        self.nside, self.lmax = nside, lmax
        z, _, _, _ = ring_geometry(nside)
        self.nrings = z.size
        self.z = torch.as_tensor(z, dtype=torch.float64, device="cuda")
        self.nalm = (lmax + 1) * (lmax + 2) // 2
        self.F = torch.empty(self.nrings, lmax + 1, dtype=torch.complex128, device="cuda")

    def map2alm_once(self, m):
        """Packed a_lm (device, complex128) of a device FP64 map."""
        import torch

        from ._lib import call, stream_ptr

        call("jfli_sht_ring_analysis", stream_ptr(), m.data_ptr(), self.nside, self.lmax, self.F.data_ptr())
        alm = torch.empty(self.nalm, dtype=torch.complex128, device="cuda")
        call("jfli_sht_map2alm", stream_ptr(), self.F.data_ptr(), self.z.data_ptr(), self.nrings, self.lmax,
             4.0 * math.pi / m.numel(), alm.data_ptr())
        return alm

    def alm2map(self, alm):
        """Device FP64 map of packed device a_lm."""
        import torch

        from ._lib import call, stream_ptr

        call("jfli_sht_alm2map", stream_ptr(), alm.data_ptr(), self.z.data_ptr(), self.nrings, self.lmax,
             self.F.data_ptr())
        out = torch.empty(12 * self.nside * self.nside, dtype=torch.float64, device="cuda")
        call("jfli_sht_ring_synthesis", stream_ptr(), self.F.data_ptr(), self.nside, self.lmax, out.data_ptr())
        return out


def packed_offsets(lmax: int) -> np.ndarray:
    """Start of each m in the packed a_lm array (a[m][l - m])."""
    m = np.arange(lmax + 2, dtype=np.int64)
    return m * (lmax + 1) - m * (m - 1) // 2


def map2alm_gpu(m: np.ndarray, lmax: int | None = None, iter: int = 3) -> np.ndarray:
    """Packed a_lm (complex128, (lmax + 1)(lmax + 2) / 2) with the GPU Legendre stages."""
    m = np.asarray(m, dtype=np.float64)
    nside = int(round(math.sqrt(m.size / 12)))
    if 12 * nside * nside != m.size:
        raise ValueError("map size is not 12 nside^2")
    lmax = 3 * nside - 1 if lmax is None else int(lmax)
    import torch

    eng = _GpuSht(nside, lmax)
    md = torch.as_tensor(m, dtype=torch.float64, device="cuda")
    alm = eng.map2alm_once(md)
    for _ in range(iter):
        alm = alm + eng.map2alm_once(md - eng.alm2map(alm))
    return alm.cpu().numpy()


def packed_to_dict(alm: np.ndarray, lmax: int) -> dict:
    off = packed_offsets(lmax)
    return {mm: alm[off[mm]:off[mm + 1]] for mm in range(lmax + 1)}


def alm2cl_packed(alm: np.ndarray, lmax: int) -> np.ndarray:
    off = packed_offsets(lmax)
    p = np.abs(alm) ** 2
    cl = p[off[0]:off[1]].copy()
    for mm in range(1, lmax + 1):
        cl[mm:] += 2.0 * p[off[mm]:off[mm + 1]]
    return cl / (2.0 * np.arange(lmax + 1) + 1.0)


def anafast(m: np.ndarray, lmax: int | None = None, iter: int = 3, engine: str = "gpu") -> np.ndarray:
    """C_l, l = 0..lmax, of a RING-ordered HEALPix map (healpy.anafast defaults)."""
    m = np.asarray(m, dtype=np.float64)
    nside = int(round(math.sqrt(m.size / 12)))
    lmax = 3 * nside - 1 if lmax is None else int(lmax)
    if engine == "gpu":
        return alm2cl_packed(map2alm_gpu(m, lmax, iter), lmax)
    if engine != "host":
        raise ValueError(f"unknown engine {engine!r} (gpu, host)")
    return alm2cl(map2alm(m, lmax, iter), lmax)


def alm2cl_cross_packed(a1: np.ndarray, a2: np.ndarray, lmax: int) -> np.ndarray:
    """Cross C_l of two packed a_lm sets: (Re a1_l0 a2_l0* + 2 sum_{m>0} Re a1_lm a2_lm*) / (2l + 1)."""
    off = packed_offsets(lmax)
    p = (a1 * np.conj(a2)).real
    cl = p[off[0]:off[1]].copy()
    for mm in range(1, lmax + 1):
        cl[mm:] += 2.0 * p[off[mm]:off[mm + 1]]
    return cl / (2.0 * np.arange(lmax + 1) + 1.0)


def cross_cls(maps, lmax: int | None = None, iter: int = 3) -> np.ndarray:
    """All auto and cross C_l of B maps (B, npix), each map analysed once (GPU engine), in
    healpy's alm2cl order: the diagonal first (11, 22, ...), then the first off-diagonal
    (12, 23, ...), and so on. -> (B (B + 1) / 2, lmax + 1)."""
    maps = np.atleast_2d(np.asarray(maps, dtype=np.float64))
    nside = int(round(math.sqrt(maps.shape[1] / 12)))
    lmax = 3 * nside - 1 if lmax is None else int(lmax)
    alms = [map2alm_gpu(m, lmax, iter) for m in maps]
    b = len(alms)
    return np.stack([alm2cl_cross_packed(alms[i], alms[i + d], lmax) for d in range(b) for i in range(b - d)])
