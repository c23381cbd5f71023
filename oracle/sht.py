"""Spherical harmonic analysis of HEALPix RING maps (FP64) on the CPU -- TEST
INFRASTRUCTURE ONLY.

Only tests/ and the fixture generators under tests/golden/ import this module, as the
checker of the library's GPU SHT; the product never does.

The reference computes angular power spectra with healpy.anafast
(_src/power/_compute.py:175-191 -> hp.anafast / jhp.anafast; healpy and jax-healpy are not
installed here). This module restates that published algorithm in NumPy:

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

Pinned by scipy's sph_harm_y, band-limited analysis/synthesis round trips and the spectra
of constant and Y_10 maps (tests/test_sht.py).
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


def _packed_offsets(lmax):
    m = np.arange(lmax + 2, dtype=np.int64)
    return m * (lmax + 1) - m * (m - 1) // 2


def _map2alm_once(m, nside, lmax):
    """One analysis: the ring FFTs in NumPy, the Legendre stage in the C restatement
    (oracle/sht.c) of the recursion above."""
    from . import clib

    z, _, _, _ = ring_geometry(nside)
    F = _ring_ffts(m, nside, lmax)
    packed = clib.sht_analysis(F, z, lmax, 4.0 * math.pi / m.size)
    off = _packed_offsets(lmax)
    return {mm: packed[off[mm]:off[mm + 1]] for mm in range(lmax + 1)}


def _map2alm_once_np(m, nside, lmax):
    """_map2alm_once with the Legendre stage in NumPy (the C stage is tested against it)."""
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
    from . import clib

    z, _, _, _ = ring_geometry(nside)
    packed = np.concatenate([np.asarray(alm[mm], np.complex128) for mm in range(lmax + 1)])
    return _ring_synth(clib.sht_synthesis(packed, z, lmax), nside, lmax)


def alm2map_np(alm: dict, nside: int, lmax: int) -> np.ndarray:
    """alm2map with the Legendre stage in NumPy."""
    z, _, _, _ = ring_geometry(nside)
    sint = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    G = np.zeros((z.size, lmax + 1), dtype=np.complex128)
    for mm in range(lmax + 1):
        lam = _lambda_m(mm, lmax, z, sint)
        G[:, mm] = alm[mm] @ lam
    return _ring_synth(G, nside, lmax)


def alm2cl(alm: dict, lmax: int) -> np.ndarray:
    cl = np.zeros(lmax + 1)
    for l in range(lmax + 1):
        s = abs(alm[0][l]) ** 2
        acc = [abs(alm[mm][l - mm]) ** 2 for mm in range(1, l + 1)]
        cl[l] = (s + 2.0 * math.fsum(acc)) / (2 * l + 1)
    return cl


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


def anafast(m: np.ndarray, lmax: int | None = None, iter: int = 3) -> np.ndarray:
    """C_l, l = 0..lmax, of a RING-ordered HEALPix map (healpy.anafast defaults)."""
    m = np.asarray(m, dtype=np.float64)
    nside = int(round(math.sqrt(m.size / 12)))
    lmax = 3 * nside - 1 if lmax is None else int(lmax)
    return alm2cl(map2alm(m, lmax, iter), lmax)


def alm2cl_cross(a1: dict, a2: dict, lmax: int) -> np.ndarray:
    """Cross C_l of two a_lm dicts: (Re a1_l0 a2_l0* + 2 sum_{m>0} Re a1_lm a2_lm*) / (2l + 1)."""
    cl = np.zeros(lmax + 1)
    for l in range(lmax + 1):
        acc = [float((a1[mm][l - mm] * np.conj(a2[mm][l - mm])).real) for mm in range(1, l + 1)]
        cl[l] = (float((a1[0][l] * np.conj(a2[0][l])).real) + 2.0 * math.fsum(acc)) / (2 * l + 1)
    return cl
