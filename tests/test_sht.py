"""Spherical harmonic transform behind SphericalDensity.angular_cl (healpy.anafast
restated): the oracle's host restatement against scipy, analysis/synthesis round trips and
known maps (CPU); the library's GPU engine against the oracle (gpu)."""

import math

import numpy as np
import pytest
from scipy.special import sph_harm_y

from jfli_b200 import sht
from oracle import sht as osht


@pytest.mark.parametrize("m", [0, 1, 7, 30])
def test_legendre_matches_scipy(m):
    z, _, _, _ = osht.ring_geometry(32)
    lam = osht._lambda_m(m, 80, z, np.sqrt(1 - z * z))
    ref = np.array([sph_harm_y(l, m, np.arccos(z), 0.0).real for l in range(m, 81)])
    assert np.abs(lam - ref).max() < 1e-12


def test_ring_geometry_covers_the_sphere():
    for nside in (1, 2, 8, 32):
        z, npr, phi0, start = sht.ring_geometry(nside)
        zo, npo, phio, so = osht.ring_geometry(nside)
        assert np.array_equal(z, zo) and np.array_equal(npr, npo) and np.array_equal(phi0, phio)
        assert npr.sum() == 12 * nside * nside
        assert np.all(np.diff(z) < 0)
        assert start[-1] + npr[-1] == 12 * nside * nside


def test_band_limited_round_trip():
    nside, lmax = 16, 32
    rng = np.random.default_rng(0)
    alm = {m: rng.standard_normal(lmax - m + 1) + 1j * rng.standard_normal(lmax - m + 1) for m in range(lmax + 1)}
    alm[0] = alm[0].real.astype(complex)
    mp = osht.alm2map(alm, nside, lmax)
    back = osht.map2alm(mp, lmax, iter=10)
    assert max(np.abs(back[m] - alm[m]).max() for m in alm) < 1e-8
    cl = osht.alm2cl(alm, lmax)
    assert np.allclose(osht.anafast(mp, lmax, iter=10), cl, rtol=1e-8)


def test_known_maps():
    nside = 16
    npix = 12 * nside * nside
    c = osht.anafast(np.full(npix, 2.0), iter=0)
    # HEALPix quadrature aliases ~1e-7 of C_0 into multipoles near 3 nside
    assert abs(c[0] / (4 * math.pi * 4.0) - 1) < 1e-12 and np.abs(c[1:]).max() < 1e-6 * c[0]
    z, npr, _, start = osht.ring_geometry(nside)
    zz = np.repeat(z, npr)
    y10 = math.sqrt(3 / (4 * math.pi)) * zz  # Y_10: C_1 = 1 for a_10 = 1
    cl = osht.anafast(y10, lmax=8, iter=3)
    assert abs(cl[1] / (1.0 / 3.0) - 1) < 1e-3 and cl[[0, 2, 3, 4]].max() < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("nside,lmax", [(8, 23), (32, 64), (64, 191)])
def test_gpu_legendre_stages_match_host(nside, lmax):
    """The GPU Legendre stages against the host recursion: packed a_lm of one analysis and
    one synthesis, and the iterated C_ell."""
    import torch

    rng = np.random.default_rng(nside)
    m = rng.standard_normal(12 * nside * nside)
    eng = sht._GpuSht(nside, lmax)
    a_gpu = eng.map2alm_once(torch.as_tensor(m, device="cuda")).cpu().numpy()
    a_host = osht._map2alm_once(m, nside, lmax)
    off = sht.packed_offsets(lmax)
    d = {mm: a_gpu[off[mm]:off[mm + 1]] for mm in range(lmax + 1)}
    scale = max(np.abs(v).max() for v in a_host.values())
    assert max(np.abs(d[k] - a_host[k]).max() for k in a_host) < 1e-12 * scale
    back_gpu = eng.alm2map(torch.as_tensor(a_gpu, device="cuda")).cpu().numpy()
    back_host = osht.alm2map(a_host, nside, lmax)
    assert np.abs(back_gpu - back_host).max() < 1e-11 * np.abs(back_host).max()
    cg = sht.anafast(torch.as_tensor(m, device="cuda"), lmax)
    assert cg.is_cuda and cg.dtype == torch.float64
    ch = osht.anafast(m, lmax)
    np.testing.assert_allclose(cg.cpu().numpy(), ch, rtol=1e-9)
    # the device alm2cl against the oracle's on the same a_lm
    np.testing.assert_allclose(sht.alm2cl(torch.as_tensor(a_gpu, device="cuda"), lmax).cpu().numpy(),
                               osht.alm2cl(d, lmax), rtol=1e-12)


@pytest.mark.gpu
def test_gpu_sht_large_lmax_round_trip():
    """nside 256, lmax 500: band-limited a_lm -> map -> a_lm with 3 iterations."""
    nside, lmax = 256, 500
    rng = np.random.default_rng(5)
    n = (lmax + 1) * (lmax + 2) // 2
    alm = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    off = sht.packed_offsets(lmax)
    alm[off[0]:off[1]] = alm[off[0]:off[1]].real
    import torch

    eng = sht._GpuSht(nside, lmax)
    mp = eng.alm2map(torch.as_tensor(alm, device="cuda")).cpu().numpy()
    back = sht.map2alm(mp, lmax, iter=3).cpu().numpy()
    err = np.abs(back - alm).max() / np.abs(alm).max()
    print(f"nside 256 lmax 500 round trip max rel err {err:.2e}")
    assert err < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("nside,lmax", [(4, 40), (16, 47), (64, 300)])
def test_gpu_ring_transforms_match_host_ffts(nside, lmax):
    """The device ring transforms against numpy's ring FFTs: analysis with m beyond the ring
    lengths (aliasing), and synthesis (the host folds m onto the ring's FFT bins)."""
    import torch

    from jfli_b200._lib import call, stream_ptr

    rng = np.random.default_rng(7)
    m = rng.standard_normal(12 * nside * nside)
    nr = 4 * nside - 1
    F = torch.empty(nr, lmax + 1, dtype=torch.complex128, device="cuda")
    call("jfli_sht_ring_analysis", stream_ptr(), torch.as_tensor(m, device="cuda").data_ptr(), nside, lmax,
         F.data_ptr())
    ref = osht._ring_ffts(m, nside, lmax)
    err = np.abs(F.cpu().numpy() - ref).max() / np.abs(ref).max()
    G = rng.standard_normal((nr, lmax + 1)) + 1j * rng.standard_normal((nr, lmax + 1))
    out = torch.empty(12 * nside * nside, dtype=torch.float64, device="cuda")
    call("jfli_sht_ring_synthesis", stream_ptr(), torch.as_tensor(G, device="cuda").data_ptr(), nside, lmax,
         out.data_ptr())
    back = osht._ring_synth(G, nside, lmax)
    err2 = np.abs(out.cpu().numpy() - back).max() / np.abs(back).max()
    print(f"nside {nside} lmax {lmax}: analysis {err:.2e}, synthesis {err2:.2e}")
    assert err < 1e-12 and err2 < 1e-12


@pytest.mark.gpu
def test_cross_cl_and_healpy_ordering():
    """Cross C_l: a map with itself gives its auto spectrum; two maps made from known,
    band-limited a_lm give Re(sum_m a1 a2*) / (2l + 1); the all-pairs form follows
    healpy's alm2cl order (diagonal first, then successive off-diagonals)."""
    import torch

    import jfli_b200 as jf

    nside, lmax = 32, 40
    rng = np.random.default_rng(11)
    n = (lmax + 1) * (lmax + 2) // 2
    off = sht.packed_offsets(lmax)
    alms = []
    for _ in range(3):
        a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        a[off[0]:off[1]] = a[off[0]:off[1]].real
        alms.append(a)
    eng = sht._GpuSht(nside, lmax)
    maps = [eng.alm2map(torch.as_tensor(a, device="cuda")).cpu().numpy() for a in alms]
    _, auto = jf.angular_cl_spherical(maps[0], lmax=lmax)
    _, same = jf.angular_cl_spherical(maps[0], maps[0], lmax=lmax)
    assert auto.is_cuda and same.is_cuda
    auto, same = auto.cpu().numpy(), same.cpu().numpy()
    np.testing.assert_allclose(same, auto, rtol=1e-10)
    _, c01 = jf.angular_cl_spherical(maps[0], maps[1], lmax=lmax)
    c01 = c01.cpu().numpy()
    dicts = [{mm: a[off[mm]:off[mm + 1]] for mm in range(lmax + 1)} for a in alms]
    expect = osht.alm2cl_cross(dicts[0], dicts[1], lmax)
    err = np.abs(c01 - expect).max() / np.abs(expect).max()
    print(f"cross C_l vs a_lm: {err:.2e}")
    assert err < 1e-4
    _, cls = jf.cross_angular_cl_spherical(np.stack(maps), lmax=lmax)
    assert cls.shape == (6, lmax + 1)
    cls = cls.cpu().numpy()
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]
    for row, (i, j) in zip(cls, pairs):
        ref = osht.alm2cl_cross(dicts[i], dicts[j], lmax)
        assert np.abs(row - ref).max() < 1e-4 * np.abs(ref).max()


@pytest.mark.parametrize("nside,lmax", [(8, 23), (16, 60)])
def test_oracle_c_legendre_matches_numpy(nside, lmax):
    """The oracle's C Legendre stages (oracle/sht.c) against its NumPy recursion."""
    rng = np.random.default_rng(nside)
    m = rng.standard_normal(12 * nside * nside)
    a_c = osht._map2alm_once(m, nside, lmax)
    a_np = osht._map2alm_once_np(m, nside, lmax)
    scale = max(np.abs(v).max() for v in a_np.values())
    assert max(np.abs(a_c[k] - a_np[k]).max() for k in a_np) < 1e-13 * scale
    back_c = osht.alm2map(a_np, nside, lmax)
    back_np = osht.alm2map_np(a_np, nside, lmax)
    assert np.abs(back_c - back_np).max() < 1e-12 * np.abs(back_np).max()
