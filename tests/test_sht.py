"""Host spherical harmonic transform behind SphericalDensity.angular_cl (healpy.anafast
restated): Legendre functions against scipy, analysis/synthesis round trips, known maps."""

import math

import numpy as np
import pytest
from scipy.special import sph_harm_y

from jfli_b200 import sht


@pytest.mark.parametrize("m", [0, 1, 7, 30])
def test_legendre_matches_scipy(m):
    z, _, _, _ = sht.ring_geometry(32)
    lam = sht._lambda_m(m, 80, z, np.sqrt(1 - z * z))
    ref = np.array([sph_harm_y(l, m, np.arccos(z), 0.0).real for l in range(m, 81)])
    assert np.abs(lam - ref).max() < 1e-12


def test_ring_geometry_covers_the_sphere():
    for nside in (1, 2, 8, 32):
        z, npr, phi0, start = sht.ring_geometry(nside)
        assert npr.sum() == 12 * nside * nside
        assert np.all(np.diff(z) < 0)
        assert start[-1] + npr[-1] == 12 * nside * nside


def test_band_limited_round_trip():
    nside, lmax = 16, 32
    rng = np.random.default_rng(0)
    alm = {m: rng.standard_normal(lmax - m + 1) + 1j * rng.standard_normal(lmax - m + 1) for m in range(lmax + 1)}
    alm[0] = alm[0].real.astype(complex)
    mp = sht.alm2map(alm, nside, lmax)
    back = sht.map2alm(mp, lmax, iter=10)
    assert max(np.abs(back[m] - alm[m]).max() for m in alm) < 1e-8
    cl = sht.alm2cl(alm, lmax)
    assert np.allclose(sht.anafast(mp, lmax, iter=10), cl, rtol=1e-8)


def test_known_maps():
    nside = 16
    npix = 12 * nside * nside
    c = sht.anafast(np.full(npix, 2.0), iter=0)
    # HEALPix quadrature aliases ~1e-7 of C_0 into multipoles near 3 nside
    assert abs(c[0] / (4 * math.pi * 4.0) - 1) < 1e-12 and np.abs(c[1:]).max() < 1e-6 * c[0]
    z, npr, _, start = sht.ring_geometry(nside)
    zz = np.repeat(z, npr)
    y10 = math.sqrt(3 / (4 * math.pi)) * zz  # Y_10: C_1 = 1 for a_10 = 1
    cl = sht.anafast(y10, lmax=8, iter=3)
    assert abs(cl[1] / (1.0 / 3.0) - 1) < 1e-3 and cl[[0, 2, 3, 4]].max() < 1e-6
