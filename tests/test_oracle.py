"""Pins of the CPU oracle (CPU only): published known answers and the reference's own
portable test statements."""

from __future__ import annotations

import json
import math
import os

import numpy as np
import pytest

from oracle import cosmology as ocosmo
from oracle import healpix as oh
from oracle import pm as opm
from tests.conftest import rel_l2

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


# ------------------------------------------------------------------------ HEALPix geometry
def test_healpix_ang2pix_matches_published_examples():
    doc = json.load(open(os.path.join(GOLDEN, "healpix_docs.json")))
    for case in doc["ang2pix"]:
        assert int(oh.ang2pix(case["nside"], case["theta"], case["phi"])) == case["pix"]


def test_healpix_interp_weights_match_published_example():
    doc = json.load(open(os.path.join(GOLDEN, "healpix_docs.json")))
    for case in doc["get_interp_weights"]:
        pix, w = oh.get_interp_weights(case["nside"], case["theta"], case["phi"])
        assert list(pix[:, 0]) == case["pix"]
        np.testing.assert_allclose(w[:, 0], case["weights"], atol=1e-15)


@pytest.mark.parametrize("nside", [1, 2, 8, 32])
def test_healpix_pixel_centres_roundtrip(nside):
    pix = np.arange(oh.nside2npix(nside))
    th, ph = oh.pix2ang(nside, pix)
    np.testing.assert_array_equal(oh.ang2pix(nside, th, ph), pix)


@pytest.mark.parametrize("nside", [1, 4, 64])
def test_healpix_interp_weights_partition_unity(nside):
    rng = np.random.default_rng(nside)
    th = np.arccos(rng.uniform(-1, 1, 20000))
    ph = rng.uniform(-np.pi, 3 * np.pi, 20000)
    pix, w = oh.get_interp_weights(nside, th, ph)
    np.testing.assert_allclose(w.sum(0), 1.0, atol=1e-12)
    assert (w >= -1e-12).all()
    assert pix.min() >= 0 and pix.max() < oh.nside2npix(nside)


def test_healpix_interp_at_pixel_centre_is_that_pixel():
    nside = 16
    pix = np.arange(oh.nside2npix(nside))[::7]
    th, ph = oh.pix2ang(nside, pix)
    p, w = oh.get_interp_weights(nside, th, ph)
    away_from_poles = (th > 0.3) & (th < np.pi - 0.3)
    picked = p[np.argmax(w, axis=0), np.arange(p.shape[1])]
    np.testing.assert_array_equal(picked[away_from_poles], pix[away_from_poles])
    np.testing.assert_allclose(w.max(0)[away_from_poles], 1.0, atol=1e-9)


# ---------------------------------------------------------------------- CIC and kernels
def test_cic_conserves_mass_and_reads_back_constants():
    rng = np.random.default_rng(1)
    disp = rng.normal(0, 3.0, (16, 16, 16, 3))
    rho = opm.cic_paint(disp)
    assert abs(rho.sum() - 16**3) < 1e-9
    const = np.full((16, 16, 16), 2.5)
    np.testing.assert_allclose(opm.cic_read(const, disp), 2.5, atol=1e-12)


def test_cic_zero_displacement_is_identity():
    mesh = np.random.default_rng(2).normal(size=(8, 8, 8))
    np.testing.assert_allclose(opm.cic_read(mesh, np.zeros((8, 8, 8, 3))), mesh, atol=1e-14)
    np.testing.assert_allclose(opm.cic_paint(np.zeros((8, 8, 8, 3))), 1.0, atol=1e-14)


def test_fd_gradient_is_the_four_point_stencil():
    """i(8 sin k - sin 2k)/6 in k-space equals [8(f+1 - f-1) - (f+2 - f-2)]/12 in real space."""
    f = np.random.default_rng(3).normal(size=(16, 12, 10))
    kvec = opm.fftk(f.shape)
    for ax in range(3):
        spec = np.fft.ifftn(opm.gradient_kernel(kvec, ax) * np.fft.fftn(f)).real
        r = lambda s: np.roll(f, -s, axis=ax)
        real = (8 * (r(1) - r(-1)) - (r(2) - r(-2))) / 12
        np.testing.assert_allclose(spec, real, atol=1e-12)


def _plane_wave(n, m, A=0.01, axis=0):
    x = np.arange(n)
    wave = A * np.cos(2 * np.pi * m * x / n)
    s = [1, 1, 1]
    s[axis] = n
    return np.broadcast_to(wave.reshape(s), (n, n, n)).copy()


@pytest.mark.parametrize("m", [1, 3, 7])
def test_lpt_plane_wave_closed_form(m):
    """1LPT of delta = A cos(k x): dx_x = -D1 A a(k)/k^2 sin(k x), a(k) = (8 sin k - sin 2k)/6;
    the second-order source of a single plane wave vanishes."""
    n, A = 16, 0.01
    ic = _plane_wave(n, m, A)
    k = 2 * np.pi * m / n
    a = (8 * np.sin(k) - np.sin(2 * k)) / 6
    x = np.arange(n)
    expect = -A * a / k**2 * np.sin(k * x)
    for order in (1, 2):
        dx, p = opm.lpt(ic, 0.7, 0.3, 2.0, 5.0, order=order)
        np.testing.assert_allclose(dx[..., 0], 0.7 * expect[:, None, None] * np.ones((1, n, n)), atol=1e-14)
        np.testing.assert_allclose(dx[..., 1:], 0.0, atol=1e-14)
        np.testing.assert_allclose(p, 2.0 * dx, atol=1e-14)


def test_power_single_mode_closed_form():
    n, L, m, A = 16, 100.0, 2, 0.5
    mesh = _plane_wave(n, m, A)
    kf = 2 * np.pi / L
    kedges = np.array([0.5, 1.5, 2.5, 3.5]) * kf
    k, pk = opm.power(mesh, (L, L, L), kedges)
    # bins [1:-1] -> bins 1..3 ; the mode sits at |k| = 2 kf (bin 2 of digitize -> index 1)
    kmesh = np.sqrt(sum((2 * np.pi * n / L * np.fft.fftfreq(n).reshape(s)) ** 2
                        for s in ([n, 1, 1], [1, n, 1], [1, 1, n])))
    count = np.count_nonzero(np.digitize(kmesh.ravel(), kedges) == 2)
    expect = 2 * (A**2 * n**3 / 4) / count * (L / n) ** 3
    np.testing.assert_allclose(pk[1], expect, rtol=1e-12)
    np.testing.assert_allclose(pk[[0, 2]], 0.0, atol=1e-20)


def test_forces_of_uniform_grid_vanish():
    f = opm.pm_forces(np.zeros((16, 16, 16, 3)))
    assert np.abs(f).max() < 1e-12


# ---------------------------------------------------------------- reference test statements
def test_reversible_roundtrip_fp64(cosmo):
    """reverse(step(y)) == y at 1e-10 (reference tests/test_against_fpm.py:177-216)."""
    from jfli_b200.pm.solvers import ReversibleDoubleKickDrift

    rng = np.random.default_rng(4)
    ic = rng.normal(size=(16, 16, 16))
    dx, p = opm.lpt(ic, 0.1, 0.0, 0.5, 0.0)
    c = ReversibleDoubleKickDrift.step_coefficients(cosmo, 0.1, 0.11, 0.01, 0.1)
    x1, v1 = opm.kkd_step(dx, p, c.kick, c.drift)
    x0, v0 = opm.kkd_reverse(x1, v1, c.kick, c.drift)
    np.testing.assert_allclose(x0, dx, rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(v0, p, rtol=1e-10, atol=1e-10)


# ---------------------------------------------------------------------- cosmology tables
def test_growth_tables_match_closed_form(cosmo):
    from jfli_b200 import cosmology as cj

    om = cosmo.Omega_m
    tab = cj.growth_table(cosmo)
    for i in (10, 60, 100, 120, 127):  # at the table nodes the ODE solution is exact
        a = float(tab.a[i])
        assert abs(tab.g[i] / ocosmo.growth(om, a) - 1) < 1e-9
        assert abs(tab.f[i] / ocosmo.growth_rate(om, a) - 1) < 1e-7
    # between nodes the 128-point table is read by linear interpolation (as in the reference)
    for a in (0.05, 0.1, 0.3, 0.7, 1.0):
        assert abs(float(cj.growth_factor(cosmo, a)) / ocosmo.growth(om, a) - 1) < 5e-4
        assert abs(float(cj.growth_rate(cosmo, a)) / ocosmo.growth_rate(om, a) - 1) < 5e-4
        assert abs(float(cj.dGfa(cosmo, a)) / ocosmo.dGfa(om, a) - 1) < 1e-3
    dtab = cj.distance_table(cosmo)
    for i in (50, 200, 250):
        assert abs(dtab.chi[i] / ocosmo.chi(om, float(dtab.a[i])) - 1) < 1e-9
    for a in (0.3, 0.6, 0.9):
        assert abs(float(cj.radial_comoving_distance(cosmo, a)) / ocosmo.chi(om, a) - 1) < 1e-3


def test_sigma8_normalisation(cosmo):
    from jfli_b200 import cosmology as cj

    k = np.logspace(-5, 3, 20000)
    pk = cj.linear_matter_power(cosmo, k)
    x = k * 8.0
    w = 3 * (np.sin(x) - x * np.cos(x)) / x**3
    s2 = np.trapezoid(k**3 * pk * w**2 / (2 * np.pi**2), np.log(k))
    assert abs(math.sqrt(s2) / cosmo.sigma8 - 1) < 1e-3


def test_oracle_fp32_matches_fp64_forces():
    rng = np.random.default_rng(5)
    dx, _ = opm.lpt(rng.normal(size=(32, 32, 32)), 1.0, 0.0, 1.0, 0.0)
    f64 = opm.pm_forces(dx, np.float64)
    f32 = opm.pm_forces(dx.astype(np.float32), np.float32)
    assert rel_l2(f32, f64) < 1e-5


def test_flat_oracle_self_consistency():
    """The flat-sky oracle: 2D CIC conserves weight inside the slab, and the flat C_ell of a
    single cosine puts its power in the bin of its |ell| (Parseval with the (px py)/(nx ny)
    normalisation)."""
    from oracle import flat as of

    rng = np.random.default_rng(0)
    pos = rng.uniform(-5, 40, (2000, 3))
    m = of.paint_2d(pos, (16, 24), 5.0, 20.0, (32, 32, 32))
    inside = ((pos[:, 2] > 5.0) & (pos[:, 2] <= 20.0)).sum()
    assert abs(m.sum() - inside) < 1e-9 * inside
    nx, ny, px = 64, 64, 1e-3
    x = np.arange(nx)[:, None] * np.ones((1, ny))
    cosmap = np.cos(2 * np.pi * 5 * x / nx)
    ell, cl = of.flat_cl(cosmap, px=px, py=px)
    target = 2 * np.pi * 5 / (nx * px)
    b = np.argmax(cl)
    assert abs(ell[b] - target) < 0.6 * (ell[1] - ell[0])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_c_cic_matches_numpy_form(dtype):
    """The OpenMP restatement (oracle/cic.c) does the NumPy form's arithmetic: FP32 paint
    and readout bit for bit, FP64 to summation order."""
    n = 20
    rng = np.random.default_rng(1)
    x = (3 * rng.standard_normal((n, n, n, 3))).astype(dtype)
    np.testing.assert_allclose(opm.cic_paint(x), opm.cic_paint_np(x), rtol=0, atol=1e-13)
    m = rng.standard_normal((n, n, n)).astype(dtype)
    assert np.array_equal(opm.cic_read(m, x), opm.cic_read_np(m, x))
    stack = rng.standard_normal((3, n, n, n)).astype(dtype)
    both = opm.cic_read(stack, x)
    for q in range(3):
        assert np.array_equal(both[..., q], opm.cic_read_np(stack[q], x))
    w = rng.uniform(0, 1, (n, n, n)).astype(dtype)
    xa = rng.uniform(-3, n + 3, (n, n, n, 3)).astype(dtype)
    np.testing.assert_allclose(opm.cic_paint(xa, absolute=True, weight=w),
                               opm.cic_paint_np(xa, absolute=True, weight=w), rtol=0, atol=1e-12)
    if dtype == np.float32:
        assert np.array_equal(opm.cic_paint(x), opm.cic_paint_np(x))
