"""Parity of the CUDA path (through the C-ABI) against the CPU oracle on seeded inputs.

Tolerances: FP32 kernels against the FP64 oracle, relative L2 over the field
(np.linalg.norm(gpu - ref) / np.linalg.norm(ref)):
  FFT 2e-6; CIC paint/readout 1e-6; potential, forces, LPT, ICs 1e-5;
  P(k) 1e-4 per bin; N-body density after 10 KDK steps 1e-4 (chaotic growth of FP32
  rounding, measured against the oracle's own FP32-vs-FP64 gap in the same test).
"""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest
import torch

import jfli_b200 as jf
from jfli_b200 import ops
from oracle import healpix as oh
from oracle import pm as opm
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def lpt_disp(n, scale, seed=0):
    rng = np.random.default_rng(seed)
    dx, _ = opm.lpt(rng.normal(size=(n, n, n)), scale, 0.0, 1.0, 0.0)
    return dx


# ----------------------------------------------------------------------------------- FFT
@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 32, 64), (64, 64, 64), (48, 96, 24), (128, 128, 128),
                                   (8, 6, 4)])
def test_rfft3d_matches_numpy(shape):
    x = np.random.default_rng(1).normal(size=shape)
    spec = host(ops.rfft3d(dev(x)))
    ref = np.fft.rfftn(x)
    assert rel_l2(spec, ref) < 2e-6
    back = host(ops.irfft3d(torch.as_tensor(ref.astype(np.complex64), device="cuda"), shape[2]))
    assert rel_l2(back, x) < 2e-6


def test_rfft3d_batched_matches_single():
    x = np.random.default_rng(2).normal(size=(3, 32, 32, 32))
    both = host(ops.rfft3d(dev(x)))
    for b in range(3):
        np.testing.assert_array_equal(both[b], host(ops.rfft3d(dev(x[b]))))


# ----------------------------------------------------------------------------------- CIC
@pytest.mark.parametrize("n,sigma", [(16, 0.5), (32, 3.0), (64, 8.0)])
def test_paint_matches_oracle(n, sigma):
    disp = np.random.default_rng(n).normal(0, sigma, (n, n, n, 3)).astype(np.float32)
    rho = host(ops.paint_cic(dev(disp)))
    ref = opm.cic_paint(disp.astype(np.float64))
    assert rel_l2(rho, ref) < 1e-6
    assert abs(rho.sum(dtype=np.float64) - n**3) < 1e-3 * n**3 * 1e-3


def test_paint_absolute_and_weights():
    n = 32
    rng = np.random.default_rng(7)
    pos = rng.uniform(-40, 80, (n, n, n, 3)).astype(np.float32)
    w = rng.uniform(0.5, 2.0, (n, n, n)).astype(np.float32)
    rho = host(ops.paint_cic(dev(pos), absolute=True, weights=dev(w), weight=0.5))
    ref = opm.cic_paint(pos.astype(np.float64), absolute=True, weight=0.5 * w.astype(np.float64))
    assert rel_l2(rho, ref) < 1e-6


@pytest.mark.parametrize("n", [16, 64])
def test_readout_matches_oracle(n):
    rng = np.random.default_rng(n + 1)
    disp = rng.normal(0, 4, (n, n, n, 3)).astype(np.float32)
    mesh = rng.normal(size=(n, n, n)).astype(np.float32)
    out = host(ops.readout_cic(dev(disp), dev(mesh)))
    ref = opm.cic_read(mesh.astype(np.float64), disp.astype(np.float64))
    assert rel_l2(out, ref) < 1e-6


# ------------------------------------------------------------------------ Poisson / forces
def test_poisson_potential_matches_oracle():
    rho = 1.0 + 0.3 * np.random.default_rng(3).normal(size=(32, 32, 32))
    pot = host(ops.poisson_potential(dev(rho), rho_mean=1.0))
    ref = opm.potential_real(rho)
    assert rel_l2(pot, ref) < 1e-5


@pytest.mark.parametrize("n,scale", [(32, 2.0), (64, 5.0)])
def test_pm_forces_matches_oracle(n, scale):
    disp = lpt_disp(n, scale, seed=n).astype(np.float32)
    f = host(ops.pm_forces(dev(disp), scale=1.5))
    ref = 1.5 * opm.pm_forces(disp.astype(np.float64))
    assert rel_l2(f, ref) < 1e-5


# (12, 12, 12) and (6, 18, 20): 432 and 540 groups of 4 cells, so the last warp is partial
@pytest.mark.parametrize("shape", [(32, 32, 32), (16, 24, 36), (12, 20, 42), (8, 8, 4), (16, 16, 64),
                                   (48, 32, 128), (64, 64, 64), (12, 12, 12), (6, 18, 20)])
def test_force_mesh_matches_stencil(shape):
    """Force mesh -D pot: the four-cell vectorised path (nz % 4 == 0, nz >= 8, 16-byte
    aligned buffers) and the scalar path otherwise."""
    pot = np.random.default_rng(sum(shape)).normal(size=shape)
    F = host(ops.force_mesh(dev(pot), scale=2.0))
    for ax in range(3):
        r = lambda s: np.roll(pot, -s, axis=ax)
        ref = -2.0 * (8 * (r(1) - r(-1)) - (r(2) - r(-2))) / 12
        np.testing.assert_allclose(F[..., ax], ref, rtol=1e-5, atol=1e-5)
    assert np.all(F[..., 3] == 0)


def test_readout_gradient_absolute_equals_relative():
    n = 32
    disp = lpt_disp(n, 3.0, seed=11).astype(np.float32)
    absol = (disp + opm.grid((n, n, n), np.float32)).astype(np.float32)
    rho = ops.paint_cic(dev(disp))
    pot = ops.poisson_potential(rho, 1.0)
    a = host(ops.readout_gradient(dev(disp), pot))
    b = host(ops.readout_gradient(dev(absol), pot, absolute=True))
    assert rel_l2(a, b) < 1e-5


# ------------------------------------------------------------------------------- ICs / LPT
def test_ic_filter_matches_oracle(cosmo):
    from jfli_b200 import cosmology as cj

    n, L = 32, 128.0
    noise = np.random.default_rng(0).standard_normal((n, n, n)).astype(np.float32)
    k, pk = cj.pk_table(cosmo, 128)
    for zmo in (False, True):
        out = host(ops.ic_filter(dev(noise), dev(k), dev(pk), (L, L, L), zero_mode_one=zmo))
        ref = opm.ic_filter(noise.astype(np.float64), (L, L, L), k, pk, zero_mode_one=zmo)
        assert rel_l2(out, ref) < 1e-5


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("n", [32, 64])
def test_lpt_matches_oracle(order, n, cosmo):
    from jfli_b200.pm.lpt import lpt_coefficients

    ic = (0.8 * np.random.default_rng(n).standard_normal((n, n, n))).astype(np.float32)
    c = lpt_coefficients(cosmo, 0.1)
    dx, p = ops.lpt(dev(ic), order, *c)
    rdx, rp = opm.lpt(ic.astype(np.float64), *c, order=order)
    assert rel_l2(host(dx), rdx) < 1e-5
    assert rel_l2(host(p), rp) < 1e-5


def test_lpt_api_matches_oracle(cosmo):
    n, L = 32, 256.0
    noise = jf.white_noise(0, (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo)
    dx, p = jf.lpt(cosmo, ic, ts=0.1, order=2)
    from jfli_b200 import cosmology as cj
    from jfli_b200.pm.lpt import lpt_coefficients

    k, pk = cj.pk_table(cosmo, 128)
    ric = opm.ic_filter(noise.astype(np.float64), (L, L, L), k, pk)
    rdx, rp = opm.lpt(ric, *lpt_coefficients(cosmo, 0.1), order=2)
    assert rel_l2(host(dx.array), rdx) < 1e-5
    assert rel_l2(host(p.array), rp) < 1e-5
    assert dx.status == jf.FieldStatus.LPT2 and dx.unit == jf.PositionUnit.GRID_RELATIVE


# ------------------------------------------------------------------------------------ P(k)
@pytest.mark.parametrize("n", [32, 64])
def test_power_matches_oracle(n):
    L = 4.0 * n
    disp = lpt_disp(n, 3.0, seed=5).astype(np.float32)
    rho = ops.paint_cic(dev(disp))
    mesh = host(rho).astype(np.float64)
    kedges = np.geomspace(2 * np.pi / L * (1 - 1e-6), np.pi * n / L, 33)
    k, pk = jf.power(rho, box_shape=(L, L, L), kedges=kedges)
    rk, rpk = opm.power(mesh, (L, L, L), kedges)
    k, pk = host(k), host(pk)
    ok = rpk > 0
    assert np.abs(pk[ok] / rpk[ok] - 1).max() < 1e-4
    np.testing.assert_allclose(k, rk, rtol=1e-6)


def test_power_default_bins_and_batch():
    n, L = 32, 100.0
    x = 1 + 0.2 * np.random.default_rng(9).normal(size=(2, n, n, n))
    k, pk = jf.power(dev(x), box_shape=(L, L, L))
    from jfli_b200.power import default_kedges

    ke = default_kedges((n, n, n), (L, L, L))
    for b in range(2):
        # default bins put many modes exactly on an edge: bin them with the reference's
        # float32 |k| grid, as the kernel does
        _, rpk = opm.power(x[b], (L, L, L), ke, kdtype=np.float32)
        assert np.abs(host(pk[b]) / rpk - 1).max() < 1e-4


# --------------------------------------------------------------------------------- HEALPix
@pytest.mark.parametrize("scheme", ["ngp", "bilinear"])
@pytest.mark.parametrize("nside", [8, 64])
def test_healpix_paint_matches_oracle(scheme, nside):
    n, L = 32, 200.0
    disp = lpt_disp(n, 2.0, seed=3).astype(np.float32)
    obs = (100.0, 100.0, 100.0)
    # positions as the kernel forms them: FP64 from the FP32 displacements
    g = opm.grid((n, n, n), np.float64)
    pos = (g + disp.astype(np.float64)) * (L / n) - np.asarray(obs, np.float64)
    r64 = np.sqrt((pos * pos).sum(-1))
    rmin, rmax = 40.0, 90.0
    out = host(ops.healpix_paint(dev(disp), nside, (L, L, L), obs, rmin, rmax, scheme=scheme))
    sel = (r64 > rmin) & (r64 <= rmax)
    v = pos[sel]
    r = r64[sel]
    th = np.arccos(np.clip(v[:, 2] / r, -1, 1))
    ph = np.arctan2(v[:, 1], v[:, 0])
    npix = 12 * nside * nside
    if scheme == "ngp":
        ref = np.bincount(oh.ang2pix(nside, th, ph), minlength=npix).astype(np.float64)
        np.testing.assert_array_equal(out, ref)
    else:
        p, w = oh.get_interp_weights(nside, th, ph)
        ref = np.bincount(p.ravel(), weights=w.ravel(), minlength=npix)
        # the kernel may contract the FP64 arithmetic into fused multiply-adds; the weights
        # move continuously with it
        assert rel_l2(out, ref) < 2e-5
    assert abs(out.sum() - sel.sum()) < 1e-3 * max(sel.sum(), 1)


@pytest.mark.parametrize("scheme", ["ngp", "bilinear", "rbf_neighbor"])
def test_healpix_paint_shells_one_pass(scheme):
    """jfli_healpix_paint_shells (S shells of one particle set in one pass) against one
    jfli_healpix_paint per shell: per-particle weights, overlapping shells, and 70 shells
    (more than one launch's 64)."""
    n, L, nside = 32, 200.0, 16
    disp = dev(lpt_disp(n, 2.0, seed=5).astype(np.float32))
    w = dev(np.random.default_rng(6).uniform(0.5, 1.5, (n, n, n)).astype(np.float32))
    obs = (100.0, 100.0, 100.0)
    edges = np.linspace(5.0, 100.0, 71)
    rmin = np.concatenate([edges[:-1], [30.0]])  # the last shell overlaps several others
    rmax = np.concatenate([edges[1:], [60.0]])
    scale = np.linspace(0.5, 2.0, rmin.size)
    maps = host(ops.healpix_paint_shells(disp, nside, (L, L, L), obs, rmin, rmax, scale, scheme=scheme, weights=w,
                                         weight=0.75))
    worst = 0.0
    for s in range(rmin.size):
        ref = host(ops.healpix_paint(disp, nside, (L, L, L), obs, rmin[s], rmax[s], scheme=scheme, weights=w,
                                     weight=0.75 * float(np.float32(scale[s]))))
        if ref.sum() == 0:
            assert maps[s].sum() == 0
            continue
        worst = max(worst, rel_l2(maps[s], ref))
    print(f"{scheme}: {rmin.size} shells in one pass vs one pass per shell: worst {worst:.2e}")
    assert worst < 1e-6


def test_healpix_paint_at_paint_nside():
    """paint_nside: ngp counts painted at nside 32 and graded to 8 on the GPU (power -2 keeps
    the counts, so the result is exact) equal the oracle's counts graded by the ring geometry;
    the field method equals grading the map it paints at nside 32."""
    from jfli_b200 import healpix_order as ho

    n, L = 32, 200.0
    disp = lpt_disp(n, 2.0, seed=3).astype(np.float32)
    obs = (100.0, 100.0, 100.0)
    cell = np.float32(L / n)
    g = opm.grid((n, n, n), np.float32)
    pos = ((g + disp) * cell - np.asarray(obs, np.float32)).astype(np.float32)
    r32 = np.sqrt((pos * pos).sum(-1, dtype=np.float32), dtype=np.float32)
    rmin, rmax = 40.0, 90.0
    sel = (r32 > np.float32(rmin)) & (r32 <= np.float32(rmax))
    v = pos[sel].astype(np.float64)
    r = r32[sel].astype(np.float64)
    th = np.arccos(np.clip(v[:, 2] / r, -1, 1))
    ph = np.arctan2(v[:, 1], v[:, 0])
    fine = ops.healpix_paint(dev(disp), 32, (L, L, L), obs, rmin, rmax, scheme="ngp")
    coarse = host(ho.ud_grade(fine, 8, power=-2.0))
    counts = np.bincount(oh.ang2pix(32, th, ph), minlength=12 * 32 * 32).astype(np.float64)
    np.testing.assert_array_equal(coarse, oh.ud_grade_ring(counts, 8, power=-2.0))

    field = jf.ParticleField(array=dev(disp), mesh_size=(n, n, n), box_size=(L, L, L),
                             observer_position=(0.5, 0.5, 0.5), nside=8, unit=jf.PositionUnit.GRID_RELATIVE,
                             status=jf.FieldStatus.PARTICLES)
    a = field.paint_spherical(65.0, 50.0, scheme="ngp", paint_nside=32)
    b = field.replace(nside=32).paint_spherical(65.0, 50.0, scheme="ngp")
    assert a.nside == 8 and tuple(a.array.shape) == (12 * 64,)
    np.testing.assert_allclose(host(a.array), host(ho.ud_grade(b.array, 8)), rtol=1e-5)


# -------------------------------------------------------------------------------- stepping
def test_kick_drift_paint_matches_unfused(cosmo):
    from jfli_b200._lib import JFLI_STEP_DRIFT, JFLI_STEP_KICK, JFLI_STEP_PAINT

    n = 32
    x0 = lpt_disp(n, 3.0, seed=2).astype(np.float32)
    v0 = (0.5 * x0).astype(np.float32)
    kick, drift = 0.37, 0.81
    # fused on the GPU
    x, v = dev(x0), dev(v0)
    force = ops.poisson_force(ops.paint_cic(x), 1.0)
    rho = torch.zeros(n, n, n, device="cuda")
    ops.kick_drift_paint(x, v, force, kick, drift, JFLI_STEP_KICK | JFLI_STEP_DRIFT | JFLI_STEP_PAINT, rho)
    # oracle
    rv = v0.astype(np.float64) + kick * opm.pm_forces(x0.astype(np.float64))
    rx = x0.astype(np.float64) + drift * rv
    assert rel_l2(host(v) - v0, rv - v0) < 1e-5
    assert rel_l2(host(x) - x0, rx - x0) < 1e-5
    assert rel_l2(host(rho), opm.cic_paint(rx)) < 1e-5


@pytest.mark.parametrize("spread", [0.3, 6.0, 14.0])
def test_kick_drift_paint_small_and_large_displacements(spread):
    """Displacements from a fraction of a cell to many cells (periodic wrap of the CIC
    corners and of the force meshes). Meshes: 32^3 and 12 x 16 x 64 walk 8 x 32 bricks along
    x (the latter with a short last chunk of planes), 40^3 takes the grid-stride walk."""
    from jfli_b200._lib import JFLI_STEP_DRIFT, JFLI_STEP_KICK, JFLI_STEP_PAINT

    for shape in ((32, 32, 32), (40, 40, 40), (12, 16, 64)):
        rng = np.random.default_rng(int(spread * 10) + shape[0])
        x0 = rng.uniform(-spread, spread, (*shape, 3)).astype(np.float32)
        v0 = rng.normal(0, 1.0, (*shape, 3)).astype(np.float32)
        kick, drift = 0.25, 0.5
        pot64 = opm.potential_real(1.0 + 0.3 * rng.normal(size=shape))
        x, v = dev(x0), dev(v0)
        rho = torch.zeros(shape, device="cuda")
        force = ops.force_mesh(dev(pot64))
        ops.kick_drift_paint(x, v, force, kick, drift, JFLI_STEP_KICK | JFLI_STEP_DRIFT | JFLI_STEP_PAINT, rho)
        kvec = opm.fftk(shape)
        pk = np.fft.fftn(pot64)
        F = np.stack([opm.cic_read(-np.fft.ifftn(opm.gradient_kernel(kvec, i) * pk).real, x0.astype(np.float64))
                      for i in range(3)], -1)
        rv = v0 + kick * F
        rx = x0 + drift * rv
        assert rel_l2(host(v) - v0, rv - v0) < 1e-5
        assert rel_l2(host(x), rx) < 1e-6
        assert rel_l2(host(rho), opm.cic_paint(rx)) < 1e-5


def _config1(cosmo, n=64, L=256.0, steps=10):
    noise = jf.white_noise(0, (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo)
    dx, p = jf.lpt(cosmo, ic, ts=0.1, order=1)
    dt0 = 0.9 / steps
    return noise, dx, p, dt0


def test_nbody_config1_matches_oracle(cosmo):
    """64^3, L=256, 1LPT to a=0.1, EfficientDriftDoubleKick dt0=0.09 to a=1 (10 steps)."""
    from jfli_b200 import cosmology as cj
    from jfli_b200.pm.integrate import time_events
    from jfli_b200.pm.lpt import lpt_coefficients
    from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK

    n, L = 64, 256.0
    noise, dx, p, dt0 = _config1(cosmo, n, L)
    solver = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="density")))
    res, run = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=dt0, solver=solver, return_state=True)
    assert run.steps == 10
    gpu = host(res.array)
    # oracle with identical inputs and coefficients
    k, pk = cj.pk_table(cosmo, 128)
    ric = opm.ic_filter(noise.astype(np.float64), (L, L, L), k, pk)
    c = lpt_coefficients(cosmo, 0.1)
    steps = [(e[1], e[2]) for e in time_events(0.1, [1.0], dt0) if e[0] == "step"]
    coeffs = dict(init_kick=EDK.init_kick(cosmo, 0.1, 0.1 + dt0),
                  steps=[(EDK.step_coefficients(cosmo, a, b, dt0).kick, EDK.step_coefficients(cosmo, a, b, dt0).drift)
                         for a, b in steps])
    results = {}
    for dt in (np.float64, np.float32):
        rdx, rp = opm.lpt(ric.astype(dt), *c, order=1, dtype=dt)
        _, _, snaps = opm.kdk_run(rdx, rp, coeffs, dtype=dt, snapshot_after={len(steps) - 1})
        results[dt] = snaps[0].astype(np.float64)
    err64 = rel_l2(gpu, results[np.float64])
    err32 = rel_l2(gpu, results[np.float32])
    gap = rel_l2(results[np.float32], results[np.float64])
    print(f"64^3, 10 steps: density vs FP64 oracle {err64:.2e}, vs FP32 oracle {err32:.2e} "
          f"(FP32-vs-FP64 oracle gap {gap:.2e})")
    # the field tolerance, 1e-5 relative L2, against both oracle precisions
    assert err64 < 1e-5 and err32 < 1e-5, (err64, err32, gap)
    kedges = np.geomspace(2 * np.pi / L * (1 - 1e-6), np.pi * n / L, 33)
    _, pk_gpu = res.power(kedges=kedges).wavenumber, res.power(kedges=kedges).array
    _, pk_ref = opm.power(results[np.float64], (L, L, L), kedges)
    ok = pk_ref > 0
    assert np.abs(host(pk_gpu)[ok] / pk_ref[ok] - 1).max() < 1e-4


def test_fused_loop_equals_stepwise_loop(cosmo):
    from jfli_b200.pm.integrate import run_fused, run_stepwise

    n, L = 32, 128.0
    noise, dx, p, dt0 = _config1(cosmo, n, L, steps=5)
    for solver_cls in (jf.EfficientDriftDoubleKick, jf.ReversibleDoubleKickDrift):
        solver = solver_cls(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="density")))
        ts = np.array([0.4, 1.0])
        solver = dataclasses.replace(
            solver, interp_kernel=solver.interp_kernel.update_geometry(ts, np.zeros(2), np.zeros(2), 1e9))
        a = run_fused(solver, dx, p, cosmo, ts, 0.1, dt0)
        b = run_stepwise(solver, dx, p, cosmo, ts, 0.1, dt0)
        assert a.steps == b.steps
        for sa, sb in zip(a.snapshots, b.snapshots):
            assert rel_l2(host(sa.array), host(sb.array)) < 1e-5
        assert rel_l2(host(a.vel), host(b.vel)) < 1e-5


def test_reversible_roundtrip_gpu(cosmo):
    """reverse(step(y)) ~= y (reference tests/test_against_fpm.py:177-216) in FP32."""
    n, L = 32, 256.0
    _, dx, p, _ = _config1(cosmo, n, L)
    interp = jf.NoInterp(painting=jf.PaintingOptions(target="density")).update_geometry(
        np.array([1.0]), np.zeros(1), np.ones(1), 1.0)
    solver = jf.ReversibleDoubleKickDrift(interp_kernel=interp)
    t0, dt = 0.1, 0.01
    d0, p0, st = solver.init(dx, p, t0, t0 + dt, dt, cosmo)
    d1, p1, st1 = solver.step(d0, p0, t0, t0 + dt, dt, st, cosmo)
    d2, p2, _ = solver.reverse(d1, p1, t0, t0 + dt, dt, st1, cosmo)
    x0, v0 = host(d0.array), host(p0.array)
    assert np.abs(host(d2.array) - x0).max() < 2e-6 * max(1.0, np.abs(x0).max())
    assert rel_l2(host(p2.array), v0) < 1e-6


def test_spherical_shells_nbody(cosmo):
    """nb_shells lightcone: 4 equal-width shells, bilinear; each map against the oracle
    painter on the GPU's own particle positions at the shell time (the particle snapshots
    of the same run, read back), divided by the pixel volume."""
    from oracle import healpix as oh

    n, L, nside = 32, 200.0, 16
    noise = jf.white_noise(1, (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo, nside=nside)
    dx, p = jf.lpt(cosmo, ic, ts=0.1, order=2)
    solver = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="spherical")))
    lc = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=0.1, nb_shells=4, solver=solver)
    maps = host(lc.array)
    assert maps.shape == (4, 12 * nside * nside)
    assert np.all(np.diff(lc.comoving_centers) > 0)  # near -> far
    assert np.isfinite(maps).all() and (maps >= 0).all() and maps.sum() > 0
    # the same schedule with particle snapshots at the shell times
    psolver = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="particles")))
    snaps = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=0.1, ts=np.sort(np.asarray(lc.scale_factors, np.float64)), solver=psolver)
    pos_all = host(snaps.array).astype(np.float64)
    obs = dx.observer_position_mpc
    g = opm.grid((n, n, n))
    for s in range(4):
        rc, wd = float(lc.comoving_centers[s]), float(lc.density_width[s])
        rmin, rmax = rc - wd / 2, rc + wd / 2
        vol = (4 * np.pi / (12 * nside * nside)) * (rmax**3 - rmin**3) / 3
        pos = (g + pos_all[s]) * (L / n)
        ref = oh.paint_shell(pos.reshape(-1, 3), obs, rmin, rmax, nside, "bilinear") / vol
        err = rel_l2(maps[s], ref)
        print(f"shell {s} ({rmin:.0f}-{rmax:.0f} Mpc/h): rel L2 vs oracle painter {err:.2e}")
        assert ref.sum() > 0 and err < 2e-5


def test_errors_surface_as_exceptions():
    from jfli_b200._lib import JfliError

    with pytest.raises(JfliError):
        ops.rfft3d(torch.zeros(10, 10, 10, device="cuda"))  # 5 is not a supported radix


# ------------------------------------------------------------------------------------ PGD
def test_pgd_correction_matches_oracle():
    """PGDKernel.apply (reference pm/correction.py:157-202) on one particle state."""
    from jfli_b200.fields import ParticleField, PositionUnit

    n = 32
    disp = lpt_disp(n, 2.0, seed=11).astype(np.float32)
    pos = ParticleField(array=dev(disp), mesh_size=(n, n, n), box_size=(128.0,) * 3, unit=PositionUnit.GRID_RELATIVE)
    for alpha, kl, ks in ((0.3, 0.3, 1.0), (0.3, 1.5 * 128.0 / n / 100.0, 8.0 * 128.0 / n)):
        out, _ = jf.PGDKernel(alpha=alpha, kl=kl, ks=ks).apply(0.5, pos, pos, 0.0)
        ref = opm.pgd_correction(disp, alpha, kl, ks)
        moved = rel_l2(ref, disp.astype(np.float64))
        err = rel_l2(host(out.array) - disp, ref - disp)
        print(f"alpha={alpha} kl={kl:.3g} ks={ks:.3g}: correction rel L2 {err:.2e} (|dx|/|x| = {moved:.2e})")
        assert moved > 1e-6
        assert err < 1e-5


def test_nbody_pgd_matches_oracle(cosmo):
    """64^3, L=256, 1LPT, EfficientDriftDoubleKick 10 steps with the PGD correction after
    every drift (reference pm/solvers.py:165-178)."""
    from jfli_b200 import cosmology as cj
    from jfli_b200.pm.integrate import time_events
    from jfli_b200.pm.lpt import lpt_coefficients
    from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK

    n, L = 64, 256.0
    alpha, kl, ks = 0.3, 0.3, 1.0
    noise, dx, p, dt0 = _config1(cosmo, n, L)
    solver = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="density")),
                                         pgd_kernel=jf.PGDKernel(alpha=alpha, kl=kl, ks=ks))
    res = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=dt0, solver=solver)
    gpu = host(res.array)
    k, pk = cj.pk_table(cosmo, 128)
    ric = opm.ic_filter(noise.astype(np.float64), (L, L, L), k, pk)
    c = lpt_coefficients(cosmo, 0.1)
    steps = [(e[1], e[2]) for e in time_events(0.1, [1.0], dt0) if e[0] == "step"]
    coeffs = dict(init_kick=EDK.init_kick(cosmo, 0.1, 0.1 + dt0),
                  steps=[(EDK.step_coefficients(cosmo, a, b, dt0).kick, EDK.step_coefficients(cosmo, a, b, dt0).drift)
                         for a, b in steps])
    rdx, rp = opm.lpt(ric, *c, order=1)
    _, _, snaps = opm.kdk_run(rdx, rp, coeffs, snapshot_after={len(steps) - 1}, pgd=(alpha, kl, ks))
    _, _, plain = opm.kdk_run(rdx, rp, coeffs, snapshot_after={len(steps) - 1})
    err = rel_l2(gpu, snaps[0])
    effect = rel_l2(plain[0], snaps[0])
    print(f"PGD run: density rel L2 vs oracle {err:.2e}; PGD changes the density by {effect:.2e}")
    assert effect > 1e-3
    assert err < 1e-4
    kedges = np.geomspace(2 * np.pi / L * (1 - 1e-6), np.pi * n / L, 33)
    pk_gpu = host(res.power(kedges=kedges).array)
    _, pk_ref = opm.power(snaps[0], (L, L, L), kedges)
    ok = pk_ref > 0
    assert np.abs(pk_gpu[ok] / pk_ref[ok] - 1).max() < 1e-4


@pytest.mark.parametrize("cross,poles,los", [(False, (0, 2, 4), (0.0, 0.0, 1.0)), (True, 0, (0.0, 0.0, 1.0)),
                                             (True, (0, 1, 2), (1.0, 1.0, 0.0)), (False, (1, 3), (0.0, 1.0, 1.0))])
def test_power_cross_and_multipoles_match_oracle(cross, poles, los):
    """Cross spectra and Legendre multipoles against the full-grid FP64 restatement of the
    reference's _power: every bin within 1e-4 of the monopole's scale (multipoles of a
    nearly isotropic field are close to zero, so their own relative error is meaningless)."""
    from oracle import pm as opm

    rng = np.random.default_rng(9)
    n, L = 32, 200.0
    a = rng.standard_normal((n, n, n)).astype(np.float32)
    a = np.cumsum(a, axis=2).astype(np.float32)  # anisotropic along z: nonzero even multipoles
    b = (0.6 * a + rng.standard_normal((n, n, n))).astype(np.float32)
    edges = np.geomspace(2 * np.pi / L * 1.5, np.pi * n / L, 12)
    k, pk = jf.power(torch.as_tensor(a, device="cuda"), torch.as_tensor(b, device="cuda") if cross else None,
                     box_shape=(L, L, L), kedges=edges, multipoles=poles, los=los)
    kr, pr = opm.power_poles(a, b if cross else None, (L, L, L), edges, poles, los)
    pk = np.atleast_2d(pk.cpu().numpy())
    pr = np.atleast_2d(pr)
    scale = np.abs(opm.power_poles(a, None, (L, L, L), edges, 0)[1])[None, :]  # the auto monopole
    err = np.max(np.abs(pk - pr) / scale)
    print(f"cross {cross} poles {poles} los {los}: max |GPU - oracle| / scale {err:.2e}")
    np.testing.assert_allclose(k.cpu().numpy(), kr, rtol=1e-6)
    assert err < 1e-4


def test_transfer_and_coherence():
    rng = np.random.default_rng(12)
    a = torch.as_tensor(rng.standard_normal((32, 32, 32)).astype(np.float32), device="cuda")
    edges = np.geomspace(0.05, 0.45, 8)
    _, t = jf.transfer(a, 2.0 * a, box_shape=(200.0,) * 3, kedges=edges)
    _, c = jf.coherence(a, 2.0 * a, box_shape=(200.0,) * 3, kedges=edges)
    np.testing.assert_allclose(t.cpu().numpy(), 2.0, rtol=1e-5)
    np.testing.assert_allclose(c.cpu().numpy(), 1.0, rtol=1e-5)
    b = torch.as_tensor(rng.standard_normal((32, 32, 32)).astype(np.float32), device="cuda")
    _, c2 = jf.coherence(a, b, box_shape=(200.0,) * 3, kedges=edges)
    assert np.all(np.abs(c2.cpu().numpy()) < 0.5)  # independent fields: weakly coherent


@pytest.mark.parametrize("nside,width,interp", [(16, None, "fwhm"), (32, 90.0, "fwhm"), (32, 40.0, "sigma")])
def test_healpix_rbf_neighbor_matches_oracle(cosmo, nside, width, interp):
    """The rbf_neighbor scheme (Gaussian weights of the 4 surrounding pixel centres,
    normalised per particle) against the oracle's restatement, through
    ParticleField.paint_spherical; each particle's weight sums to one."""
    from oracle import healpix as oh

    n, L = 32, 200.0
    disp = lpt_disp(n, 2.0, seed=21).astype(np.float32)
    field = jf.ParticleField(array=dev(disp), mesh_size=(n,) * 3, box_size=(L,) * 3, nside=nside)
    rc, wd = 60.0, 40.0
    m = host(field.paint_spherical(rc, wd, scheme="rbf_neighbor", kernel_width_arcmin=width,
                                   smoothing_interpretation=interp).array).astype(np.float64)
    sigma = ops.rbf_sigma(nside, width, interp)
    obs = field.observer_position_mpc
    pos = (opm.grid((n, n, n)) + disp.astype(np.float64)) * (L / n)
    rmin, rmax = rc - wd / 2, rc + wd / 2
    vol = (4 * np.pi / (12 * nside * nside)) * (rmax**3 - rmin**3) / 3
    ref = oh.paint_shell(pos.reshape(-1, 3), obs, rmin, rmax, nside, "rbf_neighbor", sigma=sigma) / vol
    r = np.linalg.norm(pos.reshape(-1, 3) - np.asarray(obs), axis=1)
    inside = int(((r > rmin) & (r <= rmax)).sum())
    err = rel_l2(m, ref)
    print(f"nside {nside}, width {width} ({interp}): rel L2 {err:.2e}; total {m.sum() * vol:.1f} of {inside}")
    assert inside > 0 and err < 2e-5
    assert abs(m.sum() * vol / inside - 1) < 1e-5
