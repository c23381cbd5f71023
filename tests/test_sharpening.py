"""SharpeningKernel (reference pm/correction.py:214-333), the reversible PGD-style velocity
boost: in the fused loops of both solvers, in the stepwise solver methods, through the
reversible reverse step and through the differentiable run, against the FP64 oracle
(oracle/pm.py kkd_step / kdk_run with `sharpen`).

The reversible step boosts with alpha F_pgd(x) / (its full drift factor) at the positions it
kicks at (pm/solvers.py:292-318); the efficient step with alpha F_pgd(x) / (its bare drift
factor) at the drifted positions, before its kick (pm/solvers.py:164-195). The library
folds each boost into the kick it shares positions with: one combined potential,
(-1/k^2)(kick + boost PGD filter), read out with factor 1 (jfli_sharpen_potential)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import pm as opm

# alpha 0.03: the boost stays in the velocity and drifts in every later step (as in the
# reference), so at alpha 0.3 it moves particles by ~10 cells over 10 steps and the FP32
# trajectory parts from the FP64 one; at 0.03 it changes the final density by several
# per cent and the runs stay comparable
ALPHA, KL, KS = 0.03, 0.3, 1.0


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-30)


def _rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_oracle_sharpened_step_is_reversible():
    """The oracle's sharpened KKD step and its reverse are inverses in FP64 (the property
    the reference's reverse adjoint relies on, pm/solvers.py:339-411)."""
    rng = np.random.default_rng(0)
    n = 16
    x0 = 0.8 * rng.standard_normal((n, n, n, 3))
    v0 = 0.3 * rng.standard_normal((n, n, n, 3))
    steps = [(0.3, 0.5), (0.25, 0.4), (0.2, 0.3)]
    x, v = x0.copy(), v0.copy()
    for k, d in steps:
        x, v = opm.kkd_step(x, v, k, d, np.float64, (ALPHA, KL, KS))
    moved = np.abs(x - x0).max()
    for k, d in steps[::-1]:
        x, v = opm.kkd_reverse(x, v, k, d, np.float64, (ALPHA, KL, KS))
    assert moved > 0.5
    assert np.abs(x - x0).max() < 1e-12 and np.abs(v - v0).max() < 1e-12


def _setup(n, box, seed, t0=0.1):
    import jfli_b200 as jf

    cosmo = jf.Planck18()
    ic = jf.interpolate_initial_conditions(jf.white_noise(seed, (n,) * 3), (n,) * 3, (box,) * 3, cosmo=cosmo)
    dx, p = jf.lpt(cosmo, ic, ts=t0, order=2)
    return jf, cosmo, dx, p


def _solver(jf, name, sharpen=True):
    interp = jf.NoInterp(painting=jf.PaintingOptions(target="density"))
    corr = jf.SharpeningKernel(alpha=ALPHA, kl=KL, ks=KS) if sharpen else jf.NoCorrection()
    if name == "kkd":
        return jf.ReversibleDoubleKickDrift(interp_kernel=interp, pgd_kernel=corr)
    return jf.EfficientDriftDoubleKick(interp_kernel=interp, pgd_kernel=corr)


def _oracle_final(cosmo, solver_name, x, v, t0, t1, dt0, sharpen=True):
    """Final positions of the oracle loop on the schedule the library uses."""
    from jfli_b200.pm.integrate import time_events
    from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK
    from jfli_b200.pm.solvers import ReversibleDoubleKickDrift as KKD

    steps = [(e[1], e[2]) for e in time_events(t0, [t1], dt0) if e[0] == "step"]
    ta, tb = [a for a, _ in steps], [b for _, b in steps]
    if solver_name == "kkd":
        cs = [KKD.step_coefficients(cosmo, a, b, dt0, t0) for a, b in steps]
        xf, _, _ = opm.kkd_run(x, v, [(c.kick, c.drift) for c in cs], np.float64,
                               sharpen=(ALPHA, KL, KS) if sharpen else None)
        return xf
    kicks, drifts = EDK.schedule_arrays(cosmo, ta, tb, dt0)
    coeffs = dict(init_kick=EDK.init_kick(cosmo, t0, t0 + dt0), steps=list(zip(kicks, drifts)))
    bare = np.atleast_1d(EDK.bare_drift(cosmo, ta, tb))
    xf, _, _ = opm.kdk_run(x, v, coeffs, np.float64, sharpen=(ALPHA, KL, KS, bare) if sharpen else None)
    return xf


@pytest.mark.gpu
@pytest.mark.parametrize("solver_name", ["kkd", "edk"])
def test_sharpened_nbody_matches_oracle(solver_name):
    """64^3 in 256 Mpc/h, 2LPT to a = 0.1, 10 steps to a = 1 with SharpeningKernel(0.03, 0.3,
    1.0): the fused loop's final density against the FP64 oracle loop from the same initial
    particles, the stepwise solver methods (solver.step, the reference's own loop shape)
    against the fused loop, and the size of the boost's effect on the density."""
    import dataclasses

    from jfli_b200.pm.integrate import integrate
    from jfli_b200.pm.lpt import resolve_ts_geometry

    n, box, t0, t1, dt0 = 64, 256.0, 0.1, 1.0, 0.09
    jf, cosmo, dx, p = _setup(n, box, 5, t0)
    solver = _solver(jf, solver_name)
    rho = jf.nbody(cosmo, dx, p, t0=t0, t1=t1, dt0=dt0, solver=solver).array.cpu().numpy()
    # the same run through solver.init / step / save_at (the geometry nbody gives the interp)
    ts, rc, wd, _ = resolve_ts_geometry(cosmo, dx, painting=solver.interp_kernel.painting, ts=np.array([t1]),
                                        nb_shells=None, density_widths=None, equal_vol=False, min_width=50.0)
    interp = solver.interp_kernel.update_geometry(ts=ts, r_centers=rc, density_widths=wd,
                                                  max_comoving_distance=dx.max_comoving_radius)
    lc, _ = integrate(dx, p, cosmo, ts, dataclasses.replace(solver, interp_kernel=interp), t0, t1, dt0, fused=False)
    step = lc.array.reshape(rho.shape).cpu().numpy()
    x64 = dx.array.cpu().numpy().astype(np.float64)
    v64 = p.array.cpu().numpy().astype(np.float64)
    ref = opm.cic_paint(_oracle_final(cosmo, solver_name, x64, v64, t0, t1, dt0))
    plain = opm.cic_paint(_oracle_final(cosmo, solver_name, x64, v64, t0, t1, dt0, sharpen=False))
    err, err_step, effect = _rel_l2(rho, ref), _rel_l2(step, rho), _rel_l2(plain, ref)
    print(f"{solver_name} + SharpeningKernel: density rel L2 vs the FP64 oracle {err:.2e}; stepwise vs fused "
          f"{err_step:.2e}; the boost changes the density by {effect:.2e}")
    assert effect > 1e-3
    assert err < 1e-4
    assert err_step < 1e-5


@pytest.mark.gpu
def test_sharpened_reverse_recovers_initial_state():
    """jfli_kkd_run_sharpened then jfli_kkd_adjoint_sharpened (zero cotangents) bring random
    64^3 particles back to their start, and ReversibleDoubleKickDrift.reverse undoes .step
    with the boost (the reverse takes it off at the un-drifted positions)."""
    import jfli_b200 as jf
    from jfli_b200.fields import ParticleField, PositionUnit
    from jfli_b200.pm import adjoint as adj
    from jfli_b200.pm.solvers import NBodyState

    n = 64
    rng = np.random.default_rng(2)
    x0 = torch.as_tensor(1.0 * rng.standard_normal((n, n, n, 3)), dtype=torch.float32, device="cuda")
    v0 = torch.as_tensor(0.3 * rng.standard_normal((n, n, n, 3)), dtype=torch.float32, device="cuda")
    kicks = np.linspace(0.2, 0.4, 10)
    drifts = np.linspace(0.5, 0.2, 10)
    sharpen = (ALPHA / drifts, KL, KS)
    x, v = x0.clone(), v0.clone()
    rho = torch.empty(n, n, n, device="cuda")
    adj.kkd_forward(x, v, kicks, drifts, rho, sharpen=sharpen)
    moved = float((x - x0).abs().max())
    x_plain, v_plain = x0.clone(), v0.clone()
    adj.kkd_forward(x_plain, v_plain, kicks, drifts, rho)
    boost_effect = float((x - x_plain).abs().max())
    adj.kkd_reverse_adjoint(x, v, torch.zeros_like(x), torch.zeros_like(v), kicks, drifts, sharpen=sharpen)
    ex, ev = float((x - x0).abs().max()), float((v - v0).abs().max())

    cosmo = jf.Planck18()
    solver = _solver(jf, "kkd")
    f = ParticleField(array=x0.clone(), mesh_size=(n,) * 3, box_size=(256.0,) * 3, unit=PositionUnit.GRID_RELATIVE)
    state = NBodyState(interp_state=solver.interp_kernel.init(), t_initial=0.5)
    d1, v1, s1 = solver.step(f, f.replace(array=v0.clone()), 0.5, 0.6, 0.1, state, cosmo)
    d0, vr, _ = solver.reverse(d1, v1, 0.5, 0.6, 0.1, s1, cosmo)
    sx, sv = float((d0.array - x0).abs().max()), float((vr.array - v0).abs().max())
    print(f"moved {moved:.3f} cells (the boost {boost_effect:.3f}); after the sharpened sweep |dx| {ex:.2e}, "
          f"|dv| {ev:.2e}; solver.reverse(step) |dx| {sx:.2e} |dv| {sv:.2e}")
    assert moved > 0.5 and boost_effect > 1e-3
    assert ex < 1e-4 and ev < 1e-4
    assert sx < 1e-5 and sv < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("solver_name", ["kkd", "edk"])
def test_sharpened_gradient_matches_oracle_fd(solver_name):
    """nbody with SharpeningKernel on displacements and momenta that require grad (the
    reversible adjoint over the combined kick-and-boost force): the density equals the fused
    loop's, and the directional derivative of <a, rho(final)> matches central differences
    of the FP64 oracle loop.

    The boosted run moves particles far enough that perturbations of 1e-5..3e-7 cells carry
    many of them across CIC cell faces, where the painted density has kinks: with white-noise
    weights `a` the oracle's own central differences vary by 1.5% between those steps. With
    `a` smoothed over 4 cells (each kink's slope jump scales with the cell-to-cell change
    of `a`) they vary by 1.5e-4 (ReversibleDoubleKickDrift) and 1.2e-3
    (EfficientDriftDoubleKick); the bound is 2e-3."""
    n, box, t0, t1, dt0 = 32, 128.0, 0.1, 1.0, 0.15
    jf, cosmo, dx, p = _setup(n, box, 21, t0)
    x0, v0 = dx.array.detach().contiguous().clone(), p.array.detach().contiguous().clone()
    rng = np.random.default_rng(22)
    a = rng.standard_normal((n, n, n))
    k = np.fft.fftfreq(n) * 2 * np.pi
    kk = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    a = np.real(np.fft.ifftn(np.fft.fftn(a) * np.exp(-0.5 * kk * 16.0)))  # Gaussian, sigma 4 cells
    a /= a.std()
    r = rng.standard_normal((n, n, n, 3))
    s = rng.standard_normal((n, n, n, 3))
    solver = _solver(jf, solver_name)
    xg, vg = x0.clone().requires_grad_(True), v0.clone().requires_grad_(True)
    rho = jf.nbody(cosmo, dx.replace(array=xg), p.replace(array=vg), t0=t0, t1=t1, dt0=dt0, solver=solver)
    loss = (rho.array.double() * torch.as_tensor(a, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(xg.grad.cpu().numpy() * r) + np.sum(vg.grad.cpu().numpy() * s))
    with torch.no_grad():
        rho_f = jf.nbody(cosmo, dx.replace(array=x0), p.replace(array=v0), t0=t0, t1=t1, dt0=dt0, solver=solver)
    e_fwd = float((rho.array.detach() - rho_f.array).norm() / rho_f.array.norm())

    def oracle_loss(x, v):
        return float(np.sum(a * opm.cic_paint(_oracle_final(cosmo, solver_name, x, v, t0, t1, dt0))))

    x64, v64 = x0.cpu().numpy().astype(np.float64), v0.cpu().numpy().astype(np.float64)
    eps = 1e-6
    fd = (oracle_loss(x64 + eps * r, v64 + eps * s) - oracle_loss(x64 - eps * r, v64 - eps * s)) / (2 * eps)
    L0 = oracle_loss(x64, v64)
    print(f"{solver_name} + SharpeningKernel: density vs the fused loop {e_fwd:.2e}; loss GPU "
          f"{float(loss.detach()):.8e} oracle {L0:.8e}; directional derivative {g_dir:.6e} vs oracle central "
          f"difference {fd:.6e}")
    assert e_fwd < 1e-5
    assert _rel(float(loss.detach()), L0) < 1e-4
    assert _rel(g_dir, fd) < 2e-3
