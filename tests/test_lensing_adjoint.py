"""Adjoints of the shell painter (jfli_healpix_paint_shells_adjoint) and of Born
(jfli_born_adjoint), and a lensing-map loss differentiated through both: gradients from
autograd against central differences of the FP64 oracle (oracle/healpix.py painting, Born
restated in NumPy FP64) along random directions.

The painted map is piecewise linear in the particle directions (bilinear weights) and has
steps where a particle crosses a shell edge or a pixel-bracket edge of zero weight; with
displacement steps of 1e-6 cells over 32^3 particles no particle crosses an edge, so the
central difference is the derivative."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import healpix as oh
from oracle import pm as opm

pytestmark = pytest.mark.gpu

N, L, NSIDE = 32, 200.0, 16
OBS = (100.0, 100.0, 100.0)
SHELLS = ((30.0, 50.0), (50.0, 70.0), (60.0, 90.0))  # the last overlaps the second


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-30)


def _setup(seed=3):
    from tests.test_gpu_parity import lpt_disp

    disp = lpt_disp(N, 2.0, seed=seed).astype(np.float32)
    rng = np.random.default_rng(seed + 100)
    a = rng.standard_normal((len(SHELLS), 12 * NSIDE * NSIDE))
    r = rng.standard_normal((N, N, N, 3))
    return disp, a, r


def _scales():
    from jfli_b200.painting import shell_volume_per_pixel

    return np.array([1.0 / shell_volume_per_pixel(NSIDE, lo, hi) for lo, hi in SHELLS])


def _oracle_maps(disp64, weights=None):
    g = opm.grid((N, N, N), np.float64)
    pos = (g + disp64) * (L / N)
    sc = _scales()
    out = []
    for (lo, hi), s in zip(SHELLS, sc):
        if weights is None:
            m = oh.paint_shell(pos.reshape(-1, 3), OBS, lo, hi, NSIDE, "bilinear")
        else:  # per-particle weights: the painter's bilinear deposit, weighted
            v = pos.reshape(-1, 3) - np.asarray(OBS)
            rr = np.sqrt((v ** 2).sum(-1))
            sel = (rr > lo) & (rr <= hi)
            th = np.arccos(np.clip(v[sel, 2] / rr[sel], -1, 1))
            ph = np.arctan2(v[sel, 1], v[sel, 0])
            pix, w = oh.get_interp_weights(NSIDE, th, ph)
            ww = w * weights.reshape(-1)[sel][None, :]
            m = np.bincount(pix.ravel(), weights=ww.ravel(), minlength=12 * NSIDE * NSIDE)
        out.append(m * s)
    return np.stack(out)


def _gpu_maps(disp_t, weights_t=None):
    from jfli_b200 import painting
    from jfli_b200.fields import ParticleField, PositionUnit

    f = ParticleField(array=disp_t, mesh_size=(N,) * 3, box_size=(L,) * 3, observer_position=(0.5, 0.5, 0.5),
                      nside=NSIDE, unit=PositionUnit.GRID_RELATIVE)
    c = np.array([(lo + hi) / 2 for lo, hi in SHELLS])
    w = np.array([hi - lo for lo, hi in SHELLS])
    return painting.paint_shells(f, c, w, "bilinear", weights_t)


def test_paint_shells_adjoint_matches_oracle_fd():
    disp, a, r = _setup()
    x = torch.as_tensor(disp, device="cuda").requires_grad_(True)
    maps = _gpu_maps(x)
    loss = (maps.double() * torch.as_tensor(a, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(x.grad.cpu().numpy().astype(np.float64) * r))
    d64 = disp.astype(np.float64)
    eps = 1e-6
    fd = (np.sum(a * _oracle_maps(d64 + eps * r)) - np.sum(a * _oracle_maps(d64 - eps * r))) / (2 * eps)
    L0 = float(np.sum(a * _oracle_maps(d64)))
    print(f"shell paint: loss GPU {float(loss):.8e} oracle {L0:.8e}; directional derivative {g_dir:.6e} vs oracle "
          f"central difference {fd:.6e}")
    assert _rel(float(loss), L0) < 1e-5
    assert _rel(g_dir, fd) < 1e-4


def test_paint_shells_adjoint_weights():
    """Per-particle weights: the position cotangent carries them, and the weight cotangent is
    the derivative of the (linear) map in the weights."""
    disp, a, r = _setup(seed=4)
    rng = np.random.default_rng(7)
    wts = rng.uniform(0.5, 1.5, (N, N, N))
    q = rng.standard_normal((N, N, N))
    x = torch.as_tensor(disp, device="cuda").requires_grad_(True)
    wt = torch.as_tensor(wts.astype(np.float32), device="cuda").requires_grad_(True)
    loss = (_gpu_maps(x, wt).double() * torch.as_tensor(a, device="cuda")).sum()
    loss.backward()
    g_x = float(np.sum(x.grad.cpu().numpy().astype(np.float64) * r))
    g_w = float(np.sum(wt.grad.cpu().numpy().astype(np.float64) * q))
    d64 = disp.astype(np.float64)
    w64 = wts.astype(np.float32).astype(np.float64)
    eps = 1e-6
    fd_x = (np.sum(a * _oracle_maps(d64 + eps * r, w64)) - np.sum(a * _oracle_maps(d64 - eps * r, w64))) / (2 * eps)
    fd_w = (np.sum(a * _oracle_maps(d64, w64 + 1e-3 * q)) - np.sum(a * _oracle_maps(d64, w64 - 1e-3 * q))) / 2e-3
    print(f"weighted shell paint: positions {g_x:.6e} vs {fd_x:.6e}; weights {g_w:.6e} vs {fd_w:.6e}")
    assert _rel(g_x, fd_x) < 1e-4
    assert _rel(g_w, fd_w) < 1e-5


def test_paint_shells_ngp_gradients():
    """ngp: the map is a step function of the positions (zero position cotangent); the
    weight cotangent is the cotangent map at each particle's pixel."""
    from jfli_b200 import ops

    disp, a, _ = _setup(seed=5)
    x = torch.as_tensor(disp, device="cuda")
    mb = torch.as_tensor(a.astype(np.float32), device="cuda")
    rmin = np.array([s[0] for s in SHELLS])
    rmax = np.array([s[1] for s in SHELLS])
    sc = _scales()
    wbar = torch.zeros(N, N, N, device="cuda")
    pbar = ops.healpix_paint_shells_adjoint(x, mb, NSIDE, (L,) * 3, OBS, rmin, rmax, sc, scheme="ngp", weights=None,
                                            weights_bar=wbar)
    assert float(pbar.abs().max()) == 0.0
    g = opm.grid((N, N, N), np.float64)
    v = ((g + disp.astype(np.float64)) * (L / N) - np.asarray(OBS)).reshape(-1, 3)
    rr = np.sqrt((v ** 2).sum(-1))
    ref = np.zeros(N ** 3)
    pix = oh.ang2pix(NSIDE, np.arccos(np.clip(v[:, 2] / rr, -1, 1)), np.arctan2(v[:, 1], v[:, 0]))
    for s, (lo, hi) in enumerate(SHELLS):
        sel = (rr > lo) & (rr <= hi)
        ref[sel] += sc[s] * a.astype(np.float32).astype(np.float64)[s, pix[sel]]
    err = float(np.abs(wbar.cpu().numpy().reshape(-1) - ref).max() / np.abs(ref).max())
    print(f"ngp weight cotangent vs oracle: {err:.2e}")
    assert err < 1e-6


def _born_np(maps, W):
    """kappa = W (maps / mean - 1), FP64 (the Born combination of oracle/lensing.py)."""
    mean = maps.mean(axis=1, keepdims=True)
    return W @ (maps / mean - 1.0)


def test_born_adjoint_matches_fd():
    from jfli_b200 import lensing

    rng = np.random.default_rng(11)
    P, K, npix = 5, 2, 12 * 16 * 16
    maps = rng.uniform(0.5, 2.0, (P, npix)).astype(np.float32)
    W = rng.uniform(0.0, 1e-2, (K, P))
    b = rng.standard_normal((K, npix))
    r = rng.standard_normal((P, npix))
    m = torch.as_tensor(maps, device="cuda").requires_grad_(True)
    kappa = lensing.born_maps(m, W)
    loss = (kappa.double() * torch.as_tensor(b, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(m.grad.cpu().numpy().astype(np.float64) * r))
    m64 = maps.astype(np.float64)
    eps = 1e-4
    fd = (np.sum(b * _born_np(m64 + eps * r, W)) - np.sum(b * _born_np(m64 - eps * r, W))) / (2 * eps)
    print(f"Born: directional derivative {g_dir:.8e} vs FP64 central difference {fd:.8e}")
    assert _rel(g_dir, fd) < 1e-5


def test_lensing_loss_gradient_matches_oracle_fd():
    """particles -> ParticleField.paint_spherical (three shells, bilinear) -> Born -> a
    linear loss of the convergence map, differentiated with respect to the displacements."""
    from jfli_b200 import lensing
    from jfli_b200.fields import ParticleField, PositionUnit

    disp, _, r = _setup(seed=6)
    rng = np.random.default_rng(12)
    W = rng.uniform(0.0, 1e-2, (1, len(SHELLS)))
    b = rng.standard_normal((1, 12 * NSIDE * NSIDE))
    x = torch.as_tensor(disp, device="cuda").requires_grad_(True)
    f = ParticleField(array=x, mesh_size=(N,) * 3, box_size=(L,) * 3, observer_position=(0.5, 0.5, 0.5), nside=NSIDE,
                      unit=PositionUnit.GRID_RELATIVE)
    c = np.array([(lo + hi) / 2 for lo, hi in SHELLS])
    w = np.array([hi - lo for lo, hi in SHELLS])
    shells = f.paint_spherical(center=c, density_plane_width=w, scheme="bilinear")
    kappa = lensing.born_maps(shells.array, W)
    loss = (kappa.double() * torch.as_tensor(b, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(x.grad.cpu().numpy().astype(np.float64) * r))
    d64 = disp.astype(np.float64)
    eps = 1e-6

    def oracle_loss(d):
        return float(np.sum(b * _born_np(_oracle_maps(d), W)))

    fd = (oracle_loss(d64 + eps * r) - oracle_loss(d64 - eps * r)) / (2 * eps)
    print(f"lensing loss: GPU {float(loss):.8e} oracle {oracle_loss(d64):.8e}; directional derivative {g_dir:.6e} "
          f"vs oracle central difference {fd:.6e}")
    assert _rel(float(loss), oracle_loss(d64)) < 1e-4
    assert _rel(g_dir, fd) < 1e-4


def test_nbody_shells_gradient_matches_oracle_fd():
    """nbody(EfficientDriftDoubleKick, NoInterp spherical shells, nb_shells=3) on displacements
    and momenta that require grad: the shells equal the fused loop's, and the directional
    derivative of a linear loss of the shells matches central differences of an FP64 oracle
    loop (oracle/pm.py forces, FastPM steps, oracle/healpix.py painting at each snapshot)."""
    import jfli_b200 as jf
    from jfli_b200.painting import shell_volume_per_pixel
    from jfli_b200.pm.integrate import time_events
    from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK

    n, box, nside, t0, t1, dt0 = 32, 200.0, 16, 0.1, 1.0, 0.15
    cosmo = jf.Planck18()
    ic = jf.interpolate_initial_conditions(jf.white_noise(41, (n,) * 3), (n,) * 3, (box,) * 3, cosmo=cosmo,
                                           nside=nside)
    dx, p = jf.lpt(cosmo, ic, ts=t0, order=2)
    x0, v0 = dx.array.detach().contiguous().clone(), p.array.detach().contiguous().clone()
    solver = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="spherical")))
    kw = dict(t0=t0, t1=t1, dt0=dt0, nb_shells=3, solver=solver)
    xg, vg = x0.clone().requires_grad_(True), v0.clone().requires_grad_(True)
    lc = jf.nbody(cosmo, dx.replace(array=xg), p.replace(array=vg), **kw)
    rng = np.random.default_rng(42)
    b = rng.standard_normal(tuple(lc.array.shape))
    r = rng.standard_normal((n, n, n, 3))
    s = rng.standard_normal((n, n, n, 3))
    loss = (lc.array.double() * torch.as_tensor(b, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(xg.grad.cpu().numpy() * r) + np.sum(vg.grad.cpu().numpy() * s))
    with torch.no_grad():
        lc_f = jf.nbody(cosmo, dx.replace(array=x0), p.replace(array=v0), **kw)
    e_fwd = float((lc.array.detach() - lc_f.array).norm() / lc_f.array.norm())

    # the oracle loop on the same schedule (snapshot times ascending, as the loop meets them)
    ts = np.asarray(lc.scale_factors, np.float64)[::-1]
    rc = np.asarray(lc.comoving_centers, np.float64)[::-1]
    wd = np.asarray(lc.density_width, np.float64)[::-1]
    events = time_events(t0, ts, dt0)
    steps = [(e[1], e[2]) for e in events if e[0] == "step"]
    kicks, drifts = EDK.schedule_arrays(cosmo, [q for q, _ in steps], [q for _, q in steps], dt0)
    k_init = EDK.init_kick(cosmo, t0, t0 + dt0)
    g = opm.grid((n, n, n), np.float64)
    obs = np.asarray(dx.observer_position_mpc, np.float64)

    def oracle_shells(x, v):
        x, v = x.copy(), v.copy()
        v += opm.pm_forces(x, np.float64) * k_init
        maps, si = [], 0
        for ev in events:
            if ev[0] == "step":
                x += v * drifts[si]
                v += opm.pm_forces(x, np.float64) * kicks[si]
                si += 1
            else:
                i = ev[1]
                lo, hi = rc[i] - wd[i] / 2, rc[i] + wd[i] / 2
                m = oh.paint_shell(((g + x) * (box / n)).reshape(-1, 3), obs, lo, hi, nside, "bilinear")
                maps.append(m / shell_volume_per_pixel(nside, lo, hi))
        return np.stack(maps[::-1])  # near -> far, as nbody returns them

    x64, v64 = x0.cpu().numpy().astype(np.float64), v0.cpu().numpy().astype(np.float64)
    eps = 1e-6
    fd = (np.sum(b * oracle_shells(x64 + eps * r, v64 + eps * s))
          - np.sum(b * oracle_shells(x64 - eps * r, v64 - eps * s))) / (2 * eps)
    L0 = float(np.sum(b * oracle_shells(x64, v64)))
    print(f"nbody shells: vs the fused loop {e_fwd:.2e}; loss GPU {float(loss):.8e} oracle {L0:.8e}; directional "
          f"derivative {g_dir:.6e} vs oracle central difference {fd:.6e}")
    assert e_fwd < 1e-5
    assert _rel(float(loss), L0) < 1e-3
    assert _rel(g_dir, fd) < 1e-3


def test_tiled_paint_adjoint_matches_oracle_fd():
    """jfli_healpix_paint_tiled_adjoint: one shell beyond the box (120-160 Mpc/h, box 200)
    from 27 rotated, shifted replicas drifted to the light cone at t = 0.7 (OnionTiler), the
    directional derivative of a linear loss in the displacements and velocities against
    central differences of the FP64 oracle's replica painter. The oracle's dGfa is the
    closed form where the kernel reads a dense table, so the drift's derivative differs at
    the table's interpolation error (~1e-6)."""
    import jfli_b200 as jf
    from jfli_b200 import cosmology as cj
    from jfli_b200 import painting
    from jfli_b200.fields import ParticleField, PositionUnit
    from jfli_b200.pm.interp import get_all_47_symmetries, tile_shifts

    cosmo = jf.Planck18()
    disp, _, r = _setup(seed=8)
    rng = np.random.default_rng(9)
    vel = (0.3 * rng.standard_normal((N, N, N, 3))).astype(np.float32)
    s = rng.standard_normal((N, N, N, 3))
    rot = get_all_47_symmetries()[rng.integers(0, 47, 27)]
    rot[0] = np.eye(3, dtype=rot.dtype)
    shifts = tile_shifts((0.5, 0.5, 0.5), (L, L, L))
    t, lo, hi = 0.7, 120.0, 160.0
    b = rng.standard_normal(12 * NSIDE * NSIDE)
    x = torch.as_tensor(disp, device="cuda").requires_grad_(True)
    v = torch.as_tensor(vel, device="cuda").requires_grad_(True)
    f = ParticleField(array=x, mesh_size=(N,) * 3, box_size=(L,) * 3, observer_position=(0.5, 0.5, 0.5), nside=NSIDE,
                      unit=PositionUnit.GRID_RELATIVE)
    m = painting.paint_shell_tiled(f, v, (lo + hi) / 2, hi - lo, rot, shifts, t=t, cosmo=cosmo)
    loss = (m.double() * torch.as_tensor(b, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(x.grad.cpu().numpy() * r) + np.sum(v.grad.cpu().numpy() * s))
    scale = 1.0 / painting.shell_volume_per_pixel(NSIDE, lo, hi)
    fn = dict(a_of_chi=lambda q: cj.a_of_chi(cosmo, q), Gp=lambda a: cj.Gp(cosmo, a), dGfa=lambda a: cj.dGfa(cosmo, a))

    def oracle_loss(d, w):
        return float(np.sum(b * scale * oh.paint_shell_tiled(d, w, (L, L, L), OBS, lo, hi, NSIDE, rot, shifts, t=t,
                                                              **fn)))

    d64, v64 = disp.astype(np.float64), vel.astype(np.float64)
    eps = 1e-6
    fd = (oracle_loss(d64 + eps * r, v64 + eps * s) - oracle_loss(d64 - eps * r, v64 - eps * s)) / (2 * eps)
    L0 = oracle_loss(d64, v64)
    print(f"tiled paint with drift: loss GPU {float(loss):.8e} oracle {L0:.8e}; directional derivative {g_dir:.6e} vs "
          f"oracle central difference {fd:.6e}")
    assert _rel(float(loss), L0) < 1e-4
    assert _rel(g_dir, fd) < 1e-3


@pytest.mark.parametrize("tiler,solver_name", [("onion", "edk"), ("drift", "edk"), ("onion", "kkd"),
                                               ("onion", "edk_sharp")])
def test_nbody_drifted_shells_gradient_matches_oracle_fd(tiler, solver_name):
    """nbody with light-cone-drifted HEALPix shells (OnionTiler: the shell inside the box from
    the particles drifted to the light cone, the two beyond it from 27 rotated replicas;
    DriftInterp: every shell from the drifted particles) on displacements and momenta that
    require grad: the shells equal the fused loop's, and the directional derivative of a
    linear loss of the shells matches central differences of an FP64 oracle loop (oracle/pm.py
    forces, the solver's steps, oracle/healpix.py's replica painter at each snapshot with the
    velocities there; under EfficientDriftDoubleKick those include the pending kick, which the
    loop applies before a velocity-dependent paint; with SharpeningKernel, "edk_sharp", that
    pending kick carries the sharpening boost, whose VJP adds boost J_pgd^T).

    The central differences take steps of 3e-7: at 1e-6 a particle of the nearest shell
    crosses a kink of the bilinear weights along the velocity direction under
    EfficientDriftDoubleKick (the difference moves by 7e-3 of the derivative; at 3e-7 it
    agrees with the adjoint to 7e-6)."""
    import jfli_b200 as jf
    from jfli_b200 import cosmology as cj
    from jfli_b200.painting import shell_volume_per_pixel
    from jfli_b200.pm.integrate import time_events
    from jfli_b200.pm.interp import get_all_47_symmetries, tile_shifts
    from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK

    n, box, nside, t0, t1, dt0 = 32, 200.0, 16, 0.1, 1.0, 0.15
    cosmo = jf.Planck18()
    ic = jf.interpolate_initial_conditions(jf.white_noise(43, (n,) * 3), (n,) * 3, (box,) * 3, cosmo=cosmo,
                                           nside=nside)
    dx, p = jf.lpt(cosmo, ic, ts=t0, order=2)
    x0, v0 = dx.array.detach().contiguous().clone(), p.array.detach().contiguous().clone()
    rng = np.random.default_rng(44)
    ridx = tuple(int(i) for i in rng.integers(0, 47, 27))
    painting = jf.PaintingOptions(target="spherical")
    interp = (jf.OnionTiler(painting=painting, rotation_indices=ridx) if tiler == "onion"
              else jf.DriftInterp(painting=painting))
    sharp = (0.03, 0.3, 1.0)  # SharpeningKernel(alpha, kl, ks) for "edk_sharp"
    if solver_name == "kkd":
        solver = jf.ReversibleDoubleKickDrift(interp_kernel=interp)
    else:
        solver = jf.EfficientDriftDoubleKick(interp_kernel=interp, pgd_kernel=jf.SharpeningKernel(*sharp)
                                             if solver_name == "edk_sharp" else jf.NoCorrection())
    edges = np.array([170.0, 110.0, 60.0, 20.0])  # far -> near; the box holds a sphere of 100 Mpc/h
    centres = 0.5 * (edges[1:] + edges[:-1])
    kw = dict(t0=t0, t1=t1, dt0=dt0, solver=solver, ts=np.asarray(cj.a_of_chi(cosmo, centres), np.float64),
              density_widths=edges[:-1] - edges[1:])
    xg, vg = x0.clone().requires_grad_(True), v0.clone().requires_grad_(True)
    lc = jf.nbody(cosmo, dx.replace(array=xg), p.replace(array=vg), **kw)
    b = rng.standard_normal(tuple(lc.array.shape))
    r = rng.standard_normal((n, n, n, 3))
    s = rng.standard_normal((n, n, n, 3))
    loss = (lc.array.double() * torch.as_tensor(b, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(xg.grad.cpu().numpy() * r) + np.sum(vg.grad.cpu().numpy() * s))
    with torch.no_grad():
        lc_f = jf.nbody(cosmo, dx.replace(array=x0), p.replace(array=v0), **kw)
    e_fwd = float((lc.array.detach() - lc_f.array).norm() / lc_f.array.norm())

    ts = np.asarray(lc.scale_factors, np.float64)[::-1]
    rc = np.asarray(lc.comoving_centers, np.float64)[::-1]
    wd = np.asarray(lc.density_width, np.float64)[::-1]
    events = time_events(t0, ts, dt0)
    steps = [(e[1], e[2]) for e in events if e[0] == "step"]
    if solver_name != "kkd":
        kicks, drifts = EDK.schedule_arrays(cosmo, [q for q, _ in steps], [q for _, q in steps], dt0)
        k_init = EDK.init_kick(cosmo, t0, t0 + dt0)
        bare = np.atleast_1d(EDK.bare_drift(cosmo, [q for q, _ in steps], [q for _, q in steps]))
    else:
        cs = [solver.step_coefficients(cosmo, a, q, dt0, t0) for a, q in steps]
        kicks, drifts = [c.kick for c in cs], [c.drift for c in cs]
    obs = np.asarray(dx.observer_position_mpc, np.float64)
    rot27 = get_all_47_symmetries()[list(ridx)]
    sh27 = tile_shifts(dx.observer_position, dx.box_size)
    fn = dict(a_of_chi=lambda q: cj.a_of_chi(cosmo, q), Gp=lambda a: cj.Gp(cosmo, a), dGfa=lambda a: cj.dGfa(cosmo, a))

    def oracle_shells(x, v):
        x, v = x.copy(), v.copy()
        if solver_name != "kkd":
            v += opm.pm_forces(x, np.float64) * k_init
        maps, si = [], 0
        for ev in events:
            if ev[0] == "step":
                if solver_name != "kkd":
                    x += v * drifts[si]
                    if solver_name == "edk_sharp":
                        v += opm.sharpening_boost(x, *sharp, bare[si], np.float64)
                    v += opm.pm_forces(x, np.float64) * kicks[si]
                else:
                    v += opm.pm_forces(x, np.float64) * kicks[si]
                    x += v * drifts[si]
                si += 1
            else:
                i = ev[1]
                lo, hi = rc[i] - wd[i] / 2, rc[i] + wd[i] / 2
                rot, sh = ((rot27, sh27) if (tiler == "onion" and hi > box / 2)
                           else (np.eye(3)[None], np.zeros((1, 3))))
                m = oh.paint_shell_tiled(x, v, (box,) * 3, obs, lo, hi, nside, rot, sh, t=float(ev[2]), **fn)
                maps.append(m / shell_volume_per_pixel(nside, lo, hi))
        return np.stack(maps[::-1])  # near -> far, as nbody returns them

    x64, v64 = x0.cpu().numpy().astype(np.float64), v0.cpu().numpy().astype(np.float64)
    eps = 3e-7
    fd = (np.sum(b * oracle_shells(x64 + eps * r, v64 + eps * s))
          - np.sum(b * oracle_shells(x64 - eps * r, v64 - eps * s))) / (2 * eps)
    L0 = float(np.sum(b * oracle_shells(x64, v64)))
    print(f"nbody {tiler} shells ({solver_name}): vs the fused loop {e_fwd:.2e}; loss GPU {float(loss.detach()):.8e} "
          f"oracle {L0:.8e}; directional derivative {g_dir:.6e} vs oracle central difference {fd:.6e}")
    assert e_fwd < 1e-5
    assert _rel(float(loss.detach()), L0) < 1e-3
    assert _rel(g_dir, fd) < 1e-3
