"""Adjoint kernels and the reversible-adjoint gradient against finite differences.

Small cases compare the CUDA adjoints (FP32) with central differences of the FP64 oracle
(oracle/pm.py) along random directions; the 128^3 case (the differentiation
configuration: ReversibleDoubleKickDrift, 20 steps from a = 0.1, box 500 Mpc/h, 2LPT,
loss = sum over 32 bins of (log P - log P_target)^2) compares with central differences
of the GPU forward model at eps = 1e-3."""

import numpy as np
import pytest
import torch

from oracle import pm as opm

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.as_tensor(np.asarray(a, np.float32), device="cuda")


def _kedges(n, box):
    return np.geomspace(2 * np.pi / box * (1 - 1e-6), np.pi * n / box, 33)


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-30)


# --------------------------------------------------------------------------- KKD steps
def test_kkd_step_vjp_matches_oracle_fd():
    from jfli_b200.pm import adjoint as adj

    n = 32
    rng = np.random.default_rng(1)
    x0 = (1.5 * rng.standard_normal((n, n, n, 3))).astype(np.float32)
    v0 = (0.5 * rng.standard_normal((n, n, n, 3))).astype(np.float32)
    kicks, drifts = np.array([0.3, 0.25, 0.35]), np.array([0.4, 0.5, 0.3])
    a = rng.standard_normal(x0.shape)
    b = rng.standard_normal(x0.shape)
    r = rng.standard_normal(x0.shape)
    s = rng.standard_normal(x0.shape)

    x, v = _dev(x0), _dev(v0)
    rho = torch.empty(n, n, n, device="cuda")
    force = torch.empty(n, n, n, 4, device="cuda")
    pot = torch.empty_like(rho)
    adj.kkd_forward(x, v, kicks, drifts, rho, force, pot)
    lam_x, lam_v = _dev(a), _dev(b)
    sens = adj.kkd_reverse_adjoint(x, v, lam_x, lam_v, kicks, drifts).cpu().numpy()
    g_dir = float(np.sum(lam_x.cpu().numpy() * r) + np.sum(lam_v.cpu().numpy() * s))

    def loss(xi, vi, ks=kicks, ds=drifts):
        xf, vf, _ = opm.kkd_run(xi, vi, list(zip(ks, ds)), np.float64)
        return float(np.sum(a * xf) + np.sum(b * vf))

    eps = 1e-5
    x64, v64 = x0.astype(np.float64), v0.astype(np.float64)
    fd = (loss(x64 + eps * r, v64 + eps * s) - loss(x64 - eps * r, v64 - eps * s)) / (2 * eps)
    print(f"direction: adjoint {g_dir:.8e} fd {fd:.8e}")
    assert _rel(g_dir, fd) < 1e-4
    for i in range(len(kicks)):
        kp, km = kicks.copy(), kicks.copy()
        kp[i] += eps
        km[i] -= eps
        fdk = (loss(x64, v64, ks=kp) - loss(x64, v64, ks=km)) / (2 * eps)
        dp, dm = drifts.copy(), drifts.copy()
        dp[i] += eps
        dm[i] -= eps
        fdd = (loss(x64, v64, ds=dp) - loss(x64, v64, ds=dm)) / (2 * eps)
        print(f"step {i}: dkick {sens[i, 0]:.6e} vs {fdk:.6e}; ddrift {sens[i, 1]:.6e} vs {fdd:.6e}")
        assert _rel(sens[i, 0], fdk) < 1e-4
        assert _rel(sens[i, 1], fdd) < 1e-4


def test_reverse_recovers_initial_state():
    from jfli_b200.pm import adjoint as adj

    n = 64
    rng = np.random.default_rng(2)
    x0 = _dev(1.0 * rng.standard_normal((n, n, n, 3)))
    v0 = _dev(0.3 * rng.standard_normal((n, n, n, 3)))
    kicks = np.linspace(0.2, 0.4, 10)
    drifts = np.linspace(0.5, 0.2, 10)
    x, v = x0.clone(), v0.clone()
    rho = torch.empty(n, n, n, device="cuda")
    force = torch.empty(n, n, n, 4, device="cuda")
    adj.kkd_forward(x, v, kicks, drifts, rho, force, torch.empty_like(rho))
    moved = float((x - x0).abs().max())
    adj.kkd_reverse_adjoint(x, v, torch.zeros_like(x), torch.zeros_like(v), kicks, drifts)
    ex, ev = float((x - x0).abs().max()), float((v - v0).abs().max())
    print(f"max displacement change {moved:.3f} cells; after reverse |dx| {ex:.2e}, |dv| {ev:.2e}")
    assert moved > 0.5
    assert ex < 1e-4 and ev < 1e-4


def test_stored_potentials_match_recomputed_sweep():
    """jfli_kkd_run_stored / jfli_kkd_adjoint_stored: the forward results are jfli_kkd_run's
    (to the run-to-run spread of the FP32 atomic paint's order), and the reverse sweep
    over the kept potentials gives the cotangents, the dL/dkick, dL/ddrift and the
    recovered initial state of the recomputing sweep. The stored forces are the forward
    pass's own, the recomputed ones those at positions reconstructed to FP32 rounding; on
    this random state (displacements of a cell, velocities of a third) the two sweeps'
    CIC weight gradients, which jump at cell faces, then differ for the particles that
    rounding puts on the other side of a face, so the sweeps agree to 1e-3, not to FP32.
    Each is checked against the FP64 oracle's finite differences (1e-4) on its own."""
    from jfli_b200 import ops
    from jfli_b200.pm import adjoint as adj

    n = 64
    rng = np.random.default_rng(3)
    x0 = _dev(1.0 * rng.standard_normal((n, n, n, 3)))
    v0 = _dev(0.3 * rng.standard_normal((n, n, n, 3)))
    kicks = np.linspace(0.2, 0.4, 10)
    drifts = np.linspace(0.5, 0.2, 10)
    a, b = _dev(rng.standard_normal((n, n, n, 3))), _dev(rng.standard_normal((n, n, n, 3)))
    out = {}
    for mode in ("recompute", "stored"):
        x, v = x0.clone(), v0.clone()
        rho = torch.empty(n, n, n, device="cuda")
        pots = torch.empty(len(kicks), n, n, n, device="cuda") if mode == "stored" else None
        ops.kkd_run(x, v, kicks, drifts, rho, pots=pots)
        fwd = (x.clone(), v.clone(), rho.clone())
        lx, lv = a.clone(), b.clone()
        sens = ops.kkd_adjoint(x, v, lx, lv, kicks, drifts, pots=pots)
        out[mode] = (fwd, lx, lv, sens.cpu().numpy(), x, v)
    (f0, lx0, lv0, s0, xr0, vr0), (f1, lx1, lv1, s1, xr1, vr1) = out["recompute"], out["stored"]
    for name, t0, t1 in zip(("positions", "momenta", "density"), f0, f1):
        e = float((t1 - t0).norm() / t0.norm())
        print(f"forward {name}: stored vs recomputed {e:.2e}")
        assert e < 1e-5
    e_lx = float((lx1 - lx0).norm() / lx0.norm())
    e_lv = float((lv1 - lv0).norm() / lv0.norm())
    e_s = float(np.abs(s1 - s0).max() / np.abs(s0).max())
    e_x = float((xr1 - x0).abs().max())
    print(f"stored vs recomputed: lam_x {e_lx:.2e}, lam_v {e_lv:.2e}, sensitivities {e_s:.2e}; "
          f"initial state recovered to {e_x:.2e} cells (recomputing sweep {float((xr0 - x0).abs().max()):.2e})")
    assert e_lx < 1e-3 and e_lv < 1e-3 and e_s < 1e-3
    assert e_x < 1e-4


@pytest.mark.parametrize("shape,batch", [((32, 48, 64), 1), ((24, 36, 32), 1), ((32, 32, 32), 2)])
def test_stored_sweep_shapes_and_batch(shape, batch):
    """The stored-potential loop and sweep on non-cubic meshes (the brick walk of the
    cotangent paint where ny % 8 == 0 and nz % 32 == 0, the grid-stride walk otherwise) and
    with two particle sets at once, against the recomputing sweep."""
    from jfli_b200 import ops

    rng = np.random.default_rng(sum(shape) + batch)
    lead = (batch,) if batch > 1 else ()
    x0 = _dev(0.7 * rng.standard_normal(lead + shape + (3,)))
    v0 = _dev(0.2 * rng.standard_normal(lead + shape + (3,)))
    a, b = _dev(rng.standard_normal(lead + shape + (3,))), _dev(rng.standard_normal(lead + shape + (3,)))
    kicks, drifts = np.linspace(0.2, 0.3, 5), np.linspace(0.4, 0.3, 5)
    out = {}
    for mode in ("recompute", "stored"):
        x, v = x0.clone(), v0.clone()
        rho = torch.empty(lead + shape, device="cuda")
        pots = torch.empty((len(kicks),) + lead + shape, device="cuda") if mode == "stored" else None
        ops.kkd_run(x, v, kicks, drifts, rho, pots=pots)
        fwd = rho.clone()
        lx, lv = a.clone(), b.clone()
        sens = ops.kkd_adjoint(x, v, lx, lv, kicks, drifts, pots=pots)
        out[mode] = (fwd, lx, lv, sens, x)
    (r0, lx0, lv0, s0, xr0), (r1, lx1, lv1, s1, xr1) = out["recompute"], out["stored"]
    e_rho = float((r1 - r0).norm() / r0.norm())
    e_lx = float((lx1 - lx0).norm() / lx0.norm())
    e_s = float((s1 - s0).abs().max() / s0.abs().max())
    e_x = float((xr1 - x0).abs().max())
    print(f"{shape} x{batch}: density {e_rho:.2e}, lam_x {e_lx:.2e}, sensitivities {e_s:.2e}, initial state {e_x:.2e}")
    assert e_rho < 1e-5 and e_lx < 1e-3 and e_s < 1e-3 and e_x < 1e-4


def test_kkd_step_vjp_stored_matches_oracle_fd():
    from jfli_b200 import ops

    n = 32
    rng = np.random.default_rng(1)
    x0 = (1.5 * rng.standard_normal((n, n, n, 3))).astype(np.float32)
    v0 = (0.5 * rng.standard_normal((n, n, n, 3))).astype(np.float32)
    kicks, drifts = np.array([0.3, 0.25, 0.35]), np.array([0.4, 0.5, 0.3])
    a = rng.standard_normal(x0.shape)
    b = rng.standard_normal(x0.shape)
    r = rng.standard_normal(x0.shape)
    s = rng.standard_normal(x0.shape)
    x, v = _dev(x0), _dev(v0)
    rho = torch.empty(n, n, n, device="cuda")
    pots = torch.empty(len(kicks), n, n, n, device="cuda")
    ops.kkd_run(x, v, kicks, drifts, rho, pots=pots)
    lam_x, lam_v = _dev(a), _dev(b)
    sens = ops.kkd_adjoint(x, v, lam_x, lam_v, kicks, drifts, pots=pots).cpu().numpy()
    g_dir = float(np.sum(lam_x.cpu().numpy() * r) + np.sum(lam_v.cpu().numpy() * s))

    def loss(xi, vi, ks=kicks, ds=drifts):
        xf, vf, _ = opm.kkd_run(xi, vi, list(zip(ks, ds)), np.float64)
        return float(np.sum(a * xf) + np.sum(b * vf))

    eps = 1e-5
    x64, v64 = x0.astype(np.float64), v0.astype(np.float64)
    fd = (loss(x64 + eps * r, v64 + eps * s) - loss(x64 - eps * r, v64 - eps * s)) / (2 * eps)
    print(f"direction (stored potentials): adjoint {g_dir:.8e} fd {fd:.8e}")
    assert _rel(g_dir, fd) < 1e-4
    for i in range(len(kicks)):
        kp, km = kicks.copy(), kicks.copy()
        kp[i] += eps
        km[i] -= eps
        fdk = (loss(x64, v64, ks=kp) - loss(x64, v64, ks=km)) / (2 * eps)
        assert _rel(sens[i, 0], fdk) < 1e-4


# --------------------------------------------------------------------------- P(k), LPT, ICs
def test_power_adjoint_matches_oracle_fd():
    from jfli_b200.pm import adjoint as adj

    n, box = 32, 128.0
    rng = np.random.default_rng(3)
    m0 = (1.0 + 0.3 * rng.standard_normal((n, n, n))).astype(np.float32)
    ke = _kedges(n, box)
    g = rng.standard_normal(len(ke) - 1)
    r = rng.standard_normal(m0.shape)
    mesh = _dev(m0).requires_grad_(True)
    pk = adj.PowerSpectrum.apply(mesh, ke, (box,) * 3)
    (pk * torch.as_tensor(g, device="cuda")).sum().backward()
    g_dir = float(np.sum(mesh.grad.cpu().numpy() * r))

    def loss(m):
        return float(np.sum(g * opm.power(m, (box,) * 3, ke, kdtype=np.float32)[1]))

    eps = 1e-3
    fd = (loss(m0.astype(np.float64) + eps * r) - loss(m0.astype(np.float64) - eps * r)) / (2 * eps)
    print(f"P(k) adjoint {g_dir:.8e} fd {fd:.8e}")
    assert _rel(g_dir, fd) < 1e-4


@pytest.mark.parametrize("order", [1, 2])
def test_lpt_adjoint_matches_oracle_fd(order):
    from jfli_b200.pm import adjoint as adj

    n = 32
    rng = np.random.default_rng(4 + order)
    ic0 = (0.5 * rng.standard_normal((n, n, n))).astype(np.float32)
    coeffs = (1.3, -0.4, 2.1, 3.5)
    tables = adj.ForwardTables(ktab=None, ptab=None, lpt=coeffs, kicks=None, drifts=None)
    a = rng.standard_normal((n, n, n, 3))
    b = rng.standard_normal((n, n, n, 3))
    r = rng.standard_normal(ic0.shape)
    ic = _dev(ic0).requires_grad_(True)
    dx, p = adj.LPT.apply(ic, None, order, tables)
    (torch.sum(dx * _dev(a)) + torch.sum(p * _dev(b))).backward()
    g_dir = float(np.sum(ic.grad.cpu().numpy() * r))

    def loss(f):
        dxo, po = opm.lpt(f, *coeffs, order=order, dtype=np.float64)
        return float(np.sum(a * dxo) + np.sum(b * po))

    eps = 1e-3
    f64 = ic0.astype(np.float64)
    fd = (loss(f64 + eps * r) - loss(f64 - eps * r)) / (2 * eps)
    print(f"LPT{order} adjoint {g_dir:.8e} fd {fd:.8e}")
    assert _rel(g_dir, fd) < 1e-4


def test_ic_filter_gradients_match_oracle_fd():
    from jfli_b200.pm import adjoint as adj

    n, box = 32, 128.0
    rng = np.random.default_rng(7)
    w0 = rng.standard_normal((n, n, n)).astype(np.float32)
    a = rng.standard_normal((n, n, n))
    r = rng.standard_normal((n, n, n))
    oc, s8 = 0.27, 0.79
    tab = adj.forward_tables(oc, s8, t0=0.1, t1=1.0, dt0=0.45)
    w = _dev(w0).requires_grad_(True)
    om = torch.tensor(oc, dtype=torch.float64, requires_grad=True)
    sg = torch.tensor(s8, dtype=torch.float64, requires_grad=True)
    delta = adj.ICFilter.apply(w, om, sg, tab, (box,) * 3)
    torch.sum(delta * _dev(a)).backward()

    def loss(wi, oci=oc, s8i=s8):
        t = adj.forward_tables(oci, s8i, t0=0.1, t1=1.0, dt0=0.45, derivatives=False)
        return float(np.sum(a * opm.ic_filter(wi, (box,) * 3, t.ktab, t.ptab, dtype=np.float64)))

    w64 = w0.astype(np.float64)
    fd_w = (loss(w64 + r) - loss(w64 - r)) / 2.0  # linear in w
    g_w = float(np.sum(w.grad.cpu().numpy() * r))
    h = 1e-4
    fd_s8 = (loss(w64, s8i=s8 + h) - loss(w64, s8i=s8 - h)) / (2 * h)
    fd_oc = (loss(w64, oci=oc + h) - loss(w64, oci=oc - h)) / (2 * h)
    print(f"noise {g_w:.6e} vs {fd_w:.6e}; sigma8 {float(sg.grad):.6e} vs {fd_s8:.6e}; "
          f"Omega_c {float(om.grad):.6e} vs {fd_oc:.6e}")
    assert _rel(g_w, fd_w) < 1e-4
    assert _rel(float(sg.grad), fd_s8) < 1e-4
    assert _rel(float(om.grad), fd_oc) < 1e-3


# --------------------------------------------------------------------------- whole chain
def _oracle_loss(w, oc, s8, *, n, box, t0, dt0, order, kedges, pk_target):
    from jfli_b200.pm import adjoint as adj

    t = adj.forward_tables(oc, s8, t0=t0, t1=1.0, dt0=dt0, derivatives=False)
    ic = opm.ic_filter(w, (box,) * 3, t.ktab, t.ptab, dtype=np.float64)
    dx, p = opm.lpt(ic, *t.lpt, order=order, dtype=np.float64)
    x, _, _ = opm.kkd_run(dx, p, list(zip(t.kicks, t.drifts)), np.float64)
    pk = opm.power(opm.cic_paint(x), (box,) * 3, kedges, kdtype=np.float32)[1]
    m = (pk_target > 0) & (pk > 0)
    return float(np.sum((np.log(pk[m]) - np.log(pk_target[m])) ** 2))


def test_full_chain_gradient_matches_oracle_fd():
    from jfli_b200.pm import adjoint as adj

    n, box, t0, dt0, order = 32, 128.0, 0.1, 0.225, 2
    ke = _kedges(n, box)
    rng = np.random.default_rng(8)
    w0 = rng.standard_normal((n, n, n)).astype(np.float32)
    wt = np.random.default_rng(9).standard_normal((n, n, n)).astype(np.float32)
    oc, s8 = 0.2607, 0.8102
    with torch.no_grad():
        pk_t = adj.forward_model_pk(_dev(wt), torch.tensor(oc), torch.tensor(s8), box=(box,) * 3, kedges=ke, t0=t0,
                                    dt0=dt0, lpt_order=order)
    w = _dev(w0).requires_grad_(True)
    om = torch.tensor(oc, dtype=torch.float64, requires_grad=True)
    sg = torch.tensor(s8, dtype=torch.float64, requires_grad=True)
    pk = adj.forward_model_pk(w, om, sg, box=(box,) * 3, kedges=ke, t0=t0, dt0=dt0, lpt_order=order)
    loss = adj.pk_log_loss(pk, pk_t)
    loss.backward()
    r = rng.standard_normal((n, n, n))
    g_w = float(np.sum(w.grad.cpu().numpy() * r))
    kw = dict(n=n, box=box, t0=t0, dt0=dt0, order=order, kedges=ke, pk_target=pk_t.cpu().numpy())
    w64 = w0.astype(np.float64)
    L0 = _oracle_loss(w64, oc, s8, **kw)
    e = 1e-4
    fd_w = (_oracle_loss(w64 + e * r, oc, s8, **kw) - _oracle_loss(w64 - e * r, oc, s8, **kw)) / (2 * e)
    fd_oc = (_oracle_loss(w64, oc + e, s8, **kw) - _oracle_loss(w64, oc - e, s8, **kw)) / (2 * e)
    fd_s8 = (_oracle_loss(w64, oc, s8 + e, **kw) - _oracle_loss(w64, oc, s8 - e, **kw)) / (2 * e)
    print(f"loss GPU {float(loss):.8e} oracle {L0:.8e}")
    print(f"noise {g_w:.6e} vs {fd_w:.6e}; Omega_c {float(om.grad):.6e} vs {fd_oc:.6e}; "
          f"sigma8 {float(sg.grad):.6e} vs {fd_s8:.6e}")
    assert _rel(float(loss), L0) < 1e-3
    assert _rel(g_w, fd_w) < 2e-3
    assert _rel(float(om.grad), fd_oc) < 2e-3
    assert _rel(float(sg.grad), fd_s8) < 2e-3


def test_differentiation_config_128_matches_gpu_fd():
    """128^3, box 500, 20 KKD steps from a = 0.1, 2LPT, 32-bin log-P loss against a
    second seed; gradients (sixteen random white-noise directions, Omega_c, sigma8) vs central
    differences (eps = 1e-3) of the GPU forward."""
    import time

    from jfli_b200.pm import adjoint as adj

    n, box, t0, order = 128, 500.0, 0.1, 2
    dt0 = 0.9 / 20
    ke = _kedges(n, box)
    rng = np.random.default_rng(10)
    w0 = _dev(rng.standard_normal((n, n, n)))
    wt = _dev(np.random.default_rng(11).standard_normal((n, n, n)))
    oc, s8 = 0.2607, 0.8102
    kw = dict(box=(box,) * 3, kedges=ke, t0=t0, dt0=dt0, lpt_order=order)

    def loss_at(w, o, s):
        with torch.no_grad():
            return float(adj.pk_log_loss(adj.forward_model_pk(w, torch.tensor(o), torch.tensor(s), **kw), pk_t))

    with torch.no_grad():
        pk_t = adj.forward_model_pk(wt, torch.tensor(oc), torch.tensor(s8), **kw)
    for it in range(2):  # second iteration timed (tables and workspaces warm)
        w = w0.clone().requires_grad_(True)
        om = torch.tensor(oc, dtype=torch.float64, requires_grad=True)
        sg = torch.tensor(s8, dtype=torch.float64, requires_grad=True)
        torch.cuda.synchronize()
        t_start = time.perf_counter()
        loss = adj.pk_log_loss(adj.forward_model_pk(w, om, sg, **kw), pk_t)
        loss.backward()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t_start
    e = 1e-3
    gen = torch.Generator(device="cuda").manual_seed(12)
    pairs = []
    for _ in range(16):  # sixteen random white-noise directions
        r = torch.randn(n, n, n, device="cuda", generator=gen)
        g_w = float(torch.sum(w.grad.double() * r.double()))
        fd_w = (loss_at(w0 + e * r, oc, s8) - loss_at(w0 - e * r, oc, s8)) / (2 * e)
        pairs.append((g_w, fd_w))
    fd_oc = (loss_at(w0, oc + e, s8) - loss_at(w0, oc - e, s8)) / (2 * e)
    fd_s8 = (loss_at(w0, oc, s8 + e) - loss_at(w0, oc, s8 - e)) / (2 * e)
    print(f"128^3 gradient iteration {wall * 1e3:.1f} ms; loss {float(loss):.6e}")
    # a direction r ~ N(0, I) gives g.r ~ N(0, |g|^2): the noise-direction error is stated
    # against |g|, the spread of directional derivatives, so that a direction whose derivative
    # happens to be near zero is not judged by the FP32 difference noise alone
    gnorm = float(w.grad.double().norm())
    errs = [abs(g_w - fd_w) / gnorm for g_w, fd_w in pairs]
    print("noise directions " + "; ".join(f"{g:.6e} vs {f:.6e}" for g, f in pairs) + f"; |g| {gnorm:.4e}")
    print("noise-direction errors / |g| " + ", ".join(f"{e:.2e}" for e in errs))
    print(f"Omega_c {float(om.grad):.6e} vs {fd_oc:.6e}; sigma8 {float(sg.grad):.6e} vs {fd_s8:.6e}")
    for e in errs:
        assert e < 1e-2
    assert _rel(float(om.grad), fd_oc) < 1e-2
    assert _rel(float(sg.grad), fd_s8) < 1e-2


def test_edk_density_gradient_matches_oracle_fd():
    """nbody with EfficientDriftDoubleKick (the reference's default solver, adjoint
    "checkpointed") on displacements and momenta that require grad: the density equals the
    fused loop's, and the directional derivative of <a, rho(final)> with respect to
    (dx, p) matches central differences of the FP64 oracle's FastPM loop (oracle/pm.py
    kdk_run) driven by the same host coefficients."""
    import jfli_b200 as jf
    from jfli_b200.pm.integrate import time_events
    from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK

    n, box, t0, t1, dt0 = 32, 128.0, 0.1, 1.0, 0.15
    cosmo = jf.Planck18()
    ic = jf.interpolate_initial_conditions(jf.white_noise(21, (n,) * 3), (n,) * 3, (box,) * 3, cosmo=cosmo)
    dx, p = jf.lpt(cosmo, ic, ts=t0, order=2)
    x0, v0 = dx.array.detach().contiguous().clone(), p.array.detach().contiguous().clone()
    rng = np.random.default_rng(22)
    a = rng.standard_normal((n, n, n))
    r = rng.standard_normal((n, n, n, 3))
    s = rng.standard_normal((n, n, n, 3))
    solver = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="density")))
    xg, vg = x0.clone().requires_grad_(True), v0.clone().requires_grad_(True)
    rho = jf.nbody(cosmo, dx.replace(array=xg), p.replace(array=vg), t0=t0, t1=t1, dt0=dt0, solver=solver)
    loss = (rho.array.double() * torch.as_tensor(a, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(xg.grad.cpu().numpy() * r) + np.sum(vg.grad.cpu().numpy() * s))
    with torch.no_grad():
        rho_f = jf.nbody(cosmo, dx.replace(array=x0), p.replace(array=v0), t0=t0, t1=t1, dt0=dt0, solver=solver)
    e_fwd = float((rho.array.detach() - rho_f.array).norm() / rho_f.array.norm())

    steps = [(e[1], e[2]) for e in time_events(t0, [t1], dt0) if e[0] == "step"]
    kicks, drifts = EDK.schedule_arrays(cosmo, [q for q, _ in steps], [q for _, q in steps], dt0)
    coeffs = dict(init_kick=EDK.init_kick(cosmo, t0, t0 + dt0), steps=list(zip(kicks, drifts)))

    def oracle_loss(x, v):
        xf, _, _ = opm.kdk_run(x, v, coeffs, np.float64)
        return float(np.sum(a * opm.cic_paint(xf)))

    x64, v64 = x0.cpu().numpy().astype(np.float64), v0.cpu().numpy().astype(np.float64)
    eps = 1e-5
    fd = (oracle_loss(x64 + eps * r, v64 + eps * s) - oracle_loss(x64 - eps * r, v64 - eps * s)) / (2 * eps)
    L0 = oracle_loss(x64, v64)
    print(f"EDK: density vs the fused loop {e_fwd:.2e}; loss GPU {float(loss):.8e} oracle {L0:.8e}; "
          f"directional derivative {g_dir:.6e} vs oracle central difference {fd:.6e}")
    assert e_fwd < 1e-5
    assert _rel(float(loss), L0) < 1e-4
    assert _rel(g_dir, fd) < 1e-3


def test_pgd_adjoint_matches_oracle_fd():
    """PGDKernel.apply on displacements that require grad: the directional derivative of
    <a, x' - x> (the correction alone: the identity part of x' is exact and would cancel
    most of the signal) through jfli_pgd_adjoint against central differences of the FP64
    oracle's PGD correction (oracle/pm.py pgd_correction, reference pm/correction.py:157-202)."""
    import jfli_b200 as jf
    from jfli_b200.fields import ParticleField, PositionUnit

    n = 32
    rng = np.random.default_rng(31)
    disp, _ = opm.lpt(rng.normal(size=(n, n, n)), 2.0, 0.0, 1.0, 0.0)
    disp = disp.astype(np.float32)
    a = rng.standard_normal((n, n, n, 3))
    r = rng.standard_normal((n, n, n, 3))
    results = []
    for alpha, kl, ks in ((0.3, 0.3, 1.0), (0.3, 1.5 * 128.0 / n / 100.0, 8.0 * 128.0 / n)):
        x = _dev(disp).requires_grad_(True)
        pos = ParticleField(array=x, mesh_size=(n,) * 3, box_size=(128.0,) * 3, unit=PositionUnit.GRID_RELATIVE)
        out, _ = jf.PGDKernel(alpha=alpha, kl=kl, ks=ks).apply(0.5, pos, pos, 0.0)
        loss = ((out.array - x).double() * torch.as_tensor(a, device="cuda")).sum()
        loss.backward()
        g_dir = float(np.sum(x.grad.cpu().numpy().astype(np.float64) * r))
        d64 = disp.astype(np.float64)

        def oracle_loss(d):
            return float(np.sum(a * (opm.pgd_correction(d, alpha, kl, ks) - d)))

        # the correction has kinks wherever a particle or a CIC corner crosses a cell face;
        # at steps of 1e-5 cells some of the 98k particles cross one (the difference moves by
        # 2e-4), at 1e-6 none does
        fd, fd_coarse = [(oracle_loss(d64 + e * r) - oracle_loss(d64 - e * r)) / (2 * e) for e in (1e-6, 1e-4)]
        print(f"PGD alpha={alpha} kl={kl:.3g} ks={ks:.3g}: directional derivative {g_dir:.8e} vs oracle central "
              f"difference {fd:.8e} (step 1e-4: {fd_coarse:.8e})")
        results.append(_rel(g_dir, fd))
    assert max(results) < 1e-4, results


def test_public_api_gradient_equals_forward_model():
    """interpolate_initial_conditions -> lpt -> nbody(ReversibleDoubleKickDrift) -> power
    through the public API with a noise field that requires grad gives the same gradient
    as forward_model_pk."""
    import jfli_b200 as jf
    from jfli_b200.pm import adjoint as adj

    n, box, t0, dt0 = 32, 128.0, 0.1, 0.225
    ke = _kedges(n, box)
    rng = np.random.default_rng(13)
    w0 = _dev(rng.standard_normal((n, n, n)))
    with torch.no_grad():
        pk_t = adj.forward_model_pk(_dev(rng.standard_normal((n, n, n))), torch.tensor(0.2607),
                                    torch.tensor(0.8102), box=(box,) * 3, kedges=ke, t0=t0, dt0=dt0)
    cosmo = jf.Planck18()
    noise = w0.clone().requires_grad_(True)
    ic = jf.interpolate_initial_conditions(noise, (n,) * 3, (box,) * 3, cosmo=cosmo)
    dx, p = jf.lpt(cosmo, ic, ts=t0, order=2)
    solver = jf.ReversibleDoubleKickDrift(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="density")))
    rho = jf.nbody(cosmo, dx, p, t0=t0, t1=1.0, dt0=dt0, solver=solver)
    _, pk = jf.power(rho.array, box_shape=(box,) * 3, kedges=ke)
    loss = adj.pk_log_loss(pk, pk_t)
    loss.backward()

    w2 = w0.clone().requires_grad_(True)
    loss2 = adj.pk_log_loss(adj.forward_model_pk(w2, torch.tensor(0.2607), torch.tensor(0.8102), box=(box,) * 3,
                                                 kedges=ke, t0=t0, dt0=dt0), pk_t)
    loss2.backward()
    assert abs(float(loss) - float(loss2)) <= 1e-6 * abs(float(loss2))
    err = float(torch.linalg.norm(noise.grad - w2.grad) / torch.linalg.norm(w2.grad))
    print(f"public API vs forward_model_pk gradient rel L2 {err:.2e}")
    assert err < 1e-5


@pytest.mark.parametrize("solver_name", ["kkd", "edk"])
def test_density_snapshots_gradient_matches_oracle_fd(solver_name):
    """nbody painting density snapshots at a = 0.4, 0.7 and 1 with weight 2 (the reference
    differentiates any snapshot list, pm/integrate.py:109-145) on displacements and momenta
    that require grad: the snapshots equal the fused loop's, and the directional derivative
    of sum_j <a_j, rho_j> matches central differences of the FP64 oracle loop painting at
    the same (clipped) snapshot times.

    The painted densities are piecewise linear in the positions, with kinks where a
    particle crosses a cell face. With this seed a step of 1e-5 cells crosses enough of them
    that the oracle's central difference for the final snapshot is 1% below the slope
    (1286.3 against 1301.7, 1300.9 and 1298.9 at steps 3e-6, 1e-6 and 3e-7, measured with
    the oracle alone); the test takes steps of 3e-7, and the bound is 2e-3."""
    import jfli_b200 as jf
    from jfli_b200.pm.integrate import time_events
    from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK
    from jfli_b200.pm.solvers import ReversibleDoubleKickDrift as KKD

    n, box, t0, dt0, w = 32, 128.0, 0.1, 0.15, 2.0
    ts = [0.4, 0.7, 1.0]
    cosmo = jf.Planck18()
    ic = jf.interpolate_initial_conditions(jf.white_noise(23, (n,) * 3), (n,) * 3, (box,) * 3, cosmo=cosmo)
    dx, p = jf.lpt(cosmo, ic, ts=t0, order=2)
    x0, v0 = dx.array.detach().contiguous().clone(), p.array.detach().contiguous().clone()
    rng = np.random.default_rng(24)
    a = rng.standard_normal((len(ts), n, n, n))
    r = rng.standard_normal((n, n, n, 3))
    s = rng.standard_normal((n, n, n, 3))
    interp = jf.NoInterp(painting=jf.PaintingOptions(target="density", weights=w))
    solver = (jf.ReversibleDoubleKickDrift(interp_kernel=interp) if solver_name == "kkd"
              else jf.EfficientDriftDoubleKick(interp_kernel=interp))
    kw = dict(t0=t0, t1=1.0, dt0=dt0, ts=np.asarray(ts), solver=solver)
    xg, vg = x0.clone().requires_grad_(True), v0.clone().requires_grad_(True)
    rho = jf.nbody(cosmo, dx.replace(array=xg), p.replace(array=vg), **kw)
    loss = (rho.array.double() * torch.as_tensor(a, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(xg.grad.cpu().numpy() * r) + np.sum(vg.grad.cpu().numpy() * s))
    with torch.no_grad():
        rho_f = jf.nbody(cosmo, dx.replace(array=x0), p.replace(array=v0), **kw)
    e_fwd = float((rho.array.detach() - rho_f.array).norm() / rho_f.array.norm())

    ts_run = np.asarray(rho.scale_factors, np.float64)[::-1]  # ascending, as the loop meets them
    events = time_events(t0, ts_run, dt0)
    steps = [(e[1], e[2]) for e in events if e[0] == "step"]
    after, count = set(), 0
    for ev in events:
        if ev[0] == "step":
            count += 1
        else:
            after.add(count - 1)
    if solver_name == "kkd":
        cs = [KKD.step_coefficients(cosmo, q, u, dt0, t0) for q, u in steps]

        def oracle_snaps(x, v):
            return opm.kkd_run(x, v, [(c.kick, c.drift) for c in cs], np.float64, snapshot_after=after)[2]
    else:
        kicks, drifts = EDK.schedule_arrays(cosmo, [q for q, _ in steps], [q for _, q in steps], dt0)
        coeffs = dict(init_kick=EDK.init_kick(cosmo, t0, t0 + dt0), steps=list(zip(kicks, drifts)))

        def oracle_snaps(x, v):
            return opm.kdk_run(x, v, coeffs, np.float64, snapshot_after=after)[2]

    def oracle_loss(x, v):
        snaps = np.stack(oracle_snaps(x, v)[::-1]) * w  # latest first, as nbody returns them
        return float(np.sum(a * snaps))

    x64, v64 = x0.cpu().numpy().astype(np.float64), v0.cpu().numpy().astype(np.float64)
    eps = 3e-7
    fd = (oracle_loss(x64 + eps * r, v64 + eps * s) - oracle_loss(x64 - eps * r, v64 - eps * s)) / (2 * eps)
    L0 = oracle_loss(x64, v64)
    print(f"{solver_name} density snapshots {len(ts)}: vs the fused loop {e_fwd:.2e}; loss GPU "
          f"{float(loss.detach()):.8e} oracle {L0:.8e}; directional derivative {g_dir:.6e} vs oracle central "
          f"difference {fd:.6e}")
    assert tuple(rho.array.shape) == (len(ts), n, n, n)
    assert e_fwd < 1e-5
    assert _rel(float(loss.detach()), L0) < 1e-4
    assert _rel(g_dir, fd) < 2e-3


def test_cross_power_gradient_matches_oracle_fd():
    """power(mesh, mesh2) with both meshes requiring grad: the cross spectrum equals the
    FP64 oracle's (oracle/pm.py power_poles, the reference's _power with mesh2), and the
    directional derivative of sum_b c_b P_b matches central differences of the oracle (the
    spectrum is quadratic in the meshes, so steps of 1e-3 are exact up to rounding)."""
    import jfli_b200 as jf

    n, box = 32, (100.0, 100.0, 100.0)
    rng = np.random.default_rng(31)
    m1 = rng.standard_normal((n, n, n))
    m2 = 0.6 * m1 + 0.8 * rng.standard_normal((n, n, n))  # correlated: no bin sum near zero
    r1, r2 = rng.standard_normal((n, n, n)), rng.standard_normal((n, n, n))
    kedges = np.linspace(0.05, 1.5, 12)
    t1 = torch.as_tensor(m1, dtype=torch.float32, device="cuda").requires_grad_(True)
    t2 = torch.as_tensor(m2, dtype=torch.float32, device="cuda").requires_grad_(True)
    _, pk = jf.power(t1, t2, box_shape=box, kedges=kedges)
    c = rng.standard_normal(pk.shape[-1])
    loss = (pk * torch.as_tensor(c, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(t1.grad.cpu().numpy() * r1) + np.sum(t2.grad.cpu().numpy() * r2))
    _, ref = opm.power_poles(m1, m2, box, kedges)
    ref = np.asarray(ref).reshape(-1)
    err = float(np.abs(pk.detach().cpu().numpy() - ref).max() / np.abs(ref).max())

    def oracle_loss(a, b):
        return float(np.sum(c * np.asarray(opm.power_poles(a, b, box, kedges)[1]).reshape(-1)))

    eps = 1e-3
    fd = (oracle_loss(m1 + eps * r1, m2 + eps * r2) - oracle_loss(m1 - eps * r1, m2 - eps * r2)) / (2 * eps)
    print(f"cross P(k): vs the oracle {err:.2e}; directional derivative {g_dir:.8e} vs oracle central difference "
          f"{fd:.8e}")
    assert err < 1e-5
    assert _rel(g_dir, fd) < 1e-4


def test_power_multipoles_gradient_matches_oracle_fd():
    """power(mesh, multipoles=(0, 1, 2, 4), los) with the mesh requiring grad: the
    multipoles equal the FP64 oracle's (oracle/pm.py power_poles), and the directional
    derivative of sum c_l,b P_l,b matches central differences of the oracle (the multipoles
    are quadratic in the mesh; the odd one cancels between k and -k except on the grid's
    Nyquist planes, which the adjoint's partner-averaged weight carries)."""
    import jfli_b200 as jf

    n, box = 32, (100.0, 120.0, 90.0)
    poles, los = (0, 1, 2, 4), (0.3, -0.2, 0.9)
    rng = np.random.default_rng(33)
    m = rng.standard_normal((n, n, n))
    r = rng.standard_normal((n, n, n))
    kedges = np.linspace(0.05, 1.5, 12)
    t = torch.as_tensor(m, dtype=torch.float32, device="cuda").requires_grad_(True)
    _, pk = jf.power(t, box_shape=box, kedges=kedges, multipoles=poles, los=los)
    c = rng.standard_normal(tuple(pk.shape))
    loss = (pk * torch.as_tensor(c, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(t.grad.cpu().numpy() * r))
    ref = np.asarray(opm.power_poles(m, None, box, kedges, multipoles=poles, los=los)[1]).reshape(pk.shape)
    err = float(np.abs(pk.detach().cpu().numpy() - ref).max() / np.abs(ref).max())

    def oracle_loss(a):
        return float(np.sum(c * np.asarray(opm.power_poles(a, None, box, kedges, multipoles=poles,
                                                           los=los)[1]).reshape(c.shape)))

    eps = 1e-3
    fd = (oracle_loss(m + eps * r) - oracle_loss(m - eps * r)) / (2 * eps)
    print(f"multipoles {poles}: vs the oracle {err:.2e}; directional derivative {g_dir:.8e} vs oracle central "
          f"difference {fd:.8e}")
    assert tuple(pk.shape) == (len(poles), len(kedges) - 1)
    assert err < 1e-5
    assert _rel(g_dir, fd) < 1e-4


def test_cross_multipoles_gradient_matches_oracle_fd():
    """power(mesh, mesh2, multipoles=(0, 1, 2, 3), los) with both meshes requiring grad: the
    cross multipoles equal the FP64 oracle's, and the directional derivative of
    sum c_l,b P_l,b matches central differences of the oracle (the odd cross multipoles are
    moduli of imaginary sums, whose adjoint takes the imaginary part of the per-bin phase)."""
    import jfli_b200 as jf

    n, box = 32, (100.0, 120.0, 90.0)
    poles, los = (0, 1, 2, 3), (0.3, -0.2, 0.9)
    rng = np.random.default_rng(35)
    m1 = rng.standard_normal((n, n, n))
    m2 = 0.5 * m1 + rng.standard_normal((n, n, n))
    r1, r2 = rng.standard_normal((n, n, n)), rng.standard_normal((n, n, n))
    kedges = np.linspace(0.05, 1.5, 12)
    t1 = torch.as_tensor(m1, dtype=torch.float32, device="cuda").requires_grad_(True)
    t2 = torch.as_tensor(m2, dtype=torch.float32, device="cuda").requires_grad_(True)
    _, pk = jf.power(t1, t2, box_shape=box, kedges=kedges, multipoles=poles, los=los)
    c = rng.standard_normal(tuple(pk.shape))
    loss = (pk * torch.as_tensor(c, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(t1.grad.cpu().numpy() * r1) + np.sum(t2.grad.cpu().numpy() * r2))
    ref = np.asarray(opm.power_poles(m1, m2, box, kedges, multipoles=poles, los=los)[1]).reshape(pk.shape)
    err = float(np.abs(pk.detach().cpu().numpy() - ref).max() / np.abs(ref).max())

    def oracle_loss(a, b):
        return float(np.sum(c * np.asarray(opm.power_poles(a, b, box, kedges, multipoles=poles,
                                                           los=los)[1]).reshape(c.shape)))

    eps = 1e-3
    fd = (oracle_loss(m1 + eps * r1, m2 + eps * r2) - oracle_loss(m1 - eps * r1, m2 - eps * r2)) / (2 * eps)
    print(f"cross multipoles {poles}: vs the oracle {err:.2e}; directional derivative {g_dir:.8e} vs oracle "
          f"central difference {fd:.8e}")
    assert err < 1e-5
    assert _rel(g_dir, fd) < 1e-4


def test_cic_readout_gradient_matches_oracle_fd():
    """ParticleField.read_out with positions and mesh that require grad (painting.CICReadout):
    the values equal the FP64 oracle's CIC readout, and the directional derivative of
    <a, read_out> in (positions, mesh) matches central differences of the oracle (linear in
    the mesh; steps of 1e-6 cells keep the particles inside their cells)."""
    from jfli_b200.fields import ParticleField, PositionUnit

    n = 32
    rng = np.random.default_rng(51)
    x = 0.7 * rng.standard_normal((n, n, n, 3))
    m = rng.standard_normal((n, n, n))
    a, r, q = rng.standard_normal((n, n, n)), rng.standard_normal((n, n, n, 3)), rng.standard_normal((n, n, n))
    xt = torch.as_tensor(x, dtype=torch.float32, device="cuda").requires_grad_(True)
    mt = torch.as_tensor(m, dtype=torch.float32, device="cuda").requires_grad_(True)
    f = ParticleField(array=xt, mesh_size=(n,) * 3, box_size=(128.0,) * 3, unit=PositionUnit.GRID_RELATIVE)
    vals = f.read_out(mt)
    loss = (vals.array.double() * torch.as_tensor(a, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(xt.grad.cpu().numpy() * r) + np.sum(mt.grad.cpu().numpy() * q))
    x32 = xt.detach().cpu().numpy().astype(np.float64)
    ref = opm.cic_read(m, x32)
    err = float(np.abs(vals.array.detach().cpu().numpy() - ref).max() / np.abs(ref).max())

    def oracle_loss(xx, mm):
        return float(np.sum(a * opm.cic_read(mm, xx)))

    eps = 1e-6
    fd = (oracle_loss(x32 + eps * r, m + eps * q) - oracle_loss(x32 - eps * r, m - eps * q)) / (2 * eps)
    print(f"CIC readout: vs the oracle {err:.2e}; directional derivative {g_dir:.8e} vs oracle central difference "
          f"{fd:.8e}")
    assert err < 1e-5
    assert _rel(g_dir, fd) < 1e-3


def test_flat_plane_gradient_matches_oracle_fd():
    """paint_2d of displacements that require grad (painting.PaintFlat, backward
    jfli_paint_flat_adjoint): two planes, the directional derivative of sum <a_j, plane_j>
    matches central differences of the FP64 oracle's flat painter (oracle/flat.py) with the
    same pixel-volume normalisation (steps of 1e-6 cells keep particles in their pixels and
    slabs)."""
    from jfli_b200.fields import ParticleField, PositionUnit
    from oracle import flat as ofl

    n, L, npix = 32, 128.0, (48, 40)
    rng = np.random.default_rng(61)
    x = 0.8 * rng.standard_normal((n, n, n, 3))
    centers, widths = np.array([40.0, 90.0]), np.array([30.0, 40.0])
    a = rng.standard_normal((2,) + npix)
    r = rng.standard_normal((n, n, n, 3))
    xt = torch.as_tensor(x, dtype=torch.float32, device="cuda").requires_grad_(True)
    f = ParticleField(array=xt, mesh_size=(n,) * 3, box_size=(L,) * 3, flatsky_npix=npix,
                      unit=PositionUnit.GRID_RELATIVE)
    planes = f.paint_2d(centers, widths)
    loss = (planes.array.double() * torch.as_tensor(a, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(xt.grad.cpu().numpy() * r))
    x32 = xt.detach().cpu().numpy().astype(np.float64)
    grid = np.stack(np.meshgrid(*[np.arange(n, dtype=np.float64)] * 3, indexing="ij"), axis=-1)

    def oracle_planes(xx):
        out = []
        for c, w in zip(centers, widths):
            cg, wg = c * n / L, w * n / L
            vol = (L / npix[0]) * (L / npix[1]) * w
            out.append(ofl.paint_2d(grid + xx, npix, cg - wg / 2, cg + wg / 2, (n, n, n)) / vol)
        return np.stack(out)

    err = float(np.abs(planes.array.detach().cpu().numpy() - oracle_planes(x32)).max() /
                np.abs(oracle_planes(x32)).max())
    eps = 1e-6
    fd = (np.sum(a * oracle_planes(x32 + eps * r)) - np.sum(a * oracle_planes(x32 - eps * r))) / (2 * eps)
    print(f"flat planes: vs the oracle {err:.2e}; directional derivative {g_dir:.8e} vs oracle central difference "
          f"{fd:.8e}")
    assert err < 1e-5
    assert _rel(g_dir, fd) < 1e-3
