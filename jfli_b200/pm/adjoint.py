"""Reverse-mode gradients of the forward model with the reversible adjoint.

The reference differentiates `lpt -> nbody -> power` with jax.grad; with
`adjoint="reverse"` its N-body part is a custom VJP (pm/integrate.py:147-535) whose
backward loop steps the ReversibleDoubleKickDrift solver backwards (solver.reverse,
pm/solvers.py:327-411) and pulls the cotangents through the VJP of each step, so the
trajectory is recomputed instead of stored.

Here every stage is a torch.autograd.Function whose backward runs the B200 adjoint
kernels, so `torch.autograd.grad(loss, [noise, omega_c, sigma8])` plays the role of
jax.grad:

* `ICFilter`    white noise -> linear density (initial.py:167-182). The filter is a real
                even Fourier multiplier, hence symmetric: its VJP is the filter itself.
                Cosmology: d/dsigma8 exactly (delta is proportional to sigma8), d/dOmega_c
                with the tangent kernel along dP_lin/dOmega_c.
* `LPT`         linear density -> (dx, p) (pm/lpt.py:119), VJP by `jfli_lpt_adjoint`.
* `ReversibleNBody`  (dx, p) -> final CIC density after the KKD steps. Backward: per step
                un-drift + paint, force meshes at the previous positions, then
                un-kick + adjoint paint, P(div), and the CIC-gradient gather
                (`jfli_adjoint_*`); dL/dkick_n and dL/ddrift_n come out as FP64 sums.
* `PowerSpectrum` density -> P(k) per bin (_src/power/_compute.py:68-119).

Gradients with respect to the cosmology go through the FP64 host tables the kernels
consume (kick/drift factors, LPT factors, the P_lin table): the adjoint gives dL/d(each
scalar) and the host differentiates the scalars by central differences of the FP64
tables (the growth ODE is solved to rtol 1e-12, so a step of 1e-5 gives ~1e-7 relative
accuracy).

One deliberate difference from the reference: its reverse step un-drifts with a factor
built from dGfa while the forward step drifts with gp (pm/solvers.py:309 vs 364), so its
backward loop linearises around slightly different positions than the forward pass
visited. Here the reverse drift uses the forward factor, so reverse(step(y)) == y up to
FP32 rounding and the gradient is the gradient of the forward model.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np
import torch

from .. import cosmology as cj
from .. import ops
from .._lib import JFLI_STEP_DRIFT, JFLI_STEP_KICK, JFLI_STEP_PAINT
from .integrate import time_events
from .lpt import lpt_coefficients
from .solvers import ReversibleDoubleKickDrift

OMEGA_C_STEP = 1e-5


# ----------------------------------------------------------------------------- host tables
@dataclasses.dataclass
class ForwardTables:
    """FP64 host tables of one cosmology and their Omega_c derivatives."""

    ktab: np.ndarray
    ptab: np.ndarray
    lpt: tuple  # (c1x, c2x, c1p, c2p)
    kicks: np.ndarray
    drifts: np.ndarray
    dptab: np.ndarray | None = None
    dlpt: np.ndarray | None = None
    dkicks: np.ndarray | None = None
    ddrifts: np.ndarray | None = None
    sharpen: tuple | None = None  # SharpeningKernel: (per-step boost factors, kl, ks)

    def sharpen_slice(self, s0: int, s1: int):
        """The sharpening triple of steps s0..s1-1 (None without sharpening)."""
        if self.sharpen is None:
            return None
        boosts, kl, ks = self.sharpen
        return np.asarray(boosts, np.float64)[s0:s1], kl, ks


def kkd_schedule(cosmo, t0: float, t1: float, dt0: float):
    """(kicks, drifts) of the ReversibleDoubleKickDrift steps from t0 to t1."""
    ev = [(e[1], e[2]) for e in time_events(t0, [t1], dt0) if e[0] == "step"]
    if not ev:
        return np.zeros(0), np.zeros(0)
    t0s, t1s = zip(*ev)
    kicks, drifts = ReversibleDoubleKickDrift.schedule_arrays(cosmo, t0s, t1s, dt0, t0)
    return np.asarray(kicks, np.float64), np.asarray(drifts, np.float64)


def forward_tables(omega_c: float, sigma8: float, *, t0: float, t1: float, dt0: float, n_table: int = 128,
                   derivatives: bool = True, **cosmo_kw) -> ForwardTables:
    def build(oc):
        c = cj.Planck18(Omega_c=float(oc), sigma8=float(sigma8), **cosmo_kw)
        k, pk = cj.pk_table(c, n_table)
        kicks, drifts = kkd_schedule(c, t0, t1, dt0)
        return k, pk, np.asarray(lpt_coefficients(c, t0), np.float64), kicks, drifts

    k, pk, lc, kicks, drifts = build(omega_c)
    tab = ForwardTables(ktab=k, ptab=pk, lpt=tuple(float(v) for v in lc), kicks=kicks, drifts=drifts)
    if derivatives:
        h = OMEGA_C_STEP
        _, pk_p, lc_p, k_p, d_p = build(omega_c + h)
        _, pk_m, lc_m, k_m, d_m = build(omega_c - h)
        tab.dptab = (pk_p - pk_m) / (2 * h)
        tab.dlpt = (lc_p - lc_m) / (2 * h)
        tab.dkicks = (k_p - k_m) / (2 * h)
        tab.ddrifts = (d_p - d_m) / (2 * h)
    return tab


def _dev(a) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device="cuda", dtype=torch.float32).contiguous()
    return torch.as_tensor(np.asarray(a, np.float32), device="cuda")


def _dot(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    return torch.sum(a.double() * b.double())


def _scalar(t) -> float | None:
    if t is None:
        return None
    return float(t.detach()) if isinstance(t, torch.Tensor) else float(t)


def _like(value, param) -> torch.Tensor:
    """A gradient value as a tensor with the dtype and device of the parameter."""
    if isinstance(value, torch.Tensor):
        value = float(value.detach().double())
    return torch.as_tensor(value, dtype=param.dtype, device=param.device)


# ----------------------------------------------------------------------------- functions
class ICFilter(torch.autograd.Function):
    """noise -> sqrt(P_lin(|k|) M / V) filtered field (FP32 kernels, FP64 tables)."""

    @staticmethod
    def forward(ctx, noise, omega_c, sigma8, tables: ForwardTables, box):
        kt, pt = _dev(tables.ktab), _dev(tables.ptab)
        delta = ops.ic_filter(noise.contiguous(), kt, pt, box)
        ctx.tables, ctx.box = tables, box
        ctx.sigma8 = _scalar(sigma8)
        ctx.params = (omega_c, sigma8)
        ctx.save_for_backward(noise, delta)
        return delta

    @staticmethod
    def backward(ctx, gdelta):
        noise, delta = ctx.saved_tensors
        t = ctx.tables
        g = gdelta.contiguous()
        kt, pt = _dev(t.ktab), _dev(t.ptab)
        gnoise = ops.ic_filter(g, kt, pt, ctx.box) if ctx.needs_input_grad[0] else None
        gom = gs8 = None
        if ctx.needs_input_grad[1]:
            tang = ops.ic_filter_tangent(noise.contiguous(), kt, pt, _dev(t.dptab), ctx.box)
            gom = _like(_dot(g, tang), ctx.params[0])
        if ctx.needs_input_grad[2]:
            gs8 = _like(_dot(g, delta) / ctx.sigma8, ctx.params[1])
        return gnoise, gom, gs8, None, None


class LPT(torch.autograd.Function):
    """linear density -> (dx, p) at the grid points (order 1 or 2)."""

    @staticmethod
    def forward(ctx, ic, omega_c, order: int, tables: ForwardTables):
        ic = ic.contiguous()
        dx, p = ops.lpt(ic, order, *tables.lpt)
        ctx.order, ctx.tables = order, tables
        ctx.omega_c = omega_c
        ctx.save_for_backward(ic)
        return dx, p

    @staticmethod
    def backward(ctx, lam_x, lam_v):
        (ic,) = ctx.saved_tensors
        t = ctx.tables
        c1x, c2x, c1p, c2p = t.lpt
        lam_x = lam_x.contiguous()
        lam_v = lam_v.contiguous()
        gic = ops.lpt_adjoint(ic, ctx.order, c1x, c2x, c1p, c2p, lam_x, lam_v) if ctx.needs_input_grad[0] else None
        gom = None
        if ctx.needs_input_grad[1]:
            f1 = ops.lpt(ic, 1, 1.0, 0.0, 0.0, 0.0)[0]
            x1, v1 = _dot(lam_x, f1), _dot(lam_v, f1)
            dc = [x1 + c1p * v1, 0.0, c1x * v1, 0.0]
            if ctx.order == 2:
                f2 = ops.lpt(ic, 2, 0.0, 1.0, 0.0, 0.0)[0]
                x2, v2 = _dot(lam_x, f2), _dot(lam_v, f2)
                dc[1] = x2 + c2p * v2
                dc[3] = c2x * v2
            gom = _like(sum(float(t.dlpt[i]) * dc[i] for i in range(4)), ctx.omega_c)
        return gic, gom, None, None


# Device bytes the forward pass may keep for its backward sweep: each step's potential
# (4 bytes per cell), from which the reverse sweep rebuilds the forces instead of
# un-drifting, painting and solving for them again (about a third of a reverse step).
# Runs whose potentials need more (or more than a quarter of the free device memory)
# recompute them. 0 turns the store off.
POTENTIAL_STORE_BYTES = 4 << 30


def potential_store(nsteps: int, x: torch.Tensor) -> torch.Tensor | None:
    """An (nsteps, mesh) float32 buffer for the run's potentials, or None when it does not
    fit POTENTIAL_STORE_BYTES or a quarter of the free device memory."""
    need = 4 * nsteps * (x.numel() // 3)
    if need == 0 or need > POTENTIAL_STORE_BYTES:
        return None
    if need > (256 << 20):  # the free-memory query costs a millisecond: only for large stores
        free, _ = torch.cuda.mem_get_info(x.device)
        if need > free // 4:
            return None
    return torch.empty(nsteps, *x.shape[:-1], dtype=torch.float32, device=x.device)


def kkd_forward(x: torch.Tensor, v: torch.Tensor, kicks, drifts, rho: torch.Tensor, force: torch.Tensor | None = None,
                pot: torch.Tensor | None = None, pots: torch.Tensor | None = None, sharpen=None) -> None:
    """The ReversibleDoubleKickDrift loop in place: per step kick with the force at the
    current positions, drift, paint; rho ends as the CIC density of the final positions.
    One library call (`jfli_kkd_run`, or `jfli_kkd_run_stored` keeping every step's
    potential in `pots`); force and pot are accepted for callers that pass buffers and are
    not used (the library keeps its own in its workspace). `sharpen` = (boosts, kl, ks) adds
    SharpeningKernel's boost to each step's kick (jfli_kkd_run_sharpened)."""
    ops.kkd_run(x, v, kicks, drifts, rho, pots=pots, sharpen=sharpen)


def kkd_reverse_adjoint(x: torch.Tensor, v: torch.Tensor, lam_x: torch.Tensor, lam_v: torch.Tensor, kicks, drifts,
                        pots: torch.Tensor | None = None, sharpen=None):
    """Backward sweep of kkd_forward, in place on (x, v, lam_x, lam_v): on return (x, v) is
    the recomputed initial state and (lam_x, lam_v) the cotangent at it. Returns the FP64
    (dL/dkick_n, dL/ddrift_n) arrays. One library call (`jfli_kkd_adjoint`): per step
    un-drift + paint, force mesh, un-kick + adjoint paint, P(div), CIC-gradient gather;
    with the forward pass's `pots` (`jfli_kkd_adjoint_stored`) the force mesh comes from
    the stored potential and the un-drift is part of the un-kick."""
    return ops.kkd_adjoint(x, v, lam_x, lam_v, kicks, drifts, pots=pots, sharpen=sharpen)


class ReversibleNBody(torch.autograd.Function):
    """(dx, p) -> final CIC density of the ReversibleDoubleKickDrift loop."""

    @staticmethod
    def forward(ctx, dx, p, omega_c, tables: ForwardTables):
        x = dx.detach().contiguous().clone()
        v = p.detach().contiguous().clone()
        rho = torch.empty(x.shape[:-1], dtype=torch.float32, device=x.device)
        pots = potential_store(len(tables.kicks), x) if any(ctx.needs_input_grad[:3]) else None
        kkd_forward(x, v, tables.kicks, tables.drifts, rho, pots=pots, sharpen=tables.sharpen)
        ctx.tables = tables
        ctx.omega_c = omega_c
        ctx.pots = pots
        ctx.save_for_backward(x, v)
        return rho

    @staticmethod
    def backward(ctx, grho):
        x, v = ctx.saved_tensors
        t = ctx.tables
        x = x.clone()
        v = v.clone()
        lam_x = torch.zeros_like(x)
        lam_v = torch.zeros_like(v)
        ops.adjoint_position(x, lam_x, rho_bar=grho.contiguous())  # adjoint of the final paint
        if ctx.needs_input_grad[2] and t.sharpen is not None:
            raise NotImplementedError("d/dOmega_c of a run with SharpeningKernel: the sweep's sensitivities are "
                                      "those of the combined kick and boost")
        sens = kkd_reverse_adjoint(x, v, lam_x, lam_v, t.kicks, t.drifts, pots=ctx.pots, sharpen=t.sharpen)
        ctx.pots = None
        gom = None
        if ctx.needs_input_grad[2]:
            sk, sd = sens[:, 0].cpu().numpy(), sens[:, 1].cpu().numpy()
            gom = _like(float(np.dot(sk, t.dkicks) + np.dot(sd, t.ddrifts)), ctx.omega_c)
        ctx.sensitivities = sens
        return lam_x, lam_v, gom, None


class ReversibleNBodyShells(torch.autograd.Function):
    """(dx, p) -> snapshots painted at their times along the KKD loop: HEALPix shells
    (S, npix) or CIC densities (S, *mesh; geom["out_shape"] the mesh).

    The loop runs in segments: `segments[j]` steps, then snapshot j painted from the state
    there by `painters[j]`, a dict with a scale and its kind: "density" (the CIC density
    times scale), or, with rmin and rmax, "sphere" (the particles as they are) or "tiled" (replicas `rot`, `shifts`, `telephoto`, drifted
    to the light cone at time `t` with the velocities when `vel` is set; `kick` is the
    kick the EfficientDriftDoubleKick loop applies before a velocity paint, so the painted
    velocity is v + kick F(x) while the loop's state stays in the reversible form). The
    backward walks the segments in reverse: at each shell the painter's adjoint adds its
    cotangent to lambda_x (and lambda_v, with k J^T of it through the force for a kicked
    paint) at the reconstructed state, then the segment's steps are reversed
    (jfli_kkd_adjoint, over the potentials kept by the forward when they fit)."""

    @staticmethod
    def _painted_velocity(x, v, pt, tables):
        if not pt.get("vel"):
            return None
        if not pt.get("kick"):
            return v
        vp = v.clone()
        rho = ops.paint_cic(x)
        if pt.get("boost"):  # kick F + boost F_pgd, one combined force
            from .correction import sharpen_potential

            _, kl, ks = tables.sharpen
            force = ops.force_mesh(sharpen_potential(rho, float(pt["kick"]), float(pt["boost"]), kl, ks, 1.0))
            ops.kick_drift_paint(x, vp, force, 1.0, 0.0, JFLI_STEP_KICK)
            return vp
        force = torch.empty(x.shape[:-1] + (4,), dtype=torch.float32, device=x.device)
        ops.poisson_force(rho, 1.0, out=force, pot=torch.empty_like(rho))
        ops.kick_drift_paint(x, vp, force, float(pt["kick"]), 0.0, JFLI_STEP_KICK)
        return vp

    @staticmethod
    def forward(ctx, dx, p, tables: ForwardTables, segments, geom):
        x = dx.detach().contiguous().clone()
        v = p.detach().contiguous().clone()
        n_all = int(sum(segments))
        pots = potential_store(n_all, x) if any(ctx.needs_input_grad[:2]) else None
        rho = torch.empty(x.shape[:-1], dtype=torch.float32, device=x.device)
        shape = geom.get("out_shape") or (12 * geom["nside"] ** 2,)
        maps = torch.empty(len(segments), *shape, dtype=torch.float32, device=x.device)
        s0 = 0
        for j, c in enumerate(segments):
            if c > 0:
                kkd_forward(x, v, tables.kicks[s0:s0 + c], tables.drifts[s0:s0 + c], rho,
                            pots=None if pots is None else pots[s0:s0 + c], sharpen=tables.sharpen_slice(s0, s0 + c))
            _paint(x, ReversibleNBodyShells._painted_velocity(x, v, geom["painters"][j], tables), geom, j,
                   maps[j:j + 1])
            s0 += c
        ctx.tables, ctx.segments, ctx.geom, ctx.pots = tables, list(segments), geom, pots
        ctx.save_for_backward(x, v)
        return maps

    @staticmethod
    def backward(ctx, maps_bar):
        geom = ctx.geom
        x, v = ctx.saved_tensors
        x = x.clone()
        v = v.clone()
        t, pots = ctx.tables, ctx.pots
        lam_x = torch.zeros_like(x)
        lam_v = torch.zeros_like(v)
        mb = maps_bar.contiguous()
        s1 = int(sum(ctx.segments))
        for j in range(len(ctx.segments) - 1, -1, -1):
            pt = geom["painters"][j]
            vp = ReversibleNBodyShells._painted_velocity(x, v, pt, t)
            vp_bar = torch.zeros_like(v) if vp is not None else None
            _paint_adjoint(x, vp, geom, j, mb[j:j + 1], lam_x, vp_bar)
            if vp_bar is not None:
                lam_v += vp_bar
                if pt.get("kick"):
                    ops.force_adjoint(x, vp_bar, float(pt["kick"]), lam_x)
                    if pt.get("boost"):  # the sharpening boost's share: boost J_pgd^T vp_bar
                        _, kl, ks = t.sharpen
                        ops.pgd_adjoint(x, vp_bar, float(pt["boost"]), kl, ks, lam_x)
            c = ctx.segments[j]
            if c > 0:
                s0 = s1 - c
                kkd_reverse_adjoint(x, v, lam_x, lam_v, t.kicks[s0:s1], t.drifts[s0:s1],
                                    pots=None if pots is None else pots[s0:s1], sharpen=t.sharpen_slice(s0, s1))
                s1 = s0
        ctx.pots = None
        return lam_x, lam_v, None, None, None


def _paint(x, vp, geom, j, out):
    pt = geom["painters"][j]
    if pt["kind"] == "density":
        ops.paint_cic(x, weight=pt["scale"], out=out[0])
    elif pt["kind"] == "sphere":
        ops.healpix_paint_shells(x, geom["nside"], geom["box"], geom["obs"], [pt["rmin"]], [pt["rmax"]], [pt["scale"]],
                                 scheme=geom["scheme"], out=out)
    else:
        ops.healpix_paint_tiled(x, geom["nside"], geom["box"], geom["obs"], pt["rmin"], pt["rmax"], pt["rot"],
                                pt["shifts"], vel=vp, t=pt.get("t"), cosmo=geom.get("cosmo"),
                                telephoto=pt.get("telephoto", False), scheme=geom["scheme"], weight=pt["scale"],
                                out=out[0])


def _paint_adjoint(x, vp, geom, j, map_bar, lam_x, vp_bar):
    pt = geom["painters"][j]
    if pt["kind"] == "density":
        ops.adjoint_position(x, lam_x, rho_bar=map_bar[0].contiguous(), scale=pt["scale"])
    elif pt["kind"] == "sphere":
        ops.healpix_paint_shells_adjoint(x, map_bar, geom["nside"], geom["box"], geom["obs"], [pt["rmin"]],
                                         [pt["rmax"]], [pt["scale"]], scheme=geom["scheme"], pos_bar=lam_x)
    else:
        ops.healpix_paint_tiled_adjoint(x, map_bar[0], geom["nside"], geom["box"], geom["obs"], pt["rmin"], pt["rmax"],
                                        pt["rot"], pt["shifts"], vel=vp, t=pt.get("t"), cosmo=geom.get("cosmo"),
                                        telephoto=pt.get("telephoto", False), scheme=geom["scheme"],
                                        weight=pt["scale"], pos_bar=lam_x, vel_bar=vp_bar)


class PowerSpectrum(torch.autograd.Function):
    """density -> P(k) in the kept bins (FP64), the jax-fli `power` estimator."""

    @staticmethod
    def forward(ctx, mesh, kedges: np.ndarray, box):
        mesh = mesh.contiguous()
        ke = _dev(kedges)
        sums = ops.power_sums(mesh, ke, box)
        cnt = sums[1]
        vol = float(np.prod(np.asarray(box, np.float64) / np.asarray(mesh.shape[-3:], np.float64)))
        norm = torch.where(cnt > 0, cnt, torch.ones_like(cnt))
        pk = (sums[0] / norm)[1:-1] * vol
        ctx.save_for_backward(mesh, ke, cnt)
        ctx.vol, ctx.box = vol, box
        return pk

    @staticmethod
    def backward(ctx, gpk):
        mesh, ke, cnt = ctx.saved_tensors
        w = torch.zeros(ke.numel() + 1, dtype=torch.float64, device=mesh.device)
        c = cnt[1:-1]
        w[1:-1] = torch.where(c > 0, 2.0 * gpk * ctx.vol / torch.where(c > 0, c, torch.ones_like(c)),
                              torch.zeros_like(c))
        return ops.power_adjoint(mesh, ke, w.float(), ctx.box), None, None


class PowerPoles(torch.autograd.Function):
    """mesh -> Legendre multipoles of its auto spectrum in the kept bins (FP64): for each l
    the real part of the binned sum of (2l + 1) L_l(mu) |F|^2 over the mode count, times
    prod(L/N) (reference _src/power/_compute.py:68-119 with multipoles). The gradient is the
    auto spectrum's adjoint with each mode weighted by sum_l w_l[bin] (2l + 1) L_l(mu),
    averaged with the mode's conjugate partner (jfli_power_poles_adjoint): odd multipoles
    cancel between k and -k except on the grid's Nyquist planes, where the partner has the
    same frequency -n/2."""

    @staticmethod
    def forward(ctx, mesh, kedges: np.ndarray, box, poles, los):
        from ..power import poles_sums

        out, nell = poles_sums(mesh, None, box, kedges, poles, los)
        re, cnt = out[0, 0:2 * nell:2], out[0, 2 * nell]
        vol = float(np.prod(np.asarray(box, np.float64) / np.asarray(mesh.shape[-3:], np.float64)))
        norm = torch.where(cnt > 0, cnt, torch.ones_like(cnt))
        pk = (re / norm[None, :])[:, 1:-1] * vol
        ctx.save_for_backward(mesh, _dev(kedges), cnt)
        ctx.vol, ctx.box, ctx.poles, ctx.los = vol, box, tuple(int(p) for p in poles), los
        return pk[0] if nell == 1 else pk

    @staticmethod
    def backward(ctx, gpk):
        mesh, ke, cnt = ctx.saved_tensors
        g = gpk.reshape(len(ctx.poles), -1)
        c = cnt[1:-1]
        w = torch.zeros(len(ctx.poles), ke.numel() + 1, dtype=torch.float64, device=mesh.device)
        for e in range(len(ctx.poles)):
            w[e, 1:-1] = torch.where(c > 0, 2.0 * g[e] * ctx.vol / torch.where(c > 0, c, torch.ones_like(c)),
                                     torch.zeros_like(c))
        lv = np.asarray(ctx.los, np.float64)
        out = ops.power_poles_adjoint(mesh, ke, w.float().contiguous(), list(ctx.poles), ctx.box,
                                      tuple(lv / np.linalg.norm(lv)))
        return out, None, None, None, None


class LPTLightcone(torch.autograd.Function):
    """ic -> (dx, p, a) of light-cone-mode LPT (jfli_lpt_lightcone; reference pm/lpt.py:110-130
    with utils.py:234-244): each particle at the scale factor a_p of its own light-cone
    crossing, fixed by its Lagrangian position. The map is jfli_lpt's with per-particle
    coefficients (c1x, c2x, c1p, c2p)(a_p), so its VJP is jfli_lpt_adjoint with the
    cotangents weighted per particle, u1 = c1x lam_x + c1p c1x lam_v and u2 = c2x lam_x +
    c2p c2x lam_v, passed as lam_x = u1, lam_v = u2 - u1 with unit coefficients (c1x = 1,
    c1p = 0, c2x = c2p = 1). a passes no gradient."""

    @staticmethod
    def forward(ctx, ic, order: int, cosmo, box, observer):
        dx, p, a = ops.lpt_lightcone(ic.contiguous(), order, cosmo, box, observer)
        ctx.save_for_backward(ic.contiguous(), a)
        ctx.order, ctx.cosmo = int(order), cosmo
        ctx.mark_non_differentiable(a)
        return dx, p, a

    @staticmethod
    def backward(ctx, gdx, gp, ga):
        ic, a = ctx.saved_tensors
        gdx = torch.zeros(a.shape + (3,), dtype=torch.float32, device=a.device) if gdx is None else gdx
        gp = torch.zeros_like(gdx) if gp is None else gp
        av = a.double().cpu().numpy()
        c = ctx.cosmo
        d1, f1 = cj.growth_factor(c, av), cj.growth_rate(c, av)
        d2, f2 = cj.growth_factor_second(c, av), cj.growth_rate_second(c, av)
        ea = cj.E(c, av)
        coef = [torch.as_tensor(np.asarray(v, np.float64), device=a.device)[..., None]
                for v in (d1, 3.0 / 7.0 * d2, av * av * f1 * ea, av * av * f2 * ea)]
        c1x, c2x, c1p, c2p = coef
        gx, gv = gdx.double(), gp.double()
        u1 = c1x * gx + c1p * c1x * gv
        u2 = c2x * gx + c2p * c2x * gv
        out = ops.lpt_adjoint(ic, ctx.order, 1.0, 1.0, 0.0, 1.0, u1.float().contiguous(), (u2 - u1).float().contiguous())
        return out, None, None, None, None


class CrossPoles(torch.autograd.Function):
    """(mesh, mesh2) -> Legendre multipoles of the cross spectrum (FP64): |S_l,b| over the
    mode count times prod(L/N), S_l,b the binned sum of (2l + 1) L_l(mu) F1 conj(F2)
    (reference _src/power/_compute.py:68-119 with mesh2 and multipoles). With u = S / |S|,
    dL/dmesh1 is the multipole adjoint on mesh2 with the complex factors c = u dL/dP
    prod(L/N) / count, and dL/dmesh2 the same on mesh1 with conj(c)."""

    @staticmethod
    def forward(ctx, mesh, mesh2, kedges: np.ndarray, box, poles, los):
        from ..power import poles_sums

        out, nell = poles_sums(mesh, mesh2, box, kedges, poles, los)
        re, im, cnt = out[0, 0:2 * nell:2], out[0, 1:2 * nell:2], out[0, 2 * nell]
        mod = torch.sqrt(re**2 + im**2)
        vol = float(np.prod(np.asarray(box, np.float64) / np.asarray(mesh.shape[-3:], np.float64)))
        norm = torch.where(cnt > 0, cnt, torch.ones_like(cnt))
        pk = (mod / norm[None, :])[:, 1:-1] * vol
        safe = torch.where(mod > 0, mod, torch.ones_like(mod))
        ure, uim = torch.where(mod > 0, re / safe, torch.zeros_like(re)), torch.where(mod > 0, im / safe,
                                                                                       torch.zeros_like(im))
        ctx.save_for_backward(mesh, mesh2, _dev(kedges), cnt, ure, uim)
        ctx.vol, ctx.box, ctx.poles, ctx.los = vol, box, tuple(int(p) for p in poles), los
        return pk[0] if nell == 1 else pk

    @staticmethod
    def backward(ctx, gpk):
        mesh, mesh2, ke, cnt, ure, uim = ctx.saved_tensors
        g = gpk.reshape(len(ctx.poles), -1)
        c = cnt[1:-1]
        s = torch.zeros(len(ctx.poles), ke.numel() + 1, dtype=torch.float64, device=mesh.device)
        s[:, 1:-1] = torch.where(c > 0, g * ctx.vol / torch.where(c > 0, c, torch.ones_like(c)), torch.zeros_like(c))
        lv = np.asarray(ctx.los, np.float64)
        los = tuple(lv / np.linalg.norm(lv))

        def adj(m, sign):
            w = torch.stack([s * ure, sign * s * uim]).float().contiguous()
            return ops.power_poles_adjoint(m, ke, w, list(ctx.poles), ctx.box, los, complex_weights=True)

        g1 = adj(mesh2, 1.0) if ctx.needs_input_grad[0] else None
        g2 = adj(mesh, -1.0) if ctx.needs_input_grad[1] else None
        return g1, g2, None, None, None, None


class CrossPowerSpectrum(torch.autograd.Function):
    """(mesh, mesh2) -> cross P(k) in the kept bins (FP64): the modulus of the binned sum of
    F1 conj(F2) over the mode count, times prod(L/N) (reference _src/power/_compute.py:68-119
    with mesh2). For real meshes the imaginary parts cancel between k and -k, so
    d|S_b| = sign(Re S_b) d Re S_b, and d Re S_b / d mesh is the other mesh through the auto
    spectrum's adjoint with half its weight (the auto spectrum's factor 2 comes from
    |F|^2): dL/dmesh = power_adjoint(mesh2, w / 2), dL/dmesh2 = power_adjoint(mesh, w / 2)."""

    @staticmethod
    def forward(ctx, mesh, mesh2, kedges: np.ndarray, box):
        from ..power import poles_sums

        out, _ = poles_sums(mesh, mesh2, box, kedges, (0,), (0.0, 0.0, 1.0))
        re, im, cnt = out[0, 0], out[0, 1], out[0, 2]
        vol = float(np.prod(np.asarray(box, np.float64) / np.asarray(mesh.shape[-3:], np.float64)))
        norm = torch.where(cnt > 0, cnt, torch.ones_like(cnt))
        pk = (torch.sqrt(re**2 + im**2) / norm)[1:-1] * vol
        ctx.save_for_backward(mesh, mesh2, _dev(kedges), cnt, torch.sign(re))
        ctx.vol, ctx.box = vol, box
        return pk

    @staticmethod
    def backward(ctx, gpk):
        mesh, mesh2, ke, cnt, sgn = ctx.saved_tensors
        w = torch.zeros(ke.numel() + 1, dtype=torch.float64, device=mesh.device)
        c = cnt[1:-1]
        w[1:-1] = torch.where(c > 0, gpk * ctx.vol * sgn[1:-1] / torch.where(c > 0, c, torch.ones_like(c)),
                              torch.zeros_like(c))
        g1 = ops.power_adjoint(mesh2, ke, w.float(), ctx.box) if ctx.needs_input_grad[0] else None
        g2 = ops.power_adjoint(mesh, ke, w.float(), ctx.box) if ctx.needs_input_grad[1] else None
        return g1, g2, None, None


# ----------------------------------------------------------------------------- model
def forward_model_pk(noise: torch.Tensor, omega_c: torch.Tensor, sigma8: torch.Tensor, *, box, kedges, t0: float = 0.1,
                     t1: float = 1.0, dt0: float, lpt_order: int = 2, tables: ForwardTables | None = None):
    """P(k) of the final density of noise -> ICs -> LPT -> ReversibleDoubleKickDrift,
    differentiable in noise, omega_c and sigma8 (0-d tensors) through the B200 adjoints."""
    if tables is None:
        tables = forward_tables(_scalar(omega_c), _scalar(sigma8), t0=t0, t1=t1, dt0=dt0,
                                derivatives=bool(getattr(omega_c, "requires_grad", False)))
    box = tuple(float(b) for b in box)
    delta = ICFilter.apply(noise, omega_c, sigma8, tables, box)
    dx, p = LPT.apply(delta, omega_c, lpt_order, tables)
    rho = ReversibleNBody.apply(dx, p, omega_c, tables)
    return PowerSpectrum.apply(rho, np.asarray(kedges, np.float64), box)


def pk_log_loss(pk: torch.Tensor, pk_target: torch.Tensor) -> torch.Tensor:
    """sum over bins of (log P - log P_target)^2; bins without modes are left out."""
    mask = (pk_target > 0) & (pk.detach() > 0)
    return torch.sum((torch.log(pk[mask]) - torch.log(pk_target[mask])) ** 2)
