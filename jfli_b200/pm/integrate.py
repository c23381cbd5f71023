"""Time integration (reference pm/integrate.py:17-279).

The loop structure is the reference's: an outer scan over the snapshot times `ts`, an
inner loop of `dt0` steps clipped to each snapshot time (tolerance 1e-6 for FP32 state,
1e-10 for FP64), `solver.save_at` after each inner loop.

On the GPU the loop runs as fused particle passes. With the FastPM KDK scheme the kick
that ends step n and the drift that starts step n+1 read and write the particles once:

    paint(x0) -> Poisson
    for each step: [kick(prev) + drift + paint]  -> Poisson      (one particle pass)
    final kick

and with the reversible KKD scheme each step is [kick + drift + paint] -> Poisson. The
density painted for the force at a snapshot time is the snapshot's density, so a
"density" snapshot is a copy of that mesh.
"""

from __future__ import annotations

import dataclasses
import math
from typing import Any, Literal

import numpy as np
import torch

from .. import ops
from .._lib import JFLI_STEP_CLEAR, JFLI_STEP_CORRECT, JFLI_STEP_DRIFT, JFLI_STEP_KICK, JFLI_STEP_PAINT
from ..fields import ParticleField, PositionUnit
from .correction import NoCorrection, PGDKernel, SharpeningKernel, pgd_potential, sharpen_potential
from .solvers import (AbstractNBodySolver, EfficientDriftDoubleKick, NBodyState, ReversibleDoubleKickDrift,
                      StepCoefficients)


def _clip_to_end(t_next, t1, tol):
    return t1 if t_next > t1 - tol else t_next


def time_events(t0: float, ts, dt0: float, dtype=np.float32):
    """Events of the reference loop: ("step", t_curr, t_next) and ("save", i, t_target).

    Times are accumulated in `dtype` (the precision of the reference's time variables)."""
    dt = np.dtype(dtype).type
    tol = 1e-10 if np.dtype(dtype) == np.float64 else 1e-6
    events = []
    t = dt(t0)
    for i, target in enumerate(np.atleast_1d(np.asarray(ts, dtype=np.float64))):
        tgt = dt(target)
        while t < tgt:
            tn = dt(t + dt(dt0))
            tn = _clip_to_end(tn, tgt, tol)
            events.append(("step", float(t), float(tn)))
            t = tn
        events.append(("save", i, float(tgt)))
    return events


@dataclasses.dataclass
class RunResult:
    snapshots: list
    disp: torch.Tensor
    vel: torch.Tensor
    steps: int


def _scalar_weight(w):
    if w is None:
        return 1.0
    if isinstance(w, (int, float)):
        return float(w)
    if isinstance(w, torch.Tensor) and w.ndim == 0:
        return float(w)
    return None


def run_fused(solver: AbstractNBodySolver, dx: ParticleField, p: ParticleField, cosmo, ts, t0: float, dt0: float,
              dtype=np.float32) -> RunResult:
    """Run the loop with fused particle passes; returns the snapshots and final state."""
    efficient = isinstance(solver, EfficientDriftDoubleKick)
    if not efficient and not isinstance(solver, ReversibleDoubleKickDrift):
        raise NotImplementedError(f"{type(solver).__name__} has no fused GPU schedule")
    pgd = solver.pgd_kernel if (efficient and isinstance(solver.pgd_kernel, PGDKernel)) else None
    sharpen = solver.pgd_kernel if isinstance(solver.pgd_kernel, SharpeningKernel) else None
    if not isinstance(solver.pgd_kernel, (NoCorrection, PGDKernel, SharpeningKernel)):
        raise NotImplementedError(f"{type(solver.pgd_kernel).__name__} is not on the B200 path")
    interp = solver.interp_kernel
    if dx.unit != PositionUnit.GRID_RELATIVE:
        dx = dx.to(PositionUnit.GRID_RELATIVE)
    x = dx.array.contiguous().clone()
    v = p.array.contiguous().clone()
    rho = torch.empty(x.shape[:-1], dtype=torch.float32, device=x.device)
    pot = torch.empty_like(rho)
    force = torch.empty(tuple(rho.shape) + (4,), dtype=torch.float32, device=x.device)
    events = time_events(t0, ts, dt0, dtype)
    n_steps = sum(1 for e in events if e[0] == "step")
    state = NBodyState(interp_state=interp.init(), t_initial=t0)
    # every step's FP64 factors up front (one vectorised evaluation of the growth tables),
    # so that the host only enqueues kernels inside the loop
    step_ts = [(e[1], e[2]) for e in events if e[0] == "step"]
    if step_ts:
        ta_all, tb_all = [a for a, _ in step_ts], [b for _, b in step_ts]
        if efficient:
            kicks_all, drifts_all = EfficientDriftDoubleKick.schedule_arrays(cosmo, ta_all, tb_all, dt0)
        else:
            kicks_all, drifts_all = ReversibleDoubleKickDrift.schedule_arrays(cosmo, ta_all, tb_all, dt0, t0)
        if sharpen is not None:
            # the boost factor per step: alpha / the drift factor the reference hands to the
            # correction (the bare one in the efficient step, the full one in the reversible)
            fd = (EfficientDriftDoubleKick.bare_drift(cosmo, ta_all, tb_all) if efficient
                  else np.asarray(drifts_all, np.float64))
            boosts_all = float(sharpen.alpha) / np.asarray(fd, np.float64)

    def sharpened_force(i):
        """Force mesh of step i's kick plus its sharpening boost, from the density in rho."""
        sharpen_potential(rho, float(kicks_all[i]), float(boosts_all[i]), sharpen.kl, sharpen.ks, 1.0, out=pot)
        ops.force_mesh(pot, out=force)

    tgt = interp.painting.target if interp.painting is not None else "particles"
    w_snap = _scalar_weight(interp.painting.weights) if interp.painting is not None else 1.0
    density_from_force_mesh = tgt == "density" and w_snap == 1.0

    # force at the initial positions (every paint clears the density mesh right before it)
    ops.kick_drift_paint(x, v, None, 0.0, 0.0, JFLI_STEP_PAINT | JFLI_STEP_CLEAR, rho)
    if sharpen is not None and not efficient and n_steps:
        sharpened_force(0)
    else:
        ops.poisson_force(rho, 1.0, out=force, pot=pot)
    pending = EfficientDriftDoubleKick.init_kick(cosmo, t0, t0 + dt0) if efficient else None
    rho_is_current = True  # rho holds the paint of the current positions

    snapshots = []
    step_i = 0
    for ev in events:
        if ev[0] == "step":
            _, ta, tb = ev
            c = StepCoefficients(kick=float(kicks_all[step_i]), drift=float(drifts_all[step_i]), kick_first=not efficient)
            step_i += 1
            if efficient:
                flags = JFLI_STEP_DRIFT | JFLI_STEP_PAINT | JFLI_STEP_CLEAR
                kick = 0.0
                if pending is not None:
                    flags |= JFLI_STEP_KICK
                    kick = pending
                if pgd is not None:
                    ops.kick_drift_paint(x, v, force, kick, c.drift, flags, rho)
                    pgd_potential(rho, pgd.kl, pgd.ks, 1.0, out=pot)
                    ops.force_mesh(pot, out=force)
                    ops.kick_drift_paint(x, v, force, pgd.alpha, 0.0,
                                         JFLI_STEP_CORRECT | JFLI_STEP_PAINT | JFLI_STEP_CLEAR, rho)
                else:
                    ops.kick_drift_paint(x, v, force, kick, c.drift, flags, rho)
                if sharpen is not None:  # the boost and the kick at the drifted positions
                    sharpened_force(step_i - 1)
                    pending = 1.0
                else:
                    ops.poisson_force(rho, 1.0, out=force, pot=pot)
                    pending = c.kick
            else:
                ops.kick_drift_paint(x, v, force, 1.0 if sharpen is not None else c.kick, c.drift,
                                     JFLI_STEP_KICK | JFLI_STEP_DRIFT | JFLI_STEP_PAINT | JFLI_STEP_CLEAR, rho)
                if step_i < n_steps:
                    if sharpen is not None:
                        sharpened_force(step_i)
                    else:
                        ops.poisson_force(rho, 1.0, out=force, pot=pot)
            rho_is_current = True
            state = NBodyState(interp_state=interp.advance(state.interp_state, tb), t_initial=t0)
        else:
            _, i, t_target = ev
            if efficient and pending is not None and interp.needs_velocity():
                ops.kick_drift_paint(x, v, force, pending, 0.0, JFLI_STEP_KICK)
                pending = None
            xf = dx.replace(array=x, scale_factors=t_target)
            vf = p.replace(array=v, scale_factors=t_target)
            if density_from_force_mesh and rho_is_current and not interp.needs_velocity():
                from ..fields import DensityField, DensityUnit, FieldStatus

                snap = DensityField(array=rho.clone(), **xf._meta_for_density(FieldStatus.DENSITY_FIELD))
                r_center = float(interp.r_centers[state.interp_state.shell_idx])
                width = float(interp.density_widths[state.interp_state.shell_idx])
                snap = snap.replace(scale_factors=t_target, comoving_centers=r_center, density_width=width)
            else:
                snap = solver.save_at(xf, vf, t_target, dt0, state, cosmo)
                if tgt == "particles":
                    snap = snap.replace(array=snap.array.clone())
            snapshots.append(snap)
    if efficient and pending is not None:
        ops.kick_drift_paint(x, v, force, pending, 0.0, JFLI_STEP_KICK)
    return RunResult(snapshots=snapshots, disp=x, vel=v, steps=n_steps)


def run_differentiable(solver, dx: ParticleField, p: ParticleField, cosmo, ts, t0: float, dt0: float,
                       dtype=np.float32) -> RunResult:
    """The N-body loop as one autograd node whose backward is the reversible adjoint
    (pm/adjoint.py), for inputs that require gradients. The reference's equivalents are
    nbody(..., adjoint="reverse") and nbody(..., adjoint="checkpointed") under jax.grad
    (pm/integrate.py:109-535). Covers density snapshots and HEALPix shells, with
    NoCorrection or SharpeningKernel.

    EfficientDriftDoubleKick takes the same route: its fused step kicks with the pending
    factor (the initial half kick at step 0, step i-1's kick after that) and then drifts,
    v' = v + k_i F(x), x' = x + d_i v', which is the reversible step with the kick array
    shifted by one; its last kick only touches the final velocities, not the density."""
    from .adjoint import ForwardTables, ReversibleNBody
    from .interp import DriftInterp, NoInterp, OnionTiler

    interp = solver.interp_kernel
    tgt = interp.painting.target if interp.painting is not None else "particles"
    ts_arr = np.atleast_1d(np.asarray(ts))
    efficient = isinstance(solver, EfficientDriftDoubleKick)
    solver_ok = (efficient or isinstance(solver, ReversibleDoubleKickDrift)) and isinstance(
        solver.pgd_kernel, (NoCorrection, SharpeningKernel))
    sharpen = solver.pgd_kernel if isinstance(solver.pgd_kernel, SharpeningKernel) else None
    pt = interp.painting
    shells_ok = (solver_ok and tgt == "spherical" and pt.scheme in ("ngp", "bilinear") and pt.paint_nside is None
                 and isinstance(pt.weights, (type(None), int, float)) and bool(np.all(np.diff(ts_arr) > 0))
                 and (isinstance(interp, NoInterp) or (isinstance(interp, (DriftInterp, OnionTiler))
                                                       and dx.array.dim() == 4)))
    density_ok = (solver_ok and isinstance(interp, NoInterp) and tgt == "density"
                  and isinstance(pt.weights, (type(None), int, float)) and bool(np.all(np.diff(ts_arr) > 0)))
    if not shells_ok and not density_ok:
        raise NotImplementedError(
            "gradients run through the reversible adjoint: ReversibleDoubleKickDrift or EfficientDriftDoubleKick "
            "with NoCorrection or SharpeningKernel, painting density snapshots (NoInterp, scalar weights) or HEALPix "
            "shells (ngp or bilinear; NoInterp, DriftInterp or OnionTiler) at increasing times")
    if dx.unit != PositionUnit.GRID_RELATIVE:
        raise NotImplementedError("differentiable integration takes GRID_RELATIVE displacements")
    steps = [(e[1], e[2]) for e in time_events(t0, ts, dt0, dtype) if e[0] == "step"]
    paint_kicks = paint_boosts = boosts = None
    if efficient:
        ta, tb = [a for a, _ in steps], [b for _, b in steps]
        kicks, drifts = EfficientDriftDoubleKick.schedule_arrays(cosmo, ta, tb, dt0)
        # the kick pending at a snapshot after s steps: the initial half kick, then step s-1's
        paint_kicks = np.concatenate([[EfficientDriftDoubleKick.init_kick(cosmo, t0, t0 + dt0)],
                                      np.asarray(kicks, np.float64)])
        kicks = paint_kicks[:-1]
        if sharpen is not None:
            # the boost rides with the kick it shares positions with (none on the initial half kick)
            b = float(sharpen.alpha) / np.asarray(EfficientDriftDoubleKick.bare_drift(cosmo, ta, tb), np.float64)
            paint_boosts = np.concatenate([[0.0], np.atleast_1d(b)])
            boosts = paint_boosts[:-1]
    else:
        cs = [solver.step_coefficients(cosmo, a, b, dt0, t0) for a, b in steps]
        kicks, drifts = np.array([c.kick for c in cs]), np.array([c.drift for c in cs])
        if sharpen is not None:
            boosts = np.array([sharpen.boost(c.drift) for c in cs], np.float64)
    tables = ForwardTables(ktab=None, ptab=None, lpt=None, kicks=np.asarray(kicks, np.float64),
                           drifts=np.asarray(drifts, np.float64),
                           sharpen=None if sharpen is None else (boosts, float(sharpen.kl), float(sharpen.ks)))
    if shells_ok:
        return _run_differentiable_shells(interp, dx, p, cosmo, t0, ts, dt0, dtype, tables, paint_kicks, paint_boosts)
    if ts_arr.size > 1 or _scalar_weight(interp.painting.weights) != 1.0:
        return _run_differentiable_densities(interp, dx, p, t0, ts, dt0, dtype, tables)
    rho = ReversibleNBody.apply(dx.array.contiguous(), p.array.contiguous(), None, tables)
    from ..fields import DensityField, FieldStatus

    t_target = float(ts_arr[0])
    state = NBodyState(interp_state=interp.init(), t_initial=t0)
    snap = DensityField(array=rho, **dx.replace(scale_factors=t_target)._meta_for_density(FieldStatus.DENSITY_FIELD))
    snap = snap.replace(scale_factors=t_target, comoving_centers=float(interp.r_centers[state.interp_state.shell_idx]),
                        density_width=float(interp.density_widths[state.interp_state.shell_idx]))
    return RunResult(snapshots=[snap], disp=None, vel=None, steps=len(steps))


def _run_differentiable_densities(interp, dx: ParticleField, p: ParticleField, t0: float, ts, dt0: float, dtype,
                                  tables) -> RunResult:
    """Density snapshots at several times (or with a scalar weight) along the loop as one
    autograd node (adjoint.ReversibleNBodyShells with density painters): snapshot j is the
    CIC density of the positions at the j-th snapshot time times the weight, as the fused
    loop paints it (NoInterp.paint -> ParticleField.paint); the backward adds each
    snapshot's CIC gradient at the reconstructed positions before reversing the steps that
    led there."""
    from ..fields import DensityField, FieldStatus
    from .adjoint import ReversibleNBodyShells

    events = time_events(t0, ts, dt0, dtype)
    segments, count = [], 0
    for ev in events:
        if ev[0] == "step":
            count += 1
        else:
            segments.append(count)
            count = 0
    saves = [ev for ev in events if ev[0] == "save"]
    w = float(_scalar_weight(interp.painting.weights))
    geom = dict(painters=[dict(kind="density", scale=w)] * len(segments), out_shape=tuple(dx.array.shape[:-1]))
    rhos = ReversibleNBodyShells.apply(dx.array.contiguous(), p.array.contiguous(), tables, segments, geom)
    snaps = []
    for j, ev in enumerate(saves):
        t_j = float(ev[2])
        snap = DensityField(array=rhos[j], **dx.replace(scale_factors=t_j)._meta_for_density(FieldStatus.DENSITY_FIELD))
        snaps.append(snap.replace(scale_factors=t_j, comoving_centers=float(interp.r_centers[j]),
                                  density_width=float(interp.density_widths[j])))
    return RunResult(snapshots=snaps, disp=None, vel=None, steps=int(sum(segments)))


def _run_differentiable_shells(interp, dx: ParticleField, p: ParticleField, cosmo, t0: float, ts, dt0: float, dtype,
                               tables, paint_kicks, paint_boosts=None) -> RunResult:
    """HEALPix shells along the loop as one autograd node (adjoint.ReversibleNBodyShells):
    shell j is painted at the j-th snapshot time from the state there, with the geometry,
    painter and normalisation of the fused loop's shells. NoInterp paints the particles as
    they are (paint_spherical); DriftInterp, and OnionTiler inside the box, paint one
    identity replica drifted to the light cone; OnionTiler beyond the box paints the 27
    rotated replicas, drifted when drift_on_lightcone. Under EfficientDriftDoubleKick a
    drifted shell is painted with the velocities after the pending kick, as the fused loop
    applies it before a velocity-dependent paint (`paint_kicks[s]` after s steps)."""
    from ..painting import shell_volume_per_pixel
    from .adjoint import ReversibleNBodyShells
    from .interp import DriftInterp, NoInterp, _spherical_result, tile_shifts

    events = time_events(t0, ts, dt0, dtype)
    segments, count = [], 0
    for ev in events:
        if ev[0] == "step":
            count += 1
        else:
            segments.append(count)
            count = 0
    nshell = len(segments)
    saves = [ev for ev in events if ev[0] == "save"]
    rc = np.asarray(interp.r_centers, np.float64)[:nshell]
    wd = np.asarray(interp.density_widths, np.float64)[:nshell]
    rmin, rmax = rc - wd / 2.0, rc + wd / 2.0
    ws = _scalar_weight(interp.painting.weights)
    vol = np.array([shell_volume_per_pixel(dx.nside, a, b) for a, b in zip(rmin, rmax)])
    scale = np.where(vol > 0, ws / np.where(vol > 0, vol, 1.0), ws)
    drift = isinstance(interp, DriftInterp) or (not isinstance(interp, NoInterp) and interp.drift_on_lightcone)
    rotations = interp.init().rotations if not isinstance(interp, (NoInterp, DriftInterp)) else None
    painters, done = [], 0
    for j in range(nshell):
        done += segments[j]
        pj = dict(rmin=float(rmin[j]), rmax=float(rmax[j]), scale=float(scale[j]))
        beyond = rotations is not None and rmax[j] > interp.max_comoving_distance
        if not drift and not beyond:
            pj["kind"] = "sphere"
        else:
            pj.update(kind="tiled", t=float(saves[j][2]), vel=drift,
                      kick=float(paint_kicks[done]) if (drift and paint_kicks is not None) else None,
                      boost=float(paint_boosts[done]) if (drift and paint_boosts is not None) else None)
            if beyond:
                pj.update(rot=rotations, shifts=tile_shifts(dx.observer_position, dx.box_size))
            else:
                pj.update(rot=np.eye(3)[None], shifts=np.zeros((1, 3)))
        painters.append(pj)
    geom = dict(nside=int(dx.nside), box=tuple(dx.box_size), obs=tuple(dx.observer_position_mpc),
                scheme=interp.painting.scheme, cosmo=cosmo, painters=painters)
    maps = ReversibleNBodyShells.apply(dx.array.contiguous(), p.array.contiguous(), tables, segments, geom)
    template = dx.replace(array=dx.array.detach()).paint_spherical(center=rc[0], density_plane_width=wd[0],
                                                                   scheme=interp.painting.scheme)
    snaps = [_spherical_result(template.replace(array=maps[j]), float(saves[j][2]), float(rc[j]), float(wd[j]))
             for j in range(nshell)]
    return RunResult(snapshots=snaps, disp=None, vel=None, steps=int(sum(segments)))


def run_stepwise(solver, dx, p, cosmo, ts, t0, dt0, dtype=np.float32) -> RunResult:
    """The reference loop driven through solver.init/step/save_at (unfused)."""
    disp, vel, state = solver.init(dx, p, t0, t0 + dt0, dt0, cosmo)
    snapshots = []
    n = 0
    for ev in time_events(t0, ts, dt0, dtype):
        if ev[0] == "step":
            disp, vel, state = solver.step(disp, vel, ev[1], ev[2], dt0, state, cosmo)
            n += 1
        else:
            snapshots.append(solver.save_at(disp, vel, ev[2], dt0, state, cosmo))
    return RunResult(snapshots=snapshots, disp=disp.array, vel=vel.array, steps=n)


def _stack(snapshots):
    first = snapshots[0]
    arr = torch.stack([s.array for s in snapshots])
    meta = {}
    for key in ("scale_factors", "comoving_centers", "density_width"):
        vals = [getattr(s, key) for s in snapshots]
        meta[key] = None if any(v is None for v in vals) else np.asarray([float(np.asarray(v).reshape(-1)[0])
                                                                         for v in vals])
    return first.replace(array=arr, **meta)


AdjointType = Literal["reverse", "checkpointed"]  # the adjoint modes of integrate (reference pm/integrate.py:14)


def integrate(displacements, velocities, cosmo, ts, solver, t0, t1, dt0, adjoint="checkpointed", checkpoints=None,
              fused: bool = True):
    """Snapshots at each time in ts (reference pm/integrate.py:55-118), stacked on axis 0."""
    if adjoint == "reverse" and not solver.pgd_kernel.reversible:
        raise ValueError(
            f"Cannot use adjoint='reverse' with {type(solver.pgd_kernel).__name__}. "
            f"Use SharpeningKernel for reversible integration, or use adjoint='checkpointed'.")
    if adjoint not in ("checkpointed", "reverse", "lax"):
        raise ValueError(f"Unknown adjoint type: {adjoint}")
    if torch.is_grad_enabled() and (displacements.array.requires_grad or velocities.array.requires_grad):
        res = run_differentiable(solver, displacements, velocities, cosmo, ts, t0, dt0)
    else:
        run = run_fused if fused else run_stepwise
        res = run(solver, displacements, velocities, cosmo, ts, t0, dt0)
    out = _stack(res.snapshots)
    return out, res
