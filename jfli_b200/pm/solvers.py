"""N-body steppers (reference pm/solvers.py:35-411).

Time-step coefficients are computed in FP64 on the host from the growth tables
(`jfli_b200.cosmology`) and passed to the kernels as FP32 scalars. Each solver exposes

* the reference's per-step protocol `init / step / save_at / reverse`, implemented with
  the B200 kernels, for callers that drive the loop themselves; and
* `init_coefficients / step_coefficients`, which `integrate` uses to run the whole loop
  as fused particle passes (kick of one step + drift of the next + paint in one kernel).
"""

from __future__ import annotations

import dataclasses
import math
from typing import Any

import numpy as np
import torch

from .. import cosmology as cj
from .. import ops
from .._lib import JFLI_STEP_DRIFT, JFLI_STEP_KICK
from ..fields import PositionUnit
from .correction import AbstractCorrection, NoCorrection, PGDKernel, SharpeningKernel, sharpen_potential
from .interp import AbstractInterp, InterpTilerState


@dataclasses.dataclass(frozen=True)
class NBodyState:
    interp_state: InterpTilerState
    t_initial: float


def _force_mesh(x: torch.Tensor) -> torch.Tensor:
    """Force meshes (without 1.5 Omega_m) of the CIC density of relative positions x."""
    rho = ops.paint_cic(x)
    return ops.poisson_force(rho, rho_mean=1.0)


def _step_force(x: torch.Tensor, kick: float, corr, boost: float = 0.0):
    """(force mesh, factor) of a kick at relative positions x: kick F, or with a
    SharpeningKernel the combined kick F + boost F_pgd as one force applied with factor 1."""
    if isinstance(corr, SharpeningKernel):
        rho = ops.paint_cic(x)
        return ops.force_mesh(sharpen_potential(rho, kick, boost, corr.kl, corr.ks, 1.0)), 1.0
    return _force_mesh(x), kick


def _rel(field):
    return field if field.unit == PositionUnit.GRID_RELATIVE else field.to(PositionUnit.GRID_RELATIVE)


@dataclasses.dataclass(frozen=True)
class StepCoefficients:
    """One step's scalars. kick multiplies F = -grad_FD(pot) (1.5 Omega_m included)."""

    kick: float
    drift: float
    kick_first: bool  # True: force at the current position, then drift (reversible KKD)


@dataclasses.dataclass(frozen=True)
class AbstractNBodySolver:
    interp_kernel: AbstractInterp
    pgd_kernel: AbstractCorrection = NoCorrection()

    def init(self, displacement, velocities, t0, t1, dt, cosmo):
        raise NotImplementedError

    def step(self, displacement, velocities, t0, t1, dt, state, cosmo):
        raise NotImplementedError

    def save_at(self, displacement, velocities, t1, dt, state, cosmo):
        return self.interp_kernel.paint(state.interp_state, t1, (displacement, velocities), cosmo)

    def reverse(self, displacement, velocities, t0, t1, dt, state, cosmo):
        raise NotImplementedError(f"{type(self).__name__} is not reversible.")


@dataclasses.dataclass(frozen=True)
class EfficientDriftDoubleKick(AbstractNBodySolver):
    """FastPM KDK scheme (reference pm/solvers.py:118-225)."""

    @staticmethod
    def init_kick(cosmo, t0, t1) -> float:
        t0t1 = math.sqrt(t0 * t1)
        ai, ac, af = t0, t0, t0t1
        kf = (cj.Gf(cosmo, af) - cj.Gf(cosmo, ai)) / cj.dGfa(cosmo, ac)
        return float(1.5 * cosmo.Omega_m * kf / (ac**2 * cj.E(cosmo, ac)))

    @staticmethod
    def bare_drift(cosmo, t0, t1):
        """(Gp(t1) - Gp(t0)) / gp(sqrt(t0 t1)): the drift factor without its 1/(a^3 E)
        prefactor, which the reference's step hands to the correction kernel
        (pm/solvers.py:164-175). Scalars or arrays."""
        t0t1 = np.sqrt(np.asarray(t0, np.float64) * np.asarray(t1, np.float64))
        return (cj.Gp(cosmo, t1) - cj.Gp(cosmo, t0)) / cj.gp(cosmo, t0t1)

    @staticmethod
    def step_coefficients(cosmo, t0, t1, dt, t_initial=None) -> StepCoefficients:
        t0t1 = math.sqrt(t0 * t1)
        ai, ac, af = t0, t0t1, t1
        drift = (cj.Gp(cosmo, af) - cj.Gp(cosmo, ai)) / cj.gp(cosmo, ac) / (ac**3 * cj.E(cosmo, ac))
        t2 = t1 + dt
        t1t2 = math.sqrt(t1 * t2)
        ac = t1
        k1 = (cj.Gf(cosmo, t1) - cj.Gf(cosmo, t0t1)) / cj.dGfa(cosmo, ac)
        k2 = (cj.Gf(cosmo, t1t2) - cj.Gf(cosmo, t1)) / cj.dGfa(cosmo, ac)
        kick = 1.5 * cosmo.Omega_m * (k1 + k2) / (ac**2 * cj.E(cosmo, ac))
        return StepCoefficients(kick=float(kick), drift=float(drift), kick_first=False)

    @staticmethod
    def schedule_arrays(cosmo, t0s, t1s, dt, t_initial=None):
        """Vectorised step_coefficients over arrays of step boundaries -> (kicks, drifts)."""
        t0s = np.asarray(t0s, np.float64)
        t1s = np.asarray(t1s, np.float64)
        t0t1 = np.sqrt(t0s * t1s)
        drift = (cj.Gp(cosmo, t1s) - cj.Gp(cosmo, t0s)) / cj.gp(cosmo, t0t1) / (t0t1**3 * cj.E(cosmo, t0t1))
        t1t2 = np.sqrt(t1s * (t1s + dt))
        dg = cj.dGfa(cosmo, t1s)
        k1 = (cj.Gf(cosmo, t1s) - cj.Gf(cosmo, t0t1)) / dg
        k2 = (cj.Gf(cosmo, t1t2) - cj.Gf(cosmo, t1s)) / dg
        kick = 1.5 * cosmo.Omega_m * (k1 + k2) / (t1s**2 * cj.E(cosmo, t1s))
        return kick, drift

    def init(self, displacement, velocities, t0, t1, dt, cosmo):
        state = NBodyState(interp_state=self.interp_kernel.init(), t_initial=t0)
        x = _rel(displacement).array.contiguous()
        v = velocities.array.contiguous().clone()
        force = _force_mesh(x)
        ops.kick_drift_paint(x, v, force, self.init_kick(cosmo, t0, t1), 0.0, JFLI_STEP_KICK)
        return displacement, velocities.replace(array=v, scale_factors=math.sqrt(t0 * t1)), state

    def step(self, displacement, velocities, t0, t1, dt, state, cosmo):
        c = self.step_coefficients(cosmo, t0, t1, dt)
        disp = _rel(displacement)
        x = disp.array.contiguous().clone()
        v = velocities.array.contiguous().clone()
        ops.kick_drift_paint(x, v, None, 0.0, c.drift, JFLI_STEP_DRIFT)
        if isinstance(self.pgd_kernel, SharpeningKernel):
            # the boost and the kick act at the same (drifted) positions: one combined force
            boost = self.pgd_kernel.boost(float(self.bare_drift(cosmo, t0, t1)))
            xf = disp.replace(array=x, scale_factors=t1)
            force, factor = _step_force(x, c.kick, self.pgd_kernel, boost)
        else:
            xf, vf = self.pgd_kernel.apply(t1, disp.replace(array=x, scale_factors=t1), velocities.replace(array=v),
                                           full_drift_factor=c.drift)
            x = xf.array.contiguous()
            force, factor = _force_mesh(x), c.kick
        ops.kick_drift_paint(x, v, force, factor, 0.0, JFLI_STEP_KICK)
        new_state = NBodyState(interp_state=self.interp_kernel.advance(state.interp_state, t1),
                               t_initial=state.t_initial)
        return xf.replace(array=x, scale_factors=t1), velocities.replace(array=v, scale_factors=t1), new_state


@dataclasses.dataclass(frozen=True)
class ReversibleDoubleKickDrift(AbstractNBodySolver):
    """Reversible KKD scheme (reference pm/solvers.py:228-411). The reverse step undoes the
    drift with the same growth factor gp the forward step uses, so reverse(step(y)) == y."""

    @staticmethod
    def step_coefficients(cosmo, t0, t1, dt, t_initial=None) -> StepCoefficients:
        t_prev = max(t0 - dt, t_initial if t_initial is not None else t0)
        ai_1 = math.sqrt(t_prev * t0)
        af_2 = math.sqrt(t0 * t1)
        k1 = (cj.Gf(cosmo, t0) - cj.Gf(cosmo, ai_1)) / cj.dGfa(cosmo, t0)
        k2 = (cj.Gf(cosmo, af_2) - cj.Gf(cosmo, t0)) / cj.dGfa(cosmo, t0)
        kick = 1.5 * cosmo.Omega_m * (k1 + k2) / (t0**2 * cj.E(cosmo, t0))
        drift = (cj.Gp(cosmo, t1) - cj.Gp(cosmo, t0)) / cj.gp(cosmo, af_2) / (af_2**3 * cj.E(cosmo, af_2))
        return StepCoefficients(kick=float(kick), drift=float(drift), kick_first=True)

    @staticmethod
    def schedule_arrays(cosmo, t0s, t1s, dt, t_initial):
        """Vectorised step_coefficients over arrays of step boundaries -> (kicks, drifts)."""
        t0s = np.asarray(t0s, np.float64)
        t1s = np.asarray(t1s, np.float64)
        t_prev = np.maximum(t0s - dt, t_initial)
        ai_1 = np.sqrt(t_prev * t0s)
        af_2 = np.sqrt(t0s * t1s)
        dg = cj.dGfa(cosmo, t0s)
        k1 = (cj.Gf(cosmo, t0s) - cj.Gf(cosmo, ai_1)) / dg
        k2 = (cj.Gf(cosmo, af_2) - cj.Gf(cosmo, t0s)) / dg
        kick = 1.5 * cosmo.Omega_m * (k1 + k2) / (t0s**2 * cj.E(cosmo, t0s))
        drift = (cj.Gp(cosmo, t1s) - cj.Gp(cosmo, t0s)) / cj.gp(cosmo, af_2) / (af_2**3 * cj.E(cosmo, af_2))
        return kick, drift

    def _boost(self, c: StepCoefficients) -> float:
        """The sharpening boost factor of a step (alpha / its full drift factor), 0 without one."""
        return self.pgd_kernel.boost(c.drift) if isinstance(self.pgd_kernel, SharpeningKernel) else 0.0

    def init(self, displacement, velocities, t0, t1, dt, cosmo):
        return displacement, velocities, NBodyState(interp_state=self.interp_kernel.init(), t_initial=t0)

    def step(self, displacement, velocities, t0, t1, dt, state, cosmo):
        if isinstance(self.pgd_kernel, PGDKernel):
            # The reference applies PGD here but then drifts from the uncorrected position,
            # so the correction has no effect on the trajectory (pm/solvers.py:314-318).
            pass
        elif not isinstance(self.pgd_kernel, (NoCorrection, SharpeningKernel)):
            raise NotImplementedError(f"{type(self.pgd_kernel).__name__} is not on the B200 path")
        c = self.step_coefficients(cosmo, t0, t1, dt, state.t_initial)
        disp = _rel(displacement)
        x = disp.array.contiguous().clone()
        v = velocities.array.contiguous().clone()
        # kick, then the sharpening boost at the same x (one combined force), then the drift
        force, factor = _step_force(x, c.kick, self.pgd_kernel, self._boost(c))
        ops.kick_drift_paint(x, v, force, factor, c.drift, JFLI_STEP_KICK | JFLI_STEP_DRIFT)
        new_state = NBodyState(interp_state=self.interp_kernel.advance(state.interp_state, t1),
                               t_initial=state.t_initial)
        return (disp.replace(array=x, scale_factors=t1), velocities.replace(array=v, scale_factors=math.sqrt(t0 * t1)),
                new_state)

    def reverse(self, displacement, velocities, t0, t1, dt, state, cosmo):
        c = self.step_coefficients(cosmo, t0, t1, dt, state.t_initial)
        disp = _rel(displacement)
        x = disp.array.contiguous().clone()
        v = velocities.array.contiguous().clone()
        ops.kick_drift_paint(x, v, None, 0.0, -c.drift, JFLI_STEP_DRIFT)
        force, factor = _step_force(x, c.kick, self.pgd_kernel, self._boost(c))
        ops.kick_drift_paint(x, v, force, -factor, 0.0, JFLI_STEP_KICK)
        ts = self.interp_kernel.ts
        t1c = min(t1, float(ts[-1])) if ts is not None else t1
        prev = NBodyState(interp_state=self.interp_kernel.rewind(state.interp_state, t1c), t_initial=state.t_initial)
        return disp.replace(array=x, scale_factors=t0), velocities.replace(array=v), prev
