"""Snapshot painters (reference pm/interp.py:46-318).

`NoInterp` paints the particles as they are at the snapshot time; `DriftInterp` first
drifts every particle to the scale factor at which its distance from the observer
crosses the light cone. The shell index advances at each snapshot time.
"""

from __future__ import annotations

import dataclasses
import warnings
from typing import Any

import numpy as np
import torch

from .. import cosmology as cj
from ..fields import PaintingOptions, PositionUnit


@dataclasses.dataclass(frozen=True)
class InterpTilerState:
    rotation_idx: int = -1
    shell_idx: int = -1
    rotations: Any = None


@dataclasses.dataclass(frozen=True)
class AbstractInterp:
    painting: PaintingOptions
    ts: Any = None
    r_centers: Any = None
    density_widths: Any = None
    max_comoving_distance: float | None = None

    def update_geometry(self, ts, r_centers, density_widths, max_comoving_distance):
        return dataclasses.replace(self, ts=np.asarray(ts, np.float64), r_centers=np.asarray(r_centers, np.float64),
                                   density_widths=np.asarray(density_widths, np.float64),
                                   max_comoving_distance=max_comoving_distance)

    def init(self) -> InterpTilerState:
        if self.r_centers is not None and self.max_comoving_distance is not None:
            furthest = float(self.r_centers[0] + self.density_widths[0] / 2)
            if furthest > self.max_comoving_distance:
                warnings.warn(
                    f"{type(self).__name__} does not support tiling. Your furthest shell is at {furthest:.2f} Mpc/h, "
                    f"but your box only extends to {self.max_comoving_distance:.2f} Mpc/h. Your simulations will run "
                    f"but will have artifacts for the far shells.")
        return InterpTilerState(rotation_idx=-1, shell_idx=-1, rotations=None)

    def _is_snapshot(self, t) -> bool:
        return self.ts is not None and bool(np.isin(np.float64(t), np.asarray(self.ts, np.float64)))

    def advance(self, state: InterpTilerState, t) -> InterpTilerState:
        return dataclasses.replace(state, shell_idx=state.shell_idx + 1) if self._is_snapshot(t) else state

    def rewind(self, state: InterpTilerState, t) -> InterpTilerState:
        return dataclasses.replace(state, shell_idx=state.shell_idx - 1) if self._is_snapshot(t) else state

    def paint(self, state, t, y, cosmo):
        raise NotImplementedError

    def needs_velocity(self) -> bool:
        return False

    def _paint_target(self, dx, r_center, width):
        tgt = self.painting.target if self.painting is not None else "particles"
        if tgt == "particles":
            return dx
        if tgt == "spherical":
            p = self.painting
            return dx.paint_spherical(center=r_center, density_plane_width=width, scheme=p.scheme, weights=p.weights,
                                      kernel_width_arcmin=p.kernel_width_arcmin,
                                      smoothing_interpretation=p.smoothing_interpretation, paint_nside=p.paint_nside,
                                      ud_grade_power=p.ud_grade_power, ud_grade_order_in=p.ud_grade_order_in,
                                      ud_grade_order_out=p.ud_grade_order_out, ud_grade_pess=p.ud_grade_pess,
                                      batch_size=p.batch_size)
        if tgt == "density":
            return dx.paint(weights=self.painting.weights, chunk_size=self.painting.chunk_size,
                            batch_size=self.painting.batch_size)
        raise NotImplementedError(f"painting target {tgt!r} is not on the B200 path")


@dataclasses.dataclass(frozen=True)
class NoInterp(AbstractInterp):
    """Paint without tiling (reference pm/interp.py:124-209)."""

    def paint(self, state, t, y, cosmo):
        dx, p = y
        r_center = float(self.r_centers[state.shell_idx])
        width = float(self.density_widths[state.shell_idx])
        res = self._paint_target(dx, r_center, width)
        return res.replace(scale_factors=t, comoving_centers=r_center, density_width=width)


@dataclasses.dataclass(frozen=True)
class DriftInterp(AbstractInterp):
    """Drift each particle to its light-cone crossing before painting (reference
    pm/interp.py:212-318): a_t = a(|x - observer|), x += v (D(a_t) - D(t)) / dGfa(sqrt(t a_t)),
    with x in Mpc/h as the reference does."""

    def needs_velocity(self) -> bool:
        return True

    def paint(self, state, t, y, cosmo):
        dx, p = y
        r_center = float(self.r_centers[state.shell_idx])
        width = float(self.density_widths[state.shell_idx])
        drifted = drift_to_lightcone(dx, p, float(t), cosmo)
        res = self._paint_target(drifted, r_center, width)
        return res.replace(scale_factors=t, comoving_centers=r_center, density_width=width)


def drift_to_lightcone(dx, p, t: float, cosmo):
    """Particles drifted to their light-cone crossing, as a MPC_H ParticleField (GPU kernel)."""
    from .. import ops

    return ops.lightcone_drift(dx, p, t, cosmo)


@dataclasses.dataclass(frozen=True)
class OnionTiler(AbstractInterp):
    """27-tile spherical painting (reference pm/interp.py:321-504); not on the B200 path yet."""

    drift_on_lightcone: bool = True

    def paint(self, state, t, y, cosmo):
        raise NotImplementedError("OnionTiler is not on the B200 path")


@dataclasses.dataclass(frozen=True)
class TelephotoInterp(AbstractInterp):
    def paint(self, state, t, y, cosmo):
        raise NotImplementedError("TelephotoInterp is not on the B200 path")
