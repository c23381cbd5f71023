"""Snapshot painters (reference pm/interp.py:46-699).

`NoInterp` paints the particles as they are at the snapshot time; `DriftInterp` first
drifts every particle to the scale factor at which its distance from the observer
crosses the light cone. `OnionTiler` and `TelephotoInterp` paint shells beyond the box
from rotated and shifted replicas of it. The shell index advances at each snapshot time.
"""

from __future__ import annotations

import dataclasses
import itertools
import math
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
        """Whether t is one of the snapshot times. Compared in FP32, the precision of the
        reference's time variables and of jnp.isin on its FP32 ts (pm/interp.py:148): the
        time loop clips each step to the FP32 value of the next snapshot time, so the FP64
        shell times (from the distance table) only match after the same rounding."""
        return self.ts is not None and bool(np.isin(np.float32(t), np.asarray(self.ts, np.float32)))

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
        if tgt == "flat":
            return dx.paint_2d(center=r_center, density_plane_width=width, weights=self.painting.weights,
                               batch_size=self.painting.batch_size)
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
        res = _drifted_shell(dx, p, t, cosmo, r_center, width, self.painting)
        if res is None:
            res = self._paint_target(drift_to_lightcone(dx, p, float(t), cosmo), r_center, width)
        else:
            res = _spherical_result(res, t, r_center, width)
        return res.replace(scale_factors=t, comoving_centers=r_center, density_width=width)


def _drifted_shell(dx, p, t, cosmo, r_center: float, width: float, painting):
    """The spherical shell of the particles drifted to their light-cone crossing, drifted
    and painted in one pass by the replica painter with a single identity replica, which
    places each particle and tests the shell edges in FP64. (A drifted copy of the
    positions in FP32 Mpc/h rounds them by ~1e-5 Mpc/h at a few hundred Mpc/h, enough to
    move particles near an edge across it.) None when the painting options need the
    general path: another target, a scheme the replica painter does not have, or a batch
    of particle sets (painted one shell per set by paint_spherical)."""
    if painting is None or painting.target != "spherical" or painting.scheme not in ("ngp", "bilinear") or \
            dx.array.ndim != 4:
        return None
    from ..fields import SphericalDensity
    from ..painting import paint_shell_tiled

    m = paint_shell_tiled(_at_paint_nside(dx, painting), p.array, r_center, width, np.eye(3)[None], np.zeros((1, 3)),
                          telephoto=False, t=float(t), cosmo=cosmo, scheme=painting.scheme, weights=painting.weights)
    return SphericalDensity.FromDensityMetadata(array=_regrade(m, dx, painting), field=dx)


def drift_to_lightcone(dx, p, t: float, cosmo):
    """Particles drifted to their light-cone crossing, as a MPC_H ParticleField (GPU kernel)."""
    from .. import ops

    return ops.lightcone_drift(dx, p, t, cosmo)


def get_all_47_symmetries() -> np.ndarray:
    """The 47 non-identity signed permutation matrices of the cube, (47, 3, 3) int
    (reference pm/interp.py:31-43): sign triples in itertools.product((1, -1)) order outer,
    axis permutations in itertools.permutations order inner, row i holding sign s_i in
    column p_i; the first (the identity) is dropped. The order defines which matrix a
    rotation index names."""
    mats = []
    for s in itertools.product([1, -1], repeat=3):
        for p in itertools.permutations([0, 1, 2]):
            m = np.zeros((3, 3), dtype=np.int16)
            for i in range(3):
                m[i, p[i]] = s[i]
            mats.append(m)
    return np.array(mats)[1:]


def tile_shifts(observer_position, box_size) -> np.ndarray:
    """(27, 3) Mpc/h shifts of the 27 replicas (reference pm/interp.py:441-444): the
    offsets itertools.product((0, 1, -1), repeat=3), moved by +1 on axes where the
    observer sits at fraction 0 and by -1 where it sits at 1, times the box size."""
    sh = np.array(list(itertools.product([0, 1, -1], repeat=3)), dtype=np.int64)
    obs = np.asarray(observer_position, dtype=np.float64)
    sh = np.where(obs == 0, sh + 1, sh)
    sh = np.where(obs == 1, sh - 1, sh)
    return sh * np.asarray(box_size, dtype=np.float64)


def _at_paint_nside(dx, painting):
    """The particles to paint, at PaintingOptions.paint_nside when it is given."""
    return dx if painting.paint_nside is None else dx.replace(nside=int(painting.paint_nside))


def _regrade(m, dx, painting):
    """A map painted at paint_nside brought to the particles' nside (healpy's ud_grade)."""
    from ..painting import regrade

    return regrade(m, dx.nside, painting.paint_nside, power=painting.ud_grade_power,
                   order_in=painting.ud_grade_order_in, order_out=painting.ud_grade_order_out,
                   pess=painting.ud_grade_pess)


def _spherical_result(res, t, r_center, width):
    from ..fields import DensityUnit, FieldStatus

    return res.replace(status=FieldStatus.LIGHTCONE, unit=DensityUnit.DENSITY, scale_factors=t,
                       comoving_centers=r_center, density_width=width)


@dataclasses.dataclass(frozen=True)
class OnionTiler(AbstractInterp):
    """27-replica spherical painting with random cube symmetries (reference
    pm/interp.py:321-504). A shell inside the box (outer edge within the largest sphere
    around the observer that the box holds) is painted from the particles as they are;
    a shell beyond it from the 27 replicas of the box around the observer, replica i
    rotated by its own symmetry. All replicas are painted in one pass over the particles.
    With drift_on_lightcone each particle (each replica) is first drifted to its
    light-cone crossing.

    The reference draws the 27 rotation indices with jax.random.randint(PRNGKey(42), (27,),
    0, 47); JAX is not available here, so `rotation_indices` takes them explicitly (for
    maps identical to the reference's, pass those indices) and otherwise they are drawn
    with numpy.random.default_rng(rotation_seed)."""

    drift_on_lightcone: bool = True
    rotation_indices: tuple | None = None
    rotation_seed: int = 42

    def needs_velocity(self) -> bool:
        return self.drift_on_lightcone

    def init(self) -> InterpTilerState:
        if self.painting is None or self.painting.target != "spherical":
            raise ValueError("OnionTiler only supports spherical painting.")
        if self.rotation_indices is not None:
            idx = np.asarray(self.rotation_indices, dtype=np.int64)
            if idx.shape != (27,) or idx.min() < 0 or idx.max() > 46:
                raise ValueError("rotation_indices must be 27 integers in [0, 46]")
        else:
            idx = np.random.default_rng(self.rotation_seed).integers(0, 47, size=27)
        return InterpTilerState(rotation_idx=-1, shell_idx=-1, rotations=get_all_47_symmetries()[idx])

    def paint(self, state, t, y, cosmo):
        dx, p = y
        r_center = float(self.r_centers[state.shell_idx])
        width = float(self.density_widths[state.shell_idx])
        pt = self.painting
        if r_center + width / 2 <= self.max_comoving_distance:
            res = _drifted_shell(dx, p, t, cosmo, r_center, width, pt) if self.drift_on_lightcone else None
            if res is None:
                src = drift_to_lightcone(dx, p, float(t), cosmo) if self.drift_on_lightcone else dx
                res = self._paint_target(src, r_center, width)
        else:
            from ..fields import SphericalDensity
            from ..painting import paint_shell_tiled

            shifts = tile_shifts(dx.observer_position, dx.box_size)
            m = paint_shell_tiled(_at_paint_nside(dx, pt), p.array if self.drift_on_lightcone else None, r_center,
                                  width, state.rotations, shifts, telephoto=False, t=float(t), cosmo=cosmo,
                                  scheme=pt.scheme, weights=pt.weights)
            res = SphericalDensity.FromDensityMetadata(array=_regrade(m, dx, pt), field=dx)
        return _spherical_result(res, t, r_center, width)


@dataclasses.dataclass(frozen=True)
class TelephotoInterp(AbstractInterp):
    """One rotated and shifted replica per shell beyond the box, for narrow fields of view
    (reference pm/interp.py:507-699). The rotation index advances at each snapshot whose
    shell centre lies beyond the box; the replica is the box rotated by the index's cube
    symmetry (of the 47, cyclically) and pushed along z by floor(r / R) R, R the largest
    radius the box holds. The drift distance is measured as the reference measures it,
    from the observer-centred replica minus the observer's position. Spherical shells and
    flat-sky planes, inside the box and beyond it."""

    drift_on_lightcone: bool = True

    def needs_velocity(self) -> bool:
        return self.drift_on_lightcone

    def init(self) -> InterpTilerState:
        tgt = self.painting.target if self.painting is not None else None
        if tgt not in ("spherical", "flat"):
            raise ValueError("TelephotoInterp only supports projections (flat or spherical).")
        if tgt == "spherical":
            warnings.warn("TelephotoInterp is designed for narrow FOV flat-sky projections. Using it for spherical "
                          "painting will cause significant artifacts. use for illustriative purposes only.")
        return InterpTilerState(rotation_idx=-1, shell_idx=-1, rotations=get_all_47_symmetries())

    def advance(self, state, t):
        if not self._is_snapshot(t):
            return state
        nxt = state.shell_idx + 1
        inside = float(self.r_centers[nxt]) <= self.max_comoving_distance
        return dataclasses.replace(state, shell_idx=nxt, rotation_idx=state.rotation_idx + (0 if inside else 1))

    def rewind(self, state, t):
        if not self._is_snapshot(t):
            return state
        rc = float(self.r_centers[state.shell_idx])
        wd = float(self.density_widths[state.shell_idx])
        outside = rc + wd / 2 > self.max_comoving_distance
        return dataclasses.replace(state, shell_idx=state.shell_idx - 1,
                                   rotation_idx=state.rotation_idx - (1 if outside else 0))

    def paint(self, state, t, y, cosmo):
        dx, p = y
        r_center = float(self.r_centers[state.shell_idx])
        width = float(self.density_widths[state.shell_idx])
        pt = self.painting
        if r_center <= self.max_comoving_distance:
            src = drift_to_lightcone(dx, p, float(t), cosmo) if self.drift_on_lightcone else dx
            res = self._paint_target(src, r_center, width)
        else:
            from ..fields import SphericalDensity
            from ..painting import paint_shell_tiled

            rot = state.rotations[state.rotation_idx % 47][None]
            R = self.max_comoving_distance
            shift = np.array([[0.0, 0.0, math.floor(r_center / R) * R]])
            if pt.target == "flat":  # the replica's positions, then the flat-sky painter
                from .. import ops

                rel = dx if dx.unit != PositionUnit.MPC_H else dx.to(PositionUnit.GRID_ABSOLUTE)
                pos = ops.replica_positions(rel.array.contiguous(), dx.box_size, dx.observer_position_mpc, rot[0],
                                            shift[0], absolute=rel.unit == PositionUnit.GRID_ABSOLUTE,
                                            vel=p.array.contiguous() if self.drift_on_lightcone else None,
                                            t=float(t), cosmo=cosmo, telephoto=True)
                res = dx.replace(array=pos, unit=PositionUnit.MPC_H).paint_2d(
                    center=r_center, density_plane_width=width, weights=pt.weights, batch_size=pt.batch_size)
                return res.replace(scale_factors=t, comoving_centers=r_center, density_width=width)
            m = paint_shell_tiled(_at_paint_nside(dx, pt), p.array if self.drift_on_lightcone else None, r_center,
                                  width, rot, shift, telephoto=True, t=float(t), cosmo=cosmo, scheme=pt.scheme,
                                  weights=pt.weights)
            res = SphericalDensity.FromDensityMetadata(array=_regrade(m, dx, pt), field=dx)
        return res.replace(scale_factors=t, comoving_centers=r_center, density_width=width)
