"""N-body entry point (reference pm/nbody.py:28-171)."""

from __future__ import annotations

import dataclasses

import numpy as np

from .. import cosmology as cj
from ..fields import FieldStatus, PaintingOptions
from .integrate import integrate
from .interp import NoInterp
from .lpt import resolve_ts_geometry
from .solvers import EfficientDriftDoubleKick

_DEFAULT_SOLVER = EfficientDriftDoubleKick(interp_kernel=NoInterp(painting=PaintingOptions(target="particles")))


def nbody(cosmo, dx_field, p_field, *, t0: float = 0.1, t1: float = 1.0, dt0: float = 0.05, ts=None, nb_shells=None,
          density_widths=None, solver=_DEFAULT_SOLVER, adjoint: str = "checkpointed", checkpoints=None,
          equal_vol: bool = False, min_width: float = 50.0, return_state: bool = False):
    """Evolve LPT particles and return the snapshots / lightcone (near-to-far order).

    With return_state=True also returns the run record (final positions and velocities,
    number of steps taken)."""
    if dx_field.status not in (FieldStatus.LPT1, FieldStatus.LPT2):
        raise AssertionError("dx_field must have status FieldStatus.LPT1 or FieldStatus.LPT2.")
    if p_field.status not in (FieldStatus.LPT1, FieldStatus.LPT2):
        raise AssertionError("p_field must have status FieldStatus.LPT1 or FieldStatus.LPT2.")
    if dx_field.mesh_size != p_field.mesh_size:
        raise ValueError("dx_field and p_field must have matching mesh_size")
    if dx_field.box_size != p_field.box_size:
        raise ValueError("dx_field and p_field must have matching box_size")
    lpt_t0 = np.atleast_1d(np.asarray(dx_field.scale_factors, dtype=np.float64)).squeeze()
    if lpt_t0.ndim != 0:
        raise ValueError("Starting scale factor t0 and LPT fields' scale factor must be scalars.")
    if np.float32(lpt_t0) != np.float32(t0):
        raise ValueError(f"Starting scale factor t0={t0} does not match LPT fields' scale factor {float(lpt_t0)}.")
    if ts is None and nb_shells is None:
        ts = np.array([t1])
    ts_resolved, r_centers, widths, _ = resolve_ts_geometry(
        cosmo, dx_field, painting=solver.interp_kernel.painting, ts=ts, nb_shells=nb_shells,
        density_widths=density_widths, equal_vol=equal_vol, min_width=min_width)
    interp = solver.interp_kernel.update_geometry(ts=ts_resolved, r_centers=r_centers, density_widths=widths,
                                                  max_comoving_distance=dx_field.max_comoving_radius)
    solver = dataclasses.replace(solver, interp_kernel=interp)
    lightcone, run = integrate(dx_field, p_field, cosmo, ts_resolved, solver, t0, t1, dt0, adjoint=adjoint,
                               checkpoints=checkpoints)
    r_c, wd = np.asarray(r_centers, np.float64), np.asarray(widths, np.float64)
    if np.asarray(ts_resolved).size == 1:
        lightcone = lightcone.replace(array=lightcone.array[0])
        sf = lightcone.scale_factors
        lightcone = lightcone.replace(scale_factors=None if sf is None else np.asarray(sf).reshape(-1)[0])
        r_c, wd = r_c.reshape(-1)[0], wd.reshape(-1)[0]
    else:
        lightcone = lightcone.replace(array=lightcone.array.flip(0),
                                      scale_factors=np.asarray(lightcone.scale_factors)[::-1].copy())
        r_c, wd = r_c[::-1].copy(), wd[::-1].copy()
    sf = lightcone.scale_factors
    lightcone = lightcone.replace(z_sources=None if sf is None else cj.a2z(sf), comoving_centers=r_c,
                                  density_width=wd, status=FieldStatus.LIGHTCONE)
    return (lightcone, run) if return_state else lightcone
