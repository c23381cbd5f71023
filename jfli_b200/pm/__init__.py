"""Particle-mesh module: LPT, N-body stepping and snapshot painting."""

from .correction import AbstractCorrection, NoCorrection, PGDKernel, SharpeningKernel
from .integrate import AdjointType, integrate, run_fused, run_stepwise, time_events
from .interp import (AbstractInterp, DriftInterp, InterpTilerState, NoInterp, OnionTiler, TelephotoInterp,
                     get_all_47_symmetries)
from .lpt import lpt, resolve_ts_geometry
from .nbody import nbody
from .solvers import AbstractNBodySolver, EfficientDriftDoubleKick, NBodyState, ReversibleDoubleKickDrift

__all__ = [
    "lpt", "nbody", "integrate", "AdjointType", "run_fused", "run_stepwise", "time_events", "resolve_ts_geometry",
    "EfficientDriftDoubleKick", "ReversibleDoubleKickDrift", "AbstractNBodySolver", "NBodyState",
    "PGDKernel", "SharpeningKernel", "NoCorrection", "AbstractCorrection",
    "OnionTiler", "TelephotoInterp", "NoInterp", "DriftInterp", "InterpTilerState", "AbstractInterp",
    "get_all_47_symmetries",
]
