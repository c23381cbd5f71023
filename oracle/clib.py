"""ctypes binding of oracle/cic.c and oracle/sht.c -- TEST INFRASTRUCTURE ONLY.

The C restatements of the oracle's CIC paint and readout and of its SHT Legendre stages
(OpenMP over the host's cores). `build()` compiles them with gcc into oracle/liboracle.so;
`_load()` builds it on first use when the file is missing or older than its sources (gcc
is part of the image). Only tests/, the fixture generators, the smoke check and bench.py's
CPU legs reach this module, through oracle.pm and oracle.sht.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRCS = [HERE / "cic.c", HERE / "sht.c"]
LIB = HERE / "liboracle.so"
_lib = None


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < max(p.stat().st_mtime for p in SRCS):
        tmp = LIB.with_suffix(f".{os.getpid()}.tmp")
        subprocess.run(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=gnu11", *map(str, SRCS), "-o", str(tmp),
                        "-lm"], check=True)
        os.replace(tmp, LIB)
    return LIB


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(str(build()))
        i64, vp, ci = ctypes.c_int64, ctypes.c_void_p, ctypes.c_int
        for t, ct in (("f64", ctypes.c_double), ("f32", ctypes.c_float)):
            f = getattr(lib, f"oracle_cic_paint_{t}")
            f.argtypes = [vp, i64, i64, i64, i64, ci, vp, ct, vp]
            f.restype = ci
            g = getattr(lib, f"oracle_cic_read_{t}")
            g.argtypes = [vp, ci, vp, i64, i64, i64, i64, ci, vp]
            g.restype = ci
        lib.oracle_threads.restype = ci
        lib.oracle_sht_analysis.argtypes = [vp, vp, ci, ci, ctypes.c_double, vp]
        lib.oracle_sht_analysis.restype = ci
        lib.oracle_sht_synthesis.argtypes = [vp, vp, ci, ci, vp]
        lib.oracle_sht_synthesis.restype = ci
        _lib = lib
    return _lib


def threads() -> int:
    return int(_load().oracle_threads())


def _suffix(a: np.ndarray) -> str:
    return {np.dtype(np.float64): "f64", np.dtype(np.float32): "f32"}[a.dtype]


def paint(pos: np.ndarray, shape, absolute: bool, weights, weight: float, mesh: np.ndarray) -> None:
    """mesh <- CIC paint of pos (P, 3) (C-contiguous, dtype of mesh)."""
    lib = _load()
    t = _suffix(mesh)
    assert pos.dtype == mesh.dtype and pos.flags.c_contiguous and mesh.flags.c_contiguous
    wp = None
    if weights is not None:
        assert weights.dtype == mesh.dtype and weights.size == pos.shape[0]
        wp = weights.ctypes.data
    rc = getattr(lib, f"oracle_cic_paint_{t}")(pos.ctypes.data, pos.shape[0], *shape, int(bool(absolute)), wp,
                                               float(weight), mesh.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle_cic_paint_{t} failed ({rc})")


def read(meshes: np.ndarray, pos: np.ndarray, absolute: bool, out: np.ndarray) -> None:
    """out (P, C) <- CIC readout of C meshes (C, nx, ny, nz) at pos (P, 3)."""
    lib = _load()
    t = _suffix(out)
    assert meshes.dtype == pos.dtype == out.dtype and meshes.flags.c_contiguous and pos.flags.c_contiguous
    c, nx, ny, nz = meshes.shape
    rc = getattr(lib, f"oracle_cic_read_{t}")(meshes.ctypes.data, c, pos.ctypes.data, pos.shape[0], nx, ny, nz,
                                              int(bool(absolute)), out.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle_cic_read_{t} failed ({rc})")


def sht_analysis(F: np.ndarray, z: np.ndarray, lmax: int, w: float) -> np.ndarray:
    """Packed a_lm (complex128) = w sum_r lambda_lm(z_r) F[r][m], F (nrings, lmax + 1) complex128."""
    F = np.ascontiguousarray(F, dtype=np.complex128)
    z = np.ascontiguousarray(z, dtype=np.float64)
    alm = np.empty((lmax + 1) * (lmax + 2) // 2, dtype=np.complex128)
    _load().oracle_sht_analysis(F.ctypes.data, z.ctypes.data, z.size, lmax, float(w), alm.ctypes.data)
    return alm


def sht_synthesis(alm: np.ndarray, z: np.ndarray, lmax: int) -> np.ndarray:
    """G (nrings, lmax + 1) complex128 = sum_l a_lm lambda_lm(z_r), a_lm packed by m."""
    alm = np.ascontiguousarray(alm, dtype=np.complex128)
    z = np.ascontiguousarray(z, dtype=np.float64)
    G = np.empty((z.size, lmax + 1), dtype=np.complex128)
    _load().oracle_sht_synthesis(alm.ctypes.data, z.ctypes.data, z.size, lmax, G.ctypes.data)
    return G
