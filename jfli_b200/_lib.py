"""ctypes binding of libjfli_b200.so (the C-ABI declared in include/jfli_b200.h).

The library is loaded once, lazily. There is no fallback: if the shared library is
missing, or no sm_100 CUDA device is present, every entry point raises.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import torch

_LIB_PATH = Path(__file__).resolve().parent / "libjfli_b200.so"
_lock = threading.Lock()
_lib = None

c_int = ctypes.c_int
c_float = ctypes.c_float
c_size_t = ctypes.c_size_t
c_void_p = ctypes.c_void_p
c_char_p = ctypes.c_char_p
c_longlong = ctypes.c_longlong

JFLI_STEP_KICK = 1
JFLI_STEP_DRIFT = 2
JFLI_STEP_PAINT = 4
JFLI_STEP_FORCE = 8
JFLI_STEP_CORRECT = 16
JFLI_STEP_CLEAR = 32
JFLI_HEALPIX_NGP = 0
JFLI_HEALPIX_BILINEAR = 1

_ERR = [c_char_p, c_size_t]
_DIMS = [c_int, c_int, c_int, c_int]

# name -> (restype, argtypes) ; argtypes exclude the trailing (err, errlen)
_SIGNATURES = {
    "jfli_version": (c_char_p, []),
    "jfli_launch_count": (c_longlong, []),
    "jfli_device_check": (c_int, _ERR),
    "jfli_mesh_supported": (c_int, [c_int, c_int, c_int]),
    "jfli_spectrum_elems": (c_longlong, [c_int, c_int, c_int]),
    "jfli_rfft3d": (c_int, [c_void_p, c_void_p, c_void_p, *_DIMS, *_ERR]),
    "jfli_irfft3d": (c_int, [c_void_p, c_void_p, c_void_p, *_DIMS, *_ERR]),
    "jfli_paint_cic": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_float, c_void_p, c_int, *_DIMS, *_ERR]),
    "jfli_readout_cic": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, *_DIMS, *_ERR]),
    "jfli_poisson_workspace_bytes": (c_size_t, _DIMS),
    "jfli_poisson_potential": (c_int, [c_void_p, c_void_p, c_float, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR]),
    "jfli_pgd_potential": (
        c_int,
        [c_void_p, c_void_p, c_float, c_float, c_float, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_readout_gradient": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_float, c_void_p, *_DIMS, *_ERR]),
    "jfli_pm_forces_workspace_bytes": (c_size_t, _DIMS),
    "jfli_pm_forces": (c_int, [c_void_p, c_void_p, c_int, c_float, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR]),
    "jfli_force_mesh": (c_int, [c_void_p, c_void_p, c_float, c_void_p, *_DIMS, *_ERR]),
    "jfli_pm_step_workspace_bytes": (c_size_t, _DIMS),
    "jfli_kick_drift_paint": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_float, c_int, c_float, c_void_p, *_DIMS, *_ERR],
    ),
    "jfli_pm_step": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_float, c_float, c_int, c_void_p, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_pm_step_slots": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, *_DIMS,
         *_ERR],
    ),
    "jfli_ic_filter": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_float, c_float, c_float, c_int, c_void_p,
         c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_lpt_workspace_bytes": (c_size_t, _DIMS),
    "jfli_lpt": (
        c_int,
        [c_void_p, c_void_p, c_int, c_float, c_float, c_float, c_float, c_void_p, c_void_p, c_void_p, c_size_t,
         *_DIMS, *_ERR],
    ),
    "jfli_power_spectrum_workspace_bytes": (c_size_t, [*_DIMS, c_int]),
    "jfli_power_spectrum": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_int, c_float, c_float, c_float, c_void_p, c_void_p, c_size_t, *_DIMS,
         *_ERR],
    ),
    "jfli_power_spectrum_noalloc": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_int, c_float, c_float, c_float, c_void_p, *_DIMS, *_ERR],
    ),
    "jfli_replica_positions": (
        c_int,
        [c_void_p, c_void_p, c_int, c_void_p, c_float, c_float, c_float, c_float, c_float, c_float,
         ctypes.POINTER(ctypes.c_byte), ctypes.POINTER(c_float), c_int, c_float, c_float, c_void_p, c_void_p, c_int,
         c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_void_p, *_DIMS, *_ERR],
    ),
    "jfli_power_poles_workspace_bytes": (c_size_t, [c_int, c_int, c_int, c_int, c_int, c_int, c_int]),
    "jfli_power_poles": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_float, c_float, c_float, c_float, c_float, c_float,
         ctypes.POINTER(c_int), c_int, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_paint_flat": (
        c_int,
        [c_void_p, c_void_p, c_int, c_void_p, c_float, c_float, c_float, c_int, c_int, c_void_p, c_int, *_DIMS, *_ERR],
    ),
    "jfli_flat_cl_workspace_bytes": (c_size_t, [c_int, c_int, c_int, c_int, c_int]),
    "jfli_flat_cl": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_float, c_float, c_void_p, c_int, c_void_p, c_void_p,
         c_size_t, *_ERR],
    ),
    "jfli_healpix_paint_tiled": (
        c_int,
        [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_float, c_float, c_float, c_float, c_float, c_float, c_float,
         c_int, ctypes.POINTER(ctypes.c_byte), ctypes.POINTER(c_float), c_int, c_float, c_float, c_float, c_float,
         c_float, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_int, c_int,
         c_void_p, c_int, *_DIMS, *_ERR],
    ),
    "jfli_healpix_paint_tiled_adjoint": (
        c_int,
        [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_float, c_float, c_float, c_float, c_float, c_float, c_float,
         c_int, ctypes.POINTER(ctypes.c_byte), ctypes.POINTER(c_float), c_int, c_float, c_float, c_float, c_float,
         c_float, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_int, c_int,
         c_void_p, c_void_p, c_void_p, c_void_p, *_DIMS, *_ERR],
    ),
    "jfli_lightcone_drift": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_float, c_float, c_float, c_float, c_float, c_float,
         c_float, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, *_DIMS, *_ERR],
    ),
    "jfli_sht_map2alm": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, ctypes.c_double, c_void_p, *_ERR]),
    "jfli_sht_ring_analysis": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, *_ERR]),
    "jfli_sht_ring_synthesis": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, *_ERR]),
    "jfli_sht_alm2map": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, *_ERR]),
    "jfli_sht_alm2cl": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, *_ERR]),
    "jfli_set_fft_x_pass": (c_int, [c_int, *_ERR]),
    "jfli_zero": (c_int, [c_void_p, c_void_p, ctypes.c_longlong, *_ERR]),
    "jfli_healpix_paint_rbf": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_float, c_float, c_float, c_float,
                                       c_float, c_float, c_float, c_float, c_float, c_int, c_float, c_void_p, c_int,
                                       *_DIMS, *_ERR]),
    "jfli_lpt_lightcone_workspace_bytes": (c_size_t, _DIMS),
    "jfli_lpt_lightcone": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_void_p, c_float, c_float,
                                   c_float, c_float, c_float, c_float, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_size_t, *_DIMS, *_ERR]),
    "jfli_device_status": (c_int, [c_void_p, c_int, *_ERR]),
    "jfli_poisson_force": (c_int, [c_void_p, c_void_p, c_float, c_int, c_float, c_void_p, c_void_p, c_void_p,
                                   c_size_t, *_DIMS, *_ERR]),
    "jfli_born_workspace_bytes": (c_size_t, [c_int, c_longlong]),
    "jfli_born_flat": (
        c_int,
        [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t,
         *_ERR],
    ),
    "jfli_born": (c_int, [c_void_p, c_void_p, c_int, c_longlong, c_void_p, c_int, c_void_p, c_void_p, c_size_t, *_ERR]),
    "jfli_born_adjoint_workspace_bytes": (c_size_t, [c_int, c_longlong]),
    "jfli_born_adjoint": (
        c_int, [c_void_p, c_void_p, c_int, c_longlong, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_size_t, *_ERR]),
    "jfli_adjoint_partials_count": (c_size_t, _DIMS),
    "jfli_kkd_workspace_bytes": (c_size_t, _DIMS),
    "jfli_kkd_run": (
        c_int,
        [c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_float), ctypes.POINTER(c_float), c_int, c_void_p, c_void_p,
         c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_kkd_adjoint": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_float), ctypes.POINTER(c_float), c_int,
         c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_pgd_adjoint_workspace_bytes": (c_size_t, _DIMS),
    "jfli_pgd_adjoint": (
        c_int, [c_void_p, c_void_p, c_void_p, c_float, c_float, c_float, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR]),
    "jfli_force_adjoint": (
        c_int, [c_void_p, c_void_p, c_void_p, c_float, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR]),
    "jfli_kkd_run_stored": (
        c_int,
        [c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_float), ctypes.POINTER(c_float), c_int, c_void_p, c_void_p,
         c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_kkd_adjoint_stored": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_float), ctypes.POINTER(c_float), c_int,
         c_void_p, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_paint_flat_adjoint": (
        c_int,
        [c_void_p, c_void_p, c_int, c_float, c_float, c_float, c_int, c_int, c_void_p, c_void_p, *_DIMS, *_ERR],
    ),
    "jfli_power_poles_adjoint": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_int, ctypes.POINTER(c_int), c_int, c_int, c_float, c_float,
         c_float, c_float, c_float, c_float, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_kkd_run_sharpened": (
        c_int,
        [c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_float), ctypes.POINTER(c_float), ctypes.POINTER(c_float),
         c_float, c_float, c_int, c_void_p, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_kkd_adjoint_sharpened": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_float), ctypes.POINTER(c_float),
         ctypes.POINTER(c_float), c_float, c_float, c_int, c_void_p, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_sharpen_potential": (
        c_int,
        [c_void_p, c_void_p, c_float, c_float, c_float, c_float, c_float, c_void_p, c_void_p, c_size_t, *_DIMS,
         *_ERR],
    ),
    "jfli_adjoint_unkick_paint": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_float, c_void_p, c_void_p, c_size_t,
         *_DIMS, *_ERR],
    ),
    "jfli_poisson_divergence_workspace_bytes": (c_size_t, _DIMS),
    "jfli_poisson_divergence": (
        c_int,
        [c_void_p, c_void_p, c_float, c_void_p, c_float, c_int, c_float, c_void_p, c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_adjoint_position": (
        c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_void_p, *_DIMS, *_ERR]),
    "jfli_power_spectrum_adjoint": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_float, c_float, c_float, c_void_p, c_void_p, c_size_t,
         *_DIMS, *_ERR],
    ),
    "jfli_lpt_adjoint_workspace_bytes": (c_size_t, _DIMS),
    "jfli_lpt_adjoint": (
        c_int,
        [c_void_p, c_void_p, c_int, c_float, c_float, c_float, c_float, c_void_p, c_void_p, c_void_p, c_void_p,
         c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_ic_filter_tangent": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_float, c_float, c_float, c_int,
         c_void_p, c_size_t, *_DIMS, *_ERR],
    ),
    "jfli_healpix_paint_shells": (
        c_int,
        [c_void_p, c_void_p, c_int, c_void_p, c_float, c_float, c_float, c_float, c_float, c_float, c_float, c_int,
         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(c_float), c_int, c_int,
         c_float, c_void_p, c_int, *_DIMS, *_ERR],
    ),
    "jfli_healpix_paint_shells_adjoint": (
        c_int,
        [c_void_p, c_void_p, c_int, c_void_p, c_float, c_float, c_float, c_float, c_float, c_float, c_float, c_int,
         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(c_float), c_int, c_int,
         c_void_p, c_void_p, c_void_p, *_DIMS, *_ERR],
    ),
    "jfli_healpix_paint": (
        c_int,
        [c_void_p, c_void_p, c_int, c_void_p, c_float, c_float, c_float, c_float, c_float, c_float, c_float,
         c_float, c_float, c_int, c_int, c_void_p, c_int, *_DIMS, *_ERR],
    ),
}


class JfliError(RuntimeError):
    """Error returned by a libjfli_b200 entry point."""

    def __init__(self, name: str, code: int, message: str):
        super().__init__(f"{name} failed (code {code}): {message}")
        self.code = code


def library_path() -> Path:
    return _LIB_PATH


def load(check_device: bool = True):
    """Load the shared library (once). Raises if it is missing."""
    global _lib
    with _lock:
        if _lib is None:
            if not _LIB_PATH.exists():
                raise RuntimeError(
                    f"{_LIB_PATH.name} not found next to the package; build it with `python -m jfli_b200._build`"
                )
            lib = ctypes.CDLL(str(_LIB_PATH))
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    if check_device:
        _require_device()
    return _lib


_device_ok = False


def _require_device():
    global _device_ok
    if _device_ok:
        return
    if not torch.cuda.is_available():
        raise RuntimeError("jfli_b200 needs a CUDA device (sm_100a); none is available")
    torch.cuda.init()
    buf = ctypes.create_string_buffer(512)
    rc = _lib.jfli_device_check(buf, 512)
    if rc != 0:
        raise JfliError("jfli_device_check", rc, buf.value.decode(errors="replace"))
    _device_ok = True


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def call(name: str, *args):
    """Call an entry point that ends with (err, errlen); raise JfliError on failure."""
    lib = load()
    buf = ctypes.create_string_buffer(512)
    rc = getattr(lib, name)(*args, buf, 512)
    if rc != 0:
        raise JfliError(name, rc, buf.value.decode(errors="replace"))
    return rc


def query(name: str, *args):
    """Call a pure query entry point (no error buffer)."""
    return getattr(load(check_device=False), name)(*args)


def stream_ptr(stream: torch.cuda.Stream | None = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("jfli_b200 kernels take CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("jfli_b200 kernels take contiguous tensors")
    return t.data_ptr()


def launch_count() -> int:
    return int(query("jfli_launch_count"))
