"""The C-ABI library loads and exports every entry point include/jfli_b200.h declares
(CPU only: no compute calls)."""

from __future__ import annotations

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "jfli_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jfli_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from jfli_b200 import _build

    path = _build.LIB
    if not path.exists():
        _build.build()
    return ctypes.CDLL(str(path))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "jfli_pm_forces" in names and "jfli_healpix_paint" in names and len(names) >= 15


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"symbols declared in the header but not exported: {missing}"


def test_binding_covers_header():
    from jfli_b200 import _lib

    bound = set(_lib.exported_symbols())
    assert set(declared_functions()) <= bound


def test_pure_queries_without_gpu(lib):
    lib.jfli_mesh_supported.restype = ctypes.c_int
    assert lib.jfli_mesh_supported(256, 256, 256) == 1
    assert lib.jfli_mesh_supported(192, 96, 64) == 1
    assert lib.jfli_mesh_supported(100, 100, 100) == 0  # 5 is not a supported radix
    assert lib.jfli_mesh_supported(64, 64, 63) == 0  # nz must be even
    lib.jfli_spectrum_elems.restype = ctypes.c_longlong
    assert lib.jfli_spectrum_elems(256, 256, 256) == 256 * 256 * 129
    lib.jfli_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.jfli_version()
    lib.jfli_pm_forces_workspace_bytes.restype = ctypes.c_size_t
    assert lib.jfli_pm_forces_workspace_bytes(64, 64, 64, 1) >= 64**3 * 4 + 64 * 64 * 33 * 8


def test_argument_errors_are_reported_not_raised(lib):
    """Bad arguments come back as JFLI_EINVAL with a message; nothing reaches the GPU."""
    buf = ctypes.create_string_buffer(256)
    fn = lib.jfli_paint_cic
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_float,
                   ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_char_p, ctypes.c_size_t]
    rc = fn(None, None, 0, None, 1.0, None, 0, 8, 8, 8, 1, buf, 256)
    assert rc == 1 and b"null pointer" in buf.value
    rc = fn(None, None, 0, None, 1.0, None, 0, 0, 8, 8, 1, buf, 256)
    assert rc == 1 and b"invalid mesh shape" in buf.value


def test_oversized_mesh_rejected(lib):
    """A mesh whose particle offsets would overflow 32 bits ((2^32 - 1)/3 cells) is refused
    before any launch; 1024^3 is accepted by the shape check."""
    buf = ctypes.create_string_buffer(256)
    fn = lib.jfli_paint_cic
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_float,
                   ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_char_p, ctypes.c_size_t]
    rc = fn(None, ctypes.c_void_p(16), 0, None, 1.0, ctypes.c_void_p(16), 0, 1200, 1200, 1200, 1, buf, 256)
    assert rc == 1 and b"invalid mesh shape" in buf.value
    rc = fn(None, None, 0, None, 1.0, None, 0, 1024, 1024, 1024, 1, buf, 256)
    assert rc == 1 and b"null pointer" in buf.value  # shape accepted, pointers checked next


def test_force_mesh_alignment_checked(lib):
    buf = ctypes.create_string_buffer(256)
    fn = lib.jfli_force_mesh
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p] + [ctypes.c_int] * 4 + [
        ctypes.c_char_p, ctypes.c_size_t]
    rc = fn(None, ctypes.c_void_p(256), 1.0, ctypes.c_void_p(260), 16, 16, 16, 1, buf, 256)
    assert rc == 1 and b"16-byte aligned" in buf.value


def test_unsupported_fft_shape_reported(lib):
    buf = ctypes.create_string_buffer(256)
    fn = lib.jfli_rfft3d
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 4 + [ctypes.c_char_p,
                                                                                             ctypes.c_size_t]
    rc = fn(None, ctypes.c_void_p(16), ctypes.c_void_p(16), 100, 64, 64, 1, buf, 256)
    assert rc == 3 and b"unsupported" in buf.value


def test_no_cpu_fallback_in_product():
    """The product package never imports the oracle and has no CPU compute path."""
    pkg = os.path.join(ROOT, "jfli_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith(".py"):
                src = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in re.sub(r"#.*", "", src).replace('"""', ""), f


def test_tiled_paint_checks_rotations(lib):
    """jfli_healpix_paint_tiled takes signed permutation matrices only (the exactness of
    the replica rotation in FP32 rests on it), and at most 27 replicas."""
    from jfli_b200 import _lib

    res, args = _lib._SIGNATURES["jfli_healpix_paint_tiled"]
    fn = lib.jfli_healpix_paint_tiled
    fn.restype, fn.argtypes = res, args
    buf = ctypes.create_string_buffer(256)

    def call(rot, ntiles=None):
        r = (ctypes.c_byte * 9 * len(rot))(*[(ctypes.c_byte * 9)(*m) for m in rot])
        s = (ctypes.c_float * (3 * len(rot)))()
        return fn(None, ctypes.c_void_p(256), 0, None, None, 1.0, 100.0, 100.0, 100.0, 50.0, 50.0, 50.0,
                  len(rot) if ntiles is None else ntiles, ctypes.cast(r, ctypes.POINTER(ctypes.c_byte)),
                  ctypes.cast(s, ctypes.POINTER(ctypes.c_float)), 0, 10.0, 20.0, 0.0, 0.0, 0.0, None, None, 0, None,
                  None, 0, None, None, 0, 4, 1, ctypes.c_void_p(256), 0, 16, 16, 16, 1, buf, 256)

    assert call([[1, 0, 0, 0, 1, 0, 1, 0, 0]]) == 1 and b"signed permutation" in buf.value  # column used twice
    assert call([[2, 0, 0, 0, 1, 0, 0, 0, 1]]) == 1 and b"signed permutation" in buf.value
    assert call([[1, 0, 0, 0, 0, 0, 0, 0, 1]]) == 1 and b"signed permutation" in buf.value  # empty row
    assert call([[1, 0, 0, 0, 1, 0, 0, 0, 1]], ntiles=28) == 1 and b"ntiles" in buf.value


def _bound(lib, name):
    from jfli_b200 import _lib

    res, args = _lib._SIGNATURES[name]
    fn = getattr(lib, name)
    fn.restype, fn.argtypes = res, args
    return fn


def test_flat_sky_entry_points_check_sizes(lib):
    """jfli_paint_flat and jfli_flat_cl refuse bad map sizes, edge counts and workspaces
    before any launch."""
    buf = ctypes.create_string_buffer(256)
    paint = _bound(lib, "jfli_paint_flat")
    p = ctypes.c_void_p(256)
    assert paint(None, p, 0, None, 1.0, 0.0, 1.0, 0, 16, p, 0, 16, 16, 16, 1, buf, 256) == 1
    assert b"flat-sky map" in buf.value
    cl = _bound(lib, "jfli_flat_cl")
    assert cl(None, p, None, 64, 47, 1, 1.0, 1.0, p, 10, p, p, 1 << 20, buf, 256) == 3  # npy odd
    assert b"unsupported" in buf.value
    assert cl(None, p, None, 64, 64, 1, 1.0, 1.0, p, 2000, p, p, 1 << 20, buf, 256) == 1
    assert b"nedges" in buf.value
    assert cl(None, p, None, 64, 64, 1, 1.0, 1.0, p, 10, p, p, 16, buf, 256) == 1
    assert b"workspace too small" in buf.value


def test_sht_ring_entry_points_check_limits(lib):
    buf = ctypes.create_string_buffer(256)
    p = ctypes.c_void_p(256)
    for name in ("jfli_sht_ring_analysis", "jfli_sht_ring_synthesis"):
        fn = _bound(lib, name)
        assert fn(None, p, 8192, 100, p, buf, 256) == 1 and b"nside" in buf.value
        assert fn(None, p, 64, 9000, p, buf, 256) == 1 and b"lmax" in buf.value
        assert fn(None, None, 64, 100, p, buf, 256) == 1 and b"null pointer" in buf.value
