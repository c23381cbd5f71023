"""The allocation-free P(k) entry point agrees with the workspace one.

jfli_power_spectrum_noalloc exists for callers that cannot allocate device memory when
they need a power spectrum (a JAX/XLA custom-call handler in a process whose GPU memory
XLA has already reserved, or code being recorded into a CUDA graph). Its scratch is an
array compiled into the library, shared by every call, so this test makes two calls in a
row on different meshes and checks both against jfli_power_spectrum (same sums, within
the 1e-4 per-bin P(k) tolerance of the other parity tests). This file is collected last
so that a failure here stops a run only after every other test has run.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _sums(fn_name, mesh, kedges, box, use_workspace):
    from jfli_b200 import _lib

    nx, ny, nz = mesh.shape
    ne = kedges.numel()
    out = torch.full((3, ne + 1), float("nan"), dtype=torch.float64, device="cuda")
    s = _lib.stream_ptr()
    if use_workspace:
        nb = _lib.query("jfli_power_spectrum_workspace_bytes", nx, ny, nz, 1, ne)
        ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
        _lib.call(fn_name, s, _lib.ptr(mesh), _lib.ptr(kedges), ne, *box, _lib.ptr(out), _lib.ptr(ws), ws.numel(),
                  nx, ny, nz, 1)
    else:
        _lib.call(fn_name, s, _lib.ptr(mesh), _lib.ptr(kedges), ne, *box, _lib.ptr(out), nx, ny, nz, 1)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _pk(sums):
    cnt = np.where(sums[1] > 0, sums[1], 1.0)
    return (sums[0] / cnt)[1:-1], sums[1][1:-1]


def test_noalloc_matches_workspace_entry_point_twice_in_a_row():
    rng = np.random.default_rng(11)
    cases = [((64, 64, 64), 256.0), ((128, 128, 128), 500.0)]
    for (shape, L) in cases:
        mesh = torch.as_tensor((1.0 + 0.3 * rng.standard_normal(shape)).astype(np.float32), device="cuda")
        n = shape[0]
        kedges = torch.as_tensor(np.geomspace(2 * np.pi / L * (1 - 1e-6), np.pi * n / L, 33).astype(np.float32),
                                 device="cuda")
        box = (L, L, L)
        ref = _sums("jfli_power_spectrum", mesh, kedges, box, True)
        got = _sums("jfli_power_spectrum_noalloc", mesh, kedges, box, False)
        pk_ref, cnt_ref = _pk(ref)
        pk_got, cnt_got = _pk(got)
        np.testing.assert_array_equal(cnt_got, cnt_ref)
        ok = pk_ref > 0
        assert np.abs(pk_got[ok] / pk_ref[ok] - 1).max() < 1e-4


def test_noalloc_rejects_meshes_beyond_its_scratch():
    from jfli_b200 import _lib

    buf = ctypes.create_string_buffer(512)
    lib = _lib.load()
    rc = lib.jfli_power_spectrum_noalloc(None, ctypes.c_void_p(256), ctypes.c_void_p(256), 32, 100.0, 100.0, 100.0,
                                         ctypes.c_void_p(256), 192, 192, 192, 1, buf, 512)
    assert rc == 3 and b"scratch" in buf.value
