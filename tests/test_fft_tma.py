"""The TMA-staged x pass (cp.async.bulk.tensor load and store of each pencil tile) against
the register x pass: the same Poisson potential over shapes that take one box per tile,
several boxes (x length 512), partial last tiles, a batch, and a shape whose plane stride
is not a multiple of 16 bytes (it keeps the register pass)."""

import ctypes

import pytest
import torch

from jfli_b200 import ops
from jfli_b200._lib import call
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _status(reset=True):
    v = ctypes.c_uint(0)
    call("jfli_device_status", ctypes.addressof(v), int(reset))
    return v.value


@pytest.mark.parametrize("shape", [(32, 32, 32), (64, 48, 96), (128, 128, 128), (192, 192, 192), (256, 64, 64),
                                   (512, 8, 16), (384, 8, 16), (24, 3, 4), (96, 32, 24)])
def test_tma_x_pass_matches_register_pass(shape):
    g = torch.Generator(device="cuda").manual_seed(sum(shape))
    rho = 1.0 + 0.3 * torch.randn(shape, device="cuda", generator=g)
    _status()
    try:
        call("jfli_set_fft_x_pass", 0)
        ref = ops.poisson_potential(rho, 1.0).clone()
        call("jfli_set_fft_x_pass", 1)
        out = ops.poisson_potential(rho, 1.0).clone()
    finally:
        call("jfli_set_fft_x_pass", 0)
    torch.cuda.synchronize()
    err = rel_l2(out.cpu().numpy(), ref.cpu().numpy())
    print(f"{shape}: TMA vs register x pass rel L2 {err:.2e}")
    assert _status() == 0
    assert err < 1e-6


def test_tma_x_pass_batched_and_forces():
    """A batch of two meshes (the tensor map's third dimension) and the force meshes built on it."""
    shape = (2, 64, 64, 64)
    g = torch.Generator(device="cuda").manual_seed(3)
    rho = 1.0 + 0.3 * torch.randn(shape, device="cuda", generator=g)
    try:
        call("jfli_set_fft_x_pass", 0)
        ref = ops.poisson_force(rho.clone(), 1.0).clone()
        call("jfli_set_fft_x_pass", 1)
        out = ops.poisson_force(rho.clone(), 1.0).clone()
    finally:
        call("jfli_set_fft_x_pass", 0)
    assert _status() == 0
    assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) < 1e-6
