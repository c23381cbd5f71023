"""ops.device_table: small host tables cached on a device by content (CPU target here)."""

import numpy as np

from jfli_b200 import ops


def test_same_content_same_tensor_and_lru_bound():
    a = np.linspace(0.1, 1.0, 33)
    t1 = ops.device_table(a, "cpu")
    t2 = ops.device_table(a.copy(), "cpu")
    assert t1 is t2 and t1.dtype.is_floating_point and t1.shape == (33,)
    np.testing.assert_allclose(t1.numpy(), a.astype(np.float32))
    t3 = ops.device_table(a * 2, "cpu")
    assert t3 is not t1
    for i in range(80):
        ops.device_table(np.full(4, float(i)), "cpu")
    assert len(ops._TABLES) <= 64
    assert ops.device_table(a, "cpu") is not t1  # evicted, uploaded again
