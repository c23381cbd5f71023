"""Host logic of the tiled light-cone painters (reference pm/interp.py:31-43, 321-699):
the cube symmetries, the replica shifts, and the shell / rotation bookkeeping of
OnionTiler and TelephotoInterp. CPU only."""

import itertools

import numpy as np
import pytest

import jfli_b200 as jf
from jfli_b200.pm.interp import get_all_47_symmetries, tile_shifts


def test_47_symmetries():
    m = get_all_47_symmetries()
    assert m.shape == (47, 3, 3)
    flat = {tuple(x.ravel()) for x in m}
    assert len(flat) == 47 and tuple(np.eye(3, dtype=int).ravel()) not in flat
    for x in m:  # signed permutation matrices: orthogonal, det +-1
        assert np.array_equal(x @ x.T, np.eye(3))
        assert abs(round(np.linalg.det(x))) == 1
    # the order: sign triples outer, permutations inner, identity dropped
    assert m[0].tolist() == [[1, 0, 0], [0, 0, 1], [0, 1, 0]]
    assert m[4].tolist() == [[0, 0, 1], [0, 1, 0], [1, 0, 0]]
    assert m[5].tolist() == [[1, 0, 0], [0, 1, 0], [0, 0, -1]]
    assert m[-1].tolist() == [[0, 0, -1], [0, -1, 0], [-1, 0, 0]]


@pytest.mark.parametrize("obs", [(0.5, 0.5, 0.5), (0.0, 0.0, 0.0), (1.0, 0.3, 0.0)])
def test_tile_shifts_cover_the_observer(obs):
    L = np.array([100.0, 100.0, 100.0])
    sh = tile_shifts(obs, L)
    assert sh.shape == (27, 3)
    assert len({tuple(s) for s in sh}) == 27
    base = np.array(list(itertools.product([0, 1, -1], repeat=3)))
    for ax, f in enumerate(obs):
        want = base[:, ax] + (1 if f == 0 else (-1 if f == 1 else 0))
        assert np.array_equal(sh[:, ax], want * L[ax])


def _geometry(kernel, r_centers, widths, rmax):
    ts = np.linspace(0.3, 0.9, len(r_centers))
    return kernel.update_geometry(ts, np.asarray(r_centers, float), np.asarray(widths, float), rmax), ts


def test_telephoto_rotation_index_advances_beyond_the_box():
    with pytest.warns(UserWarning):
        k, ts = _geometry(jf.TelephotoInterp(painting=jf.PaintingOptions(target="spherical")),
                          [400.0, 250.0, 150.0, 90.0], [60.0] * 4, 100.0)
        st = k.init()
    assert st.rotations.shape == (47, 3, 3)
    rots = []
    for t in ts:
        st = k.advance(st, t)
        rots.append((st.shell_idx, st.rotation_idx))
    assert rots == [(0, 0), (1, 1), (2, 2), (3, 2)]  # 90 Mpc/h lies inside the box
    assert k.advance(st, 0.55) == st  # not a snapshot time
    back = []
    for t in ts[::-1]:
        st = k.rewind(st, t)
        back.append((st.shell_idx, st.rotation_idx))
    # rewinding the 90 Mpc/h shell: its outer edge (120) is beyond the box, so the
    # reference's rewind takes one rotation back there too
    assert back == [(2, 1), (1, 0), (0, -1), (-1, -2)]


def test_onion_tiler_rotations():
    k, _ = _geometry(jf.OnionTiler(painting=jf.PaintingOptions(target="spherical")), [300.0], [50.0], 100.0)
    st = k.init()
    idx = np.random.default_rng(42).integers(0, 47, size=27)
    assert np.array_equal(st.rotations, get_all_47_symmetries()[idx])
    given = tuple(range(27))
    k2, _ = _geometry(jf.OnionTiler(painting=jf.PaintingOptions(target="spherical"), rotation_indices=given),
                      [300.0], [50.0], 100.0)
    assert np.array_equal(k2.init().rotations, get_all_47_symmetries()[:27])
    with pytest.raises(ValueError):
        jf.OnionTiler(painting=jf.PaintingOptions(target="spherical"), rotation_indices=(47,) * 27).init()
    with pytest.raises(ValueError):
        jf.OnionTiler(painting=jf.PaintingOptions(target="density")).init()
    with pytest.raises(ValueError):
        jf.TelephotoInterp(painting=jf.PaintingOptions(target="density")).init()
    assert jf.TelephotoInterp(painting=jf.PaintingOptions(target="flat")).init().rotations.shape == (47, 3, 3)


def test_snapshot_times_match_after_fp32_rounding():
    """The time loop clips steps to the FP32 value of each snapshot time; the snapshot test
    must find those times among the FP64 shell times (which are not FP32 numbers)."""
    from jfli_b200.pm.integrate import time_events

    ts = np.array([0.4123456789012345, 0.7345678901234567, 0.9876543210987654])
    k, _ = _geometry(jf.NoInterp(painting=jf.PaintingOptions(target="spherical")), [300.0, 200.0, 100.0],
                     [100.0] * 3, 400.0)
    k = k.update_geometry(ts, k.r_centers, k.density_widths, 400.0)
    st = k.init()
    for ev in time_events(0.1, ts, 0.05):
        if ev[0] == "step":
            st = k.advance(st, ev[2])
    assert st.shell_idx == 2
