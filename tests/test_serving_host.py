"""Host-side logic of the serving engine: request stream, per-request tables, slot budget."""

import numpy as np
import pytest

from jfli_b200 import cosmology as cj
from jfli_b200 import serving
from jfli_b200.pm.integrate import time_events
from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK


def test_stream_is_seeded_and_in_range():
    a = serving.poisson_stream(512, rate=100.0, seed=3)
    b = serving.poisson_stream(512, rate=100.0, seed=3)
    assert a == b
    assert {r.mesh for r in a} == {64, 96, 128, 192}
    assert all(r.box == 4.0 * r.mesh for r in a)
    assert all(0.20 <= r.omega_c <= 0.35 and 0.70 <= r.sigma8 <= 0.90 for r in a)
    assert all(10 <= r.steps <= 40 for r in a)
    assert [r.seed for r in a] == list(range(512))
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) >= 0)
    # mean inter-arrival time of a rate-100 Poisson process
    assert abs(np.mean(np.diff(arr)) - 0.01) < 0.002
    frac = np.mean([r.want_grad for r in a])
    assert 0.18 < frac < 0.32


def test_stream_all_at_once():
    a = serving.poisson_stream(16, rate=0.0)
    assert all(r.arrival == 0.0 for r in a)


@pytest.mark.parametrize("steps", [10, 17, 23, 40])
def test_prepare_matches_stepwise_coefficients(steps):
    req = serving.ForwardRequest(rid=0, mesh=64, box=256.0, omega_c=0.3, sigma8=0.75, steps=steps, seed=1)
    prep = serving.prepare(req)
    c = cj.Planck18(Omega_c=0.3, sigma8=0.75)
    dt0 = (1.0 - serving.A_INIT) / steps
    ev = [e for e in time_events(serving.A_INIT, [1.0], dt0) if e[0] == "step"]
    assert len(ev) == steps == len(prep["kicks"]) == len(prep["drifts"])
    for i, (_, ta, tb) in enumerate(ev):
        sc = EDK.step_coefficients(c, ta, tb, dt0)
        assert prep["kicks"][i] == pytest.approx(sc.kick, rel=1e-12)
        assert prep["drifts"][i] == pytest.approx(sc.drift, rel=1e-12)
    assert prep["init_kick"] == pytest.approx(EDK.init_kick(c, serving.A_INIT, serving.A_INIT + dt0), rel=1e-14)
    assert prep["kedges"].shape == (33,)
    assert prep["ktab"].dtype == np.float32 and prep["ktab"].shape == (128,)


def test_slot_capacities_respect_budget():
    caps = serving.slot_capacities((64, 96, 128, 192), 32.0, 16)
    assert caps == {64: 16, 96: 16, 128: 16, 192: 16}
    caps = serving.slot_capacities((64, 96, 128, 192), 24.0, 16)
    assert caps[64] == 16 and all(c * serving.SizeGroup.bytes_per_slot(n) <= 6e9 for n, c in caps.items())
    small = serving.slot_capacities((64, 96, 128, 192), 2.0, 16)
    assert small[192] < small[128] <= small[96] <= small[64]
    for n, cap in small.items():
        assert cap == 1 or cap * serving.SizeGroup.bytes_per_slot(n) <= 2e9 / 4
    assert serving.slot_capacities((256,), 0.001, 8) == {256: 1}
