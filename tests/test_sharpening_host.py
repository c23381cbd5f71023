"""Host logic of SharpeningKernel (no GPU): the boost factors the solvers hand to the
combined potential, and the per-segment slices of the reversible tables."""

from __future__ import annotations

import math

import numpy as np


def test_bare_drift_is_the_full_drift_without_its_prefactor():
    """EfficientDriftDoubleKick.bare_drift is (Gp(t1) - Gp(t0)) / gp(sqrt(t0 t1)), the
    factor the reference's step hands to the correction (pm/solvers.py:164-175); the step's
    drift is it times 1 / (a^3 E(a)) at a = sqrt(t0 t1)."""
    import jfli_b200 as jf
    from jfli_b200 import cosmology as cj
    from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK

    cosmo = jf.Planck18()
    for t0, t1 in [(0.1, 0.25), (0.4, 0.55), (0.85, 1.0)]:
        ac = math.sqrt(t0 * t1)
        c = EDK.step_coefficients(cosmo, t0, t1, 0.15)
        bare = float(EDK.bare_drift(cosmo, t0, t1))
        assert abs(bare / (ac**3 * cj.E(cosmo, ac)) - c.drift) <= 1e-12 * abs(c.drift)
    arr = EDK.bare_drift(cosmo, [0.1, 0.4], [0.25, 0.55])
    assert np.allclose(arr, [float(EDK.bare_drift(cosmo, 0.1, 0.25)), float(EDK.bare_drift(cosmo, 0.4, 0.55))],
                       rtol=1e-14)


def test_boost_factor_and_reversible_step_boost():
    """The boost is alpha over the drift factor handed over; ReversibleDoubleKickDrift hands
    its full drift factor (pm/solvers.py:305-316), and without a SharpeningKernel its boost
    is 0."""
    import jfli_b200 as jf

    sk = jf.SharpeningKernel(alpha=0.3, kl=0.3, ks=1.0)
    assert sk.reversible
    assert abs(sk.boost(0.25) - 1.2) < 1e-15
    cosmo = jf.Planck18()
    interp = jf.NoInterp(painting=jf.PaintingOptions(target="density"))
    solver = jf.ReversibleDoubleKickDrift(interp_kernel=interp, pgd_kernel=sk)
    c = solver.step_coefficients(cosmo, 0.4, 0.55, 0.15, 0.1)
    assert abs(solver._boost(c) - 0.3 / c.drift) < 1e-12
    assert jf.ReversibleDoubleKickDrift(interp_kernel=interp)._boost(c) == 0.0


def test_forward_tables_sharpen_slice():
    """ForwardTables.sharpen_slice gives the boosts of a segment of steps with the scales."""
    from jfli_b200.pm.adjoint import ForwardTables

    t = ForwardTables(ktab=None, ptab=None, lpt=None, kicks=np.arange(5.0), drifts=np.ones(5),
                      sharpen=(np.array([0.0, 1.0, 2.0, 3.0, 4.0]), 0.3, 1.0))
    b, kl, ks = t.sharpen_slice(1, 4)
    assert np.array_equal(b, [1.0, 2.0, 3.0]) and (kl, ks) == (0.3, 1.0)
    plain = ForwardTables(ktab=None, ptab=None, lpt=None, kicks=np.arange(5.0), drifts=np.ones(5))
    assert plain.sharpen_slice(0, 2) is None
