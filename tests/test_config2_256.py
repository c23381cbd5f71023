"""The 256^3 configuration the headline metric is quoted on, against the FP64 and FP32
oracle runs of tests/golden/config2_256.npz (written by tests/golden/make_config2.py):
256^3 particles on a 256^3 mesh, box 1000 Mpc/h, seeded white noise, 2LPT to a = 0.1,
EfficientDriftDoubleKick with dt0 = 0.9/40 (reference pm/nbody.py:116-169,
pm/solvers.py:124-202), P(k) in 32 log bins (_src/power/_compute.py:68-119), and the
light cone of 4 equal-width HEALPix shells at nside 256, bilinear
(_src/fields/_painting.py:249-348), with C_ell of each shell (_compute.py:175-191).

Every error is stated against the FP64 oracle, beside the FP32 oracle's own distance from
FP64 (the precision floor of any FP32 implementation; at this mesh and step count it is
below 1e-6 for the fields and P(k), so the trajectory does not amplify FP32 rounding past
the bounds). Bounds, all against FP64:
* fields -- 2LPT displacements and momenta, forces of the 2LPT particles, the density after
  40 steps (8^3-block sums and a full-resolution plane), final displacements and momenta:
  1e-5 relative L2;
* P(k): 1e-4 per bin (the bins that hold modes; an empty bin is NaN, 0/0, as in the
  reference);
* C_ell of each shell's overdensity: 1e-4 per band of 8 multipoles, 5e-4 per multipole;
* shell maps: 1e-5 relative L2 averaged to nside 4, and printed at nside 16.
A shell map is a count of particles inside r_min < r <= r_max: a particle that a 1e-6
relative position difference moves across a shell edge moves one particle's weight in or
out of a pixel. At the 312.5 Mpc/h shell one such particle is ~1e-3 of an nside-16 pixel's
count (2e-5 relative L2 over the map) and 1e-4 of the power at the highest multipoles;
averaging over 8 multipoles or to nside 4 brings it under the bounds. The bounds hold the
fields themselves to the FP64 trajectory.
"""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch

import jfli_b200 as jf
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "config2_256.npz")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(GOLDEN):
        pytest.fail("tests/golden/config2_256.npz is missing: run tests/golden/make_config2.py")
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="module")
def lpt_state(ref):
    n, L = int(ref["mesh"]), float(ref["box"])
    cosmo = jf.Planck18()
    noise = jf.white_noise(int(ref["seed"]), (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo, nside=int(ref["nside"]))
    dx, p = jf.lpt(cosmo, ic, ts=0.1, order=2)
    return cosmo, dx, p


def _sample(t, idx):
    return t.reshape(-1, 3)[torch.as_tensor(idx, device=t.device)].double().cpu().numpy()


def test_config2_lpt_and_forces(ref, lpt_state):
    from jfli_b200 import ops

    _, dx, p = lpt_state
    idx = ref["sample"]
    e_dx = rel_l2(_sample(dx.array, idx), ref["lpt_dx_f64"])
    e_p = rel_l2(_sample(p.array, idx), ref["lpt_p_f64"])
    f = ops.pm_forces(dx.array.contiguous())
    e_f = rel_l2(_sample(f, idx), ref["force_lpt_f64"])
    print(f"2LPT at 256^3 vs FP64 oracle: displacement {e_dx:.2e}, momentum {e_p:.2e}, forces {e_f:.2e} "
          f"(FP32 oracle displacement gap {float(ref['gap_lpt_dx_f32']):.2e})")
    assert e_dx < 1e-5 and e_p < 1e-5 and e_f < 1e-5


def test_config2_density_pk_and_state(ref, lpt_state):
    cosmo, dx, p = lpt_state
    n, L = int(ref["mesh"]), float(ref["box"])
    solver = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="density")))
    rho, run = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=float(ref["dt0"]), solver=solver, return_state=True)
    assert run.steps == int(ref["steps"]) == 40
    ps = rho.power(kedges=ref["kedges"])
    pk = ps.array.double().cpu().numpy()
    ok = ref["pk_f64"] > 0  # bins holding modes
    assert np.all(~np.isfinite(pk[~ok]) | (pk[~ok] == 0))
    pk_err = np.abs(pk[ok] / ref["pk_f64"][ok] - 1)
    pk_err32 = np.abs(pk[ok] / ref["pk_f32"][ok] - 1)
    gap_pk = float(ref["gap_pk_f32"])
    r = rho.array.double()
    coarse = r.reshape(32, 8, 32, 8, 32, 8).sum(dim=(1, 3, 5)).cpu().numpy()
    plane = r[n // 2].cpu().numpy()
    e_coarse = rel_l2(coarse, ref["rho_coarse_f64"])
    e_plane = rel_l2(plane, ref["rho_plane_f64"])
    g_coarse = rel_l2(ref["rho_coarse_f32"], ref["rho_coarse_f64"])
    g_plane = rel_l2(ref["rho_plane_f32"], ref["rho_plane_f64"])
    e_dx = rel_l2(_sample(run.disp, ref["sample"]), ref["dx_f64"])
    e_p = rel_l2(_sample(run.vel, ref["sample"]), ref["p_f64"])
    print(f"256^3, 40 steps, vs FP64 oracle: P(k) max {pk_err.max():.2e} per bin (vs FP32 oracle "
          f"{pk_err32.max():.2e}; FP32-vs-FP64 oracle gap {gap_pk:.2e}); density 8^3 blocks {e_coarse:.2e} "
          f"(gap {g_coarse:.2e}), plane {e_plane:.2e} (gap {g_plane:.2e}, full-field gap "
          f"{float(ref['gap_rho_f32']):.2e}); displacements {e_dx:.2e}, momenta {e_p:.2e} (full-field "
          f"displacement gap {float(ref['gap_dx_f32']):.2e})")
    assert pk_err.max() < 1e-4
    assert e_coarse < 1e-5 and e_plane < 1e-5
    assert e_dx < 1e-5 and e_p < 1e-5


def test_config2_shells_and_cl(ref, lpt_state):
    from jfli_b200 import sht
    from jfli_b200.healpix_order import ud_grade

    cosmo, dx, p = lpt_state
    solver = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(
        painting=jf.PaintingOptions(target="spherical", scheme="bilinear")))
    shells, run = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=float(ref["dt0"]), nb_shells=4, solver=solver,
                           return_state=True)
    assert run.steps == int(ref["shell_steps"])
    np.testing.assert_allclose(np.asarray(shells.comoving_centers), ref["shell_centers"], rtol=1e-12)
    maps = shells.array.double()
    nside, lmax = int(ref["nside"]), 3 * int(ref["nside"]) - 1
    coarse_t = ud_grade(maps, int(ref["nside_coarse"]))
    coarse = coarse_t.cpu().numpy()
    c4 = ud_grade(coarse_t, 4).cpu().numpy()
    r4 = ud_grade(torch.as_tensor(ref["shells_coarse_f64"]), 4).numpy()
    for s in range(4):
        m = maps[s]
        cl = sht.anafast(m / m.mean() - 1.0, lmax).cpu().numpy()
        c64, c32 = ref["cl_f64"][s], ref["cl_f32"][s]
        e_cl = np.abs(cl[1:] / c64[1:] - 1)
        g_cl = np.abs(c32[1:] / c64[1:] - 1)
        nb = (lmax // 8) * 8
        band = lambda c: c[1:nb + 1].reshape(-1, 8).mean(axis=1)
        e_band = np.abs(band(cl) / band(c64) - 1)
        e_map = rel_l2(coarse[s], ref["shells_coarse_f64"][s])
        e_map4 = rel_l2(c4[s], r4[s])
        g_map = rel_l2(ref["shells_coarse_f32"][s], ref["shells_coarse_f64"][s])
        e_sum = abs(float(m.sum()) / float(ref["shell_sum_f64"][s]) - 1)
        print(f"shell {s} (centre {ref['shell_centers'][s]:.1f} Mpc/h) vs FP64 oracle: C_ell max {e_cl.max():.2e} "
              f"per multipole, {e_band.max():.2e} per band of 8 (FP32 oracle {g_cl.max():.2e}); map at nside "
              f"{int(ref['nside_coarse'])} {e_map:.2e} (gap {g_map:.2e}), at nside 4 {e_map4:.2e}; full-map gap "
              f"{float(ref['gap_shells_f32'][s]):.2e}; total {e_sum:.2e}")
        assert e_band.max() < 1e-4 and e_cl.max() < 5e-4
        assert e_map4 < 1e-5
