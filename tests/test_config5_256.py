"""The large light-cone chain at 256^3 against the FP64 and FP32 oracle runs of
tests/golden/config5_256.npz (written by tests/golden/make_config5.py): 2LPT, 60
EfficientDriftDoubleKick steps with the PGD correction (pm/correction.py:157-202), 16
OnionTiler shells to 1500 Mpc/h at nside 256 (pm/interp.py:321-504), Born convergence for a
tophat n(z) on 0 < z < 1 (_src/lensing/_born.py:100-130) and C_ell
(_src/power/_compute.py:175-191), through jfli_b200.pipelines.lightcone_convergence with
the oracle's white noise and rotation draw.

Every error is stated against the FP64 oracle, beside the FP32 oracle's own distance from
FP64. Bounds: C_ell of the convergence map and of shells 3, 8 and 15 within 1e-4 per
multipole where the FP64 spectrum is above 1e-3 of its largest value, and everywhere within
2x the FP32 oracle's gap + 1e-4; the maps (averaged to nside 16) and the shells' totals as
close to FP64 as the FP32 oracle (2x its gap + 1e-6).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import jfli_b200 as jf
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "config5_256.npz")


def _cl_errors(cl, c64, c32):
    big = c64[1:] > 1e-3 * c64[1:].max()
    e = np.abs(cl[1:] / c64[1:] - 1)
    g = np.abs(c32[1:] / c64[1:] - 1)
    return e, g, big


def test_config5_lightcone_chain(cosmo):
    from jfli_b200 import pipelines, sht
    from jfli_b200.healpix_order import ud_grade

    if not os.path.exists(GOLDEN):
        pytest.fail("tests/golden/config5_256.npz is missing: run tests/golden/make_config5.py")
    ref = dict(np.load(GOLDEN))
    n, L, nside = int(ref["mesh"]), float(ref["box"]), int(ref["nside"])
    noise = np.random.default_rng(int(ref["seed"])).standard_normal((n, n, n)).astype(np.float32)
    rot = np.random.default_rng(42).integers(0, 47, 27)
    res = pipelines.lightcone_convergence(cosmo, mesh=n, box=L, seed=0, nb_shells=16, nside=nside,
                                          nz_shear=[jf.tophat_nz(0.0, 1.0)], steps=60, pgd=tuple(ref["pgd"]),
                                          max_z=1.0, tiler="onion", noise=noise, rotation_indices=rot)
    assert res.steps == int(ref["steps"])
    np.testing.assert_allclose(np.asarray(res.shells.comoving_centers), ref["shell_centers"], rtol=1e-12)
    lmax, nc = int(ref["lmax"]), int(ref["nside_coarse"])
    maps = res.shells.array.double()
    kappa = res.kappa.array[0].double()
    # convergence map
    kcl = sht.anafast(kappa, lmax).cpu().numpy()
    e, g, big = _cl_errors(kcl, ref["kappa_cl_f64"], ref["kappa_cl_f32"])
    e_map = rel_l2(ud_grade(kappa, nc).cpu().numpy(), ref["kappa_coarse_f64"])
    g_map = rel_l2(ref["kappa_coarse_f32"], ref["kappa_coarse_f64"])
    rms = float(kappa.std())
    print(f"kappa vs FP64 oracle: C_ell max {e[big].max():.2e} over the {big.sum()} multipoles above 1e-3 of the "
          f"peak, {e.max():.2e} over all (FP32 oracle {g.max():.2e}); map at nside {nc} {e_map:.2e} (gap "
          f"{g_map:.2e}; full-map gap {float(ref['gap_kappa_f32']):.2e}); rms {rms:.4e} vs "
          f"{float(ref['kappa_rms_f64']):.4e}")
    assert e[big].max() < 1e-4 and np.all(e < 2 * g + 1e-4)
    assert e_map < 2 * g_map + 1e-6
    # shells
    coarse = ud_grade(maps, nc).cpu().numpy()
    sums = maps.sum(dim=1).cpu().numpy()
    e_sum = np.abs(sums / ref["shell_sum_f64"] - 1)
    g_sum = np.abs(ref["shell_sum_f32"] / ref["shell_sum_f64"] - 1)
    for s in range(16):
        e_s = rel_l2(coarse[s], ref["shells_coarse_f64"][s])
        g_s = rel_l2(ref["shells_coarse_f32"][s], ref["shells_coarse_f64"][s])
        print(f"shell {s} ({ref['shell_centers'][s]:.0f} Mpc/h): map at nside {nc} {e_s:.2e} (gap {g_s:.2e}; "
              f"full-map gap {float(ref['gap_shells_f32'][s]):.2e}), total {e_sum[s]:.2e} (gap {g_sum[s]:.2e})")
        assert e_s < 2 * g_s + 1e-6
        assert e_sum[s] < 2 * g_sum[s] + 1e-6
    for row, s in enumerate(ref["cl_shells"]):
        m = maps[int(s)]
        cl = sht.anafast(m / m.mean() - 1.0, lmax).cpu().numpy()
        e, g, big = _cl_errors(cl, ref["shell_cl_f64"][row], ref["shell_cl_f32"][row])
        print(f"shell {int(s)} C_ell vs FP64 oracle: max {e[big].max():.2e} (above 1e-3 of the peak), {e.max():.2e} "
              f"over all (FP32 oracle {g.max():.2e})")
        assert e[big].max() < 1e-4 and np.all(e < 2 * g + 1e-4)
