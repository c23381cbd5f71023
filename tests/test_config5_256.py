"""The large light-cone chain at 256^3 against the FP64 and FP32 oracle runs of
tests/golden/config5_256.npz (written by tests/golden/make_config5.py): 2LPT, 60
EfficientDriftDoubleKick steps with the PGD correction (pm/correction.py:157-202), 16
OnionTiler shells to 1500 Mpc/h at nside 256 (pm/interp.py:321-504), Born convergence for a
tophat n(z) on 0 < z < 1 (_src/lensing/_born.py:100-130) and C_ell
(_src/power/_compute.py:175-191), through jfli_b200.pipelines.lightcone_convergence with
the oracle's white noise and rotation draw.

Every error is stated against the FP64 oracle, beside the FP32 oracle's own distance from
FP64. Bounds: C_ell of the convergence map and of shells 3, 8 and 15 within 1e-4 per band
of 8 multipoles and 5e-4 per multipole (or 2x the FP32 oracle's own error where that is
larger); the shell maps averaged to nside 4 within 1e-5 relative L2 (or 2x the FP32
oracle's gap), printed at nside 16; the shells' totals within 1e-5; the convergence map
averaged to nside 4 within 2e-5 (or 2x the FP32 oracle's gap). A shell counts particles
between two radii, so a particle that rounding moves across an edge moves its whole
weight: the bands and the coarse maps average that out, the per-multipole and nside-16
figures show it. The convergence map's large scales are a small residual of all sixteen
shells (its rms at nside 4 is a seventh of the full map's), so one such particle moves it
by about 1e-5 at nside 4; its bound allows two.
"""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch

import jfli_b200 as jf
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "config5_256.npz")


def _band(c, lmax):
    nb = (lmax // 8) * 8
    return c[1:nb + 1].reshape(-1, 8).mean(axis=1)


def _check_cl(label, cl, c64, c32, lmax, failures):
    e = np.abs(cl[1:] / c64[1:] - 1)
    g = np.abs(c32[1:] / c64[1:] - 1)
    eb = np.abs(_band(cl, lmax) / _band(c64, lmax) - 1)
    gb = np.abs(_band(c32, lmax) / _band(c64, lmax) - 1)
    print(f"{label} C_ell vs FP64 oracle: max {e.max():.2e} per multipole, {eb.max():.2e} per band of 8 (FP32 "
          f"oracle {g.max():.2e}, {gb.max():.2e})")
    if not (eb.max() < max(1e-4, 2 * gb.max()) and e.max() < max(5e-4, 2 * g.max())):
        failures.append(f"{label} C_ell")


def _coarse4(m):
    from jfli_b200.healpix_order import ud_grade

    return ud_grade(torch.as_tensor(np.asarray(m, np.float64)), 4).numpy()


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
    failures = []  # every figure is printed before the test fails on any of them
    maps = res.shells.array.double()
    kappa = res.kappa.array[0].double()
    # convergence map
    kcl = sht.anafast(kappa, lmax).cpu().numpy()
    _check_cl("kappa", kcl, ref["kappa_cl_f64"], ref["kappa_cl_f32"], lmax, failures)
    kc = ud_grade(kappa, nc).cpu().numpy()
    e_map = rel_l2(kc, ref["kappa_coarse_f64"])
    e4 = rel_l2(_coarse4(kc), _coarse4(ref["kappa_coarse_f64"]))
    g4 = rel_l2(_coarse4(ref["kappa_coarse_f32"]), _coarse4(ref["kappa_coarse_f64"]))
    rms = float(kappa.std())
    print(f"kappa map vs FP64 oracle: at nside {nc} {e_map:.2e}, at nside 4 {e4:.2e} (gap {g4:.2e}; full-map gap "
          f"{float(ref['gap_kappa_f32']):.2e}); rms {rms:.4e} vs {float(ref['kappa_rms_f64']):.4e}")
    k64 = ref["kappa_coarse_f64"]
    print(f"kappa mean {float(kappa.mean()):.3e}; coarse-map projection on the FP64 one {kc @ k64 / (k64 @ k64):.8f}")
    if not e4 < max(2e-5, 2 * g4):
        failures.append("kappa map")
    # shells
    coarse = ud_grade(maps, nc).cpu().numpy()
    sums = maps.sum(dim=1).cpu().numpy()
    e_sum = np.abs(sums / ref["shell_sum_f64"] - 1)
    for s in range(16):
        e_s = rel_l2(coarse[s], ref["shells_coarse_f64"][s])
        e4 = rel_l2(_coarse4(coarse[s]), _coarse4(ref["shells_coarse_f64"][s]))
        g4 = rel_l2(_coarse4(ref["shells_coarse_f32"][s]), _coarse4(ref["shells_coarse_f64"][s]))
        print(f"shell {s} ({ref['shell_centers'][s]:.0f} Mpc/h): map at nside {nc} {e_s:.2e}, at nside 4 {e4:.2e} "
              f"(gap {g4:.2e}; full-map gap {float(ref['gap_shells_f32'][s]):.2e}), total {e_sum[s]:.2e}")
        if not (e4 < max(1e-5, 2 * g4) and e_sum[s] < 1e-5):
            failures.append(f"shell {s} map")
    for row, s in enumerate(ref["cl_shells"]):
        m = maps[int(s)]
        cl = sht.anafast(m / m.mean() - 1.0, lmax).cpu().numpy()
        _check_cl(f"shell {int(s)}", cl, ref["shell_cl_f64"][row], ref["shell_cl_f32"][row], lmax, failures)
    assert not failures, failures
