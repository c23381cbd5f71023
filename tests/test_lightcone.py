"""Light-cone drift (DriftInterp, reference pm/interp.py:110-121, 254-318) against the
FP64 oracle, and the nb_shells light cone painted with it."""

import numpy as np
import pytest
import torch

import jfli_b200 as jf
from jfli_b200 import cosmology as cj
from jfli_b200 import ops
from oracle import healpix as oh
from oracle import pm as opm
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _state(n, seed, amp=2.0):
    rng = np.random.default_rng(seed)
    disp = (amp * rng.standard_normal((n, n, n, 3))).astype(np.float32)
    vel = (0.8 * rng.standard_normal((n, n, n, 3))).astype(np.float32)
    return disp, vel


@pytest.mark.parametrize("t", [0.35, 0.8])
def test_lightcone_drift_matches_oracle(cosmo, t):
    n, L = 64, 256.0
    disp, vel = _state(n, 5)
    obs = (128.0, 128.0, 128.0)
    out = ops.lightcone_drift_array(torch.as_tensor(disp, device="cuda"), torch.as_tensor(vel, device="cuda"), t,
                                    cosmo, (L, L, L), obs).cpu().numpy()
    ref = opm.lightcone_drift(disp, vel, (L, L, L), obs, t, lambda r: cj.a_of_chi(cosmo, r),
                              lambda a: cj.Gp(cosmo, a), lambda a: cj.dGfa(cosmo, a))
    moved = np.abs(ref - opm.lightcone_drift(disp, 0 * vel, (L, L, L), obs, t, lambda r: cj.a_of_chi(cosmo, r),
                                             lambda a: cj.Gp(cosmo, a), lambda a: cj.dGfa(cosmo, a))).max()
    err = np.abs(out - ref).max()
    print(f"t={t}: max drift {moved:.3f} Mpc/h, max |GPU - oracle| {err:.2e} Mpc/h")
    assert moved > 0.1
    assert err < 2e-4 * L / 256 * 4  # FP32 positions of a 256 Mpc/h box (ulp 3e-5) plus table rounding


def test_drift_interp_shell_matches_oracle(cosmo):
    """DriftInterp.paint (spherical, bilinear) of one particle state against the oracle
    drift + HEALPix painter."""
    n, L, nside = 32, 200.0, 16
    disp, vel = _state(n, 6, amp=1.5)
    noise = jf.white_noise(1, (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo, nside=nside)
    dx, p = jf.lpt(cosmo, ic, ts=0.5, order=1)
    dx = dx.replace(array=torch.as_tensor(disp, device="cuda"))
    p = p.replace(array=torch.as_tensor(vel, device="cuda"))
    t, rc, wd = 0.5, 70.0, 40.0
    interp = jf.DriftInterp(painting=jf.PaintingOptions(target="spherical")).update_geometry(
        np.array([t]), np.array([rc]), np.array([wd]), 200.0)
    state = interp.init()
    out = interp.paint(state, t, (dx, p), cosmo).array.cpu().numpy()
    obs = dx.observer_position_mpc
    pos = opm.lightcone_drift(disp, vel, (L, L, L), obs, t, lambda r: cj.a_of_chi(cosmo, r),
                              lambda a: cj.Gp(cosmo, a), lambda a: cj.dGfa(cosmo, a))
    rmin, rmax = rc - wd / 2, rc + wd / 2
    vol = (4 * np.pi / (12 * nside * nside)) * (rmax**3 - rmin**3) / 3
    ref = oh.paint_shell(pos, obs, rmin, rmax, nside, "bilinear") / vol
    err = rel_l2(out, ref)
    print(f"shell map rel L2 vs oracle {err:.2e}; particles in shell {ref.sum() * vol:.0f}")
    assert ref.sum() > 0
    assert err < 1e-3


def test_nbody_drift_interp_lightcone(cosmo):
    n, L, nside = 32, 200.0, 16
    noise = jf.white_noise(1, (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo, nside=nside)
    dx, p = jf.lpt(cosmo, ic, ts=0.1, order=2)
    maps = {}
    for name, kernel in (("drift", jf.DriftInterp), ("plain", jf.NoInterp)):
        solver = jf.EfficientDriftDoubleKick(interp_kernel=kernel(painting=jf.PaintingOptions(target="spherical")))
        lc = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=0.1, nb_shells=4, solver=solver)
        maps[name] = lc.array.cpu().numpy()
    a, b = maps["drift"], maps["plain"]
    assert a.shape == b.shape == (4, 12 * nside * nside)
    assert np.isfinite(a).all() and (a >= 0).all()
    # the drift moves particles by a fraction of a shell width: maps differ, totals are close
    d = rel_l2(a, b)
    tot = abs(a.sum() / b.sum() - 1)
    print(f"drift vs no drift: map rel L2 {d:.3e}, total {tot:.3e}")
    assert d > 1e-4
    assert tot < 0.1


def test_angular_cl_of_gpu_shell_matches_oracle_shell(cosmo):
    """C_ell (host SHT) of a GPU-painted HEALPix shell against the same SHT of the
    oracle-painted shell: per-multipole relative difference below 1e-4."""
    from jfli_b200 import sht

    n, L, nside = 64, 400.0, 32
    disp, _ = _state(n, 9, amp=1.0)
    obs = (200.0, 200.0, 200.0)
    rmin, rmax = 80.0, 140.0
    gpu = ops.healpix_paint(torch.as_tensor(disp, device="cuda"), nside, (L, L, L), obs, rmin, rmax).cpu().numpy()
    g = opm.grid((n, n, n))
    pos = (g + disp.astype(np.float64)) * (L / n)
    ref = oh.paint_shell(pos, obs, rmin, rmax, nside, "bilinear")
    lmax = 2 * nside
    cg = sht.anafast(gpu / gpu.mean() - 1, lmax, engine="host")
    cr = sht.anafast(ref / ref.mean() - 1, lmax, engine="host")
    rel = np.abs(cg[1:] / cr[1:] - 1).max()
    print(f"C_ell GPU shell vs oracle shell: max per-ell rel {rel:.2e}")
    assert rel < 1e-4
    dens = jf.SphericalDensity(array=torch.as_tensor(gpu, device="cuda"), mesh_size=(n,) * 3, box_size=(L,) * 3,
                               nside=nside)
    np.testing.assert_allclose(dens.angular_cl(lmax=lmax), sht.anafast(gpu, lmax, engine="host"), rtol=1e-9)
