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
    """C_ell (oracle SHT) of a GPU-painted HEALPix shell against the same SHT of the
    oracle-painted shell: per-multipole relative difference below 1e-4; and the library's
    angular_cl (GPU SHT) of the GPU shell against the oracle SHT of it."""
    from oracle import sht as osht

    n, L, nside = 64, 400.0, 32
    disp, _ = _state(n, 9, amp=1.0)
    obs = (200.0, 200.0, 200.0)
    rmin, rmax = 80.0, 140.0
    gpu = ops.healpix_paint(torch.as_tensor(disp, device="cuda"), nside, (L, L, L), obs, rmin, rmax).cpu().numpy()
    g = opm.grid((n, n, n))
    pos = (g + disp.astype(np.float64)) * (L / n)
    ref = oh.paint_shell(pos, obs, rmin, rmax, nside, "bilinear")
    lmax = 2 * nside
    cg = osht.anafast(gpu / gpu.mean() - 1, lmax)
    cr = osht.anafast(ref / ref.mean() - 1, lmax)
    rel = np.abs(cg[1:] / cr[1:] - 1).max()
    print(f"C_ell GPU shell vs oracle shell: max per-ell rel {rel:.2e}")
    assert rel < 1e-4
    dens = jf.SphericalDensity(array=torch.as_tensor(gpu, device="cuda"), mesh_size=(n,) * 3, box_size=(L,) * 3,
                               nside=nside)
    ps = dens.angular_cl(lmax=lmax)
    assert ps.array.is_cuda
    np.testing.assert_allclose(ps.array.cpu().numpy(), osht.anafast(gpu, lmax), rtol=1e-9)
    assert ps.name == "cl" and ps.wavenumber[-1] == lmax


# ------------------------------------------------------------------ tiled light cones
def _funcs(cosmo):
    return dict(a_of_chi=lambda r: cj.a_of_chi(cosmo, r), Gp=lambda a: cj.Gp(cosmo, a),
                dGfa=lambda a: cj.dGfa(cosmo, a))


@pytest.mark.parametrize("observer_frac,drift,scheme", [((0.5, 0.5, 0.5), True, "bilinear"),
                                                        ((0.5, 0.5, 0.5), False, "ngp"),
                                                        ((0.0, 0.0, 0.0), True, "bilinear"),
                                                        ((1.0, 0.25, 0.0), True, "ngp")])
def test_onion_tiled_shell_matches_oracle(cosmo, observer_frac, drift, scheme):
    """27 rotated replicas (random cube symmetries, shifts by the observer rule), each
    drifted to the light cone, painted on a shell beyond the box: GPU one-pass kernel
    against the FP64 oracle that evaluates every replica."""
    from jfli_b200.pm.interp import get_all_47_symmetries, tile_shifts

    n, L, nside = 32, 200.0, 16
    disp, vel = _state(n, 21, amp=1.5)
    obs = tuple(f * L for f in observer_frac)
    rot = get_all_47_symmetries()[np.random.default_rng(3).integers(0, 47, 27)]
    sh = tile_shifts(observer_frac, (L, L, L))
    rmax_box = L / (1 + 2 * min(min(f, 1 - f) for f in observer_frac))
    rc, wd = rmax_box + 60.0, 50.0
    t = float(cj.a_of_chi(cosmo, rc))
    v = torch.as_tensor(vel, device="cuda") if drift else None
    out = ops.healpix_paint_tiled(torch.as_tensor(disp, device="cuda"), nside, (L, L, L), obs, rc - wd / 2,
                                  rc + wd / 2, rot, sh, vel=v, t=t, cosmo=cosmo, scheme=scheme).cpu().numpy()
    ref = oh.paint_shell_tiled(disp, vel if drift else None, (L, L, L), obs, rc - wd / 2, rc + wd / 2, nside, rot, sh,
                               t=t, scheme=scheme, **_funcs(cosmo))
    err = rel_l2(out, ref)
    print(f"observer {observer_frac} drift {drift} {scheme}: weight {ref.sum():.0f}, rel L2 {err:.2e}")
    assert ref.sum() > 1000
    assert err < 1e-3


def test_telephoto_replica_matches_oracle(cosmo):
    """One rotated replica pushed along z, drifted with the distance measured as the
    reference measures it (observer-centred replica minus the observer position)."""
    from jfli_b200.pm.interp import get_all_47_symmetries

    n, L, nside = 32, 200.0, 16
    disp, vel = _state(n, 22, amp=1.5)
    obs = (100.0, 100.0, 100.0)
    R = 100.0
    rc, wd = 230.0, 40.0
    rot = get_all_47_symmetries()[[5]]
    sh = np.array([[0.0, 0.0, np.floor(rc / R) * R]])
    t = float(cj.a_of_chi(cosmo, rc))
    out = ops.healpix_paint_tiled(torch.as_tensor(disp, device="cuda"), nside, (L, L, L), obs, rc - wd / 2,
                                  rc + wd / 2, rot, sh, vel=torch.as_tensor(vel, device="cuda"), t=t, cosmo=cosmo,
                                  telephoto=True).cpu().numpy()
    ref = oh.paint_shell_tiled(disp, vel, (L, L, L), obs, rc - wd / 2, rc + wd / 2, nside, rot, sh, telephoto=True,
                               t=t, **_funcs(cosmo))
    err = rel_l2(out, ref)
    print(f"telephoto: weight {ref.sum():.0f}, rel L2 {err:.2e}")
    assert ref.sum() > 100
    assert err < 1e-3


def test_tiled_skipping_changes_nothing(cosmo):
    """Replicas skipped by the drift bound could not have reached the shell: the map with
    the computed bound equals the map with skipping disabled (an enormous bound), up to
    the order of the FP32 atomic sums."""
    from jfli_b200.pm.interp import get_all_47_symmetries, tile_shifts

    n, L, nside = 48, 300.0, 32
    disp, vel = _state(n, 23, amp=2.0)
    vel *= 4.0  # large momenta: wide drift margins
    obs = (150.0, 150.0, 150.0)
    rot = get_all_47_symmetries()[np.random.default_rng(4).integers(0, 47, 27)]
    sh = tile_shifts((0.5, 0.5, 0.5), (L, L, L))
    rc, wd = 260.0, 40.0
    t = float(cj.a_of_chi(cosmo, rc))
    args = (torch.as_tensor(disp, device="cuda"), nside, (L, L, L), obs, rc - wd / 2, rc + wd / 2, rot, sh)
    kw = dict(vel=torch.as_tensor(vel, device="cuda"), t=t, cosmo=cosmo)
    a = ops.healpix_paint_tiled(*args, **kw).double()
    b = ops.healpix_paint_tiled(*args, **kw, dbound=1e30).double()
    bound = ops.drift_bound(ops.drift_tables(cosmo), t, float(cj.Gp(cosmo, t)))
    d = float((a - b).abs().max())
    print(f"drift bound {bound:.3f}; max |skipped - full| {d:.2e} of max {float(b.max()):.2e}")
    assert torch.equal(a != 0, b != 0)
    assert d <= 1e-5 * float(b.abs().max())


def test_onion_tiler_in_nbody(cosmo):
    """nbody with OnionTiler and shells past the box: shells inside the box are the
    DriftInterp shells; shells beyond it are painted from the 27 replicas and carry the
    expected mean density."""
    n, L, nside = 32, 200.0, 16
    noise = jf.white_noise(2, (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo, nside=nside)
    dx, p = jf.lpt(cosmo, ic, ts=0.1, order=2)
    r_far = np.array([260.0, 180.0, 60.0])  # 100 Mpc/h is the largest radius the box holds
    ts = np.asarray(cj.a_of_chi(cosmo, r_far), np.float64)
    widths = np.array([60.0, 60.0, 60.0])
    maps = {}
    for name, kernel in (("onion", jf.OnionTiler), ("drift", jf.DriftInterp)):
        solver = jf.EfficientDriftDoubleKick(interp_kernel=kernel(painting=jf.PaintingOptions(target="spherical")))
        lc = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=0.1, ts=ts, density_widths=widths, solver=solver)
        maps[name] = lc.array.cpu().numpy()
    on, dr = maps["onion"], maps["drift"]
    assert on.shape == (3, 12 * nside * nside)
    # near -> far: shell 0 (60 Mpc/h) lies inside the box and uses the single-box path
    assert rel_l2(on[0], dr[0]) < 1e-6
    # every replica is the same 200 Mpc/h box, so a 60 Mpc/h shell samples the box's own
    # structures: its mean departs from the box mean by the box's variance on that scale
    # (5% measured for the 180 Mpc/h shell), not by a painting error
    mean_density = n**3 / L**3
    for s in (1, 2):
        rel = abs(on[s].mean() / mean_density - 1)
        print(f"shell {s}: mean {on[s].mean():.4e} vs {mean_density:.4e} ({rel:.2e})")
        assert rel < 0.15


def test_lightcone_shells_are_their_own_shells(cosmo):
    """Each shell of an nb_shells light cone is the paint, at that shell's radius and width,
    of the particles at that shell's time: compared with the particle snapshots of the
    same run (same snapshot times, so the same steps) painted directly. The shell times
    come from the FP64 distance table while the loop clips steps to their FP32 values."""
    n, L, nside = 64, 256.0, 32
    noise = jf.white_noise(5, (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo, nside=nside)
    dx, p = jf.lpt(cosmo, ic, ts=0.1, order=2)
    sph = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="spherical")))
    lc = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=0.9 / 20, nb_shells=4, solver=sph)
    ts = np.asarray(lc.scale_factors, np.float64)[::-1]  # far -> near: the order the loop meets them
    parts = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="particles")))
    snaps = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=0.9 / 20, ts=ts, solver=parts)
    nbar = n**3 / L**3
    for s in range(4):
        rc, wd = float(lc.comoving_centers[s]), float(lc.density_width[s])
        ref = snaps[s].paint_spherical(center=rc, density_plane_width=wd).array.double().cpu().numpy()
        got = lc.array[s].double().cpu().numpy()
        err = rel_l2(got, ref)
        print(f"shell {s} at {rc:.1f} Mpc/h (a = {float(lc.scale_factors[s]):.4f}): rel L2 {err:.2e}, "
              f"mean / nbar {got.mean() / nbar:.4f}")
        # the two runs differ only in the order of the FP32 atomic deposits, which moves a
        # few particles across the shell edges
        assert err < 2e-2
        assert abs(got.mean() / ref.mean() - 1) < 2e-3


def test_replica_positions_and_telephoto_flat_plane(cosmo):
    """One rotated, pushed replica drifted to the light cone (TelephotoInterp's transform)
    against the FP64 oracle, and the flat-sky plane TelephotoInterp paints from it beyond
    the box against the oracle positions painted flat."""
    from jfli_b200.pm.interp import get_all_47_symmetries
    from oracle import flat as of

    n, L = 32, 200.0
    disp, vel = _state(n, 24, amp=1.5)
    obs = (100.0, 100.0, 100.0)
    R, shift = get_all_47_symmetries()[7], np.array([0.0, 0.0, 200.0])
    t = float(cj.a_of_chi(cosmo, 230.0))
    got = ops.replica_positions(torch.as_tensor(disp, device="cuda"), (L, L, L), obs, R, shift,
                                vel=torch.as_tensor(vel, device="cuda"), t=t, cosmo=cosmo,
                                telephoto=True).cpu().numpy().reshape(-1, 3)
    ref = oh.replica_positions(disp, vel, (L, L, L), obs, R, shift, telephoto=True, t=t, **_funcs(cosmo))
    err = np.abs(got - ref).max()
    print(f"replica positions: max |GPU - oracle| {err:.2e} Mpc/h")
    assert err < 2e-3  # FP32 positions up to ~400 Mpc/h (ulp 3e-5) plus table rounding

    noise = jf.white_noise(3, (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo, flatsky_npix=(48, 48))
    dx, p = jf.lpt(cosmo, ic, ts=0.5, order=1)
    dx = dx.replace(array=torch.as_tensor(disp, device="cuda"))
    p = p.replace(array=torch.as_tensor(vel, device="cuda"))
    rc, wd = 230.0, 40.0  # beyond the 100 Mpc/h the box holds around its centre
    interp = jf.TelephotoInterp(painting=jf.PaintingOptions(target="flat")).update_geometry(
        np.array([t]), np.array([rc]), np.array([wd]), 100.0)
    st = interp.advance(interp.init(), t)
    assert st.shell_idx == 0 and st.rotation_idx == 0
    plane = interp.paint(st, t, (dx, p), cosmo).array.cpu().numpy()
    rot = st.rotations[0]
    pos = oh.replica_positions(disp, vel, (L, L, L), obs, rot, np.array([0.0, 0.0, 200.0]), telephoto=True, t=t,
                               **_funcs(cosmo))
    cg, wg = rc * n / L, wd * n / L
    ref_plane = of.paint_2d(pos / L * n, (48, 48), cg - wg / 2, cg + wg / 2, (n, n, n)) / ((L / 48) ** 2 * wd)
    e2 = rel_l2(plane, ref_plane)
    print(f"telephoto flat plane: weight {ref_plane.sum():.3e}, rel L2 {e2:.2e}")
    assert ref_plane.sum() > 0 and e2 < 1e-3
