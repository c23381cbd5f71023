"""Born convergence (reference _src/lensing/_born.py) against the FP64 oracle."""

import numpy as np
import pytest
import torch

import jfli_b200 as jf
from jfli_b200 import cosmology as cj
from jfli_b200 import lensing
from oracle import lensing as olens
from tests.conftest import rel_l2


def test_born_weights_match_oracle_on_host(cosmo):
    """The FP64 weight matrix contracted with delta equals the oracle's Born sum."""
    rng = np.random.default_rng(0)
    P, npix = 6, 12 * 8 * 8
    maps = rng.gamma(2.0, 1.0, (P, npix))
    a = np.linspace(0.95, 0.6, P)
    r = cj.radial_comoving_distance(cosmo, a)
    rmax = 1.05 * r.max()
    chi = lambda z: cj.radial_comoving_distance(cosmo, 1.0 / (1.0 + np.asarray(z)))
    for nz in ([lensing.tophat_nz(0.0, 1.0)], [lensing.smail_nz(2.0, 1.5, 0.5, 3.0), lensing.tophat_nz(0.2, 0.8)]):
        W, _ = lensing.born_weights(cosmo, a, rmax, nz)
        delta = maps / maps.mean(1, keepdims=True) - 1
        ref = olens.born_spherical(maps, r, a, rmax / P, cosmo.Omega_m, chi, nz_list=nz)
        assert rel_l2(W @ delta, ref) < 1e-12
    W, z = lensing.born_weights(cosmo, a, rmax, [0.5, 1.0])
    ref = olens.born_spherical(maps, r, a, rmax / P, cosmo.Omega_m, chi, z_sources=[0.5, 1.0])
    assert rel_l2(W @ (maps / maps.mean(1, keepdims=True) - 1), ref) < 1e-12
    np.testing.assert_allclose(z, [0.5, 1.0])


def test_tophat_nz_is_normalised():
    nz = lensing.tophat_nz(0.0, 1.0)
    z = np.linspace(0.0, 1.0, 1001)
    assert abs(np.trapezoid(nz(z), z) - 1.0) < 1e-2


@pytest.mark.gpu
def test_born_gpu_matches_oracle(cosmo):
    import jfli_b200 as jf

    rng = np.random.default_rng(1)
    nside, P = 64, 16
    npix = 12 * nside * nside
    maps = rng.gamma(3.0, 1.0, (P, npix)).astype(np.float32)
    maps[3] = 0.0  # an empty shell: mean 0 -> eps, as the reference
    a = np.linspace(0.97, 0.5, P)
    r = cj.radial_comoving_distance(cosmo, a)
    L = 2.2 * r.max()
    lc = jf.SphericalDensity(array=torch.as_tensor(maps, device="cuda"), mesh_size=(64,) * 3, box_size=(L,) * 3,
                             nside=nside, status=jf.FieldStatus.LIGHTCONE, scale_factors=a, comoving_centers=r,
                             density_width=np.full(P, L / 2 / P))
    nz = [lensing.tophat_nz(0.0, 1.0), lensing.smail_nz(2.0, 1.5, 0.6, 3.0)]
    kappa = lensing.born(cosmo, lc, nz)
    chi = lambda z: cj.radial_comoving_distance(cosmo, 1.0 / (1.0 + np.asarray(z)))
    ref = olens.born_spherical(maps.astype(np.float64), r, a, lc.max_comoving_radius / P, cosmo.Omega_m, chi,
                               nz_list=nz)
    out = kappa.array.cpu().numpy()
    err = rel_l2(out, ref)
    print(f"Born kappa rel L2 vs oracle {err:.2e}; rms kappa {np.sqrt((ref**2).mean()):.3e}")
    assert kappa.status == jf.FieldStatus.KAPPA and out.shape == (2, npix)
    assert err < 1e-5


@pytest.mark.gpu
def test_lightcone_convergence_pipeline(cosmo):
    """White noise -> 2LPT -> KDK with PGD painting 4 shells -> Born (the large light-cone
    chain at a small size): finite maps, Born consistent with the oracle on the painted
    shells, and the PGD correction changes the shells."""
    from jfli_b200 import pipelines

    kw = dict(mesh=64, box=256.0, seed=3, nb_shells=4, nside=32, nz_shear=[lensing.tophat_nz(0.0, 1.0)], steps=10)
    res = pipelines.lightcone_convergence(cosmo, pgd=(0.3, 1.5, 8.0), **kw)
    plain = pipelines.lightcone_convergence(cosmo, pgd=None, **kw)
    maps = res.shells.array.cpu().numpy()
    kap = res.kappa.array.cpu().numpy()
    assert maps.shape == (4, 12 * 32 * 32) and kap.shape == (1, 12 * 32 * 32)
    assert np.isfinite(maps).all() and np.isfinite(kap).all() and res.steps >= 10  # + clipped steps at shells
    a = np.asarray(res.shells.scale_factors)
    r = cj.radial_comoving_distance(cosmo, a)
    chi = lambda z: cj.radial_comoving_distance(cosmo, 1.0 / (1.0 + np.asarray(z)))
    ref = olens.born_spherical(maps.astype(np.float64), r, a, res.shells.max_comoving_radius / 4, cosmo.Omega_m, chi,
                               nz_list=[lensing.tophat_nz(0.0, 1.0)], max_z=1.0)
    assert rel_l2(kap, ref) < 1e-5
    assert rel_l2(maps, plain.shells.array.cpu().numpy()) > 1e-3
    print("timings", res.timings)


@pytest.mark.gpu
def test_lightcone_pipeline_with_onion_tiler(cosmo):
    """The light-cone chain with OnionTiler: 4 shells out to three times the box's
    inscribed radius; shells beyond the box come from the 27 replicas and hold the box's
    mean density (within the box's own variance on the shell scale), and Born over them
    matches the oracle."""
    from jfli_b200 import pipelines

    res = pipelines.lightcone_convergence(cosmo, mesh=64, box=256.0, seed=4, nb_shells=4, nside=32,
                                          nz_shear=[lensing.tophat_nz(0.0, 1.0)], steps=10, tiler="onion")
    maps = res.shells.array.cpu().numpy()
    kap = res.kappa.array.cpu().numpy()
    centres = np.asarray(res.shells.comoving_centers, np.float64)
    assert maps.shape == (4, 12 * 32 * 32) and np.isfinite(maps).all() and np.isfinite(kap).all()
    assert np.allclose(np.sort(centres), [48.0, 144.0, 240.0, 336.0])
    mean_density = 64**3 / 256.0**3
    for s, rc in enumerate(centres):
        rel = abs(maps[s].mean() / mean_density - 1)
        print(f"shell at {rc:.0f} Mpc/h: mean / box mean - 1 = {rel:.2e}")
        assert rel < 0.15
    a = np.asarray(res.shells.scale_factors)
    r = cj.radial_comoving_distance(cosmo, a)
    chi = lambda z: cj.radial_comoving_distance(cosmo, 1.0 / (1.0 + np.asarray(z)))
    # the reference's born takes the plane width as the box's inscribed radius over the
    # number of planes (lensing/born.py:23-24), whatever the shells' own widths
    ref = olens.born_spherical(maps.astype(np.float64), r, a, res.shells.max_comoving_radius / 4, cosmo.Omega_m, chi,
                               nz_list=[lensing.tophat_nz(0.0, 1.0)], max_z=1.0)
    assert rel_l2(kap, ref) < 1e-5


@pytest.mark.gpu
def test_born_flat_matches_oracle(cosmo):
    """Flat-sky Born (reference _born_flat): planes sampled at the lensed grid by periodic
    bilinear interpolation, against the FP64 oracle, for a source distribution and for
    source redshifts; a FlatKappaField comes back."""
    import torch

    rng = np.random.default_rng(21)
    n0, n1, P = 48, 64, 3
    planes = (1.0 + 0.3 * rng.standard_normal((P, n0, n1))).astype(np.float32)
    a = np.array([0.85, 0.7, 0.55])
    r = cj.radial_comoving_distance(cosmo, a)
    L = (300.0, 300.0, 300.0)
    fs = (4.0, 3.0)
    lc = jf.FlatDensity(array=torch.as_tensor(planes, device="cuda"), mesh_size=(32, 32, 32), box_size=L,
                        flatsky_npix=(n0, n1), field_size=fs, status=jf.FieldStatus.LIGHTCONE, scale_factors=a,
                        comoving_centers=r, density_width=np.full(P, 50.0), unit=jf.DensityUnit.DENSITY)
    chi = lambda z: cj.radial_comoving_distance(cosmo, 1.0 / (1.0 + np.asarray(z)))
    d_r = lc.max_comoving_radius / P
    for kw, okw in ((dict(nz_shear=[lensing.tophat_nz(0.0, 1.5)]), dict(nz_list=[lensing.tophat_nz(0.0, 1.5)])),
                    (dict(nz_shear=[1.0, 2.0]), dict(z_sources=np.array([1.0, 2.0])))):
        kap = jf.born(cosmo, lc, **kw)
        assert isinstance(kap, jf.FlatKappaField) and kap.unit == jf.ConvergenceUnit.DIMENSIONLESS
        ref = olens.born_flat(planes, r, a, d_r, cosmo.Omega_m, chi, fs, L, max_z=1.5, **okw)
        err = rel_l2(kap.array.cpu().numpy(), ref)
        print(f"flat Born {list(kw.values())[0]!r}: rel L2 {err:.2e}")
        assert err < 1e-5
