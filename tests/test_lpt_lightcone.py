"""Light-cone-mode LPT (reference pm/lpt.py:110-213 with the per-particle scale factors of
utils.py:234-244) against the FP64 oracle: displacements, momenta and scale factors of
every particle, and the lightcone painted from them (HEALPix shells, density)."""

import numpy as np
import pytest
import torch

import jfli_b200 as jf
from jfli_b200 import cosmology as cj
from jfli_b200.pm.lpt import lpt_coefficients
from oracle import healpix as oh
from oracle import pm as opm
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _coefficients(cosmo):
    def coeffs(a):
        a = np.asarray(a, np.float64)
        D1 = cj.growth_factor(cosmo, a)
        f1 = cj.growth_rate(cosmo, a)
        D2 = cj.growth_factor_second(cosmo, a)
        f2 = cj.growth_rate_second(cosmo, a)
        Ea = cj.E(cosmo, a)
        return D1, 3.0 / 7.0 * D2, a * a * f1 * Ea, a * a * f2 * Ea
    return coeffs


def _setup(cosmo, n=32, L=300.0, nside=16):
    noise = jf.white_noise(4, (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo, nside=nside)
    return ic, ic.array.double().cpu().numpy()


@pytest.mark.parametrize("order", [1, 2])
def test_lightcone_lpt_particles_match_oracle(cosmo, order):
    n, L = 32, 300.0
    ic, ic64 = _setup(cosmo, n, L)
    dx, p = jf.lpt(cosmo, ic, nb_shells=4, order=order)
    assert dx.status == jf.FieldStatus.LIGHTCONE
    obs = ic.observer_position_mpc
    rdx, rp, ra = opm.lpt_lightcone(ic64, order, (L, L, L), obs, lambda r: cj.a_of_chi(cosmo, r), _coefficients(cosmo))
    e_dx = rel_l2(dx.array.double().cpu().numpy(), rdx)
    e_p = rel_l2(p.array.double().cpu().numpy(), rp)
    a = dx.scale_factors.double().cpu().numpy()
    assert a.shape == (n, n, n, 1)
    e_a = np.abs(a[..., 0] - ra).max()
    print(f"order {order}: dx {e_dx:.2e}, p {e_p:.2e} rel L2; a max abs {e_a:.2e} (a in [{ra.min():.3f}, {ra.max():.3f}])")
    assert e_dx < 1e-5 and e_p < 1e-5 and e_a < 1e-6
    # a snapshot-mode LPT at one a equals the light-cone one where that a holds: scalar coefficients
    c = lpt_coefficients(cosmo, 0.5)
    sdx, _ = opm.lpt(ic64, *c, order=order)
    assert rel_l2(jf.lpt(cosmo, ic, ts=0.5, order=order)[0].array.double().cpu().numpy(), sdx) < 1e-5


def test_lightcone_lpt_painted_shells_and_density(cosmo):
    n, L, nside = 32, 300.0, 16
    ic, ic64 = _setup(cosmo, n, L, nside)
    obs = ic.observer_position_mpc
    rdx, _, _ = opm.lpt_lightcone(ic64, 2, (L, L, L), obs, lambda r: cj.a_of_chi(cosmo, r), _coefficients(cosmo))
    shells, _ = jf.lpt(cosmo, ic, nb_shells=4, order=2, painting=jf.PaintingOptions(target="spherical"))
    maps = shells.array.double().cpu().numpy()
    assert maps.shape == (4, 12 * nside * nside)
    centres = np.asarray(shells.comoving_centers, np.float64)
    widths = np.asarray(shells.density_width, np.float64)
    np.testing.assert_allclose(np.asarray(shells.scale_factors), cj.a_of_chi(cosmo, centres), rtol=1e-12)
    pos = (opm.grid((n, n, n)) + rdx) * (L / n)
    for s in range(4):
        rmin, rmax = centres[s] - widths[s] / 2, centres[s] + widths[s] / 2
        vol = (4 * np.pi / (12 * nside * nside)) * (rmax**3 - rmin**3) / 3
        ref = oh.paint_shell(pos.reshape(-1, 3), obs, rmin, rmax, nside, "bilinear") / vol
        err = rel_l2(maps[s], ref)
        print(f"shell {s} ({rmin:.1f}-{rmax:.1f} Mpc/h): rel L2 {err:.2e}")
        assert ref.sum() > 0 and err < 2e-5
    dens, _ = jf.lpt(cosmo, ic, nb_shells=4, order=2, painting=jf.PaintingOptions(target="density"))
    assert rel_l2(dens.array.double().cpu().numpy(), opm.cic_paint(rdx)) < 1e-5


@pytest.mark.parametrize("order", [1, 2])
def test_lightcone_lpt_gradient_matches_oracle_fd(cosmo, order):
    """Light-cone-mode LPT on an initial field that requires grad (the per-particle
    coefficients applied to the cotangents of jfli_lpt_adjoint): the directional derivative
    of <r1, dx> + <r2, p> with respect to the initial field matches central differences of
    the FP64 oracle (oracle/pm.py lpt_lightcone; linear or quadratic in the field, so steps
    of 1e-3 are exact up to rounding)."""
    n, L = 32, 300.0
    ic, ic64 = _setup(cosmo, n, L)
    rng = np.random.default_rng(40 + order)
    r1, r2, s = rng.standard_normal((n, n, n, 3)), rng.standard_normal((n, n, n, 3)), rng.standard_normal((n, n, n))
    icg = ic.array.detach().clone().requires_grad_(True)
    dx, p = jf.lpt(cosmo, ic.replace(array=icg), nb_shells=4, order=order)
    loss = (dx.array.double() * torch.as_tensor(r1, device="cuda")).sum() + \
        (p.array.double() * torch.as_tensor(r2, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(icg.grad.cpu().numpy() * s))
    obs = ic.observer_position_mpc

    def oracle_loss(f):
        rdx, rp, _ = opm.lpt_lightcone(f, order, (L, L, L), obs, lambda r: cj.a_of_chi(cosmo, r), _coefficients(cosmo))
        return float(np.sum(r1 * rdx) + np.sum(r2 * rp))

    eps = 1e-3
    fd = (oracle_loss(ic64 + eps * s) - oracle_loss(ic64 - eps * s)) / (2 * eps)
    print(f"light-cone LPT order {order}: directional derivative {g_dir:.8e} vs oracle central difference {fd:.8e}")
    assert abs(g_dir - fd) / abs(fd) < 1e-4


def test_lpt_density_gradient_matches_oracle_fd(cosmo):
    """Snapshot LPT painted to a density (ParticleField.paint on displacements that require
    grad: the CIC-paint node, whose backward is jfli_adjoint_position): the directional
    derivative of <a, rho> with respect to the initial field matches central differences
    of the FP64 oracle (LPT then CIC paint; steps of 1e-6 keep the particles inside their
    cells)."""
    n, L = 32, 300.0
    ic, ic64 = _setup(cosmo, n, L)
    rng = np.random.default_rng(44)
    a, s = rng.standard_normal((n, n, n)), rng.standard_normal((n, n, n))
    icg = ic.array.detach().clone().requires_grad_(True)
    rho, _ = jf.lpt(cosmo, ic.replace(array=icg), ts=0.5, order=2, painting=jf.PaintingOptions(target="density"))
    loss = (rho.array.double() * torch.as_tensor(a, device="cuda")).sum()
    loss.backward()
    g_dir = float(np.sum(icg.grad.cpu().numpy() * s))
    c = lpt_coefficients(cosmo, 0.5)

    def oracle_loss(f):
        rdx, _ = opm.lpt(f, *c, order=2)
        return float(np.sum(a * opm.cic_paint(rdx)))

    eps = 1e-6
    fd = (oracle_loss(ic64 + eps * s) - oracle_loss(ic64 - eps * s)) / (2 * eps)
    print(f"LPT density: directional derivative {g_dir:.8e} vs oracle central difference {fd:.8e}")
    assert abs(g_dir - fd) / abs(fd) < 1e-3
