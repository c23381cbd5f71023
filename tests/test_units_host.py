"""Density unit conversions (reference fields/units.py:133-258 and the fields' .to methods):
DENSITY as the hub, the voxel / pixel volumes each field type uses, and round trips. CPU."""

import math

import numpy as np
import pytest
import torch

import jfli_b200 as jf

U = jf.DensityUnit


def _dens():
    rng = np.random.default_rng(0)
    a = torch.as_tensor(rng.uniform(0.5, 1.5, (8, 8, 8)))
    return jf.DensityField(array=a, mesh_size=(8, 8, 8), box_size=(16.0, 16.0, 32.0), unit=U.DENSITY)


def test_density_field_conversions():
    f = _dens()
    vox = 2.0 * 2.0 * 4.0
    counts = f.to(U.COUNTS)
    assert counts.unit == U.COUNTS
    torch.testing.assert_close(counts.array, f.array * vox)
    over = f.to(U.OVERDENSITY)
    torch.testing.assert_close(over.array, f.array / f.array.mean() - 1.0)
    back = over.to(U.DENSITY, mean_density=float(f.array.mean()))
    torch.testing.assert_close(back.array, f.array)
    msun = f.to(U.MSUN_H_PER_MPC3, omega_m=0.3, h=0.7)
    m_pp = 0.3 * 2.775e11 * 0.7**2 * vox / 0.7**3
    torch.testing.assert_close(msun.array, f.array * vox * m_pp * 0.7 / vox)
    torch.testing.assert_close(msun.to(U.DENSITY, omega_m=0.3, h=0.7).array, f.array)
    with pytest.raises(ValueError):
        over.to(U.DENSITY)  # mean density needed from OVERDENSITY
    with pytest.raises(ValueError):
        f.to(U.MSUN_H_PER_MPC3)
    assert f.to(U.DENSITY) is f


def test_spherical_and_flat_volumes():
    nside = 4
    maps = torch.ones(2, 12 * nside * nside, dtype=torch.float64)
    sph = jf.SphericalDensity(array=maps, mesh_size=(8, 8, 8), box_size=(100.0,) * 3, nside=nside, unit=U.DENSITY,
                              comoving_centers=np.array([20.0, 40.0]), density_width=np.array([10.0, 20.0]))
    c = sph.to(U.COUNTS).array
    vol = [4 * math.pi / (12 * nside * nside) * ((cc + w / 2) ** 3 - (cc - w / 2) ** 3) / 3
           for cc, w in ((20.0, 10.0), (40.0, 20.0))]
    torch.testing.assert_close(c[:, 0], torch.as_tensor(vol, dtype=torch.float64))
    flat = jf.FlatDensity(array=torch.ones(16, 8, dtype=torch.float64), mesh_size=(8, 8, 8),
                          box_size=(100.0, 50.0, 80.0), flatsky_npix=(16, 8), density_width=5.0, unit=U.DENSITY)
    # the reference's flat-map volume: (L_x / flatsky_npix[1]) (L_y / flatsky_npix[0]) width
    torch.testing.assert_close(flat.to(U.COUNTS).array, torch.full((16, 8), (100.0 / 8) * (50.0 / 16) * 5.0,
                                                                    dtype=torch.float64))


def test_convert_units_families():
    x = torch.zeros(4, 4, 4, 3)
    with pytest.raises(TypeError):
        jf.convert_units(x, jf.PositionUnit.GRID_RELATIVE, U.DENSITY, (4, 4, 4), (8.0,) * 3)
    mpc = jf.convert_units(x, jf.PositionUnit.GRID_RELATIVE, jf.PositionUnit.MPC_H, (4, 4, 4), (8.0,) * 3)
    assert float(mpc[1, 2, 3, 2]) == 6.0
