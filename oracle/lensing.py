"""FP64 CPU restatement of the reference's spherical Born convergence (test infrastructure
only: imported by tests/, never by the product)."""

from __future__ import annotations

import numpy as np

H0_OVER_C = 100.0 / 299792.458


def simps_weights(a, b, n):
    """reference _src/lensing/_born.py:16-27."""
    w = np.ones(n + 1)
    w[1:-1:2] = 4.0
    w[2:-2:2] = 2.0
    return w * ((b - a) / n / 3.0)


def born_core(maps, r, a, z_source, d_r, omega_m, chi_of_z):
    """reference _src/lensing/_born.py:29-97 (spherical branch): kappa for each source
    redshift in z_source, (nz, npix)."""
    maps = np.asarray(maps, np.float64)
    mean = maps.mean(axis=1, keepdims=True)
    mean = np.where(mean == 0, np.finfo(np.float32).eps, mean)
    delta = maps / mean - 1.0
    contrib = delta * (d_r * r / a)[:, None] * (1.5 * omega_m * H0_OVER_C**2)
    chi_s = np.atleast_1d(chi_of_z(np.atleast_1d(z_source)))
    eff = np.clip(1.0 - r[None, :] / chi_s[:, None], 0.0, 1000.0)  # (nz, P)
    return np.einsum("zp,pn->zn", eff, contrib)


def born_spherical(maps, r, a, d_r, omega_m, chi_of_z, nz_list=None, z_sources=None, min_z=0.01, max_z=1.5,
                   n_integrate=32):
    """reference _src/lensing/_born.py:100-130."""
    if nz_list is not None:
        zg = np.linspace(min_z, max_z, n_integrate + 1)
        kg = born_core(maps, r, a, zg, d_r, omega_m, chi_of_z)
        w = simps_weights(min_z, max_z, n_integrate)
        nzw = np.stack([nz(zg) for nz in nz_list])
        return np.einsum("kz,z,zn->kn", nzw, w, kg)
    return born_core(maps, r, a, z_sources, d_r, omega_m, chi_of_z)
