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


def _bilinear_wrap(plane, u, v):
    """Periodic bilinear sample of plane (n0, n1) at axis-0 coordinates u and axis-1
    coordinates v (jax.scipy.ndimage.map_coordinates, order 1, mode "wrap")."""
    n0, n1 = plane.shape
    fu, fv = np.floor(u), np.floor(v)
    wu, wv = u - fu, v - fv
    a0 = np.mod(fu.astype(np.int64), n0)
    b0 = np.mod(fv.astype(np.int64), n1)
    a1, b1 = (a0 + 1) % n0, (b0 + 1) % n1
    return ((1 - wu) * ((1 - wv) * plane[a0, b0] + wv * plane[a0, b1]) +
            wu * ((1 - wv) * plane[a1, b0] + wv * plane[a1, b1]))


def born_flat(planes, r, a, d_r, omega_m, chi_of_z, field_size, box, nz_list=None, z_sources=None, min_z=0.01,
              max_z=1.5, n_integrate=32):
    """reference _src/lensing/_born.py:29-97 (flat branch) and _born_flat (133-186): each
    plane's contribution delta (d_r r / a) 3/2 Omega_m (H0/c)^2 sampled at the lensed grid
    (coords = meshgrid(linspace(0, f_x, n1), linspace(0, f_y, n0)) in degrees -> radians,
    times chi over pixel_size = (L_y / n0, L_x / n1), minus 0.5), then the efficiency sum."""
    planes = np.asarray(planes, np.float64)
    p, n0, n1 = planes.shape
    fx, fy = field_size
    mean = planes.mean(axis=(1, 2), keepdims=True)
    mean = np.where(mean == 0, np.finfo(np.float32).eps, mean)
    contrib = (planes / mean - 1.0) * (d_r * r / a)[:, None, None] * (1.5 * omega_m * H0_OVER_C**2)
    xg, yg = np.meshgrid(np.arange(n1) * (fx / n1), np.arange(n0) * (fy / n0))
    cx, cy = xg * (np.pi / 180), yg * (np.pi / 180)
    ps0, ps1 = box[1] / n0, box[0] / n1
    sampled = np.stack([_bilinear_wrap(contrib[i], cx * r[i] / ps0 - 0.5, cy * r[i] / ps1 - 0.5) for i in range(p)])

    def core(zs):
        chi_s = np.atleast_1d(chi_of_z(np.atleast_1d(zs)))
        eff = np.clip(1.0 - r[None, :] / chi_s[:, None], 0.0, 1000.0)
        return np.einsum("zp,pij->zij", eff, sampled)

    if nz_list is not None:
        zg = np.linspace(min_z, max_z, n_integrate + 1)
        w = simps_weights(min_z, max_z, n_integrate)
        nzw = np.stack([nz(zg) for nz in nz_list])
        return np.einsum("kz,z,zij->kij", nzw, w, core(zg))
    return core(z_sources)
