"""Born convergence of a spherical light cone (reference lensing/born.py:14-89,
_src/lensing/_born.py:16-130, _src/lensing/_metadata.py:17-43).

The host builds, in FP64, the (sources x planes) weight matrix of the Born sum:
  W[k][p] = 3/2 Omega_m (H0/c)^2 * dr * r_p / a_p * sum_z w_z n_k(z) clip(1 - r_p/chi(z), 0, 1000)
for redshift distributions (Simpson weights w_z on n_integrate + 1 points from min_z to
max_z, as the reference's _simps_weights), or with n_k(z) w_z replaced by a single source
redshift z_k. The GPU kernel (`jfli_born`) then forms kappa_k = sum_p W[k][p] delta_p
with delta_p = map_p / mean(map_p) - 1, reading every shell map once.
"""

from __future__ import annotations

import dataclasses

import math

import numpy as np
import torch

from . import cosmology as cj
from ._lib import call, ptr, query, stream_ptr
from .fields import FieldStatus, SphericalDensity

H0_OVER_C = 100.0 / 299792.458  # h/Mpc (jax_cosmo.constants: H0 = 100 km/s/(Mpc/h), c in km/s)


def simpson_weights(a: float, b: float, n: int) -> np.ndarray:
    """Composite Simpson weights dx/3 [1, 4, 2, ..., 4, 1] on n subintervals."""
    w = np.ones(n + 1)
    w[1:-1:2] = 4.0
    w[2:-2:2] = 2.0
    return w * ((b - a) / n / 3.0)


@dataclasses.dataclass(frozen=True, eq=False)
class RedshiftDistribution:
    """n(z) normalised on [0, zmax] with Simpson's rule on 256 intervals, like
    jax_cosmo.redshift.redshift_distribution (pz_fn(z, *params) / norm), with its
    galaxy density (gals_per_arcmin2, default 1)."""

    pz_fn: object
    params: tuple = ()
    zmax: float = 10.0
    gals_per_arcmin2: float = 1.0

    @property
    def norm(self) -> float:
        z = np.linspace(0.0, self.zmax, 257)
        return float(np.sum(simpson_weights(0.0, self.zmax, 256) * self.pz_fn(z, *self.params)))

    @property
    def gals_per_steradian(self) -> float:
        return self.gals_per_arcmin2 * (180.0 * 60.0 / math.pi) ** 2

    def __call__(self, z):
        z = np.asarray(z, dtype=np.float64)
        return self.pz_fn(z, *self.params) / self.norm


def _tophat(z, zmin, zmax):
    return np.where((z >= zmin) & (z <= zmax), 1.0, 0.0)


def tophat_nz(zmin: float, zmax: float) -> RedshiftDistribution:
    return RedshiftDistribution(_tophat, (float(zmin), float(zmax)), zmax=float(zmax))


def _smail(z, a, b, z0):
    return z**a * np.exp(-((z / z0) ** b))


def smail_nz(a: float, b: float, z0: float, zmax: float = 10.0) -> RedshiftDistribution:
    return RedshiftDistribution(_smail, (float(a), float(b), float(z0)), zmax=float(zmax))


def _kde(z, zcat, weight, bw):
    """Weighted Gaussian kernel density estimate: sum_i w_i N(z; zcat_i, bw) / sum_i w_i."""
    d = (np.atleast_1d(z)[None, :] - zcat[:, None]) / bw
    k = np.exp(-0.5 * d * d) / (math.sqrt(2.0 * math.pi) * bw)
    out = weight @ k / np.sum(weight)
    return out if np.ndim(z) else out[0]


def kde_nz(zcat, weight, bw: float, zmax: float = 10.0, gals_per_arcmin2: float = 1.0) -> RedshiftDistribution:
    """n(z) as a Gaussian kernel density estimate of the samples `zcat` with weights
    `weight` and bandwidth `bw`, normalised on [0, zmax] (jax_cosmo.redshift.kde_nz, from
    the jax_cosmo fork jax-fli pins at ASKabalan/jax_cosmo@ALL-MODIF, pyproject.toml:33;
    used by io/cosmogrid.py:25-67 for the Stage-3 distributions)."""
    zcat = np.asarray(zcat, dtype=np.float64).ravel()
    weight = np.asarray(weight, dtype=np.float64).ravel()
    if zcat.shape != weight.shape or zcat.size == 0:
        raise ValueError("zcat and weight must be non-empty and of the same length")
    if not bw > 0:
        raise ValueError("bw must be positive")
    return RedshiftDistribution(_kde, (zcat, weight, float(bw)), zmax=float(zmax),
                                gals_per_arcmin2=float(gals_per_arcmin2))


def _sources(nz_shear):
    entries = list(nz_shear) if isinstance(nz_shear, (list, tuple)) else [nz_shear]
    if not entries:
        raise ValueError("nz_shear must contain at least one entry")
    if callable(entries[0]):
        if not all(callable(e) for e in entries):
            raise ValueError("Cannot mix redshift distributions with scalar sources")
        return "distribution", entries
    z = np.atleast_1d(np.asarray(entries, dtype=np.float64).squeeze())
    if z.ndim != 1:
        raise ValueError("Scalar redshift sources must be 1D array-like")
    return "redshift", z


def born_weights(cosmo, scale_factors, max_radius: float, nz_shear, min_z=0.01, max_z=1.5, n_integrate=32):
    """(W (K, P) FP64, z_eff (K,)) of the Born sum for the planes at `scale_factors`."""
    a = np.atleast_1d(np.asarray(scale_factors, dtype=np.float64))
    r = cj.radial_comoving_distance(cosmo, a)
    dr = max_radius / a.size
    base = 1.5 * cosmo.Omega_m * H0_OVER_C**2 * dr * r / a
    kind, src = _sources(nz_shear)

    def efficiency(z):
        chi_s = cj.radial_comoving_distance(cosmo, 1.0 / (1.0 + np.asarray(z, np.float64)))
        return np.clip(1.0 - r[None, :] / np.atleast_1d(chi_s)[:, None], 0.0, 1000.0)  # (nz, P)

    if kind == "distribution":
        zg = np.linspace(min_z, max_z, n_integrate + 1)
        sw = simpson_weights(min_z, max_z, n_integrate)
        eff = efficiency(zg)
        nzw = np.stack([np.asarray(nz(zg), np.float64) for nz in src])  # (K, nz)
        W = (nzw * sw[None, :]) @ eff * base[None, :]
        z_eff = np.array([np.sum(sw * zg * nz(zg)) / np.sum(sw * nz(zg)) for nz in src])
    else:
        W = efficiency(src) * base[None, :]
        z_eff = src
    return W, z_eff


class BornMaps(torch.autograd.Function):
    """kappa = W (maps / mean - 1) as an autograd node: backward jfli_born_adjoint."""

    @staticmethod
    def forward(ctx, maps, weights):
        ctx.weights = weights
        ctx.save_for_backward(maps)
        return _born_maps(maps.detach(), weights)

    @staticmethod
    def backward(ctx, kbar):
        (maps,) = ctx.saved_tensors
        maps = maps.detach().contiguous()
        squeeze = maps.ndim == 1
        m2 = maps[None] if squeeze else maps
        nplanes, npix = int(m2.shape[0]), int(m2.shape[1])
        w = torch.as_tensor(np.ascontiguousarray(ctx.weights, dtype=np.float32), device=maps.device)
        kb = kbar.contiguous()
        if tuple(kb.shape) != (w.shape[0], npix):
            raise ValueError("kappa cotangent shape differs from the convergence maps'")
        out = torch.empty_like(m2)
        from .ops import workspace

        ws = workspace(int(query("jfli_born_adjoint_workspace_bytes", nplanes, npix)), "born", maps.device)
        call("jfli_born_adjoint", stream_ptr(), ptr(m2), nplanes, npix, ptr(w), int(w.shape[0]), ptr(kb), ptr(out),
             ptr(ws), ws.numel())
        return (out[0] if squeeze else out), None


def born_maps(maps: torch.Tensor, weights: np.ndarray) -> torch.Tensor:
    """kappa (K, npix) = W @ (maps / mean - 1) on the GPU (differentiable in the maps)."""
    if maps.dtype != torch.float32 or not maps.is_cuda:
        raise TypeError("maps must be a float32 CUDA tensor")
    if torch.is_grad_enabled() and maps.requires_grad:
        return BornMaps.apply(maps, weights)
    return _born_maps(maps, weights)


def _born_maps(maps: torch.Tensor, weights: np.ndarray) -> torch.Tensor:
    maps = maps.contiguous()
    if maps.ndim == 1:
        maps = maps[None]
    nplanes, npix = int(maps.shape[0]), int(maps.shape[1])
    w = torch.as_tensor(np.ascontiguousarray(weights, dtype=np.float32), device=maps.device)
    if tuple(w.shape) != (w.shape[0], nplanes):
        raise ValueError("weights must be (sources, planes)")
    out = torch.empty(w.shape[0], npix, dtype=torch.float32, device=maps.device)
    nb = int(query("jfli_born_workspace_bytes", nplanes, npix))
    from .ops import workspace

    ws = workspace(nb, "born", maps.device)
    call("jfli_born", stream_ptr(), ptr(maps), nplanes, npix, ptr(w), int(w.shape[0]), ptr(out), ptr(ws), ws.numel())
    return out


def born_flat_maps(planes: torch.Tensor, weights: np.ndarray, s0: np.ndarray, s1: np.ndarray) -> torch.Tensor:
    """kappa (K, n0, n1) of flat planes (P, n0, n1): W @ (bilinear samples / mean - 1) on the GPU."""
    if planes.dtype != torch.float32 or not planes.is_cuda:
        raise TypeError("planes must be a float32 CUDA tensor")
    planes = planes.contiguous()
    if planes.ndim == 2:
        planes = planes[None]
    nplanes, n0, n1 = (int(v) for v in planes.shape)
    dev = planes.device
    w = torch.as_tensor(np.ascontiguousarray(weights, dtype=np.float32), device=dev)
    if tuple(w.shape) != (w.shape[0], nplanes):
        raise ValueError("weights must be (sources, planes)")
    t0 = torch.as_tensor(np.asarray(s0, np.float32), device=dev)
    t1 = torch.as_tensor(np.asarray(s1, np.float32), device=dev)
    out = torch.empty(w.shape[0], n0, n1, dtype=torch.float32, device=dev)
    nb = int(query("jfli_born_workspace_bytes", nplanes, n0 * n1))
    from .ops import workspace

    ws = workspace(nb, "born", dev)
    call("jfli_born_flat", stream_ptr(), ptr(planes), nplanes, n0, n1, ptr(w), int(w.shape[0]), ptr(t0), ptr(t1),
         ptr(out), ptr(ws), ws.numel())
    return out


def flat_sample_scales(field_size, flatsky_npix, box_size, chi):
    """Per-plane sample steps of flat Born (reference _src/lensing/_born.py:52-64, 155-160): the
    grid axis-1 angle (linspace(0, f_x, n_1) in degrees) times chi over the pixel size
    box_y / n_0 drives the plane's axis 0, and the axis-0 angle times chi over box_x / n_1
    its axis 1, as the reference pairs coords with pixel_size."""
    fx, fy = (field_size, field_size) if np.ndim(field_size) == 0 else field_size
    n0, n1 = flatsky_npix  # the reference names them (ny, nx)
    ps0, ps1 = box_size[1] / n0, box_size[0] / n1
    deg = math.pi / 180.0
    chi = np.asarray(chi, np.float64)
    return (fx / n1) * deg * chi / ps0, (fy / n0) * deg * chi / ps1


def born(cosmo, lightcone: SphericalDensity, nz_shear, min_z=0.01, max_z=1.5, n_integrate=32):
    """Born convergence maps (K, npix) of a spherical light cone (status LIGHTCONE), as a
    SphericalKappaField (unit DIMENSIONLESS) like the reference's."""
    if nz_shear is None:
        raise ValueError("nz_shear must be provided for lensing")
    if lightcone.status != FieldStatus.LIGHTCONE:
        raise ValueError(f"Expected lightcone with status=LIGHTCONE, got {lightcone.status}")
    from .fields import ConvergenceUnit, FlatDensity, FlatKappaField

    if isinstance(lightcone, FlatDensity):
        if lightcone.field_size is None:
            raise ValueError("field_size is required on lightcone for flat-sky convergence")
        if lightcone.array.ndim != 3:
            raise ValueError(f"Lightcone array must be 3D (flat), got {lightcone.array.ndim}D")
        a = np.atleast_1d(np.asarray(lightcone.scale_factors, np.float64))
        W, z_eff = born_weights(cosmo, a, lightcone.max_comoving_radius, nz_shear, min_z, max_z, n_integrate)
        s0, s1 = flat_sample_scales(lightcone.field_size, lightcone.flatsky_npix, lightcone.box_size,
                                    cj.radial_comoving_distance(cosmo, a))
        kappa = born_flat_maps(lightcone.array, W, s0, s1)
        a_src = 1.0 / (1.0 + z_eff)
        return FlatKappaField.FromDensityMetadata(
            array=kappa, field=lightcone, status=FieldStatus.KAPPA, unit=ConvergenceUnit.DIMENSIONLESS,
            z_sources=z_eff, scale_factors=a_src, comoving_centers=cj.radial_comoving_distance(cosmo, a_src),
            density_width=np.zeros_like(z_eff))
    if not isinstance(lightcone, SphericalDensity):
        raise TypeError(f"born needs a SphericalDensity or FlatDensity light cone, got {type(lightcone).__name__}")
    if lightcone.array.ndim != 2:
        raise ValueError(f"Lightcone array must be 2D (spherical), got {lightcone.array.ndim}D")
    W, z_eff = born_weights(cosmo, lightcone.scale_factors, lightcone.max_comoving_radius, nz_shear, min_z, max_z,
                            n_integrate)
    kappa = born_maps(lightcone.array, W)
    a_src = 1.0 / (1.0 + z_eff)
    from .fields import SphericalKappaField

    return SphericalKappaField.FromDensityMetadata(
        array=kappa, field=lightcone, status=FieldStatus.KAPPA, unit=ConvergenceUnit.DIMENSIONLESS, z_sources=z_eff,
        scale_factors=a_src, comoving_centers=cj.radial_comoving_distance(cosmo, a_src),
        density_width=np.zeros_like(z_eff))
