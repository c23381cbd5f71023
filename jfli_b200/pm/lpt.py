"""LPT entry point (reference pm/lpt.py:19-214) and geometry resolution
(reference pm/_resolve_geometry.py:12-114)."""

from __future__ import annotations

import numpy as np
import torch

from .. import cosmology as cj
from .. import ops
from ..fields import DensityField, FieldStatus, PaintingOptions, ParticleField, PositionUnit
from ..utils import compute_lightcone_shells, distances


def resolve_ts_geometry(cosmo, field, painting, ts=None, nb_shells=None, density_widths=None, equal_vol=False,
                        min_width=50.0):
    """(ts_resolved, r_centers, density_widths, is_lightcone) from ts / nb_shells / widths."""
    if ts is None and nb_shells is None:
        raise ValueError("Cannot specify both `ts` and `nb_shells`.")
    is_projecting = painting.target in ("flat", "spherical")
    if ts is not None and nb_shells is not None:
        raise ValueError("Cannot specify both `ts` and `nb_shells`.")
    if nb_shells is not None:
        r_centers, ts_resolved = compute_lightcone_shells(cosmo, field, nb_shells=nb_shells, equal_vol=equal_vol,
                                                          min_width=min_width)
        if density_widths is not None:
            try:
                density_widths = np.broadcast_to(np.asarray(density_widths, np.float64), r_centers.shape).copy()
            except ValueError:
                raise ValueError("density_widths must be broadcastable to the shape of r_centers.")
        else:
            density_widths = distances(r_centers, 0.0)
        return np.asarray(ts_resolved), np.asarray(r_centers), np.asarray(density_widths), True
    ts = np.asarray(ts, dtype=np.float64)
    if ts.ndim == 0 or (ts.ndim == 1 and ts.size == 1):
        ts = np.atleast_1d(ts).reshape(())
        r_center = cj.radial_comoving_distance(cosmo, ts)
        if density_widths is not None:
            dw = np.asarray(density_widths, np.float64).squeeze()
            if dw.ndim != 0:
                raise ValueError("For single-shell mode, density_widths must be a scalar.")
            density_widths = np.atleast_1d(dw)
        elif is_projecting:
            raise ValueError("Projection painting requires explicit density_widths for single-shell mode.")
        else:
            density_widths = np.array([0.0])
        return np.atleast_1d(ts), np.atleast_1d(r_center), density_widths, False
    if ts.ndim == 1:
        r_centers = cj.radial_comoving_distance(cosmo, ts)
        if density_widths is not None:
            try:
                density_widths = np.broadcast_to(np.asarray(density_widths, np.float64), r_centers.shape).copy()
            except ValueError:
                raise ValueError("density_widths must be broadcastable to the shape of ts.")
        else:
            density_widths = distances(r_centers, 0.0)
        return ts, r_centers, density_widths, True
    if ts.ndim == 2 and ts.shape[0] == 2:
        r_near, r_far = cj.radial_comoving_distance(cosmo, ts[0]), cj.radial_comoving_distance(cosmo, ts[1])
        r_centers = 0.5 * (r_near + r_far)
        return cj.a_of_chi(cosmo, r_centers), r_centers, np.abs(r_far - r_near), True
    raise ValueError(f"ts has unsupported shape {ts.shape}. Expected scalar, 1-D, or (2, N).")


def lpt_coefficients(cosmo, a: float):
    """(c1x, c2x, c1p, c2p) of JaxPM's lpt: dx = D1 F1 + 3/7 D2 F2,
    p = a^2 E (f1 D1 F1 + f2 3/7 D2 F2) (FastPM momentum)."""
    D1 = float(cj.growth_factor(cosmo, a))
    f1 = float(cj.growth_rate(cosmo, a))
    D2 = float(cj.growth_factor_second(cosmo, a))
    f2 = float(cj.growth_rate_second(cosmo, a))
    Ea = float(cj.E(cosmo, a))
    return D1, 3.0 / 7.0 * D2, a * a * f1 * Ea, a * a * f2 * Ea


def lpt(cosmo, initial_field: DensityField, *, ts=None, nb_shells=None, density_widths=None, order: int = 1,
        initial_particles=None, painting: PaintingOptions = PaintingOptions(target="particles"), equal_vol=False,
        min_width=50.0):
    """LPT displacements and momenta of a linear density field (reference pm/lpt.py:20-213)."""
    if not isinstance(initial_field, DensityField):
        raise TypeError("initial_field must be a DensityField instance.")
    if order not in (1, 2):
        raise ValueError("order must be either 1 or 2.")
    if initial_field.status != FieldStatus.INITIAL_FIELD:
        raise ValueError("initial_field must have status FieldStatus.INITIAL_FIELD.")
    if initial_particles is not None:
        raise NotImplementedError("custom initial_particles are not on the B200 path")
    ts_resolved, r_centers, widths, is_lightcone = resolve_ts_geometry(
        cosmo, initial_field, painting=painting, ts=ts, nb_shells=nb_shells, density_widths=density_widths,
        equal_vol=equal_vol, min_width=min_width)
    if is_lightcone:
        return _lpt_lightcone(cosmo, initial_field, order, painting, r_centers, widths)
    if painting.target not in ("particles", "density"):
        raise ValueError(
            f"Painting target {painting.target} is incompatible with snapshot mode. Use 'particles' or 'density'.")
    a = float(np.asarray(ts_resolved).reshape(-1)[0])
    c1x, c2x, c1p, c2p = lpt_coefficients(cosmo, a)
    ic = initial_field.array.contiguous()
    if torch.is_grad_enabled() and ic.requires_grad:
        from .adjoint import LPT, ForwardTables

        tables = ForwardTables(ktab=None, ptab=None, lpt=(c1x, c2x, c1p, c2p), kicks=None, drifts=None)
        dx, p = LPT.apply(ic, None, order, tables)
    else:
        dx, p = ops.lpt(ic, order, c1x, c2x, c1p, c2p)
    status = FieldStatus.LPT1 if order == 1 else FieldStatus.LPT2
    a_arr = np.atleast_1d(np.float64(a))
    meta = dict(status=status, scale_factors=a_arr, comoving_centers=cj.radial_comoving_distance(cosmo, a_arr),
                z_sources=cj.a2z(a_arr), unit=PositionUnit.GRID_RELATIVE)
    dx_field = ParticleField.FromDensityMetadata(array=dx, field=initial_field, **meta)
    p_field = ParticleField.FromDensityMetadata(array=p, field=initial_field, **meta)
    if painting.target == "density":
        dx_field = dx_field.paint(weights=painting.weights, chunk_size=painting.chunk_size,
                                  batch_size=painting.batch_size)
    return dx_field, p_field


def _device_interp(x: torch.Tensor, xp: np.ndarray, fp: np.ndarray) -> torch.Tensor:
    """The host `interp` (linear, end extrapolation, searchsorted side="left") on a device
    tensor, in FP64."""
    xpt = torch.as_tensor(np.asarray(xp, np.float64), device=x.device)
    fpt = torch.as_tensor(np.asarray(fp, np.float64), device=x.device)
    xd = x.double()
    i = (torch.searchsorted(xpt, xd.contiguous(), side="left") - 1).clamp(0, xpt.numel() - 2)
    slope = (fpt[i + 1] - fpt[i]) / (xpt[i + 1] - xpt[i])
    return fpt[i] + (xd - xpt[i]) * slope


def _lpt_lightcone(cosmo, initial_field, order, painting, r_centers, widths):
    """Light-cone-mode LPT (reference pm/lpt.py:110-213): each particle at the scale factor
    of its own light-cone crossing (compute_particle_scale_factors, utils.py:234-244), then
    the lightcone painted as the painting target asks (spherical shells or flat planes at
    the shell centres, a density, or the particles themselves). The fields carry the
    per-particle scale factors, shape (..., nx, ny, nz, 1), as the reference's do."""
    ic = initial_field.array.contiguous()
    if torch.is_grad_enabled() and ic.requires_grad:
        from .adjoint import LPTLightcone

        dx, p, a = LPTLightcone.apply(ic, order, cosmo, initial_field.box_size, initial_field.observer_position_mpc)
    else:
        dx, p, a = ops.lpt_lightcone(ic, order, cosmo, initial_field.box_size, initial_field.observer_position_mpc)
    a = a[..., None]
    dt = cj.distance_table(cosmo)
    chi = _device_interp(a, dt.a, dt.chi).clamp(0.0, 1e6).float()
    meta = dict(status=FieldStatus.LIGHTCONE, scale_factors=a, comoving_centers=chi, z_sources=1.0 / a - 1.0,
                unit=PositionUnit.GRID_RELATIVE)
    dx_field = ParticleField.FromDensityMetadata(array=dx, field=initial_field, **meta)
    p_field = ParticleField.FromDensityMetadata(array=p, field=initial_field, **meta)
    target = painting.target if painting is not None else "particles"
    if target in ("flat", "spherical"):
        if target == "flat":
            res = dx_field.paint_2d(center=r_centers, density_plane_width=widths, weights=painting.weights,
                                    batch_size=painting.batch_size)
        else:
            res = dx_field.paint_spherical(center=r_centers, density_plane_width=widths, scheme=painting.scheme,
                                           weights=painting.weights, kernel_width_arcmin=painting.kernel_width_arcmin,
                                           smoothing_interpretation=painting.smoothing_interpretation,
                                           paint_nside=painting.paint_nside, ud_grade_power=painting.ud_grade_power,
                                           ud_grade_order_in=painting.ud_grade_order_in,
                                           ud_grade_order_out=painting.ud_grade_order_out,
                                           ud_grade_pess=painting.ud_grade_pess, batch_size=painting.batch_size)
        a_snap = np.asarray(cj.a_of_chi(cosmo, np.asarray(r_centers, np.float64)), np.float64)
        res = res.replace(scale_factors=a_snap, z_sources=cj.a2z(a_snap))
        if res.is_batched():  # the reference returns the shells reversed: res[::-1]
            res = res.replace(array=res.array.flip(0), scale_factors=a_snap[::-1].copy(),
                              z_sources=cj.a2z(a_snap)[::-1].copy(),
                              comoving_centers=np.asarray(res.comoving_centers)[::-1].copy()
                              if np.ndim(res.comoving_centers) else res.comoving_centers,
                              density_width=np.asarray(res.density_width)[::-1].copy()
                              if np.ndim(res.density_width) else res.density_width)
        dx_field = res
    elif target not in ("density", "particles"):
        raise ValueError(f"Unknown painting target {target}.")
    if target == "density":
        dx_field = dx_field.paint(weights=painting.weights, chunk_size=painting.chunk_size,
                                  batch_size=painting.batch_size)
    return dx_field, p_field
