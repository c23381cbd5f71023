"""Spherical (HEALPix) shell painting front end (reference _src/fields/_painting.py:249-348).

A shell of centre c and width w keeps particles with c - w/2 < r <= c + w/2 around the
observer; the map holds the painted weight per pixel divided by the pixel's comoving
volume Omega_pix (r_max^3 - r_min^3) / 3, i.e. a number density in (Mpc/h)^-3, the same
normalisation the flat-sky painter applies (reference _src/fields/_painting.py:196-200).
"""

from __future__ import annotations

import math

import numpy as np
import torch

from . import ops
from .fields import PositionUnit, _weights_arg


def shell_volume_per_pixel(nside: int, rmin: float, rmax: float) -> float:
    return (4.0 * math.pi / (12 * nside * nside)) * (rmax**3 - rmin**3) / 3.0


class CICPaint(torch.autograd.Function):
    """Relative displacements -> their CIC density times a scalar weight (ParticleField.paint,
    reference fields/particles.py:119-178); the backward is the CIC gradient of the density
    cotangent at the positions (jfli_adjoint_position), the adjoint of the deposit."""

    @staticmethod
    def forward(ctx, x, weight: float):
        x = x.contiguous()
        ctx.save_for_backward(x)
        ctx.weight = float(weight)
        return ops.paint_cic(x, weight=ctx.weight)

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        lam = torch.zeros_like(x)
        ops.adjoint_position(x, lam, rho_bar=g.contiguous(), scale=ctx.weight)
        return lam, None


class CICReadout(torch.autograd.Function):
    """(relative displacements, mesh) -> the mesh's CIC interpolation at the particles
    (ParticleField.read_out, reference fields/particles.py:182-229). Backward: the mesh's
    cotangent is the CIC paint of the output cotangent g as per-particle weights; the
    positions' is g_p grad_x R_x[mesh], the u . F term of jfli_adjoint_position with the mesh
    as the first lane of a float4 mesh and u = (g, 0, 0)."""

    @staticmethod
    def forward(ctx, x, mesh):
        x, mesh = x.contiguous(), mesh.contiguous()
        ctx.save_for_backward(x, mesh)
        return ops.readout_cic(x, mesh)

    @staticmethod
    def backward(ctx, g):
        x, mesh = ctx.saved_tensors
        g = g.contiguous()
        gx = gm = None
        if ctx.needs_input_grad[1]:
            gm = ops.paint_cic(x, weights=g)
        if ctx.needs_input_grad[0]:
            m4 = torch.zeros(tuple(mesh.shape) + (4,), dtype=torch.float32, device=mesh.device)
            m4[..., 0] = mesh
            u = torch.zeros_like(x)
            u[..., 0] = g
            gx = torch.zeros_like(x)
            ops.adjoint_position(x, gx, u=u, force=m4)
        return gx, gm


class PaintFlat(torch.autograd.Function):
    """Relative displacements -> one flat-sky plane (paint_2d's 2D CIC of the particles in a
    z slab, scalar weight; reference _src/fields/_painting.py:117-202); the backward is
    jfli_paint_flat_adjoint (the CIC weights' gradient in x and y; none at the slab edges)."""

    @staticmethod
    def forward(ctx, x, npix, zlo: float, zhi: float, weight: float):
        x = x.contiguous()
        ctx.save_for_backward(x)
        ctx.zlo, ctx.zhi, ctx.weight = float(zlo), float(zhi), float(weight)
        return ops.paint_flat(x, npix, zlo, zhi, weight=weight)

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        return ops.paint_flat_adjoint(x, g.contiguous(), ctx.zlo, ctx.zhi, weight=ctx.weight), None, None, None, None


class PaintShells(torch.autograd.Function):
    """Shells of one particle set as an autograd node: forward jfli_healpix_paint_shells,
    backward its adjoint (position and per-particle weight cotangents; the shell edges are
    steps in the distance and pass nothing back)."""

    @staticmethod
    def forward(ctx, pos, wts, geom):
        nside, box, obs, rmin, rmax, scale, scheme, absolute = geom
        out = ops.healpix_paint_shells(pos.detach().contiguous(), nside, box, obs, rmin, rmax, scale, scheme=scheme,
                                       absolute=absolute, weights=None if wts is None else wts.detach().contiguous())
        ctx.geom = geom
        ctx.save_for_backward(pos, wts) if wts is not None else ctx.save_for_backward(pos)
        ctx.has_w = wts is not None
        return out

    @staticmethod
    def backward(ctx, maps_bar):
        nside, box, obs, rmin, rmax, scale, scheme, absolute = ctx.geom
        saved = ctx.saved_tensors
        pos = saved[0].detach().contiguous()
        wts = saved[1].detach().contiguous() if ctx.has_w else None
        w_bar = torch.zeros_like(wts) if (wts is not None and ctx.needs_input_grad[1]) else None
        pos_bar = ops.healpix_paint_shells_adjoint(pos, maps_bar.contiguous(), nside, box, obs, rmin, rmax, scale,
                                                   scheme=scheme, absolute=absolute, weights=wts,
                                                   weights_bar=w_bar)
        return pos_bar, w_bar, None


def paint_shells(field, centers, widths, scheme="bilinear", weights=None, out=None, sigma=None) -> torch.Tensor:
    """(S, 12 nside^2) maps of one particle set for S shells (`sigma`: the rbf_neighbor
    scheme's Gaussian width in radians)."""
    if field.unit == PositionUnit.MPC_H:
        field = field.to(PositionUnit.GRID_ABSOLUTE)
    absolute = field.unit == PositionUnit.GRID_ABSOLUTE
    w, ws = _weights_arg(weights)
    npix = 12 * field.nside * field.nside
    centers = np.atleast_1d(np.asarray(centers, dtype=np.float64))
    widths = np.atleast_1d(np.asarray(widths, dtype=np.float64))
    pos = field.array.contiguous()
    rmin, rmax = centers - widths / 2.0, centers + widths / 2.0
    vol = np.array([shell_volume_per_pixel(field.nside, a, b) for a, b in zip(rmin, rmax)])
    scale = np.where(vol > 0, ws / np.where(vol > 0, vol, 1.0), ws)
    if torch.is_grad_enabled() and (pos.requires_grad or (w is not None and w.requires_grad)):
        if pos.dim() != 4 or scheme not in ("ngp", "bilinear"):
            raise NotImplementedError("gradients of spherical painting: one particle set, ngp or bilinear")
        if out is not None:
            raise ValueError("out= is not supported when painting differentiably")
        geom = (field.nside, tuple(field.box_size), tuple(field.observer_position_mpc), rmin, rmax, scale, scheme,
                absolute)
        return PaintShells.apply(pos, w, geom)
    if out is None:
        out = torch.empty(centers.size, npix, dtype=torch.float32, device=field.array.device)
    if pos.dim() == 4 and out.is_contiguous():
        # one pass over the particles for all the shells
        ops.healpix_paint_shells(pos, field.nside, field.box_size, field.observer_position_mpc, rmin, rmax, scale,
                                 scheme=scheme, absolute=absolute, weights=w, out=out, sigma=sigma)
        return out
    for s in range(centers.size):
        ops.healpix_paint(pos, field.nside, field.box_size, field.observer_position_mpc, rmin[s], rmax[s],
                          scheme=scheme, absolute=absolute, weights=w, weight=float(scale[s]), out=out[s],
                          sigma=sigma)
    return out


def check_grade_orders(order_in: str, order_out: str) -> None:
    """ud_grade orders a painter accepts: RING in (the painters write RING maps), RING or
    NESTED out."""
    from .healpix_order import _order

    if _order(order_in) != "RING":
        raise NotImplementedError("painted maps are RING ordered: ud_grade_order_in must be 'RING'")
    _order(order_out)


def regrade(maps: torch.Tensor, nside: int, paint_nside, *, power: float = 0.0, order_in: str = "RING",
            order_out: str = "RING", pess: bool = False) -> torch.Tensor:
    """Painted RING maps (..., 12 paint_nside^2) brought to the field's nside with healpy's
    ud_grade (PaintingOptions.paint_nside and ud_grade_* options, reference
    fields/painting.py:78-96); unchanged when paint_nside is unset or equal to nside. The
    painters write RING maps, so order_in must be RING; order_out may be NESTED."""
    from .healpix_order import ud_grade

    check_grade_orders(order_in, order_out)
    if paint_nside is None or int(paint_nside) == int(nside):
        return maps
    return ud_grade(maps, int(nside), pess=bool(pess), order_in="RING", order_out=order_out,
                    power=float(power) if power else None)


def paint_shell_tiled(field, vel, center: float, width: float, rotations, shifts, *, telephoto: bool = False,
                      t: float | None = None, cosmo=None, scheme: str = "bilinear", weights=None) -> torch.Tensor:
    """(12 nside^2,) map of one shell painted from rotated and shifted replicas of the
    particles (OnionTiler / TelephotoInterp), each replica drifted to the light cone when
    `vel` is given; normalised like paint_shells (number density per pixel volume)."""
    if field.unit == PositionUnit.MPC_H:
        field = field.to(PositionUnit.GRID_ABSOLUTE)
    absolute = field.unit == PositionUnit.GRID_ABSOLUTE
    w, ws = _weights_arg(weights)
    rmin, rmax = float(center) - float(width) / 2.0, float(center) + float(width) / 2.0
    vol = shell_volume_per_pixel(field.nside, rmin, rmax)
    scale = ws / vol if vol > 0 else ws
    v = vel.contiguous() if vel is not None else None
    pos = field.array.contiguous()
    kw = dict(absolute=absolute, t=t, cosmo=cosmo, telephoto=telephoto, scheme=scheme, weight=scale)
    if torch.is_grad_enabled() and (pos.requires_grad or (v is not None and v.requires_grad)):
        if pos.dim() != 4 or w is not None:
            raise NotImplementedError("gradients of replica painting: one particle set, scalar weights")
        geom = (field.nside, tuple(field.box_size), tuple(field.observer_position_mpc), rmin, rmax, rotations, shifts,
                kw)
        return PaintShellTiled.apply(pos, v, geom)
    return ops.healpix_paint_tiled(pos, field.nside, field.box_size, field.observer_position_mpc, rmin, rmax,
                                   rotations, shifts, vel=v, weights=w, **kw)


class PaintShellTiled(torch.autograd.Function):
    """One shell of rotated, shifted (and light-cone drifted) replicas as an autograd node:
    forward jfli_healpix_paint_tiled, backward its adjoint (position and velocity
    cotangents)."""

    @staticmethod
    def forward(ctx, pos, vel, geom):
        nside, box, obs, rmin, rmax, rotations, shifts, kw = geom
        ctx.geom = geom
        ctx.has_v = vel is not None
        ctx.save_for_backward(pos, vel) if vel is not None else ctx.save_for_backward(pos)
        return ops.healpix_paint_tiled(pos.detach(), nside, box, obs, rmin, rmax, rotations, shifts,
                                       vel=None if vel is None else vel.detach(), **kw)

    @staticmethod
    def backward(ctx, map_bar):
        nside, box, obs, rmin, rmax, rotations, shifts, kw = ctx.geom
        saved = ctx.saved_tensors
        pos = saved[0].detach()
        vel = saved[1].detach() if ctx.has_v else None
        vel_bar = torch.zeros_like(vel) if vel is not None else None
        pos_bar = ops.healpix_paint_tiled_adjoint(pos, map_bar.contiguous(), nside, box, obs, rmin, rmax, rotations,
                                                  shifts, vel=vel, vel_bar=vel_bar, **kw)
        return pos_bar, vel_bar, None
