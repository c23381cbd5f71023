"""Sub-grid corrections (reference pm/correction.py:25-333)."""

from __future__ import annotations

import dataclasses

import torch

from .. import ops
from .._lib import JFLI_STEP_CORRECT, JFLI_STEP_KICK, JFLI_STEP_PAINT


class AbstractCorrection:
    reversible: bool = True

    def apply(self, t, pos, vel, full_drift_factor):
        raise NotImplementedError

    def rewind(self, t, pos, vel, full_drift_factor):
        raise NotImplementedError


@dataclasses.dataclass(frozen=True)
class NoCorrection(AbstractCorrection):
    @property
    def reversible(self) -> bool:
        return True

    def apply(self, t, pos, vel, full_drift_factor):
        return pos, vel

    def rewind(self, t, pos, vel, full_drift_factor):
        return pos, vel


@dataclasses.dataclass(frozen=True)
class PGDKernel(AbstractCorrection):
    """Potential-gradient-descent position correction (reference pm/correction.py:130-202):
    x += alpha * F_pgd(x), F_pgd the FD-gradient force of the potential filtered by
    exp(-kl^2/k^2) exp(-k^4/ks^4), k in radians per cell."""

    alpha: float = 0.2
    kl: float = 0.3
    ks: float = 1.0

    @property
    def reversible(self) -> bool:
        return False

    def pgd_potential(self, rho: torch.Tensor, rho_mean: float = 1.0) -> torch.Tensor:
        return pgd_potential(rho, self.kl, self.ks, rho_mean)

    def apply(self, t, pos, vel, full_drift_factor):
        from ..fields import PositionUnit

        if pos.unit != PositionUnit.GRID_RELATIVE:
            pos = pos.to(PositionUnit.GRID_RELATIVE)
        if torch.is_grad_enabled() and pos.array.requires_grad:
            return pos.replace(array=PgdCorrection.apply(pos.array, (self.alpha, self.kl, self.ks))), vel
        return pos.replace(array=pgd_correct(pos.array, self.alpha, self.kl, self.ks)), vel

    def rewind(self, t, pos, vel, full_drift_factor):
        raise NotImplementedError("PGDKernel is not reversible")


@dataclasses.dataclass(frozen=True)
class SharpeningKernel(AbstractCorrection):
    """Reversible PGD-style correction (reference pm/correction.py:214-333): a velocity boost
    v += alpha F_pgd(x) / full_drift_factor at the positions the next drift starts from, so
    that the drift adds alpha F_pgd(x) to x on top of v * drift; rewind takes the same boost
    off at the un-drifted positions. F_pgd as for PGDKernel. The fused loops fold the boost
    into the step's kick (one combined potential, sharpen_potential)."""

    alpha: float = 0.2
    kl: float = 0.3
    ks: float = 1.0

    @property
    def reversible(self) -> bool:
        return True

    def boost(self, full_drift_factor: float) -> float:
        """The factor of F_pgd in the velocity boost."""
        return float(self.alpha) / float(full_drift_factor)

    def _boosted(self, pos, vel, factor):
        x = pos.array.contiguous()
        v = vel.array.contiguous().clone()
        rho = ops.paint_cic(x)
        force = ops.force_mesh(pgd_potential(rho, self.kl, self.ks, 1.0))
        ops.kick_drift_paint(x, v, force, factor, 0.0, JFLI_STEP_KICK)
        return pos, vel.replace(array=v)

    def apply(self, t, pos, vel, full_drift_factor):
        return self._boosted(pos, vel, self.boost(full_drift_factor))

    def rewind(self, t, pos, vel, full_drift_factor):
        return self._boosted(pos, vel, -self.boost(full_drift_factor))


def pgd_correct(x: torch.Tensor, alpha: float, kl: float, ks: float) -> torch.Tensor:
    """x + alpha F_pgd(x) for relative displacements x (a new tensor)."""
    x = x.detach().contiguous().clone()
    rho = ops.paint_cic(x)
    force = ops.force_mesh(pgd_potential(rho, kl, ks, 1.0))
    ops.kick_drift_paint(x, torch.empty_like(x), force, alpha, 0.0, JFLI_STEP_CORRECT)
    return x


class PgdCorrection(torch.autograd.Function):
    """x -> x + alpha F_pgd(x) as an autograd node; backward jfli_pgd_adjoint (the readout
    and density parts of J^T, at the uncorrected positions)."""

    @staticmethod
    def forward(ctx, x, params):
        ctx.params = params
        ctx.save_for_backward(x)
        return pgd_correct(x, *params)

    @staticmethod
    def backward(ctx, g):
        from .._lib import call, ptr, query, stream_ptr

        (x,) = ctx.saved_tensors
        alpha, kl, ks = ctx.params
        x = x.detach().contiguous()
        u = g.contiguous()
        lam = u.clone()
        (nx, ny, nz), batch, _ = ops._mesh_dims(x, True)
        ws = ops.workspace(int(query("jfli_pgd_adjoint_workspace_bytes", nx, ny, nz, batch)), "pgd_adj", x.device)
        call("jfli_pgd_adjoint", stream_ptr(), ptr(x), ptr(u), float(alpha), float(kl), float(ks), ptr(lam), ptr(ws),
             ws.numel(), nx, ny, nz, batch)
        return lam, None


def pgd_potential(rho: torch.Tensor, kl: float, ks: float, rho_mean: float = 1.0,
                  out: torch.Tensor | None = None) -> torch.Tensor:
    from .._lib import call, ptr, query, stream_ptr

    (nx, ny, nz) = tuple(rho.shape[-3:])
    batch = rho.numel() // (nx * ny * nz)
    if out is None:
        out = torch.empty_like(rho)
    nb = query("jfli_poisson_workspace_bytes", nx, ny, nz, batch)
    ws = ops.workspace(nb, "spec", rho.device)
    call("jfli_pgd_potential", stream_ptr(), ptr(rho), float(rho_mean), float(kl), float(ks), ptr(out), ptr(ws),
         ws.numel(), nx, ny, nz, batch)
    return out


def sharpen_potential(rho: torch.Tensor, kick: float, boost: float, kl: float, ks: float, rho_mean: float = 1.0,
                      out: torch.Tensor | None = None) -> torch.Tensor:
    """The potential whose force, applied with factor 1, is kick F + boost F_pgd at the
    positions rho was painted from (jfli_sharpen_potential)."""
    from .._lib import call, ptr, query, stream_ptr

    (nx, ny, nz) = tuple(rho.shape[-3:])
    batch = rho.numel() // (nx * ny * nz)
    if out is None:
        out = torch.empty_like(rho)
    nb = query("jfli_poisson_workspace_bytes", nx, ny, nz, batch)
    ws = ops.workspace(nb, "spec", rho.device)
    call("jfli_sharpen_potential", stream_ptr(), ptr(rho), float(rho_mean), float(kick), float(boost), float(kl),
         float(ks), ptr(out), ptr(ws), ws.numel(), nx, ny, nz, batch)
    return out
