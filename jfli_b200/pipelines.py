"""End-to-end forward models built from the public API.

`lightcone_convergence` is the large light-cone chain of the reference's
`make_full_field_model` (probabilistic_models/forward_model.py:24-79) with NoInterp
spherical painting: white noise -> linear ICs -> LPT -> EfficientDriftDoubleKick (with an
optional PGD correction) painting `nb_shells` HEALPix shells during the run -> Born
convergence for the given source distributions. Every array stays on the GPU; the
white noise is drawn on the device from the seed.
"""

from __future__ import annotations

import dataclasses
import time

import numpy as np
import torch

from . import ops


@dataclasses.dataclass
class LightconeResult:
    kappa: object  # SphericalDensity (status KAPPA), (n_sources, npix)
    shells: object  # SphericalDensity (status LIGHTCONE), (nb_shells, npix), near -> far
    steps: int
    timings: dict


def pgd_scales_to_grid(kl_hmpc: float, ks_hmpc: float, mesh: int, box: float):
    """PGD scales given in h/Mpc -> the radians-per-cell units PGDKernel takes (k L / N)."""
    return kl_hmpc * box / mesh, ks_hmpc * box / mesh


def lightcone_convergence(cosmo, *, mesh: int, box: float, seed: int, nb_shells: int, nside: int, nz_shear,
                          t0: float = 0.1, t1: float = 1.0, steps: int = 60, lpt_order: int = 2, pgd=None,
                          min_z: float = 0.01, max_z: float = 1.0, n_integrate: int = 32) -> LightconeResult:
    """pgd = (alpha, kl, ks) with kl, ks in h/Mpc, or None."""
    import jfli_b200 as jf

    timings = {}
    sync = torch.cuda.synchronize
    t = time.perf_counter()
    gen = torch.Generator(device="cuda").manual_seed(int(seed))
    noise = torch.randn((mesh,) * 3, generator=gen, device="cuda", dtype=torch.float32)
    ic = jf.interpolate_initial_conditions(noise, (mesh,) * 3, (box,) * 3, cosmo=cosmo, nside=nside)
    del noise
    dx, p = jf.lpt(cosmo, ic, ts=t0, order=lpt_order)
    del ic
    ops.release_workspaces()  # the LPT scratch is the largest one; the step allocates its own
    torch.cuda.empty_cache()
    sync()
    timings["ics_lpt_s"] = time.perf_counter() - t

    correction = jf.NoCorrection()
    if pgd is not None:
        alpha, kl, ks = pgd
        kl_g, ks_g = pgd_scales_to_grid(kl, ks, mesh, box)
        correction = jf.PGDKernel(alpha=float(alpha), kl=float(kl_g), ks=float(ks_g))
    solver = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="spherical")),
                                         pgd_kernel=correction)
    t = time.perf_counter()
    shells, run = jf.nbody(cosmo, dx, p, t0=t0, t1=t1, dt0=(t1 - t0) / steps, nb_shells=nb_shells, solver=solver,
                           return_state=True)
    sync()
    timings["nbody_s"] = time.perf_counter() - t
    n_steps = run.steps
    del dx, p, run
    t = time.perf_counter()
    kappa = jf.born(cosmo, shells, nz_shear, min_z=min_z, max_z=max_z, n_integrate=n_integrate)
    sync()
    timings["born_s"] = time.perf_counter() - t
    return LightconeResult(kappa=kappa, shells=shells, steps=n_steps, timings=timings)
