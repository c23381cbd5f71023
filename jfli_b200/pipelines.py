"""End-to-end forward models built from the public API.

`lightcone_convergence` is the large light-cone chain of the reference's
`make_full_field_model` (probabilistic_models/forward_model.py:24-79) with spherical
painting (NoInterp inside the box, or OnionTiler replicas beyond it): white noise ->
linear ICs -> LPT -> EfficientDriftDoubleKick (with an optional PGD correction) painting
`nb_shells` HEALPix shells during the run -> Born convergence for the given source
distributions. Every array stays on the GPU; the
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
                          min_z: float = 0.01, max_z: float = 1.0, n_integrate: int = 32, tiler: str = "none",
                          max_radius: float | None = None, noise=None,
                          rotation_indices=None) -> LightconeResult:
    """pgd = (alpha, kl, ks) with kl, ks in h/Mpc, or None.

    noise: the (mesh,)^3 white noise (array or tensor) to start from; when None it is
    drawn on the device from `seed`. rotation_indices: OnionTiler's 27 cube-symmetry
    indices (None: its seeded draw).

    tiler "none": nb_shells equal-width shells inside the box (NoInterp; radii up to the
    largest sphere around the observer that the box holds, as nbody(nb_shells=...) gives).
    tiler "onion": nb_shells equal-width shells from 0 to `max_radius` (default three times
    that radius, which the 27 replicas cover completely around a centred observer), painted
    with OnionTiler (replicas beyond the box, light-cone drift on)."""
    import jfli_b200 as jf

    timings = {}
    sync = torch.cuda.synchronize
    t = time.perf_counter()
    if noise is None:
        gen = torch.Generator(device="cuda").manual_seed(int(seed))
        noise = torch.randn((mesh,) * 3, generator=gen, device="cuda", dtype=torch.float32)
    else:
        noise = torch.as_tensor(noise, dtype=torch.float32).to("cuda")
        if tuple(noise.shape) != (mesh,) * 3:
            raise ValueError(f"noise must have shape {(mesh,) * 3}")
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
    painting = jf.PaintingOptions(target="spherical")
    if tiler == "none":
        kernel, geom = jf.NoInterp(painting=painting), dict(nb_shells=nb_shells)
    elif tiler == "onion":
        from . import cosmology as cj

        r_max = 3.0 * dx.max_comoving_radius if max_radius is None else float(max_radius)
        edges = np.linspace(0.0, r_max, nb_shells + 1)[::-1]  # far -> near, as the time loop meets them
        centres = 0.5 * (edges[1:] + edges[:-1])
        kernel = jf.OnionTiler(painting=painting, rotation_indices=None if rotation_indices is None
                               else tuple(int(i) for i in rotation_indices))
        geom = dict(ts=np.asarray(cj.a_of_chi(cosmo, centres), np.float64), density_widths=edges[:-1] - edges[1:])
    else:
        raise ValueError(f"tiler must be 'none' or 'onion', not {tiler!r}")
    solver = jf.EfficientDriftDoubleKick(interp_kernel=kernel, pgd_kernel=correction)
    t = time.perf_counter()
    shells, run = jf.nbody(cosmo, dx, p, t0=t0, t1=t1, dt0=(t1 - t0) / steps, solver=solver, return_state=True,
                           **geom)
    sync()
    timings["nbody_s"] = time.perf_counter() - t
    n_steps = run.steps
    del dx, p, run
    t = time.perf_counter()
    kappa = jf.born(cosmo, shells, nz_shear, min_z=min_z, max_z=max_z, n_integrate=n_integrate)
    sync()
    timings["born_s"] = time.perf_counter() - t
    return LightconeResult(kappa=kappa, shells=shells, steps=n_steps, timings=timings)
