"""Tensor-level wrappers around the C-ABI kernels.

Every function takes CUDA float32 tensors (a leading batch dimension is optional),
enqueues the library's kernels on torch's current stream and returns new tensors or
fills the ones given. Shapes:

* mesh       (..., nx, ny, nz)
* particles  (..., nx, ny, nz, 3)
* spectrum   (..., nx, ny, nz//2+1) complex64
"""

from __future__ import annotations

import collections
import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr, query, stream_ptr

_workspaces: dict[tuple, torch.Tensor] = {}


def workspace(nbytes: int, key: str = "default", device=None) -> torch.Tensor:
    """A cached uint8 device buffer of at least `nbytes`, one per key, device and current
    stream, so that work enqueued on different streams never shares scratch space."""
    dev = torch.device("cuda") if device is None else torch.device(device)
    idx = dev.index if dev.index is not None else torch.cuda.current_device()
    k = (key, idx, torch.cuda.current_stream(idx).cuda_stream)
    buf = _workspaces.get(k)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)
        _workspaces[k] = buf
    return buf


_TABLES: "collections.OrderedDict[tuple, torch.Tensor]" = collections.OrderedDict()


def device_table(values, device="cuda", dtype=np.float32) -> torch.Tensor:
    """A small host table (bin edges, P(k) samples) on the device, cached by content and
    read-only for callers. A copy from pageable host memory makes the host wait until the
    stream has drained, which stalls a caller that enqueues the next request while the GPU
    works on this one: a table met before is reused, a new one goes up through pinned
    memory without blocking."""
    a = np.ascontiguousarray(np.asarray(values, dtype=dtype))
    dev = torch.device(device)
    key = (a.tobytes(), a.shape, a.dtype.str, str(dev))
    t = _TABLES.get(key)
    if t is None:
        t = torch.from_numpy(a.copy())
        t = t.pin_memory().to(dev, non_blocking=True) if dev.type == "cuda" else t.to(dev)
        _TABLES[key] = t
        if len(_TABLES) > 64:
            _TABLES.popitem(last=False)
    else:
        _TABLES.move_to_end(key)
    return t


def release_workspaces():
    _workspaces.clear()


def _mesh_dims(t: torch.Tensor, particle: bool):
    shape = tuple(t.shape)
    core = shape[-4:-1] if particle else shape[-3:]
    if len(core) != 3:
        raise ValueError(f"bad {'particle' if particle else 'mesh'} tensor shape {shape}")
    lead = shape[:-4] if particle else shape[:-3]
    batch = int(np.prod(lead)) if lead else 1
    return tuple(int(v) for v in core), batch, lead


def _check(t: torch.Tensor, name: str, dtype=torch.float32):
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def mesh_supported(nx: int, ny: int, nz: int) -> bool:
    return bool(query("jfli_mesh_supported", nx, ny, nz))


def rfft3d(mesh: torch.Tensor) -> torch.Tensor:
    _check(mesh, "mesh")
    (nx, ny, nz), batch, lead = _mesh_dims(mesh, False)
    spec = torch.empty(*lead, nx, ny, nz // 2 + 1, dtype=torch.complex64, device=mesh.device)
    call("jfli_rfft3d", stream_ptr(), ptr(mesh), ptr(spec), nx, ny, nz, batch)
    return spec


def irfft3d(spec: torch.Tensor, nz: int) -> torch.Tensor:
    """Inverse of rfft3d; the spectrum is copied first (the kernel overwrites its input)."""
    if spec.dtype != torch.complex64:
        raise TypeError("spec must be complex64")
    work = spec.contiguous().clone()
    nx, ny = int(spec.shape[-3]), int(spec.shape[-2])
    lead = tuple(spec.shape[:-3])
    batch = int(np.prod(lead)) if lead else 1
    out = torch.empty(*lead, nx, ny, nz, dtype=torch.float32, device=spec.device)
    call("jfli_irfft3d", stream_ptr(), ptr(work), ptr(out), nx, ny, nz, batch)
    return out


def paint_cic(pos: torch.Tensor, *, absolute: bool = False, weights: torch.Tensor | None = None,
              weight: float = 1.0, out: torch.Tensor | None = None, accumulate: bool = False) -> torch.Tensor:
    _check(pos, "pos")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    if weights is not None:
        _check(weights, "weights")
        if tuple(weights.shape) != tuple(pos.shape[:-1]):
            raise ValueError("weights must have the particle grid shape")
    if out is None:
        out = torch.empty(*lead, nx, ny, nz, dtype=torch.float32, device=pos.device)
        accumulate = False
    call("jfli_paint_cic", stream_ptr(), ptr(pos), int(absolute), ptr(weights), float(weight), ptr(out),
         int(accumulate), nx, ny, nz, batch)
    return out


def readout_cic(pos: torch.Tensor, mesh: torch.Tensor, *, absolute: bool = False) -> torch.Tensor:
    _check(pos, "pos")
    _check(mesh, "mesh")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    if tuple(mesh.shape[-3:]) != (nx, ny, nz):
        raise ValueError("mesh and particle grid shapes differ")
    out = torch.empty(*lead, nx, ny, nz, dtype=torch.float32, device=pos.device)
    call("jfli_readout_cic", stream_ptr(), ptr(pos), int(absolute), ptr(mesh), ptr(out), nx, ny, nz, batch)
    return out


def poisson_potential(rho: torch.Tensor, rho_mean: float = 0.0, out: torch.Tensor | None = None) -> torch.Tensor:
    _check(rho, "rho")
    (nx, ny, nz), batch, lead = _mesh_dims(rho, False)
    if out is None:
        out = torch.empty_like(rho)
    nb = query("jfli_poisson_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "spec", rho.device)
    call("jfli_poisson_potential", stream_ptr(), ptr(rho), float(rho_mean), ptr(out), ptr(ws), ws.numel(), nx, ny,
         nz, batch)
    return out


def readout_gradient(pos: torch.Tensor, pot: torch.Tensor, *, absolute: bool = False, scale: float = 1.0,
                     out: torch.Tensor | None = None) -> torch.Tensor:
    _check(pos, "pos")
    _check(pot, "pot")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    if out is None:
        out = torch.empty_like(pos)
    call("jfli_readout_gradient", stream_ptr(), ptr(pos), int(absolute), ptr(pot), float(scale), ptr(out), nx, ny,
         nz, batch)
    return out


def pm_forces(pos: torch.Tensor, *, absolute: bool = False, scale: float = 1.0) -> torch.Tensor:
    """paint -> Poisson -> -grad_FD -> readout, times `scale` (jax-fli _forces: 1.5 Omega_m)."""
    _check(pos, "pos")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    out = torch.empty_like(pos)
    nb = query("jfli_pm_forces_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "forces", pos.device)
    call("jfli_pm_forces", stream_ptr(), ptr(pos), int(absolute), float(scale), ptr(out), ptr(ws), ws.numel(), nx,
         ny, nz, batch)
    return out


def force_mesh(pot: torch.Tensor, scale: float = 1.0, out: torch.Tensor | None = None) -> torch.Tensor:
    """(..., nx, ny, nz, 4) force mesh scale * (-D pot) as (Fx, Fy, Fz, 0) per cell, D the
    4-point finite difference."""
    _check(pot, "pot")
    (nx, ny, nz), batch, lead = _mesh_dims(pot, False)
    if out is None:
        out = torch.empty(*lead, nx, ny, nz, 4, dtype=torch.float32, device=pot.device)
    elif out.numel() != 4 * batch * nx * ny * nz:
        raise ValueError("out must hold (nx, ny, nz, 4) per mesh")
    call("jfli_force_mesh", stream_ptr(), ptr(pot), float(scale), ptr(out), nx, ny, nz, batch)
    return out


def poisson_force(rho: torch.Tensor, rho_mean: float = 1.0, out: torch.Tensor | None = None,
                  pot: torch.Tensor | None = None, clear: bool = False) -> torch.Tensor:
    """Force meshes of a density: Poisson solve, then the finite-difference gradient (one
    library call). With clear=True the density mesh comes back zeroed (the forward FFT
    clears what it reads), ready for the next paint."""
    _check(rho, "rho")
    (nx, ny, nz), batch, lead = _mesh_dims(rho, False)
    if pot is None:
        pot = torch.empty_like(rho)
    if out is None:
        out = torch.empty(*lead, nx, ny, nz, 4, dtype=torch.float32, device=rho.device)
    elif out.numel() != 4 * batch * nx * ny * nz:
        raise ValueError("out must hold (nx, ny, nz, 4) per mesh")
    nb = query("jfli_poisson_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "spec", rho.device)
    call("jfli_poisson_force", stream_ptr(), ptr(rho), float(rho_mean), int(bool(clear)), 1.0, ptr(pot), ptr(out),
         ptr(ws), ws.numel(), nx, ny, nz, batch)
    return out


def kick_drift_paint(disp: torch.Tensor, vel: torch.Tensor, force: torch.Tensor | None, kick: float, drift: float,
                     flags: int, rho: torch.Tensor | None = None, weight: float = 1.0) -> None:
    """In place: [kick (or CORRECT shift) with the CIC readout of `force`] -> [drift] -> [paint]."""
    _check(disp, "disp")
    _check(vel, "vel")
    (nx, ny, nz), batch, _ = _mesh_dims(disp, True)
    if force is not None:
        _check(force, "force")
        if force.numel() != 4 * batch * nx * ny * nz:
            raise ValueError("force must hold an (nx, ny, nz, 4) force mesh per particle grid")
    call("jfli_kick_drift_paint", stream_ptr(), ptr(disp), ptr(vel), ptr(force), float(kick), float(drift),
         int(flags), float(weight), ptr(rho), nx, ny, nz, batch)


def pm_step(disp, vel, kick, drift, flags, rho, force) -> None:
    (nx, ny, nz), batch, _ = _mesh_dims(disp, True)
    nb = query("jfli_pm_step_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "pm_step", disp.device)
    call("jfli_pm_step", stream_ptr(), ptr(disp), ptr(vel), float(kick), float(drift), int(flags), ptr(rho),
         ptr(force), ptr(ws), ws.numel(), nx, ny, nz, batch)


def zero_(t: torch.Tensor) -> torch.Tensor:
    """Set a float32 CUDA tensor to zero in place with the library's kernel (jfli_zero)."""
    _check(t, "t")
    call("jfli_zero", stream_ptr(), ptr(t), int(t.numel()))
    return t


def ic_filter(noise: torch.Tensor, ktab: torch.Tensor, ptab: torch.Tensor, box_size, *,
              zero_mode_one: bool = False) -> torch.Tensor:
    _check(noise, "noise")
    _check(ktab, "ktab")
    _check(ptab, "ptab")
    (nx, ny, nz), batch, lead = _mesh_dims(noise, False)
    out = torch.empty_like(noise)
    nb = query("jfli_poisson_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "spec", noise.device)
    lx, ly, lz = (float(v) for v in box_size)
    call("jfli_ic_filter", stream_ptr(), ptr(noise), ptr(out), ptr(ktab), ptr(ptab), int(ktab.numel()), lx, ly, lz,
         int(zero_mode_one), ptr(ws), ws.numel(), nx, ny, nz, batch)
    return out


def lpt_lightcone(ic: torch.Tensor, order: int, cosmo, box_size, observer_mpc):
    """(displacement, momentum, scale factor) particle grids of light-cone-mode LPT: every
    particle at the scale factor of its Lagrangian grid point's light-cone crossing
    (jfli_lpt_lightcone), from the cosmology's FP64 distance and growth tables."""
    import numpy as np

    from . import cosmology as cj

    _check(ic, "ic")
    (nx, ny, nz), batch, lead = _mesh_dims(ic, False)
    dt = cj.distance_table(cosmo)
    gt = cj.growth_table(cosmo)
    tables = np.concatenate([dt.chi[::-1], dt.a[::-1], gt.a, gt.g, gt.f, gt.g2, gt.f2]).astype(np.float64)
    tab = torch.as_tensor(tables, device=ic.device)
    bg = (ctypes.c_double * 5)(cosmo.Omega_m, cosmo.Omega_k, cosmo.Omega_de, cosmo.w0, cosmo.wa)
    dx = torch.empty((*lead, nx, ny, nz, 3), dtype=torch.float32, device=ic.device)
    p = torch.empty_like(dx)
    a = torch.empty((*lead, nx, ny, nz), dtype=torch.float32, device=ic.device)
    nb = query("jfli_lpt_lightcone_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "lpt_lightcone", ic.device)
    lx, ly, lz = (float(v) for v in box_size)
    ox, oy, oz = (float(v) for v in observer_mpc)
    call("jfli_lpt_lightcone", stream_ptr(), ptr(ic), int(order), ptr(tab), len(dt.chi), len(gt.a), bg, lx, ly, lz,
         ox, oy, oz, ptr(dx), ptr(p), ptr(a), ptr(ws), ws.numel(), nx, ny, nz, batch)
    return dx, p, a


def lpt(ic: torch.Tensor, order: int, c1x: float, c2x: float, c1p: float, c2p: float,
        dx: torch.Tensor | None = None, p: torch.Tensor | None = None):
    """(displacement, momentum) particle grids; written into dx / p when given."""
    _check(ic, "ic")
    (nx, ny, nz), batch, lead = _mesh_dims(ic, False)
    shape = (*lead, nx, ny, nz, 3)
    for name, t in (("dx", dx), ("p", p)):
        if t is not None:
            _check(t, name)
            if tuple(t.shape) != shape:
                raise ValueError(f"{name} must have shape {shape}")
    if dx is None:
        dx = torch.empty(shape, dtype=torch.float32, device=ic.device)
    if p is None:
        p = torch.empty(shape, dtype=torch.float32, device=ic.device)
    nb = query("jfli_lpt_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "lpt", ic.device)
    call("jfli_lpt", stream_ptr(), ptr(ic), int(order), float(c1x), float(c2x), float(c1p), float(c2p), ptr(dx),
         ptr(p), ptr(ws), ws.numel(), nx, ny, nz, batch)
    return dx, p


def power_sums(mesh: torch.Tensor, kedges: torch.Tensor, box_size) -> torch.Tensor:
    """(..., 3, nedges+1) float64 sums: |delta_k|^2, mode count, |k| per digitize bin."""
    _check(mesh, "mesh")
    _check(kedges, "kedges")
    (nx, ny, nz), batch, lead = _mesh_dims(mesh, False)
    ne = int(kedges.numel())
    out = torch.empty(*lead, 3, ne + 1, dtype=torch.float64, device=mesh.device)
    nb = query("jfli_power_spectrum_workspace_bytes", nx, ny, nz, batch, ne)
    ws = workspace(nb, "power", mesh.device)
    lx, ly, lz = (float(v) for v in box_size)
    call("jfli_power_spectrum", stream_ptr(), ptr(mesh), ptr(kedges), ne, lx, ly, lz, ptr(out), ptr(ws), ws.numel(),
         nx, ny, nz, batch)
    return out


def rbf_sigma(nside: int, kernel_width_arcmin=None, smoothing_interpretation: str = "fwhm") -> float:
    """Gaussian sigma (radians) of the rbf_neighbor scheme: kernel_width_arcmin read as a
    FWHM (sigma = FWHM / sqrt(8 ln 2)) or as sigma itself; without a width, the pixel size
    sqrt(4 pi / npix) is the FWHM."""
    if smoothing_interpretation not in ("fwhm", "sigma"):
        raise ValueError(f"smoothing_interpretation must be 'fwhm' or 'sigma', got {smoothing_interpretation!r}")
    if kernel_width_arcmin is None:
        width, smoothing_interpretation = math.sqrt(4.0 * math.pi / (12 * nside * nside)), "fwhm"
    else:
        width = float(kernel_width_arcmin) * math.pi / (180.0 * 60.0)
    if not width > 0:
        raise ValueError("kernel_width_arcmin must be positive")
    return width / math.sqrt(8.0 * math.log(2.0)) if smoothing_interpretation == "fwhm" else width


def healpix_paint(pos: torch.Tensor, nside: int, box_size, observer_mpc, rmin: float, rmax: float, *,
                  scheme: str = "bilinear", absolute: bool = False, weights: torch.Tensor | None = None,
                  weight: float = 1.0, out: torch.Tensor | None = None, accumulate: bool = False,
                  sigma: float | None = None) -> torch.Tensor:
    """Shell map; `sigma` (radians) is the Gaussian width of the rbf_neighbor scheme
    (default: rbf_sigma(nside))."""
    _check(pos, "pos")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    sch = {"ngp": _lib.JFLI_HEALPIX_NGP, "bilinear": _lib.JFLI_HEALPIX_BILINEAR, "rbf_neighbor": 2}.get(scheme)
    if sch is None:
        raise NotImplementedError(f"spherical painting scheme {scheme!r} is not implemented (ngp, bilinear, "
                                  f"rbf_neighbor)")
    if out is None:
        out = torch.empty(*lead, 12 * nside * nside, dtype=torch.float32, device=pos.device)
        accumulate = False
    lx, ly, lz = (float(v) for v in box_size)
    ox, oy, oz = (float(v) for v in observer_mpc)
    if sch == 2:
        sg = rbf_sigma(nside) if sigma is None else float(sigma)
        call("jfli_healpix_paint_rbf", stream_ptr(), ptr(pos), int(absolute), ptr(weights), float(weight), lx, ly, lz,
             ox, oy, oz, float(rmin), float(rmax), int(nside), sg, ptr(out), int(accumulate), nx, ny, nz, batch)
        return out
    call("jfli_healpix_paint", stream_ptr(), ptr(pos), int(absolute), ptr(weights), float(weight), lx, ly, lz, ox,
         oy, oz, float(rmin), float(rmax), int(nside), sch, ptr(out), int(accumulate), nx, ny, nz, batch)
    return out


def healpix_paint_shells(pos: torch.Tensor, nside: int, box_size, observer_mpc, rmin, rmax, scale, *,
                         scheme: str = "bilinear", absolute: bool = False, weights: torch.Tensor | None = None,
                         weight: float = 1.0, out: torch.Tensor | None = None, accumulate: bool = False,
                         sigma: float | None = None) -> torch.Tensor:
    """(S, 12 nside^2) maps of S shells of one particle set in one pass (see
    jfli_healpix_paint_shells); rmin, rmax, scale: S values each."""
    _check(pos, "pos")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    if batch != 1:
        raise ValueError("healpix_paint_shells paints one particle set")
    sch = {"ngp": _lib.JFLI_HEALPIX_NGP, "bilinear": _lib.JFLI_HEALPIX_BILINEAR, "rbf_neighbor": 2}.get(scheme)
    if sch is None:
        raise NotImplementedError(f"spherical painting scheme {scheme!r} is not implemented (ngp, bilinear, "
                                  f"rbf_neighbor)")
    lo = np.ascontiguousarray(np.atleast_1d(np.asarray(rmin, np.float64)))
    hi = np.ascontiguousarray(np.atleast_1d(np.asarray(rmax, np.float64)))
    sc = np.ascontiguousarray(np.atleast_1d(np.asarray(scale, np.float32)))
    if not (lo.shape == hi.shape == sc.shape):
        raise ValueError("rmin, rmax and scale must have one value per shell")
    npix = 12 * nside * nside
    if out is None:
        out = torch.empty(lo.size, npix, dtype=torch.float32, device=pos.device)
        accumulate = False
    elif tuple(out.shape) != (lo.size, npix) or not out.is_contiguous():
        raise ValueError(f"out must be a contiguous ({lo.size}, {npix}) tensor")
    lx, ly, lz = (float(v) for v in box_size)
    ox, oy, oz = (float(v) for v in observer_mpc)
    sg = (rbf_sigma(nside) if sigma is None else float(sigma)) if sch == 2 else 0.0
    dp = ctypes.POINTER(ctypes.c_double)
    call("jfli_healpix_paint_shells", stream_ptr(), ptr(pos), int(absolute), ptr(weights), float(weight), lx, ly, lz,
         ox, oy, oz, int(lo.size), lo.ctypes.data_as(dp), hi.ctypes.data_as(dp),
         sc.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(nside), sch, sg, ptr(out), int(accumulate), nx, ny,
         nz, batch)
    return out


def healpix_paint_shells_adjoint(pos: torch.Tensor, maps_bar: torch.Tensor, nside: int, box_size, observer_mpc, rmin,
                                 rmax, scale, *, scheme: str = "bilinear", absolute: bool = False,
                                 weights: torch.Tensor | None = None, weight: float = 1.0,
                                 pos_bar: torch.Tensor | None = None,
                                 weights_bar: torch.Tensor | None = None) -> torch.Tensor:
    """Adjoint of healpix_paint_shells: accumulates into pos_bar (zeros when None, returned)
    and, when given, weights_bar (see jfli_healpix_paint_shells_adjoint)."""
    _check(pos, "pos")
    _check(maps_bar, "maps_bar")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    if batch != 1:
        raise ValueError("healpix_paint_shells_adjoint takes one particle set")
    sch = {"ngp": _lib.JFLI_HEALPIX_NGP, "bilinear": _lib.JFLI_HEALPIX_BILINEAR}.get(scheme)
    if sch is None:
        raise NotImplementedError(f"the shell-painting adjoint has the ngp and bilinear schemes, not {scheme!r}")
    lo = np.ascontiguousarray(np.atleast_1d(np.asarray(rmin, np.float64)))
    hi = np.ascontiguousarray(np.atleast_1d(np.asarray(rmax, np.float64)))
    sc = np.ascontiguousarray(np.atleast_1d(np.asarray(scale, np.float32)))
    npix = 12 * nside * nside
    if tuple(maps_bar.shape) != (lo.size, npix) or not maps_bar.is_contiguous():
        raise ValueError(f"maps_bar must be a contiguous ({lo.size}, {npix}) tensor")
    if pos_bar is None:
        pos_bar = torch.zeros_like(pos)
    lx, ly, lz = (float(v) for v in box_size)
    ox, oy, oz = (float(v) for v in observer_mpc)
    dp = ctypes.POINTER(ctypes.c_double)
    call("jfli_healpix_paint_shells_adjoint", stream_ptr(), ptr(pos), int(absolute), ptr(weights), float(weight), lx,
         ly, lz, ox, oy, oz, int(lo.size), lo.ctypes.data_as(dp), hi.ctypes.data_as(dp),
         sc.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(nside), sch, ptr(maps_bar), ptr(pos_bar),
         ptr(weights_bar), nx, ny, nz, batch)
    return pos_bar


def drift_tables(cosmo, n_dense: int = 4096):
    """Device FP32 copies of the FP64 host tables the light-cone drift interpolates:
    (chi ascending, a at chi), (growth a, D1), (dense a, dGfa)."""
    from . import cosmology as cj

    dt = cj.distance_table(cosmo)
    gt = cj.growth_table(cosmo)
    da = np.logspace(-3.0, 0.0, n_dense)
    tabs = (dt.chi[::-1], dt.a[::-1], gt.a, gt.g, da, cj.dGfa(cosmo, da))
    return tuple(torch.as_tensor(np.ascontiguousarray(t, dtype=np.float32), device="cuda") for t in tabs)


def replica_positions(pos: torch.Tensor, box_size, observer_mpc, rotation, shift, *, absolute: bool = False,
                      vel: torch.Tensor | None = None, t: float | None = None, cosmo=None, telephoto: bool = False,
                      tables=None) -> torch.Tensor:
    """Mpc/h positions of one rotated, shifted (and, with vel, light-cone drifted) replica
    of the particles (see jfli_replica_positions)."""
    from . import cosmology as cj

    _check(pos, "pos")
    (nx, ny, nz), batch, _ = _mesh_dims(pos, True)
    rot = np.ascontiguousarray(np.rint(np.asarray(rotation, np.float64)).astype(np.int8).reshape(9))
    sh = np.ascontiguousarray(np.asarray(shift, np.float32).reshape(3))
    tabs = (None,) * 6
    t_arg = gp_t = 0.0
    if vel is not None:
        _check(vel, "vel")
        if t is None or cosmo is None:
            raise ValueError("the light-cone drift needs the time t and the cosmology")
        tabs = drift_tables(cosmo) if tables is None else tables
        t_arg = float(t)
        gp_t = float(cj.Gp(cosmo, t_arg))
    chi, a_chi, ga, g, da, dg = tabs
    n = lambda x: int(x.numel()) if x is not None else 0
    out = torch.empty_like(pos)
    lx, ly, lz = (float(v) for v in box_size)
    ox, oy, oz = (float(v) for v in observer_mpc)
    call("jfli_replica_positions", stream_ptr(), ptr(pos), int(absolute), ptr(vel), lx, ly, lz, ox, oy, oz,
         rot.ctypes.data_as(ctypes.POINTER(ctypes.c_byte)), sh.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
         int(bool(telephoto)), t_arg, gp_t, ptr(chi), ptr(a_chi), n(chi), ptr(ga), ptr(g), n(ga), ptr(da), ptr(dg),
         n(da), ptr(out), nx, ny, nz, batch)
    return out


def paint_flat_adjoint(pos: torch.Tensor, map_bar: torch.Tensor, zlo: float, zhi: float, *, absolute: bool = False,
                       weight: float = 1.0, pos_bar: torch.Tensor | None = None) -> torch.Tensor:
    """pos_bar += the gradient of <map_bar, paint_flat(pos, ...)> in the positions (zeros when
    None; returned); scalar weight (jfli_paint_flat_adjoint)."""
    _check(pos, "pos")
    _check(map_bar, "map_bar")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    npx, npy = (int(v) for v in map_bar.shape[-2:])
    if pos_bar is None:
        pos_bar = torch.zeros_like(pos)
    call("jfli_paint_flat_adjoint", stream_ptr(), ptr(pos), int(absolute), float(weight), float(zlo), float(zhi), npx,
         npy, ptr(map_bar), ptr(pos_bar), nx, ny, nz, batch)
    return pos_bar


def paint_flat(pos: torch.Tensor, npix, zlo: float, zhi: float, *, absolute: bool = False,
               weights: torch.Tensor | None = None, weight: float = 1.0, out: torch.Tensor | None = None,
               accumulate: bool = False) -> torch.Tensor:
    """Flat-sky plane (..., npx, npy) of the particles with zlo < z <= zhi (grid units):
    raw 2D CIC sums (see jfli_paint_flat)."""
    _check(pos, "pos")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    npx, npy = (int(v) for v in npix)
    if out is None:
        out = torch.empty(*lead, npx, npy, dtype=torch.float32, device=pos.device)
        accumulate = False
    call("jfli_paint_flat", stream_ptr(), ptr(pos), int(absolute), ptr(weights), float(weight), float(zlo), float(zhi),
         npx, npy, ptr(out), int(accumulate), nx, ny, nz, batch)
    return out


def flat_cl_sums(map1: torch.Tensor, map2: torch.Tensor | None, dnx: float, dny: float,
                 ell_edges: torch.Tensor) -> torch.Tensor:
    """(batch, 3, nedges + 1) FP64 sums (power, modes, ell) of maps (..., npx, npy) binned by
    |ell| (see jfli_flat_cl); dnx, dny = n times the pixel size in radians."""
    _check(map1, "map1")
    if map2 is not None:
        _check(map2, "map2")
        if map2.shape != map1.shape:
            raise ValueError("map2 must have the shape of map1")
    npx, npy = map1.shape[-2:]
    batch = int(np.prod(map1.shape[:-2])) if map1.ndim > 2 else 1
    edges = ell_edges.to(device=map1.device, dtype=torch.float32).contiguous()
    nedges = int(edges.numel())
    nb = query("jfli_flat_cl_workspace_bytes", npx, npy, batch, nedges, int(map2 is not None))
    ws = workspace(nb, "flat_cl", map1.device)
    out = torch.empty(batch, 3, nedges + 1, dtype=torch.float64, device=map1.device)
    call("jfli_flat_cl", stream_ptr(), ptr(map1), ptr(map2), int(npx), int(npy), batch, float(dnx), float(dny),
         ptr(edges), nedges, ptr(out), ptr(ws), ws.numel())
    return out


def drift_bound(tables, t: float, gp_t: float) -> float:
    """Bound on |D| = |Gp(a_t) - Gp(t)| / dGfa(sqrt(t a_t)) as the drift kernels evaluate
    it for any distance inside the distance table: the Gp difference is at most
    max(Gp(t), 1 - Gp(t)) after the clip to [0, 1], and the interpolated dGfa is at least
    the smallest value it takes over the reachable sqrt(t a_t) (table nodes, or the linear
    extrapolation at the ends). Infinite when that minimum is not positive."""
    chi, a_chi, ga, g, da, dg = (x.double().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x, np.float64)
                                 for x in tables)
    lo, hi = math.sqrt(t * float(a_chi.min())), math.sqrt(t * float(a_chi.max()))

    def at(x):  # the kernels' linear interpolation with end extrapolation
        i = int(np.clip(np.searchsorted(da, x, side="left") - 1, 0, len(da) - 2))
        return dg[i] + (x - da[i]) * (dg[i + 1] - dg[i]) / (da[i + 1] - da[i])

    inside = dg[(da >= lo) & (da <= hi)]
    den = min([at(lo), at(hi)] + ([float(inside.min())] if inside.size else []))
    if not den > 0:
        return float("inf")
    return max(gp_t, 1.0 - gp_t) / den * 1.001 + 1e-6


def _tiled_prep(pos, rotations, shifts, scheme, vel, t, cosmo, tables, dbound):
    """(scheme code, int8 rotations (T, 9), float32 shifts (T, 3), drift tables, t, Gp(t),
    drift bound) for the replica painter and its adjoint."""
    from . import cosmology as cj

    sch = {"ngp": _lib.JFLI_HEALPIX_NGP, "bilinear": _lib.JFLI_HEALPIX_BILINEAR}.get(scheme)
    if sch is None:
        raise NotImplementedError(f"spherical painting scheme {scheme!r} is not implemented (ngp, bilinear)")
    rot = np.ascontiguousarray(np.rint(np.asarray(rotations, np.float64)).astype(np.int8).reshape(-1, 9))
    sh = np.ascontiguousarray(np.asarray(shifts, np.float32).reshape(-1, 3))
    if rot.shape[0] != sh.shape[0]:
        raise ValueError(f"{rot.shape[0]} rotations for {sh.shape[0]} shifts")
    tabs = (None,) * 6
    t_arg = gp_t = 0.0
    if vel is None:
        return sch, rot, sh, tabs, t_arg, gp_t, 0.0
    _check(vel, "vel")
    if vel.shape != pos.shape:
        raise ValueError("vel must have the shape of pos")
    if t is None or cosmo is None:
        raise ValueError("the light-cone drift needs the time t and the cosmology")
    tabs = drift_tables(cosmo) if tables is None else tables
    t_arg = float(t)
    gp_t = float(cj.Gp(cosmo, t_arg))
    if dbound is None:
        dbound = drift_bound(tabs, t_arg, gp_t)
    return sch, rot, sh, tabs, t_arg, gp_t, (dbound if math.isfinite(dbound) else 1e30)


def healpix_paint_tiled_adjoint(pos: torch.Tensor, map_bar: torch.Tensor, nside: int, box_size, observer_mpc,
                                rmin: float, rmax: float, rotations, shifts, *, absolute: bool = False,
                                vel: torch.Tensor | None = None, t: float | None = None, cosmo=None,
                                telephoto: bool = False, scheme: str = "bilinear",
                                weights: torch.Tensor | None = None, weight: float = 1.0, tables=None,
                                dbound: float | None = None, pos_bar: torch.Tensor | None = None,
                                vel_bar: torch.Tensor | None = None,
                                weights_bar: torch.Tensor | None = None) -> torch.Tensor:
    """Adjoint of healpix_paint_tiled: accumulates into pos_bar (zeros when None, returned),
    vel_bar and weights_bar (see jfli_healpix_paint_tiled_adjoint)."""
    _check(pos, "pos")
    _check(map_bar, "map_bar")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    sch, rot, sh, tabs, t_arg, gp_t, dbound = _tiled_prep(pos, rotations, shifts, scheme, vel, t, cosmo, tables, dbound)
    if tuple(map_bar.shape) != (*lead, 12 * nside * nside) or not map_bar.is_contiguous():
        raise ValueError("map_bar must be a contiguous map per particle set")
    if pos_bar is None:
        pos_bar = torch.zeros_like(pos)
    lx, ly, lz = (float(v) for v in box_size)
    ox, oy, oz = (float(v) for v in observer_mpc)
    chi, a_chi, ga, g, da, dg = tabs
    n = lambda x: int(x.numel()) if x is not None else 0
    call("jfli_healpix_paint_tiled_adjoint", stream_ptr(), ptr(pos), int(absolute), ptr(vel), ptr(weights),
         float(weight), lx, ly, lz, ox, oy, oz, int(rot.shape[0]), rot.ctypes.data_as(ctypes.POINTER(ctypes.c_byte)),
         sh.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(bool(telephoto)), float(rmin), float(rmax), t_arg,
         gp_t, float(dbound), ptr(chi), ptr(a_chi), n(chi), ptr(ga), ptr(g), n(ga), ptr(da), ptr(dg), n(da),
         int(nside), sch, ptr(map_bar), ptr(pos_bar), ptr(vel_bar), ptr(weights_bar), nx, ny, nz, batch)
    return pos_bar


def healpix_paint_tiled(pos: torch.Tensor, nside: int, box_size, observer_mpc, rmin: float, rmax: float, rotations,
                        shifts, *, absolute: bool = False, vel: torch.Tensor | None = None, t: float | None = None,
                        cosmo=None, telephoto: bool = False, scheme: str = "bilinear",
                        weights: torch.Tensor | None = None, weight: float = 1.0, out: torch.Tensor | None = None,
                        accumulate: bool = False, tables=None, dbound: float | None = None) -> torch.Tensor:
    """Shell map of the rotated and shifted replicas of `pos` (one pass; see
    jfli_healpix_paint_tiled). rotations (T, 3, 3) signed permutation matrices, shifts
    (T, 3) in Mpc/h; with `vel` the replicas are drifted to the light cone at time t.
    `dbound` replaces the computed drift bound (a larger one only skips fewer replicas)."""
    _check(pos, "pos")
    (nx, ny, nz), batch, lead = _mesh_dims(pos, True)
    sch, rot, sh, tabs, t_arg, gp_t, dbound = _tiled_prep(pos, rotations, shifts, scheme, vel, t, cosmo, tables, dbound)
    if out is None:
        out = torch.empty(*lead, 12 * nside * nside, dtype=torch.float32, device=pos.device)
        accumulate = False
    lx, ly, lz = (float(v) for v in box_size)
    ox, oy, oz = (float(v) for v in observer_mpc)
    chi, a_chi, ga, g, da, dg = tabs
    n = lambda x: int(x.numel()) if x is not None else 0
    call("jfli_healpix_paint_tiled", stream_ptr(), ptr(pos), int(absolute), ptr(vel), ptr(weights), float(weight),
         lx, ly, lz, ox, oy, oz, int(rot.shape[0]), rot.ctypes.data_as(ctypes.POINTER(ctypes.c_byte)),
         sh.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(bool(telephoto)), float(rmin), float(rmax), t_arg,
         gp_t, float(dbound), ptr(chi), ptr(a_chi), n(chi), ptr(ga), ptr(g), n(ga), ptr(da), ptr(dg), n(da),
         int(nside), sch, ptr(out), int(accumulate), nx, ny, nz, batch)
    return out


def lightcone_drift_array(disp: torch.Tensor, vel: torch.Tensor, t: float, cosmo, box_size, observer_mpc,
                          tables=None) -> torch.Tensor:
    """Drifted positions in Mpc/h of particles given as relative displacements."""
    from . import cosmology as cj

    _check(disp, "disp")
    _check(vel, "vel")
    (nx, ny, nz), batch, _ = _mesh_dims(disp, True)
    chi, a_chi, ga, g, da, dg = drift_tables(cosmo) if tables is None else tables
    out = torch.empty_like(disp)
    lx, ly, lz = (float(v) for v in box_size)
    ox, oy, oz = (float(v) for v in observer_mpc)
    gp_t = float(cj.Gp(cosmo, float(t)))
    call("jfli_lightcone_drift", stream_ptr(), ptr(disp), ptr(vel), ptr(out), lx, ly, lz, ox, oy, oz, float(t), gp_t,
         ptr(chi), ptr(a_chi), int(chi.numel()), ptr(ga), ptr(g), int(ga.numel()), ptr(da), ptr(dg), int(da.numel()),
         nx, ny, nz, batch)
    return out


def lightcone_drift(dx, p, t: float, cosmo):
    """ParticleField (MPC_H) of dx drifted to the light cone with the momenta p."""
    from .fields import PositionUnit

    rel = dx if dx.unit == PositionUnit.GRID_RELATIVE else dx.to(PositionUnit.GRID_RELATIVE)
    arr = lightcone_drift_array(rel.array.contiguous(), p.array.contiguous(), t, cosmo, dx.box_size,
                                dx.observer_position_mpc)
    return dx.replace(array=arr, unit=PositionUnit.MPC_H)


# ------------------------------------------------------------------------- adjoints
def adjoint_unkick_paint(disp: torch.Tensor, vel: torch.Tensor, lam_x: torch.Tensor, lam_v: torch.Tensor,
                         force: torch.Tensor, kick: float, drift: float, ubar: torch.Tensor | None = None):
    """Reverse kick and first half of the VJP of one reversible step (in place on vel and
    lam_v). Returns (ubar, (dL/dkick, dL/ddrift)) with ubar the (..., 3, nx, ny, nz) paint
    of the new lam_v; the two scalars are FP64 sums in a fixed order (one tensor of 2)."""
    for name, t in (("disp", disp), ("vel", vel), ("lam_x", lam_x), ("lam_v", lam_v), ("force", force)):
        _check(t, name)
    (nx, ny, nz), batch, lead = _mesh_dims(disp, True)
    if ubar is None:
        ubar = torch.empty(*lead, 3, nx, ny, nz, dtype=torch.float32, device=disp.device)
    count = int(query("jfli_adjoint_partials_count", nx, ny, nz, batch))
    partials = torch.empty(count, dtype=torch.float64, device=disp.device)
    call("jfli_adjoint_unkick_paint", stream_ptr(), ptr(disp), ptr(vel), ptr(lam_x), ptr(lam_v), ptr(force),
         float(kick), float(drift), ptr(ubar), ptr(partials), count, nx, ny, nz, batch)
    return ubar, partials.view(batch, -1, 2).sum(dim=1).reshape(*lead, 2) if lead else partials.view(-1, 2).sum(0)


def poisson_divergence(u: torch.Tensor, *, aos: bool, alpha: float = 1.0, w: torch.Tensor | None = None,
                       beta: float = 0.0, scale: float = 1.0, out: torch.Tensor | None = None) -> torch.Tensor:
    """scale * P(div_FD(alpha u + beta w)); u, w three meshes (..., 3, nx, ny, nz) or particle
    grids (..., nx, ny, nz, 3) (aos=True)."""
    _check(u, "u")
    if w is not None:
        _check(w, "w")
        if w.shape != u.shape:
            raise ValueError("u and w must have the same shape")
    if aos:
        (nx, ny, nz), batch, lead = _mesh_dims(u, True)
    else:
        if u.shape[-4] != 3:
            raise ValueError("u must hold three meshes (..., 3, nx, ny, nz)")
        nx, ny, nz = (int(v) for v in u.shape[-3:])
        lead = tuple(u.shape[:-4])
        batch = int(np.prod(lead)) if lead else 1
    if out is None:
        out = torch.empty(*lead, nx, ny, nz, dtype=torch.float32, device=u.device)
    nb = query("jfli_poisson_divergence_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "div", u.device)
    call("jfli_poisson_divergence", stream_ptr(), ptr(u), float(alpha), ptr(w), float(beta), int(aos), float(scale),
         ptr(out), ptr(ws), ws.numel(), nx, ny, nz, batch)
    return out


def adjoint_position(disp: torch.Tensor, lam_x: torch.Tensor, *, rho_bar: torch.Tensor | None = None,
                     u: torch.Tensor | None = None, force: torch.Tensor | None = None, scale: float = 1.0) -> None:
    """lam_x += scale * grad_x R_x[rho_bar + sum_a u_a force_a] (in place)."""
    _check(disp, "disp")
    _check(lam_x, "lam_x")
    (nx, ny, nz), batch, _ = _mesh_dims(disp, True)
    call("jfli_adjoint_position", stream_ptr(), ptr(disp), ptr(u), ptr(rho_bar), ptr(force), float(scale), ptr(lam_x),
         nx, ny, nz, batch)


def _host_floats(a):
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    return arr, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _check_pots(pots: torch.Tensor, nsteps: int, disp: torch.Tensor, batch: int):
    _check(pots, "pots")
    if pots.numel() != nsteps * batch * (disp.numel() // (3 * batch)):
        raise ValueError(f"pots must hold {nsteps} potentials of the particle grid's mesh")


def pgd_adjoint(disp: torch.Tensor, u: torch.Tensor, alpha: float, kl: float, ks: float,
                lam_x: torch.Tensor) -> torch.Tensor:
    """lam_x += alpha J_pgd^T u for the PGD force at the relative positions disp (in place;
    jfli_pgd_adjoint with lam_x as its accumulator)."""
    for name, t in (("disp", disp), ("u", u), ("lam_x", lam_x)):
        _check(t, name)
    (nx, ny, nz), batch, _ = _mesh_dims(disp, True)
    ws = workspace(int(query("jfli_pgd_adjoint_workspace_bytes", nx, ny, nz, batch)), "force_adj", disp.device)
    call("jfli_pgd_adjoint", stream_ptr(), ptr(disp), ptr(u), float(alpha), float(kl), float(ks), ptr(lam_x),
         ptr(ws), ws.numel(), nx, ny, nz, batch)
    return lam_x


def force_adjoint(disp: torch.Tensor, u: torch.Tensor, scale: float, lam_x: torch.Tensor) -> torch.Tensor:
    """lam_x += scale J^T u for the PM force at the relative positions disp (in place;
    jfli_force_adjoint)."""
    for name, t in (("disp", disp), ("u", u), ("lam_x", lam_x)):
        _check(t, name)
    (nx, ny, nz), batch, _ = _mesh_dims(disp, True)
    ws = workspace(int(query("jfli_pgd_adjoint_workspace_bytes", nx, ny, nz, batch)), "force_adj", disp.device)
    call("jfli_force_adjoint", stream_ptr(), ptr(disp), ptr(u), float(scale), ptr(lam_x), ptr(ws), ws.numel(), nx, ny,
         nz, batch)
    return lam_x


def _sharpen_args(sharpen, nsteps: int):
    """(boost array, its float pointer, kl, ks) of a (boosts, kl, ks) sharpening triple."""
    boosts, kl, ks = sharpen
    b_arr, b_ptr = _host_floats(boosts)
    if b_arr.size != nsteps:
        raise ValueError(f"{b_arr.size} boost factors for {nsteps} steps")
    return b_arr, b_ptr, float(kl), float(ks)


def kkd_run(disp: torch.Tensor, vel: torch.Tensor, kicks, drifts, rho: torch.Tensor,
            pots: torch.Tensor | None = None, sharpen=None) -> None:
    """The ReversibleDoubleKickDrift loop in one call (in place on disp, vel); rho receives
    the CIC density of the final positions. With `pots` (nsteps potentials, float32 on the
    device) the potential of every step is kept there for kkd_adjoint. `sharpen` = (boosts,
    kl, ks): SharpeningKernel's per-step boost factors and PGD scales
    (jfli_kkd_run_sharpened)."""
    _check(disp, "disp")
    _check(vel, "vel")
    _check(rho, "rho")
    (nx, ny, nz), batch, _ = _mesh_dims(disp, True)
    k_arr, k_ptr = _host_floats(kicks)
    d_arr, d_ptr = _host_floats(drifts)
    if k_arr.size != d_arr.size:
        raise ValueError("kicks and drifts must have the same length")
    nb = query("jfli_kkd_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "kkd", disp.device)
    if pots is not None:
        _check_pots(pots, int(k_arr.size), disp, batch)
    if sharpen is not None:
        b_arr, b_ptr, kl, ks = _sharpen_args(sharpen, k_arr.size)
        call("jfli_kkd_run_sharpened", stream_ptr(), ptr(disp), ptr(vel), k_ptr, d_ptr, b_ptr, kl, ks,
             int(k_arr.size), ptr(rho), ptr(pots), ptr(ws), ws.numel(), nx, ny, nz, batch)
        return
    if pots is not None:
        call("jfli_kkd_run_stored", stream_ptr(), ptr(disp), ptr(vel), k_ptr, d_ptr, int(k_arr.size), ptr(rho),
             ptr(pots), ptr(ws), ws.numel(), nx, ny, nz, batch)
        return
    call("jfli_kkd_run", stream_ptr(), ptr(disp), ptr(vel), k_ptr, d_ptr, int(k_arr.size), ptr(rho), ptr(ws),
         ws.numel(), nx, ny, nz, batch)


def kkd_adjoint(disp: torch.Tensor, vel: torch.Tensor, lam_x: torch.Tensor, lam_v: torch.Tensor, kicks,
                drifts, pots: torch.Tensor | None = None, sharpen=None) -> torch.Tensor:
    """Reverse sweep of kkd_run in one call (in place on all four particle grids); returns
    the (nsteps, 2) FP64 (dL/dkick, dL/ddrift) on the device. `pots`: the potentials a
    kkd_run with pots kept (the forces are then rebuilt from them, not recomputed).
    `sharpen` as for kkd_run (the first column is then dL/d of the combined force's
    factor; jfli_kkd_adjoint_sharpened)."""
    for name, t in (("disp", disp), ("vel", vel), ("lam_x", lam_x), ("lam_v", lam_v)):
        _check(t, name)
    (nx, ny, nz), batch, _ = _mesh_dims(disp, True)
    k_arr, k_ptr = _host_floats(kicks)
    d_arr, d_ptr = _host_floats(drifts)
    if k_arr.size != d_arr.size:
        raise ValueError("kicks and drifts must have the same length")
    sens = torch.zeros(k_arr.size, batch, 2, dtype=torch.float64, device=disp.device)
    nb = query("jfli_kkd_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "kkd", disp.device)
    if pots is not None:
        _check_pots(pots, int(k_arr.size), disp, batch)
    if sharpen is not None:
        b_arr, b_ptr, kl, ks = _sharpen_args(sharpen, k_arr.size)
        call("jfli_kkd_adjoint_sharpened", stream_ptr(), ptr(disp), ptr(vel), ptr(lam_x), ptr(lam_v), k_ptr, d_ptr,
             b_ptr, kl, ks, int(k_arr.size), ptr(pots), ptr(sens), ptr(ws), ws.numel(), nx, ny, nz, batch)
    elif pots is not None:
        call("jfli_kkd_adjoint_stored", stream_ptr(), ptr(disp), ptr(vel), ptr(lam_x), ptr(lam_v), k_ptr, d_ptr,
             int(k_arr.size), ptr(pots), ptr(sens), ptr(ws), ws.numel(), nx, ny, nz, batch)
    else:
        call("jfli_kkd_adjoint", stream_ptr(), ptr(disp), ptr(vel), ptr(lam_x), ptr(lam_v), k_ptr, d_ptr,
             int(k_arr.size), ptr(sens), ptr(ws), ws.numel(), nx, ny, nz, batch)
    return sens if batch > 1 else sens[:, 0, :]


def power_adjoint(mesh: torch.Tensor, kedges: torch.Tensor, weights: torch.Tensor, box_size) -> torch.Tensor:
    """dL/dmesh of the P(k) sums for per-bin weights 2 dL/dP_b prod(L/N) / count_b."""
    _check(mesh, "mesh")
    _check(kedges, "kedges")
    _check(weights, "weights")
    (nx, ny, nz), batch, lead = _mesh_dims(mesh, False)
    ne = int(kedges.numel())
    if weights.numel() != ne + 1:
        raise ValueError("weights must have nedges + 1 entries")
    out = torch.empty_like(mesh)
    nb = query("jfli_poisson_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "spec", mesh.device)
    lx, ly, lz = (float(v) for v in box_size)
    call("jfli_power_spectrum_adjoint", stream_ptr(), ptr(mesh), ptr(kedges), ptr(weights), ne, lx, ly, lz, ptr(out),
         ptr(ws), ws.numel(), nx, ny, nz, batch)
    return out


def power_poles_adjoint(mesh: torch.Tensor, kedges: torch.Tensor, weights: torch.Tensor, ells, box_size,
                        los=(0.0, 0.0, 1.0), complex_weights: bool = False) -> torch.Tensor:
    """dL/dmesh of multipole sums for per-multipole, per-bin weights (nell, nedges + 1) =
    2 dL/dP_l,b prod(L/N) / count_b of an auto spectrum, or (2, nell, nedges + 1), the real
    and imaginary parts of a cross spectrum's complex factors (jfli_power_poles_adjoint)."""
    _check(mesh, "mesh")
    _check(kedges, "kedges")
    _check(weights, "weights")
    (nx, ny, nz), batch, lead = _mesh_dims(mesh, False)
    ne = int(kedges.numel())
    ell_arr = np.ascontiguousarray(np.asarray(ells, dtype=np.int32))
    if weights.numel() != (2 if complex_weights else 1) * ell_arr.size * (ne + 1):
        raise ValueError("weights must hold nedges + 1 entries per multipole (twice that for complex weights)")
    out = torch.empty_like(mesh)
    nb = query("jfli_poisson_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "spec", mesh.device)
    lx, ly, lz = (float(v) for v in box_size)
    call("jfli_power_poles_adjoint", stream_ptr(), ptr(mesh), ptr(kedges), ptr(weights), ne,
         ell_arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(ell_arr.size), int(bool(complex_weights)), lx, ly, lz,
         *(float(v) for v in los), ptr(out), ptr(ws), ws.numel(), nx, ny, nz, batch)
    return out


def lpt_adjoint(ic: torch.Tensor, order: int, c1x: float, c2x: float, c1p: float, c2p: float, lam_x: torch.Tensor,
                lam_v: torch.Tensor) -> torch.Tensor:
    """dL/d ic of lpt() given the cotangents of its displacement and momentum."""
    _check(ic, "ic")
    _check(lam_x, "lam_x")
    _check(lam_v, "lam_v")
    (nx, ny, nz), batch, lead = _mesh_dims(ic, False)
    out = torch.empty_like(ic)
    nb = query("jfli_lpt_adjoint_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "lpt_adj", ic.device)
    call("jfli_lpt_adjoint", stream_ptr(), ptr(ic), int(order), float(c1x), float(c2x), float(c1p), float(c2p),
         ptr(lam_x), ptr(lam_v), ptr(out), ptr(ws), ws.numel(), nx, ny, nz, batch)
    return out


def ic_filter_tangent(noise: torch.Tensor, ktab: torch.Tensor, ptab: torch.Tensor, dptab: torch.Tensor, box_size, *,
                      zero_mode_one: bool = False) -> torch.Tensor:
    """Derivative of ic_filter(noise) along a change dptab of the P(k) table."""
    for name, t in (("noise", noise), ("ktab", ktab), ("ptab", ptab), ("dptab", dptab)):
        _check(t, name)
    (nx, ny, nz), batch, lead = _mesh_dims(noise, False)
    out = torch.empty_like(noise)
    nb = query("jfli_poisson_workspace_bytes", nx, ny, nz, batch)
    ws = workspace(nb, "spec", noise.device)
    lx, ly, lz = (float(v) for v in box_size)
    call("jfli_ic_filter_tangent", stream_ptr(), ptr(noise), ptr(out), ptr(ktab), ptr(ptab), ptr(dptab),
         int(ktab.numel()), lx, ly, lz, int(zero_mode_one), ptr(ws), ws.numel(), nx, ny, nz, batch)
    return out


def launch_count() -> int:
    return _lib.launch_count()
