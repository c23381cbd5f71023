"""Flat-sky planes (ParticleField.paint_2d, reference _src/fields/_painting.py:117-202) and
the flat-sky angular power spectrum (FlatDensity.angular_cl, _src/power/_compute.py:122-172)
on the GPU against the NumPy oracle (oracle/flat.py)."""

import numpy as np
import pytest
import torch

import jfli_b200 as jf
from jfli_b200 import ops
from oracle import flat as of
from oracle import pm as opm
from tests.conftest import rel_l2

MAP_TOL = 1e-5  # relative L2 of a painted plane (FP32 weights vs FP64)
CL_TOL = 1e-4  # per bin, relative


def _state(shape, seed, amp=3.0):
    rng = np.random.default_rng(seed)
    return (amp * rng.standard_normal(tuple(shape) + (3,))).astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,npix,slab", [((32, 32, 32), (64, 48), (8.0, 20.0)),
                                             ((48, 32, 64), (32, 96), (-2.0, 70.0)),
                                             ((32, 32, 32), (32, 32), (30.5, 33.0))])
def test_paint_flat_matches_oracle(shape, npix, slab):
    disp = _state(shape, 1)
    w = np.random.default_rng(2).uniform(0.5, 1.5, shape).astype(np.float32)
    out = ops.paint_flat(torch.as_tensor(disp, device="cuda"), npix, *slab,
                         weights=torch.as_tensor(w, device="cuda"), weight=0.75).cpu().numpy()
    pos = opm.grid(shape) + disp.astype(np.float64)
    # per-particle weights: the oracle's deposit rule with the weights folded in
    ref = np.zeros(npix)
    p = pos.reshape(-1, 3)
    ww = w.reshape(-1).astype(np.float64) * 0.75
    sel_z = (p[:, 2] > slab[0]) & (p[:, 2] <= slab[1])
    xy = np.mod(p[:, :2] * np.array([npix[0] / shape[0], npix[1] / shape[1]]), np.array(npix, np.float64))
    fl = np.floor(xy)
    for cx in (0.0, 1.0):
        for cy in (0.0, 1.0):
            nb = fl + np.array([cx, cy])
            k = (1 - np.abs(xy[:, 0] - nb[:, 0])) * (1 - np.abs(xy[:, 1] - nb[:, 1])) * ww * sel_z
            ix = np.mod(nb[:, 0].astype(np.int64), npix[0])
            iy = np.mod(nb[:, 1].astype(np.int64), npix[1])
            ref += np.bincount(ix * npix[1] + iy, weights=k, minlength=npix[0] * npix[1]).reshape(npix)
    plain = of.paint_2d(pos, npix, slab[0], slab[1], shape)
    out1 = ops.paint_flat(torch.as_tensor(disp, device="cuda"), npix, *slab).cpu().numpy()
    e1, e2 = rel_l2(out1, plain), rel_l2(out, ref)
    print(f"{shape} -> {npix}, slab {slab}: weight {plain.sum():.0f}, rel L2 {e1:.2e} (weighted {e2:.2e})")
    assert plain.sum() > 100
    assert e1 < MAP_TOL and e2 < MAP_TOL


@pytest.mark.gpu
def test_paint_2d_field_units_and_batches():
    """ParticleField.paint_2d: centre and width in Mpc/h along z from the box origin, density
    per pixel volume; several planes at once; a batched (S, ...) input paints every snapshot
    into every plane, as the reference's light-cone mode does."""
    shape, L, npix = (32, 32, 32), (200.0, 200.0, 100.0), (64, 64)
    disp = _state(shape, 3, amp=1.0)
    f = jf.ParticleField(array=torch.as_tensor(disp, device="cuda"), mesh_size=shape, box_size=L,
                         flatsky_npix=npix, unit=jf.PositionUnit.GRID_RELATIVE)
    centers, widths = np.array([25.0, 60.0]), np.array([10.0, 30.0])
    planes = f.paint_2d(centers, widths)
    assert isinstance(planes, jf.FlatDensity) and tuple(planes.array.shape) == (2, 64, 64)
    pos = opm.grid(shape) + disp.astype(np.float64)
    for s in range(2):
        cg, wg = centers[s] * shape[2] / L[2], widths[s] * shape[2] / L[2]
        vol = (L[0] / npix[0]) * (L[1] / npix[1]) * widths[s]
        ref = of.paint_2d(pos, npix, cg - wg / 2, cg + wg / 2, shape) / vol
        assert rel_l2(planes.array[s].cpu().numpy(), ref) < MAP_TOL
    # mean density of a plane: particles in the slab over the slab volume
    nbar = np.prod(shape) / np.prod(L)
    assert abs(planes.array[1].double().mean().item() / nbar - 1) < 0.1
    both = f.replace(array=torch.stack([f.array, f.array]))
    twice = both.paint_2d(centers, widths)
    np.testing.assert_allclose(twice.array.cpu().numpy(), 2 * planes.array.cpu().numpy(), rtol=1e-5, atol=1e-7)


@pytest.mark.gpu
@pytest.mark.parametrize("npix", [(64, 48), (96, 128), (32, 32)])
def test_flat_cl_matches_oracle(npix):
    rng = np.random.default_rng(4)
    m1 = rng.standard_normal(npix).astype(np.float32)
    m2 = (0.5 * m1 + rng.standard_normal(npix)).astype(np.float32)
    px = py = np.deg2rad(5.0 / 60.0)
    ell, cl = jf.angular_cl_flat(torch.as_tensor(m1, device="cuda"), pixel_size=(px, py))
    ell_r, cl_r = of.flat_cl(m1, px=px, py=py)
    filled = np.isfinite(cl_r) & (cl_r != 0)
    rel = np.max(np.abs(cl.cpu().numpy()[filled] / cl_r[filled] - 1))
    print(f"{npix}: {filled.sum()} bins, max per-bin rel {rel:.2e}")
    assert filled.sum() > 30 and rel < CL_TOL
    np.testing.assert_allclose(ell.cpu().numpy(), ell_r, rtol=1e-6)
    edges = np.geomspace(200.0, 0.9 * float(of.ell_grid32(*npix, px, py).max()), 12)
    _, xc = jf.angular_cl_flat(torch.as_tensor(m1, device="cuda"), torch.as_tensor(m2, device="cuda"),
                               field_size=(px * npix[0], py * npix[1]), ell_edges=edges)
    _, xr = of.flat_cl(m1, m2, px=px, py=py, ell_edges=edges)
    xc = xc.cpu().numpy()
    full = xr != 0  # bins with no modes are 0 on both sides
    assert np.all(xc[~full] == 0) and full.sum() >= 5
    assert np.max(np.abs(xc[full] / xr[full] - 1)) < CL_TOL


@pytest.mark.gpu
def test_flat_cl_batched_and_field_method():
    rng = np.random.default_rng(5)
    maps = rng.standard_normal((3, 64, 64)).astype(np.float32)
    px = np.deg2rad(2.0 / 60.0)
    fd = jf.FlatDensity(array=torch.as_tensor(maps, device="cuda"), mesh_size=(32, 32, 32),
                        box_size=(100.0, 100.0, 100.0), flatsky_npix=(64, 64))
    ps = fd.angular_cl(pixel_size=(px, px))
    assert tuple(ps.array.shape) == (3, 49)  # 50 edges: 51 bins, under/overflow dropped
    for b in range(3):
        _, one = jf.angular_cl_flat(torch.as_tensor(maps[b], device="cuda"), pixel_size=(px, px))
        np.testing.assert_allclose(ps.array[b].cpu().numpy(), one.cpu().numpy(), rtol=1e-12)


@pytest.mark.gpu
def test_flat_planes_through_nbody(cosmo):
    """A flat-sky light cone from nbody (NoInterp, target "flat"): each plane is the flat
    paint of the particles at its snapshot time (checked against the same run's particle
    snapshots painted directly)."""
    n, L = 32, 128.0
    noise = jf.white_noise(6, (n, n, n))
    ic = jf.interpolate_initial_conditions(noise, (n, n, n), (L, L, L), cosmo=cosmo, flatsky_npix=(64, 64))
    dx, p = jf.lpt(cosmo, ic, ts=0.1, order=2)
    flat = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="flat")))
    lc = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=0.9 / 10, nb_shells=3, solver=flat)
    assert tuple(lc.array.shape) == (3, 64, 64)
    ts = np.asarray(lc.scale_factors, np.float64)[::-1]
    parts = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="particles")))
    snaps = jf.nbody(cosmo, dx, p, t0=0.1, t1=1.0, dt0=0.9 / 10, ts=ts, solver=parts)
    for s in range(3):
        rc, wd = float(lc.comoving_centers[s]), float(lc.density_width[s])
        ref = snaps[s].paint_2d(rc, wd).array.double().cpu().numpy()
        err = rel_l2(lc.array[s].double().cpu().numpy(), ref)
        print(f"plane {s} at z = {rc:.1f} Mpc/h: rel L2 {err:.2e}")
        # the two runs differ only in the order of the FP32 atomic deposits
        assert err < 2e-2
