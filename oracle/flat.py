"""CPU oracle for flat-sky planes and their angular power spectrum — TEST INFRASTRUCTURE
ONLY (see oracle/pm.py): NumPy restatements that the GPU kernels are checked against.

paint_2d follows the reference's _single_paint_2d (_src/fields/_painting.py:117-202) with
jaxpm's cic_paint_2d: x, y scaled to the map and wrapped (numpy.mod), the plane selected by
zlo < z <= zhi in grid units, 2D CIC weights (1 - |x - n|) on the floor and floor + 1
neighbours, wrapped. flat_cl follows _flat_cl (_src/power/_compute.py:122-172): full
complex fft2 (FP64 here), (px py) / (nx ny) normalisation, ell = |2 pi fftfreq| on a float32
grid as the reference builds it, numpy.digitize + bincount, under/overflow bins dropped.
"""

from __future__ import annotations

import numpy as np


def paint_2d(pos_abs, npix, zlo, zhi, mesh_size, weight=1.0):
    """Raw 2D CIC sums (npx, npy) of particles given in absolute grid units (..., 3)."""
    npx, npy = npix
    nx, ny, _ = mesh_size
    p = pos_abs.reshape(-1, 3).astype(np.float64)
    sel = (p[:, 2] > zlo) & (p[:, 2] <= zhi)
    xy = p[sel, :2] * np.array([npx / nx, npy / ny])
    xy = np.mod(xy, np.array([npx, npy], np.float64))
    fl = np.floor(xy)
    out = np.zeros(npx * npy)
    for cx in (0.0, 1.0):
        for cy in (0.0, 1.0):
            n = fl + np.array([cx, cy])
            w = (1.0 - np.abs(xy[:, 0] - n[:, 0])) * (1.0 - np.abs(xy[:, 1] - n[:, 1])) * weight
            ix = np.mod(n[:, 0].astype(np.int64), npx)
            iy = np.mod(n[:, 1].astype(np.int64), npy)
            out += np.bincount(ix * npy + iy, weights=w, minlength=npx * npy)
    return out.reshape(npx, npy)


def ell_grid32(nx, ny, px, py):
    """The reference's float32 |ell| grid: 2 pi * fftfreq(n, d) (float32), squares summed."""
    def comp(n, d):
        k = np.fft.fftfreq(n) * n  # integers in fftfreq order
        f = (k.astype(np.float32) / np.float32(n * d)).astype(np.float32)
        return (np.float32(2.0 * np.pi) * f).astype(np.float32)

    lx, ly = comp(nx, px), comp(ny, py)
    LX, LY = np.meshgrid(lx, ly, indexing="ij")
    return np.sqrt((LX * LX + LY * LY).astype(np.float32)).astype(np.float32)


def flat_cl(map1, map2=None, *, px, py, ell_edges=None):
    """(ell_avg, cl) of one map (or a cross pair), FP64 FFT."""
    nx, ny = map1.shape
    m2 = map1 if map2 is None else map2
    f1 = np.fft.fft2(map1.astype(np.float64))
    f2 = np.fft.fft2(m2.astype(np.float64))
    pk = (f1 * np.conj(f2)).real * (px * py) / (nx * ny)
    ell = ell_grid32(nx, ny, px, py)
    if ell_edges is None:
        ell_edges = np.linspace(0.0, ell.max(), 50).astype(np.float32)
        ell_edges[-1] = ell.max()
    edges = np.asarray(ell_edges, np.float32)
    dig = np.digitize(ell.reshape(-1), edges)
    nb = edges.size + 1
    cnt = np.bincount(dig, minlength=nb).astype(np.float64)
    esum = np.bincount(dig, weights=ell.reshape(-1).astype(np.float64), minlength=nb)
    csum = np.bincount(dig, weights=pk.reshape(-1), minlength=nb)
    den = np.where(cnt > 0, cnt, 1.0)
    return (esum / den)[1:-1], (csum / den)[1:-1]
