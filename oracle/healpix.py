"""CPU oracle for HEALPix shell painting — TEST INFRASTRUCTURE ONLY (see oracle/pm.py).

Vectorised FP64 NumPy restatement of the published HEALPix RING geometry (Gorski et al.
2005): ang2pix, ring information and the 4-pixel bilinear interpolation weights that
healpy's get_interp_weights returns; the reference reaches them through jax_healpy /
JaxPM `paint_particles_spherical` (_src/fields/_painting.py:329). Pinned against the
worked examples of healpy's documentation (tests/golden/healpix_docs.json) and by
self-consistency (weights sum to 1, pixel centres map back to themselves).
"""

from __future__ import annotations

import numpy as np


def nside2npix(nside):
    return 12 * nside * nside


def ring_info(ring, nside):
    ring = np.asarray(ring, np.int64)
    npix = 12 * nside * nside
    ncap = 2 * nside * (nside - 1)
    north = np.where(ring > 2 * nside, 4 * nside - ring, ring)
    polar = north < nside
    tmp = north.astype(np.float64) ** 2 * (4.0 / npix)
    theta_p = np.arctan2(np.sqrt(np.maximum(tmp * (2.0 - tmp), 0.0)), 1.0 - tmp)
    theta_e = np.arccos(np.clip((2 * nside - north) * (2.0 / (3.0 * nside)), -1.0, 1.0))
    theta = np.where(polar, theta_p, theta_e)
    nr = np.where(polar, 4 * north, 4 * nside)
    shifted = np.where(polar, 1, ((north - nside) & 1) == 0).astype(np.int64)
    start = np.where(polar, 2 * north * (north - 1), ncap + (north - nside) * 4 * nside)
    south = north != ring
    theta = np.where(south, np.pi - theta, theta)
    start = np.where(south, npix - start - nr, start)
    return start, nr, theta, shifted


def ring_above(z, nside):
    z = np.asarray(z, np.float64)
    az = np.abs(z)
    eq = (nside * (2.0 - 1.5 * z)).astype(np.int64)
    ir = (nside * np.sqrt(3.0 * (1.0 - az))).astype(np.int64)
    pol = np.where(z > 0, ir, 4 * nside - ir - 1)
    return np.where(az <= 2.0 / 3.0, eq, pol)


def ang2pix(nside, theta, phi):
    theta = np.asarray(theta, np.float64)
    phi = np.asarray(phi, np.float64)
    z = np.cos(theta)
    za = np.abs(z)
    ph = np.mod(phi, 2 * np.pi)
    tt = ph / (0.5 * np.pi)
    npix = 12 * nside * nside
    ncap = 2 * nside * (nside - 1)
    t1 = nside * (0.5 + tt)
    t2 = nside * z * 0.75
    jp = (t1 - t2).astype(np.int64)
    jm = (t1 + t2).astype(np.int64)
    ir = nside + 1 + jp - jm
    kshift = 1 - (ir & 1)
    ip = np.mod((jp + jm - nside + kshift + 1) // 2, 4 * nside)
    pix_eq = ncap + (ir - 1) * 4 * nside + ip
    tp = tt - np.floor(tt)
    tmp = nside * np.sqrt(3.0 * (1.0 - za))
    jp2 = (tp * tmp).astype(np.int64)
    jm2 = ((1.0 - tp) * tmp).astype(np.int64)
    ir2 = jp2 + jm2 + 1
    ip2 = np.mod((tt * ir2).astype(np.int64), 4 * ir2)
    pix_pol = np.where(z > 0, 2 * ir2 * (ir2 - 1) + ip2, npix - 2 * ir2 * (ir2 + 1) + ip2)
    return np.where(za <= 2.0 / 3.0, pix_eq, pix_pol)


def pix2ang(nside, pix):
    """Pixel centres (theta, phi) of RING pixels."""
    pix = np.asarray(pix, np.int64)
    rings = np.arange(1, 4 * nside)
    start, nr, theta, shifted = ring_info(rings, nside)
    r = np.searchsorted(start, pix, side="right") - 1
    i = pix - start[r]
    phi = (i + 0.5 * shifted[r]) * 2 * np.pi / nr[r]
    return theta[r], phi


UNSEEN = -1.6375e30


def ring_parents(nside_in, nside_out):
    """For every RING pixel at nside_in, the RING pixel at nside_out < nside_in that holds its
    centre: the pixel hierarchy from the geometry alone, with no NESTED numbering."""
    theta, phi = pix2ang(nside_in, np.arange(nside2npix(nside_in)))
    return ang2pix(nside_out, theta, phi)


def ud_grade_ring(m, nside_out, pess=False, power=None):
    """healpy.ud_grade of one RING map (healpy's documented rules: averages of the children
    that are not UNSEEN, UNSEEN where none is (or any, with pess), power p scaling by
    (nside_out / nside_in)^p, copies when upgrading), built on ring_parents."""
    m = np.asarray(m, np.float64)
    nside_in = int(round(np.sqrt(m.size / 12)))
    ratio = (nside_out / nside_in) ** power if power else 1.0
    if nside_out == nside_in:
        return m.copy()
    if nside_out > nside_in:
        return m[ring_parents(nside_out, nside_in)] * ratio
    par = ring_parents(nside_in, nside_out)
    k = (nside_in // nside_out) ** 2
    good = ~((np.abs(m - UNSEEN) <= 1e-8 + 1e-5 * abs(UNSEEN)) | ~np.isfinite(m))
    npix_out = nside2npix(nside_out)
    total = np.bincount(par, weights=m * good, minlength=npix_out)
    nhit = np.bincount(par, weights=good.astype(np.float64), minlength=npix_out)
    out = np.where(nhit > 0, total / np.where(nhit > 0, nhit, 1.0) * ratio, total)
    return np.where((nhit < k) if pess else (nhit == 0), UNSEEN, out)


def get_interp_weights(nside, theta, phi):
    """(pix (4, N), weights (4, N)) bilinear interpolation on the RING grid."""
    theta = np.atleast_1d(np.asarray(theta, np.float64))
    ph = np.mod(np.atleast_1d(np.asarray(phi, np.float64)), 2 * np.pi)
    npix = 12 * nside * nside
    z = np.cos(theta)
    ir1 = ring_above(z, nside)
    ir2 = ir1 + 1
    pix = np.zeros((4, theta.size), np.int64)
    w = np.zeros((4, theta.size), np.float64)
    th1 = np.zeros(theta.size)
    th2 = np.zeros(theta.size)
    for ring, slot, thv in ((ir1, 0, th1), (ir2, 2, th2)):
        ok = (ring > 0) & (ring < 4 * nside)
        rr = np.where(ok, ring, 1)
        start, nr, tht, shifted = ring_info(rr, nside)
        dphi = 2 * np.pi / nr
        tmp = ph / dphi - 0.5 * shifted
        i1 = np.where(tmp < 0, tmp.astype(np.int64) - 1, tmp.astype(np.int64))
        wp = (ph - (i1 + 0.5 * shifted) * dphi) / dphi
        i2 = i1 + 1
        i1 = np.where(i1 < 0, i1 + nr, i1)
        i2 = np.where(i2 >= nr, i2 - nr, i2)
        pix[slot] = np.where(ok, start + i1, pix[slot])
        pix[slot + 1] = np.where(ok, start + i2, pix[slot + 1])
        w[slot] = np.where(ok, 1.0 - wp, 0.0)
        w[slot + 1] = np.where(ok, wp, 0.0)
        thv[:] = np.where(ok, tht, 0.0)
    north = ir1 == 0
    south = ir2 == 4 * nside
    mid = ~(north | south)
    # interior
    wt = np.where(mid, (theta - th1) / np.where(mid, th2 - th1, 1.0), 0.0)
    w_mid = np.stack([w[0] * (1 - wt), w[1] * (1 - wt), w[2] * wt, w[3] * wt])
    # north pole cap
    wtn = np.where(north, theta / np.where(north, th2, 1.0), 0.0)
    facn = (1.0 - wtn) * 0.25
    w_n = np.stack([facn, facn, w[2] * wtn + facn, w[3] * wtn + facn])
    p_n = np.stack([(pix[2] + 2) & 3, (pix[3] + 2) & 3, pix[2], pix[3]])
    # south pole cap
    wts = np.where(south, (theta - th1) / np.where(south, np.pi - th1, 1.0), 0.0)
    facs = wts * 0.25
    w_s = np.stack([w[0] * (1 - wts) + facs, w[1] * (1 - wts) + facs, facs, facs])
    p_s = np.stack([pix[0], pix[1], ((pix[0] + 2) & 3) + npix - 4, ((pix[1] + 2) & 3) + npix - 4])
    w_out = np.where(north, w_n, np.where(south, w_s, w_mid))
    p_out = np.where(north, p_n, np.where(south, p_s, pix))
    return p_out, w_out


def rbf_weights(nside, theta, phi, sigma):
    """(pixels (4, P), weights (4, P)) of the library's rbf_neighbor scheme: the 4 pixels of
    the bilinear scheme, weighted by exp(-d^2 / (2 sigma^2)) of the angle d between the
    direction and each pixel centre, normalised to sum 1 (sigma in radians)."""
    pix, _ = get_interp_weights(nside, theta, phi)
    tc, pc = pix2ang(nside, pix.ravel())
    tc, pc = tc.reshape(pix.shape), pc.reshape(pix.shape)
    u = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)])
    c = np.stack([np.sin(tc) * np.cos(pc), np.sin(tc) * np.sin(pc), np.cos(tc)])
    d = 2.0 * np.arcsin(np.minimum(1.0, 0.5 * np.linalg.norm(c - u[:, None, :], axis=0)))
    d2 = d * d
    w = np.exp(-(d2 - d2.min(axis=0)) / (2.0 * sigma * sigma))
    return pix, w / w.sum(axis=0)


def paint_shell(pos_mpc, observer, rmin, rmax, nside, scheme="bilinear", weight=1.0, sigma=None):
    """Raw weight sums per pixel of the particles with rmin < r <= rmax (FP64); `sigma`
    (radians) for the rbf_neighbor scheme."""
    v = pos_mpc.reshape(-1, 3).astype(np.float64) - np.asarray(observer, np.float64)
    r = np.sqrt((v**2).sum(-1))
    sel = (r > rmin) & (r <= rmax)
    v = v[sel]
    r = r[sel]
    z = v[:, 2] / r
    theta = np.arccos(np.clip(z, -1.0, 1.0))
    phi = np.arctan2(v[:, 1], v[:, 0])
    npix = 12 * nside * nside
    if scheme == "ngp":
        pix = ang2pix(nside, theta, phi)
        return np.bincount(pix, minlength=npix) * weight
    if scheme == "rbf_neighbor":
        pix, w = rbf_weights(nside, theta, phi, sigma)
        return np.bincount(pix.ravel(), weights=w.ravel() * weight, minlength=npix)
    pix, w = get_interp_weights(nside, theta, phi)
    return np.bincount(pix.ravel(), weights=w.ravel() * weight, minlength=npix)


def replica_positions(disp, vel, box, observer, R, shift, *, telephoto=False, t=None, a_of_chi=None, Gp=None,
                      dGfa=None):
    """Mpc/h positions (FP64, flattened to (P, 3)) of one replica: c = x - o with
    x = (grid + disp) / N * L, q = R c + s; with velocities drifted along R v by
    (Gp(a_t) - Gp(t)) / dGfa(sqrt(t a_t)), a_t = a_of_chi(distance), the distance being
    |q + o - o| (onion) or |q - o| (telephoto, as the reference measures it); the
    position q + o (+ the drift). TelephotoInterp._paint_telephoto (pm/interp.py:643-699)
    and one replica of OnionTiler._paint_tiled_27 (pm/interp.py:418-504)."""
    shape = disp.shape[:3]
    n = np.asarray(shape, np.float64)
    L = np.asarray(box, np.float64)
    o = np.asarray(observer, np.float64)
    g = np.stack(np.meshgrid(*[np.arange(k, dtype=np.float64) for k in shape], indexing="ij"), axis=-1)
    c = ((g + disp.astype(np.float64)) / n * L - o).reshape(-1, 3)
    R = np.asarray(R, np.float64)
    q = c @ R.T + np.asarray(shift, np.float64)
    if vel is None:
        return q + o
    vr = vel.astype(np.float64).reshape(-1, 3) @ R.T
    dist = np.linalg.norm(q - o, axis=-1) if telephoto else np.linalg.norm((q + o) - o, axis=-1)
    at = a_of_chi(dist)
    d = (Gp(at) - Gp(t)) / dGfa(np.sqrt(t * at))
    return (q + d[:, None] * vr) + o if telephoto else (q + o) + d[:, None] * vr


def paint_shell_tiled(disp, vel, box, observer, rmin, rmax, nside, rotations, shifts, *, telephoto=False, t=None,
                      a_of_chi=None, Gp=None, dGfa=None, scheme="bilinear", weight=1.0):
    """Raw weight sums of the rotated and shifted replicas of the particles (FP64), every
    replica evaluated (no skipping). OnionTiler._paint_tiled_27 (reference
    pm/interp.py:418-504) and TelephotoInterp._paint_telephoto (pm/interp.py:643-699):
    c = x - o with x = (grid + disp) / N * L; q = R c + s; with velocities, the replica is
    drifted by (Gp(a_t) - Gp(t)) / dGfa(sqrt(t a_t)) along R v, a_t = a_of_chi(distance),
    the distance being |q + o - o| (onion) or |q - o| (telephoto, as the reference
    measures it); the painted position is q + o (+ the drift)."""
    shape = disp.shape[:3]
    n = np.asarray(shape, np.float64)
    L = np.asarray(box, np.float64)
    o = np.asarray(observer, np.float64)
    g = np.stack(np.meshgrid(*[np.arange(k, dtype=np.float64) for k in shape], indexing="ij"), axis=-1)
    x = (g + disp.astype(np.float64)) / n * L
    c = (x - o).reshape(-1, 3)
    v = vel.astype(np.float64).reshape(-1, 3) if vel is not None else None
    npix = 12 * nside * nside
    out = np.zeros(npix)
    for R, s in zip(np.asarray(rotations, np.float64), np.asarray(shifts, np.float64)):
        q = c @ R.T + s
        if v is None:
            pos = q + o
        else:
            vr = v @ R.T
            if telephoto:
                dist = np.linalg.norm(q - o, axis=-1)
            else:
                dist = np.linalg.norm((q + o) - o, axis=-1)
            at = a_of_chi(dist)
            d = (Gp(at) - Gp(t)) / dGfa(np.sqrt(t * at))
            pos = (q + d[:, None] * vr) + o if telephoto else (q + o) + d[:, None] * vr
        out += paint_shell(pos, o, rmin, rmax, nside, scheme, weight)
    return out
