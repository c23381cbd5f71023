"""CPU oracle for the particle-mesh path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this
module, and only as the checker; the product (jfli_b200) never imports it.

NumPy/SciPy restatement, in FP64 (default) or FP32, of the algorithm the reference runs
through its un-vendored JaxPM fork (jaxpm @ ALL-MODIF, pyproject.toml:32), written from
the published method and the reference's call sites:

* cic_paint_dx / cic_read_dx     <- _src/fields/_painting.py:67, fields/particles.py:203
* pm_forces                      <- pm/solvers.py:19-32 (k-space: -1/k^2, FD-4 gradient
                                    i(8 sin k - sin 2k)/6, k = 2 pi fftfreq, one inverse
                                    complex FFT per force component, CIC readout)
* lpt (order 1, 2)               <- pm/lpt.py:119 (JaxPM lpt, FastPM momentum)
* ic_filter                      <- initial.py:167-182, infer/dist.py:43-79
* power                          <- _src/power/_compute.py:23-119 (full complex FFT,
                                    norm="ortho", digitize + bincount, [1:-1], prod(L/N))
* KDK / KKD steps and the loop   <- pm/solvers.py:118-411, pm/integrate.py:17-279

Parity status: the JaxPM fork and jax itself are not installable here, so no output of
the reference could be generated. The oracle is pinned by the reference's portable
test statements and by analytic known answers (tests/test_oracle.py): the reversible
round trip of tests/test_against_fpm.py:177-216, the shell partition invariants of
tests/test_equal_vol_shells.py, a single plane-wave mode through LPT / forces / P(k)
with closed-form results, and mass conservation of CIC. Values that only the forks
define (growth tables, P_lin normalisation) are parity unpinned.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.fft as sfft

WORKERS = -1


# ----------------------------------------------------------------------------------- CIC
def grid(shape, dtype=np.float64):
    ax = [np.arange(n, dtype=dtype) for n in shape]
    return np.stack(np.meshgrid(*ax, indexing="ij"), axis=-1)


def _cic_corners(disp, shape, absolute=False):
    """(indices (P, 8) flat, weights (P, 8)) for positions grid + disp (or absolute)."""
    dt = disp.dtype
    pos = disp.reshape(-1, 3)
    if absolute:
        base = np.zeros_like(pos, dtype=np.int64)
        f = np.floor(pos)
        frac = pos - f
        ii = f.astype(np.int64)
    else:
        g = grid(shape, np.int64).reshape(-1, 3)
        f = np.floor(pos)
        frac = (pos - f).astype(dt)
        ii = g + f.astype(np.int64)
    n = np.asarray(shape, np.int64)
    idx = []
    wts = []
    one = dt.type(1)
    for ox, oy, oz in ((0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1)):
        o = np.array([ox, oy, oz])
        c = np.mod(ii + o, n)
        w = np.ones(pos.shape[0], dtype=dt)
        for a in range(3):
            w = w * (frac[:, a] if o[a] else (one - frac[:, a]))
        idx.append((c[:, 0] * n[1] + c[:, 1]) * n[2] + c[:, 2])
        wts.append(w)
    return np.stack(idx, axis=1), np.stack(wts, axis=1)


def cic_paint_np(disp, shape=None, weight=1.0, absolute=False):
    """Trilinear deposit onto a periodic mesh; positions are grid + disp (relative).
    NumPy form (bincount accumulates in FP64); cic_paint runs the same arithmetic in C."""
    shape = tuple(disp.shape[:3]) if shape is None else tuple(shape)
    idx, w = _cic_corners(disp, shape, absolute)
    if np.ndim(weight) > 0:
        w = w * np.asarray(weight, dtype=w.dtype).reshape(-1, 1)
    else:
        w = w * w.dtype.type(weight)
    mesh = np.bincount(idx.ravel(), weights=w.ravel(), minlength=int(np.prod(shape)))
    return mesh.reshape(shape).astype(disp.dtype)


def cic_read_np(mesh, disp, absolute=False):
    """NumPy form of cic_read."""
    idx, w = _cic_corners(disp, mesh.shape, absolute)
    vals = mesh.reshape(-1)[idx]
    return (vals * w).sum(axis=1).reshape(disp.shape[:3]).astype(disp.dtype)


def _work_dtype(disp):
    return np.float32 if disp.dtype == np.float32 else np.float64


def cic_paint(disp, shape=None, weight=1.0, absolute=False):
    """Trilinear deposit onto a periodic mesh; positions are grid + disp (relative) or the
    positions themselves in cells (absolute). The arithmetic of cic_paint_np, run by the
    OpenMP restatement in oracle/cic.c."""
    from . import clib

    dt = _work_dtype(disp)
    shape = tuple(disp.shape[:3]) if shape is None else tuple(int(s) for s in shape)
    pos = np.ascontiguousarray(disp, dtype=dt).reshape(-1, 3)
    wts = None
    if np.ndim(weight) > 0:
        wts = np.ascontiguousarray(np.broadcast_to(np.asarray(weight, dtype=dt).reshape(-1), (pos.shape[0],)))
        weight = 1.0
    mesh = np.empty(shape, dtype=dt)
    clib.paint(pos, shape, absolute, wts, weight, mesh)
    return mesh.astype(disp.dtype, copy=False)


def cic_read(mesh, disp, absolute=False):
    """CIC readout of one mesh (or a stack of meshes along a leading axis) at the particles."""
    from . import clib

    dt = _work_dtype(disp)
    stack = np.ascontiguousarray(mesh, dtype=dt)
    single = stack.ndim == 3
    if single:
        stack = stack[None]
    pos = np.ascontiguousarray(disp, dtype=dt).reshape(-1, 3)
    out = np.empty((pos.shape[0], stack.shape[0]), dtype=dt)
    clib.read(stack, pos, absolute, out)
    lead = disp.shape[:3] if not absolute else disp.shape[:-1]
    if single:
        return out[:, 0].reshape(lead).astype(disp.dtype, copy=False)
    return out.reshape(*lead, stack.shape[0]).astype(disp.dtype, copy=False)


# -------------------------------------------------------------------------- k-space kernels
def fftk(shape, dtype=np.float64):
    """Wave vectors in radians per cell, broadcastable over the full complex grid."""
    out = []
    for i, n in enumerate(shape):
        k = (2 * np.pi * np.fft.fftfreq(n)).astype(dtype)
        s = [1, 1, 1]
        s[i] = n
        out.append(k.reshape(s))
    return out


def invlaplace(kvec):
    kk = sum(k**2 for k in kvec)
    safe = np.where(kk == 0, 1, kk)
    return np.where(kk == 0, 0, -1 / safe)


def gradient_kernel(kvec, i):
    w = kvec[i]
    return 1j * (8 * np.sin(w) - np.sin(2 * w)) / 6


def _ctype(dtype):
    return np.complex128 if np.dtype(dtype) == np.float64 else np.complex64


def fft3(x):
    return sfft.fftn(x, workers=WORKERS)


def ifft3(x):
    return sfft.ifftn(x, workers=WORKERS)


def potential_k(delta_k, kvec):
    return delta_k * invlaplace(kvec)


def forces_from_delta_k(delta_k, disp, dtype=np.float64):
    kvec = fftk(delta_k.shape, dtype)
    pot_k = potential_k(delta_k, kvec)
    meshes = np.stack([ifft3(-gradient_kernel(kvec, i) * pot_k).real.astype(dtype) for i in range(3)])
    return cic_read(meshes, disp.astype(dtype))


def pm_forces(disp, dtype=np.float64):
    """-grad_FD laplace^-1 of the CIC density, read out at the particles (no 1.5 Omega_m)."""
    disp = disp.astype(dtype)
    rho = cic_paint(disp)
    return forces_from_delta_k(fft3(rho), disp, dtype)


def potential_real(rho, dtype=np.float64):
    kvec = fftk(rho.shape, dtype)
    return ifft3(potential_k(fft3(rho.astype(dtype)), kvec)).real.astype(dtype)


# ------------------------------------------------------------------------------------ ICs
def interp_extrap(x, xp, fp):
    i = np.clip(np.searchsorted(xp, x) - 1, 0, len(xp) - 2)
    slope = (fp[i + 1] - fp[i]) / (xp[i + 1] - xp[i])
    return fp[i] + (x - xp[i]) * slope


def ic_filter(noise, box, ktab, ptab, zero_mode_one=False, dtype=np.float64):
    shape = noise.shape
    field = fft3(noise.astype(dtype))
    kvec = fftk(shape, dtype)
    kmesh = np.sqrt(sum((kk / box[i] * shape[i]) ** 2 for i, kk in enumerate(kvec)))
    pk = interp_extrap(kmesh.ravel(), np.asarray(ktab, dtype), np.asarray(ptab, dtype)).reshape(kmesh.shape)
    pk = pk * (np.prod(shape) / np.prod(box))
    if zero_mode_one:
        pk = np.where(kmesh == 0, 1.0, pk)
    return ifft3(field * np.sqrt(pk)).real.astype(dtype)


# ------------------------------------------------------------------------------------ LPT
def lpt_forces(ic, order=1, dtype=np.float64):
    """(F1, F2) of JaxPM lpt at the grid points: the first-order force -grad_FD laplace^-1 ic
    and, for order 2, the force of the second-order source sum_{i<j} phi_ii phi_jj - phi_ij^2
    (F2 None for order 1)."""
    ic = ic.astype(dtype)
    zeros = np.zeros(ic.shape + (3,), dtype)
    delta_k = fft3(ic)
    F1 = forces_from_delta_k(delta_k, zeros, dtype)
    if order != 2:
        return F1, None
    kvec = fftk(ic.shape, dtype)
    pot_k = potential_k(delta_k, kvec)
    delta2 = 0
    shear_acc = 0
    for i in range(3):
        shear_ii = ifft3(gradient_kernel(kvec, i) ** 2 * pot_k).real
        delta2 = delta2 + shear_ii * shear_acc
        shear_acc = shear_acc + shear_ii
        for j in range(i + 1, 3):
            delta2 = delta2 - ifft3(gradient_kernel(kvec, i) * gradient_kernel(kvec, j) * pot_k).real ** 2
    return F1, forces_from_delta_k(fft3(delta2), zeros, dtype)


def lpt_lightcone(ic, order, box, observer, a_of_chi, coefficients, dtype=np.float64):
    """Light-cone-mode LPT (reference pm/lpt.py:110-130, utils.py:234-244): every particle
    at a = a_of_chi(|x - observer|), x its grid point in Mpc/h, with the LPT coefficients
    (c1x, c2x, c1p, c2p) = coefficients(a) (arrays); returns (dx, p, a)."""
    F1, F2 = lpt_forces(ic, order, dtype)
    shape = ic.shape
    x = grid(shape) / np.asarray(shape, np.float64) * np.asarray(box, np.float64)
    a = a_of_chi(np.linalg.norm(x - np.asarray(observer, np.float64), axis=-1))
    c1x, c2x, c1p, c2p = (np.asarray(c, np.float64)[..., None] for c in coefficients(a))
    dx = c1x * F1
    p = c1p * dx
    if F2 is not None:
        dx2 = c2x * F2
        dx = dx + dx2
        p = p + c2p * dx2
    return dx.astype(dtype), p.astype(dtype), a


def lpt(ic, c1x, c2x, c1p, c2p, order=1, dtype=np.float64):
    """JaxPM lpt at the grid points: dx = c1x F1 (+ c2x F2), p = c1p c1x F1 (+ c2p c2x F2)."""
    ic = ic.astype(dtype)
    zeros = np.zeros(ic.shape + (3,), dtype)
    delta_k = fft3(ic)
    F1 = forces_from_delta_k(delta_k, zeros, dtype)
    dx = c1x * F1
    p = c1p * dx
    if order == 2:
        kvec = fftk(ic.shape, dtype)
        pot_k = potential_k(delta_k, kvec)
        delta2 = 0
        shear_acc = 0
        for i in range(3):
            shear_ii = ifft3(gradient_kernel(kvec, i) ** 2 * pot_k).real
            delta2 = delta2 + shear_ii * shear_acc
            shear_acc = shear_acc + shear_ii
            for j in range(i + 1, 3):
                delta2 = delta2 - ifft3(gradient_kernel(kvec, i) * gradient_kernel(kvec, j) * pot_k).real ** 2
        F2 = forces_from_delta_k(fft3(delta2), zeros, dtype)
        dx2 = c2x * F2
        dx = dx + dx2
        p = p + c2p * dx2
    return dx.astype(dtype), p.astype(dtype)


# ------------------------------------------------------------------------------------ P(k)
def power(mesh, box, kedges, kdtype=np.float64):
    """(kavg, pk) with jax-fli's _power conventions. `kdtype` is the precision of the
    |k| grid and of the bin edges used by digitize (float32 in the reference's default
    FP32 mode, which decides the bin of modes that sit exactly on an edge)."""
    shape = mesh.shape
    meshk = sfft.fftn(mesh.astype(np.float64), norm="ortho", workers=WORKERS)
    kvec = []
    for i, (m, b) in enumerate(zip(shape, box)):
        s = [1, 1, 1]
        s[i] = m
        kvec.append(kdtype(2 * np.pi * m / b) * np.fft.fftfreq(m).astype(kdtype).reshape(s))
    kmesh = np.sqrt(sum(k * k for k in kvec)).astype(kdtype)
    kedges = np.asarray(kedges).astype(kdtype)
    dig = np.digitize(kmesh.ravel(), kedges)
    nb = len(kedges) + 1
    cnt = np.bincount(dig, minlength=nb)
    kavg = np.bincount(dig, weights=kmesh.ravel(), minlength=nb) / np.where(cnt == 0, 1, cnt)
    ps = np.bincount(dig, weights=(meshk.real**2 + meshk.imag**2).ravel(), minlength=nb)
    pk = (ps / np.where(cnt > 0, cnt, 1))[1:-1] * np.prod(np.asarray(box) / np.asarray(shape))
    return kavg[1:-1], pk


# ------------------------------------------------------------------------------- stepping
def clip_times(t0, ts, dt0, dtype=np.float32):
    """Step list of pm/integrate.py:_fwd_loop: [(t_curr, t_next)], snapshot after each target."""
    T = np.dtype(dtype).type
    tol = 1e-10 if np.dtype(dtype) == np.float64 else 1e-6
    out = []
    t = T(t0)
    for target in np.atleast_1d(ts):
        tg = T(target)
        seg = []
        while t < tg:
            tn = T(t + T(dt0))
            if tn > tg - tol:
                tn = tg
            seg.append((float(t), float(tn)))
            t = tn
        out.append(seg)
    return out


def pgd_correction(disp, alpha, kl, ks, dtype=np.float64):
    """PGD position correction (reference pm/correction.py:157-202): paint, filter the
    potential by exp(-kl^2/k^2) exp(-k^4/ks^4) (k in rad/cell, k = 0 -> 0), read out the
    FD-gradient force and move x by alpha times it."""
    disp = disp.astype(dtype)
    kvec = fftk(disp.shape[:3], dtype)
    kk = sum(k**2 for k in kvec)
    safe = np.where(kk == 0, 1, kk)
    rng = np.where(kk == 0, 0, np.exp(-(kl**2) / safe) * np.exp(-(kk**2) / ks**4))
    pot_k = fft3(cic_paint(disp)) * invlaplace(kvec) * rng
    f = cic_read(np.stack([ifft3(-gradient_kernel(kvec, i) * pot_k).real.astype(dtype) for i in range(3)]), disp)
    return disp + dtype(alpha) * f


def sharpening_boost(disp, alpha, kl, ks, drift_factor, dtype=np.float64):
    """SharpeningKernel's velocity boost (reference pm/correction.py:293-333): the PGD
    displacement alpha F_pgd(x) divided by the drift factor the step hands over."""
    x = disp.astype(dtype)
    return (pgd_correction(x, alpha, kl, ks, dtype) - x) / dtype(drift_factor)


def kdk_run(dx, p, coeffs, dtype=np.float64, snapshot_after=None, pgd=None, sharpen=None):
    """FastPM KDK loop (EfficientDriftDoubleKick): coeffs = dict(init_kick, steps=[(kick, drift)]).
    pgd = (alpha, kl, ks) applies the PGD correction after each drift (reference
    pm/solvers.py:165-178); sharpen = (alpha, kl, ks, bare drift factors) adds the
    SharpeningKernel boost at the drifted positions before the kick (pm/solvers.py:174-195).

    Returns (x, v, snapshots) with snapshots = densities painted after the listed steps."""
    x = dx.astype(dtype).copy()
    v = p.astype(dtype).copy()
    v += pm_forces(x, dtype) * dtype(coeffs["init_kick"])
    snaps = []
    for n, (kick, drift) in enumerate(coeffs["steps"]):
        x += v * dtype(drift)
        if pgd is not None:
            x = pgd_correction(x, *pgd, dtype=dtype)
        if sharpen is not None:
            v += sharpening_boost(x, *sharpen[:3], sharpen[3][n], dtype)
        v += pm_forces(x, dtype) * dtype(kick)
        if snapshot_after is not None and n in snapshot_after:
            snaps.append(cic_paint(x))
    return x, v, snaps


def kkd_step(x, v, kick, drift, dtype=np.float64, sharpen=None):
    """One ReversibleDoubleKickDrift step: kick with the force at x, then drift. sharpen =
    (alpha, kl, ks) adds SharpeningKernel's boost at x between the kick and the drift, with
    the step's full drift factor (reference pm/solvers.py:292-318)."""
    v = v + pm_forces(x, dtype) * dtype(kick)
    if sharpen is not None:
        v = v + sharpening_boost(x, *sharpen, drift, dtype)
    x = x + v * dtype(drift)
    return x, v


def kkd_reverse(x, v, kick, drift, dtype=np.float64, sharpen=None):
    """The inverse of kkd_step: un-drift, take the boost off at the recovered positions, un-kick."""
    x = x - v * dtype(drift)
    if sharpen is not None:
        v = v - sharpening_boost(x, *sharpen, drift, dtype)
    v = v - pm_forces(x, dtype) * dtype(kick)
    return x, v


def kkd_run(dx, p, steps, dtype=np.float64, snapshot_after=None, sharpen=None):
    x = dx.astype(dtype).copy()
    v = p.astype(dtype).copy()
    snaps = []
    for n, (kick, drift) in enumerate(steps):
        x, v = kkd_step(x, v, kick, drift, dtype, sharpen)
        if snapshot_after is not None and n in snapshot_after:
            snaps.append(cic_paint(x))
    return x, v, snaps


# ------------------------------------------------------------------------ light cone
def lightcone_drift(disp, vel, box, observer, t, a_of_chi, Gp, dGfa):
    """Particles drifted to their light-cone crossing, in Mpc/h (reference
    pm/interp.py:110-121 and 284-297): x = (grid + disp) / N * L, a_t = a_of_chi(|x - o|),
    x += v (Gp(a_t) - Gp(t)) / dGfa(sqrt(t a_t)); the momentum array is added as stored.
    The cosmology functions are passed in (FP64)."""
    shape = disp.shape[:3]
    n = np.asarray(shape, np.float64)
    L = np.asarray(box, np.float64)
    x = (grid(shape) + disp.astype(np.float64)) / n * L
    r = np.linalg.norm(x - np.asarray(observer, np.float64), axis=-1)
    at = a_of_chi(r)
    drift = (Gp(at) - Gp(t)) / dGfa(np.sqrt(t * at))
    return x + drift[..., None] * vel.astype(np.float64)


def power_poles(mesh, mesh2, box, kedges, multipoles=0, los=(0.0, 0.0, 1.0)):
    """Reference _power with cross spectra and multipoles (_src/power/_compute.py:5-119):
    full complex fftn (ortho, FP64 here), k grid (2 pi m / L) fftfreq(m) in float32 as the
    reference builds it, digitize, mu = (k . los) / |k| (0 at k = 0), weights
    (2l + 1) L_l(mu) (the reference's recurrence), bincount of Re and Im; the modulus for a
    cross spectrum, the real sum for an auto one; / counts, [1:-1], * prod(L/N)."""
    shape = mesh.shape
    box = np.asarray(box, np.float64)
    poles = multipoles if isinstance(multipoles, (list, tuple)) else (multipoles,)
    f1 = np.fft.fftn(mesh.astype(np.float64), norm="ortho")
    mmk = (f1.real**2 + f1.imag**2) if mesh2 is None else f1 * np.conj(np.fft.fftn(mesh2.astype(np.float64),
                                                                                     norm="ortho"))
    kvec = []
    for i, (m, b) in enumerate(zip(shape, box)):
        fr = np.fft.fftfreq(m).astype(np.float32)
        sh = [1] * 3
        sh[i] = m
        kvec.append((np.float32(2 * np.pi * m / b) * fr).reshape(sh).astype(np.float32))
    kmesh = np.sqrt((kvec[0] ** 2 + kvec[1] ** 2 + kvec[2] ** 2).astype(np.float32)).astype(np.float32)
    kmesh = np.broadcast_to(kmesh, shape)
    edges = np.asarray(kedges, np.float32)
    dig = np.digitize(kmesh.reshape(-1), edges)
    nb = edges.size + 1
    cnt = np.bincount(dig, minlength=nb).astype(np.float64)
    kavg = (np.bincount(dig, weights=kmesh.reshape(-1).astype(np.float64), minlength=nb) / np.maximum(cnt, 1))[1:-1]
    if poles == (0,):
        mu = np.ones(shape)
    else:
        lv = np.asarray(los, np.float64) / np.linalg.norm(los)
        dot = sum(np.broadcast_to(kvec[i].astype(np.float64), shape) * lv[i] for i in range(3))
        mu = np.where(kmesh == 0, 0.0, dot / np.where(kmesh == 0, 1.0, kmesh))
    out = []
    for ell in poles:
        p0, p1 = np.ones_like(mu), mu
        if ell == 0:
            L = p0
        elif ell == 1:
            L = p1
        else:
            for n in range(2, ell + 1):
                p0, p1 = p1, ((2 * n - 1) * mu * p1 - (n - 1) * p0) / n
            L = p1
        w = (mmk * (2 * ell + 1) * L).reshape(-1)
        if mesh2 is None:
            ps = np.bincount(dig, weights=w.real, minlength=nb)
        else:
            ps = np.hypot(np.bincount(dig, weights=w.real, minlength=nb), np.bincount(dig, weights=w.imag,
                                                                                       minlength=nb))
        out.append((ps / np.maximum(cnt, 1))[1:-1] * np.prod(box / np.asarray(shape)))
    pk = np.stack(out)
    return kavg, (pk[0] if len(poles) == 1 else pk)
