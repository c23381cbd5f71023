"""Generate tests/golden/config5_256.npz: the large light-cone chain at 256^3, run by the
CPU oracle in FP64 and in FP32, for the FP64 statement of that configuration.

Workload (the large light-cone configuration, at the 256^3 size its FP64 statement is made
at): 256^3 particles on a 256^3 mesh, box 1000 Mpc/h, Planck18 (the library's FP64 tables),
white noise numpy default_rng(0).standard_normal as float32, 2LPT to a = 0.1,
EfficientDriftDoubleKick with dt0 = 0.9 / 60 and the PGD correction after every drift
(alpha 0.3, kl 1.5 h/Mpc, ks 8 h/Mpc, as k L / N in radians per cell; reference
pm/correction.py:157-202, pm/solvers.py:165-178); 16 equal-width HEALPix shells from 0 to
1500 Mpc/h around the centred observer at nside 256 (bilinear), painted at their times
with OnionTiler (reference pm/interp.py:321-504): the 4 shells inside the box from the
particles drifted to the light cone, the 12 beyond it from the 27 rotated replicas
(rotation indices numpy default_rng(42).integers(0, 47, 27), every replica evaluated, each
drifted to the light cone); Born convergence of the shells for a tophat n(z) on 0 < z < 1
(reference _src/lensing/_born.py:100-130: 33 Simpson nodes from z = 0.01 to 1, plane width
the box's inscribed radius over the number of planes); C_ell (oracle SHT, healpy anafast
algorithm, lmax 767) of the convergence map and of shells 3 (inside the box), 8 and 15.

Kept (oracle FP64 in float64; oracle FP32 where the FP32-vs-FP64 gap is stated):
  * the convergence map's C_ell, its average over 16^2-pixel blocks (nside 16), mean, rms;
  * each shell's total weight and its average over 16^2-pixel blocks (nside 16);
  * the C_ell of shells 3, 8, 15;
  * the FP32-vs-FP64 gaps over the full maps (relative L2; max per multipole).

Usage (about 40 minutes on 8 cores):  python tests/golden/make_config5.py [--mesh 256]
"""

from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from jfli_b200 import cosmology as cj  # noqa: E402  (host FP64 tables only)
from jfli_b200.lensing import tophat_nz  # noqa: E402
from jfli_b200.pm.integrate import time_events  # noqa: E402
from jfli_b200.pm.interp import get_all_47_symmetries, tile_shifts  # noqa: E402
from jfli_b200.pm.lpt import lpt_coefficients  # noqa: E402
from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK  # noqa: E402
from oracle import healpix as oh  # noqa: E402
from oracle import lensing as olens  # noqa: E402
from oracle import pm as opm  # noqa: E402
from oracle import sht as osht  # noqa: E402

SEED = 0
A0 = 0.1
STEPS = 60
NSHELLS = 16
NSIDE = 256
NSIDE_COARSE = 16
PGD = (0.3, 1.5, 8.0)  # alpha, kl, ks in h/Mpc
CL_SHELLS = (3, 8, 15)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def geometry(cosmo, L):
    """Shell centres, widths and times far to near (as the time loop meets them)."""
    r_max = 3.0 * L / 2.0
    edges = np.linspace(0.0, r_max, NSHELLS + 1)[::-1]
    centres = 0.5 * (edges[1:] + edges[:-1])
    return centres, edges[:-1] - edges[1:], np.asarray(cj.a_of_chi(cosmo, centres), np.float64)


def run(dx, p, cosmo, n, L, dtype, log):
    centres, widths, ts = geometry(cosmo, L)
    dt0 = 0.9 / STEPS
    events = time_events(A0, ts, dt0)
    steps = [(e[1], e[2]) for e in events if e[0] == "step"]
    kicks, drifts = EDK.schedule_arrays(cosmo, [a for a, _ in steps], [b for _, b in steps], dt0)
    alpha, kl, ks = PGD[0], PGD[1] * L / n, PGD[2] * L / n
    rot = get_all_47_symmetries()[np.random.default_rng(42).integers(0, 47, 27)]
    shifts = tile_shifts((0.5, 0.5, 0.5), (L, L, L))
    obs = np.full(3, L / 2.0)
    fn = dict(a_of_chi=lambda r: cj.a_of_chi(cosmo, r), Gp=lambda a: cj.Gp(cosmo, a),
              dGfa=lambda a: cj.dGfa(cosmo, a))
    x = dx.astype(dtype).copy()
    v = p.astype(dtype).copy()
    v += opm.pm_forces(x, dtype) * dtype(EDK.init_kick(cosmo, A0, A0 + dt0))
    maps = [None] * NSHELLS
    si = 0
    t0 = time.time()
    for ev in events:
        if ev[0] == "step":
            x += v * dtype(drifts[si])
            x = opm.pgd_correction(x, alpha, kl, ks, dtype=dtype)
            v += opm.pm_forces(x, dtype) * dtype(kicks[si])
            si += 1
        else:
            i, t = ev[1], float(ev[2])
            rc, wd = centres[i], widths[i]
            rmin, rmax = rc - wd / 2, rc + wd / 2
            vol = (4 * np.pi / (12 * NSIDE * NSIDE)) * (rmax**3 - rmin**3) / 3
            if rmax <= L / 2.0:
                pos = opm.lightcone_drift(x, v, (L, L, L), obs, t, **fn)
                m = oh.paint_shell(pos.reshape(-1, 3), obs, rmin, rmax, NSIDE, "bilinear")
            else:
                m = oh.paint_shell_tiled(x, v, (L, L, L), obs, rmin, rmax, NSIDE, rot, shifts, t=t, **fn)
            maps[i] = m / vol
            log(f"shell {i} ({rmin:.0f}-{rmax:.0f} Mpc/h) at step {si}, {time.time() - t0:.0f}s")
    maps = np.stack(maps[::-1])  # near -> far
    a_near = ts[::-1].copy()
    nz = [tophat_nz(0.0, 1.0)]
    kappa = olens.born_spherical(maps, np.asarray(cj.radial_comoving_distance(cosmo, a_near)), a_near,
                                 (L / 2.0) / NSHELLS, cosmo.Omega_m,
                                 lambda z: cj.radial_comoving_distance(cosmo, 1.0 / (1.0 + np.asarray(z))),
                                 nz_list=nz, min_z=0.01, max_z=1.0, n_integrate=32)[0]
    return maps, kappa, len(steps), centres[::-1].copy(), widths[::-1].copy(), a_near


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", type=int, default=256)
    ap.add_argument("--box", type=float, default=1000.0)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "config5_256.npz"))
    args = ap.parse_args()
    n, L = args.mesh, args.box
    cosmo = cj.Planck18()
    noise = np.random.default_rng(SEED).standard_normal((n, n, n)).astype(np.float32)
    ktab, ptab = cj.pk_table(cosmo, 128)
    lmax = 3 * NSIDE - 1
    out = dict(mesh=n, box=L, seed=SEED, nside=NSIDE, nside_coarse=NSIDE_COARSE, lmax=lmax,
               pgd=np.asarray(PGD), cl_shells=np.asarray(CL_SHELLS))
    full = {}
    t0 = time.time()

    def log(msg):
        print(f"[{time.time() - t0:.0f}s] {msg}", flush=True)

    for tag, dt in (("f64", np.float64), ("f32", np.float32)):
        ic = opm.ic_filter(noise.astype(np.float64), (L, L, L), ktab, ptab).astype(dt)
        dx, p = opm.lpt(ic, *lpt_coefficients(cosmo, A0), order=2, dtype=dt)
        log(f"[{tag}] 2LPT")
        maps, kappa, steps, centres, widths, a_near = run(dx, p, cosmo, n, L, dt, log)
        out.update(steps=steps, shell_centers=centres, shell_widths=widths, shell_a=a_near)
        out[f"shell_sum_{tag}"] = maps.sum(axis=1)
        out[f"shells_coarse_{tag}"] = np.stack([oh.ud_grade_ring(m, NSIDE_COARSE) for m in maps])
        out[f"kappa_coarse_{tag}"] = oh.ud_grade_ring(kappa, NSIDE_COARSE)
        out[f"kappa_mean_{tag}"] = float(kappa.mean())
        out[f"kappa_rms_{tag}"] = float(kappa.std())
        out[f"kappa_cl_{tag}"] = osht.anafast(kappa, lmax)
        out[f"shell_cl_{tag}"] = np.stack([osht.anafast(maps[s] / maps[s].mean() - 1.0, lmax) for s in CL_SHELLS])
        full[f"maps_{tag}"] = maps
        full[f"kappa_{tag}"] = kappa
        log(f"[{tag}] done")
    out["gap_shells_f32"] = np.array([rel_l2(a, b) for a, b in zip(full["maps_f32"], full["maps_f64"])])
    out["gap_kappa_f32"] = rel_l2(full["kappa_f32"], full["kappa_f64"])
    out["gap_kappa_cl_f32"] = float(np.abs(out["kappa_cl_f32"][1:] / out["kappa_cl_f64"][1:] - 1).max())
    out["gap_shell_cl_f32"] = np.abs(out["shell_cl_f32"][:, 1:] / out["shell_cl_f64"][:, 1:] - 1).max(axis=1)
    for k in sorted(out):
        if k.startswith("gap_"):
            print(k, out[k])
    np.savez_compressed(args.out, **out)
    print(f"wrote {args.out} ({os.path.getsize(args.out) / 1e6:.2f} MB) in {time.time() - t0:.0f}s")


if __name__ == "__main__":
    main()
