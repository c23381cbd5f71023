"""Generate tests/golden/config2_256.npz: the 256^3 plain-PM configuration with its
precision audit, run by the CPU oracle in FP64 and in FP32.

Workload (the configuration the headline metric is quoted on): 256^3 particles on a 256^3
mesh, box 1000 Mpc/h, Planck18, white noise numpy default_rng(0).standard_normal as
float32 (the array the GPU run receives), the library's FP64 P_lin, growth and time-step
tables (the parity harness feeds identical tables to every side), 2LPT to a = 0.1, then
EfficientDriftDoubleKick with dt0 = 0.9 / 40:

  A. density run to a = 1 (ts = [1.0], 40 steps): final CIC density, its P(k) in 32
     log-spaced bins (33 edges from 2 pi / L (1 - 1e-6) to pi N / L), final displacements
     and momenta; forces of the 2LPT particles (pm_forces, no 1.5 Omega_m factor);
  B. light-cone run, nb_shells = 4 (centred observer, equal widths of 125 Mpc/h, centres
     62.5 ... 437.5 Mpc/h), HEALPix nside 256, bilinear, each shell painted at its time
     (number density per pixel volume), near to far; C_ell of each shell's overdensity
     map / mean - 1 (oracle SHT, healpy anafast algorithm, lmax 767, iter 3).

A full-size field is 67-201 MB, so the fixture keeps reductions (oracle FP64 in float64,
oracle FP32 where the FP32-vs-FP64 gap is stated):
  * P(k) and C_ell in full;
  * densities summed over 8^3 blocks (32^3) and one full-resolution plane (x = 128);
  * shells averaged over 16^2 children per pixel (graded to nside 16, RING);
  * displacements, momenta and forces at 4096 seeded particles (FP64 only);
  * the FP32-vs-FP64 gaps over the full fields (relative L2; max per bin).

Usage (about 15 minutes on 8 cores):  python tests/golden/make_config2.py [--mesh 256]
Smaller meshes (e.g. --mesh 64 --out /tmp/c.npz) give a fast check of the script itself.
"""

from __future__ import annotations

import argparse
import os
import sys
import time
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from jfli_b200 import cosmology as cj  # noqa: E402  (host FP64 tables only)
from jfli_b200.pm.integrate import time_events  # noqa: E402
from jfli_b200.pm.lpt import lpt_coefficients  # noqa: E402
from jfli_b200.pm.solvers import EfficientDriftDoubleKick as EDK  # noqa: E402
from jfli_b200.utils import compute_lightcone_shells, distances  # noqa: E402
from oracle import healpix as oh  # noqa: E402
from oracle import pm as opm  # noqa: E402
from oracle import sht as osht  # noqa: E402

SEED = 0
A0 = 0.1
STEPS = 40
NSHELLS = 4
NSIDE = 256
NSIDE_COARSE = 16
NSAMPLE = 4096


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def block_sum(rho, b=8):
    n = rho.shape[0] // b
    return rho.astype(np.float64).reshape(n, b, n, b, n, b).sum(axis=(1, 3, 5))


def grade_ring(m, nside_out):
    return oh.ud_grade_ring(np.asarray(m, np.float64), nside_out)


def kdk_coefficients(cosmo, ts, dt0):
    steps = [(e[1], e[2]) for e in time_events(A0, ts, dt0) if e[0] == "step"]
    kicks, drifts = EDK.schedule_arrays(cosmo, [a for a, _ in steps], [b for _, b in steps], dt0)
    return dict(init_kick=EDK.init_kick(cosmo, A0, A0 + dt0), steps=list(zip(kicks, drifts))), steps


def run_shells(x0, p0, cosmo, dt0, n, L, dtype):
    """KDK from the 2LPT state with the 4 shells painted at their snapshot times (the
    reference loop: steps clipped to each shell's time, the shell painted from the
    positions there, no drift within the shell); maps near to far."""
    field = types.SimpleNamespace(max_comoving_radius=L / 2.0)
    r_c, a_c = compute_lightcone_shells(cosmo, field, nb_shells=NSHELLS)
    widths = distances(r_c, 0.0)
    events = time_events(A0, a_c, dt0)
    coeffs, _ = kdk_coefficients(cosmo, a_c, dt0)
    x = x0.astype(dtype).copy()
    v = p0.astype(dtype).copy()
    v += opm.pm_forces(x, dtype) * dtype(coeffs["init_kick"])
    obs = np.full(3, L / 2.0)
    g = opm.grid((n, n, n))
    maps = []
    si = 0
    nsteps = 0
    for ev in events:
        if ev[0] == "step":
            kick, drift = coeffs["steps"][si]
            si += 1
            nsteps += 1
            x += v * dtype(drift)
            v += opm.pm_forces(x, dtype) * dtype(kick)
        else:
            i = ev[1]
            rmin, rmax = r_c[i] - widths[i] / 2, r_c[i] + widths[i] / 2
            pos = (g + x.astype(np.float64)) * (L / n)
            vol = (4 * np.pi / (12 * NSIDE * NSIDE)) * (rmax**3 - rmin**3) / 3
            maps.append(oh.paint_shell(pos.reshape(-1, 3), obs, rmin, rmax, NSIDE, "bilinear") / vol)
    return np.stack(maps[::-1]), r_c[::-1].copy(), widths[::-1].copy(), nsteps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", type=int, default=256)
    ap.add_argument("--box", type=float, default=1000.0)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "config2_256.npz"))
    args = ap.parse_args()
    n, L = args.mesh, args.box
    cosmo = cj.Planck18()
    dt0 = 0.9 / STEPS
    noise = np.random.default_rng(SEED).standard_normal((n, n, n)).astype(np.float32)
    ktab, ptab = cj.pk_table(cosmo, 128)
    kedges = np.geomspace(2 * np.pi / L * (1 - 1e-6), np.pi * n / L, 33)
    sample = np.sort(np.random.default_rng(12345).choice(n**3, size=min(NSAMPLE, n**3), replace=False))
    out = dict(mesh=n, box=L, seed=SEED, dt0=dt0, kedges=kedges, sample=sample.astype(np.int64),
               nside=NSIDE, nside_coarse=NSIDE_COARSE, plane_x=n // 2)
    full = {}
    t0 = time.time()
    for tag, dt in (("f64", np.float64), ("f32", np.float32)):
        ic = opm.ic_filter(noise.astype(np.float64), (L, L, L), ktab, ptab).astype(dt)
        dx, p = opm.lpt(ic, *lpt_coefficients(cosmo, A0), order=2, dtype=dt)
        print(f"[{tag}] 2LPT done {time.time() - t0:.0f}s", flush=True)
        if tag == "f64":
            out["lpt_dx_f64"] = dx.reshape(-1, 3)[sample]
            out["lpt_p_f64"] = p.reshape(-1, 3)[sample]
            out["force_lpt_f64"] = opm.pm_forces(dx, dt).reshape(-1, 3)[sample]
        full[f"lpt_dx_{tag}"] = dx
        coeffs, steps = kdk_coefficients(cosmo, [1.0], dt0)
        x, v, snaps = opm.kdk_run(dx, p, coeffs, dtype=dt, snapshot_after={len(steps) - 1})
        rho = snaps[0]
        print(f"[{tag}] density run, {len(steps)} steps, done {time.time() - t0:.0f}s", flush=True)
        kavg, pk = opm.power(rho, (L, L, L), kedges, kdtype=np.float32)
        out["kavg"] = kavg
        out["steps"] = len(steps)
        out[f"pk_{tag}"] = pk
        out[f"rho_coarse_{tag}"] = block_sum(rho)
        out[f"rho_plane_{tag}"] = rho[n // 2].astype(np.float32 if tag == "f32" else np.float64)
        if tag == "f64":
            out["dx_f64"] = x.reshape(-1, 3)[sample]
            out["p_f64"] = v.reshape(-1, 3)[sample]
        full[f"rho_{tag}"] = rho
        full[f"dx_{tag}"] = x
        maps, r_c, widths, nsh = run_shells(dx, p, cosmo, dt0, n, L, dt)
        print(f"[{tag}] light-cone run, {nsh} steps, done {time.time() - t0:.0f}s", flush=True)
        out["shell_steps"] = nsh
        out["shell_centers"] = r_c
        out["shell_widths"] = widths
        out[f"shells_coarse_{tag}"] = np.stack([grade_ring(m, NSIDE_COARSE) for m in maps])
        out[f"shell_sum_{tag}"] = maps.astype(np.float64).sum(axis=1)
        out[f"cl_{tag}"] = np.stack([osht.anafast(m / m.mean() - 1.0, 3 * NSIDE - 1) for m in maps])
        print(f"[{tag}] C_ell done {time.time() - t0:.0f}s", flush=True)
        full[f"shells_{tag}"] = maps
    out["gap_lpt_dx_f32"] = rel_l2(full["lpt_dx_f32"], full["lpt_dx_f64"])
    out["gap_rho_f32"] = rel_l2(full["rho_f32"], full["rho_f64"])
    out["gap_dx_f32"] = rel_l2(full["dx_f32"], full["dx_f64"])
    out["gap_shells_f32"] = np.array([rel_l2(a, b) for a, b in zip(full["shells_f32"], full["shells_f64"])])
    ok = out["pk_f64"] > 0
    out["gap_pk_f32"] = float(np.abs(out["pk_f32"][ok] / out["pk_f64"][ok] - 1).max())
    out["gap_cl_f32"] = np.abs(out["cl_f32"][:, 1:] / out["cl_f64"][:, 1:] - 1).max(axis=1)
    for k in sorted(out):
        if k.startswith("gap_"):
            print(k, out[k])
    np.savez_compressed(args.out, **out)
    print(f"wrote {args.out} ({os.path.getsize(args.out) / 1e6:.2f} MB) in {time.time() - t0:.0f}s")


if __name__ == "__main__":
    main()
