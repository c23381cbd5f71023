/*
 * libjfli_b200 — C-ABI of the B200 (sm_100a) particle-mesh kernels behind the
 * jax-fli API. Every function takes device pointers owned by the caller, enqueues its
 * work on `stream` (a cudaStream_t passed as void*, NULL = legacy default stream) and
 * returns JFLI_OK (0) or a JFLI_E* code, with a NUL-terminated message written to
 * `err` (may be NULL) of capacity `errlen`. Nothing throws across this boundary.
 *
 * Layouts (all C order, float32 unless stated):
 *   mesh       [batch][nx][ny][nz]
 *   particles  [batch][nx][ny][nz][3]  particle (i,j,k) sits on grid point (i,j,k);
 *              "relative" positions are displacements in cell units (jax-fli
 *              PositionUnit.GRID_RELATIVE), "absolute" positions are grid coordinates
 *              (PositionUnit.GRID_ABSOLUTE)
 *   spectrum   [batch][nx][ny][nz/2+1] complex64 (interleaved float2)
 * Meshes used with an FFT need nx, ny and nz/2 of the form 2^a 3^b (<= 4096), nz even.
 * One mesh (one batch entry) holds at most (2^32 - 1) / 3 cells (about 1130^3): particle
 * offsets are 32-bit. Larger shapes return JFLI_EINVAL.
 *
 * Reference interfaces replaced (paths inside the jax-fli project):
 *   jfli_paint_cic         <- _src/fields/_painting.py:22-86 (_single_paint -> cic_paint_dx / cic_paint)
 *   jfli_readout_cic       <- fields/particles.py:182-229 (read_out -> cic_read_dx / cic_read)
 *   jfli_rfft3d/irfft3d    <- jaxpm fft3d / ifft3d as used at initial.py:175,182, pm/correction.py:174,193
 *   jfli_poisson_potential <- the invlaplace_kernel stage of jaxpm pm_forces (pm/solvers.py:22)
 *   jfli_pm_forces         <- pm/solvers.py:19-32 (_forces -> jaxpm pm_forces, times 1.5 Omega_m)
 *   jfli_force_mesh        <- the gradient_kernel stage of jaxpm pm_forces (pm/solvers.py:22)
 *   jfli_kick_drift_paint  <- pm/solvers.py:151-202 and 258-325 (the per-particle part of step())
 *   jfli_pm_step           <- one step() of EfficientDriftDoubleKick / ReversibleDoubleKickDrift
 *   jfli_kkd_run           <- the ReversibleDoubleKickDrift time loop (pm/integrate.py:196-279)
 *   jfli_ic_filter         <- initial.py:167-182 (interpolate_initial_conditions), infer/dist.py:43-79
 *   jfli_lpt               <- pm/lpt.py:119 (jaxpm lpt, order 1 and 2)
 *   jfli_power_spectrum    <- _src/power/_compute.py:23-119 (_initialize_pk + _power)
 *   jfli_power_poles       <- the same _power with mesh2 (cross) and multipoles != 0
 *   jfli_healpix_paint     <- _src/fields/_painting.py:249-348 (jaxpm paint_particles_spherical)
 *   jfli_lightcone_drift   <- pm/interp.py:110-121 (_drift_to_time) as used by DriftInterp.paint
 *                             (pm/interp.py:254-318)
 *   jfli_replica_positions <- TelephotoInterp._paint_telephoto's transformed positions
 *                             (pm/interp.py:666-685) for its flat-sky planes
 *   jfli_paint_flat        <- _src/fields/_painting.py:117-202 (_single_paint_2d, jaxpm cic_paint_2d)
 *                             behind ParticleField.paint_2d (fields/particles.py:234-320)
 *   jfli_flat_cl           <- _src/power/_compute.py:122-172 (_flat_cl) behind
 *                             FlatDensity.angular_cl (fields/lightcone.py:197-233)
 *   jfli_healpix_paint_tiled <- OnionTiler._paint_tiled_27 (pm/interp.py:418-504) and
 *                             TelephotoInterp._paint_telephoto (pm/interp.py:643-699): the
 *                             rotated, shifted (and drifted) replicas painted in one pass
 *   jfli_born              <- _src/lensing/_born.py:29-130 (_born_core_impl, _born_spherical)
 *   jfli_born_flat         <- _src/lensing/_born.py:29-97 and 133-186 (_born_flat)
 *   jfli_sht_map2alm / jfli_sht_alm2map <- the Legendre stages of healpy.anafast behind
 *                             SphericalDensity.angular_cl (_src/power/_compute.py:175-191)
 *   jfli_sht_ring_analysis / jfli_sht_ring_synthesis <- the ring FFTs along phi of the same
 * Adjoints (the reverse-mode derivatives jax.grad takes through the same code, and the
 * backward loop of the reversible adjoint, pm/integrate.py:147-535):
 *   jfli_adjoint_unkick_paint, jfli_poisson_divergence, jfli_adjoint_position, jfli_kkd_adjoint
 *                          <- _integrate_bwd (pm/integrate.py:288-535): solver.reverse
 *                             (pm/solvers.py:327-411) + VJP of ReversibleDoubleKickDrift.step
 *                             (pm/solvers.py:258-325) through _forces (pm/solvers.py:19-32)
 *   jfli_power_spectrum_adjoint <- VJP of _power (_src/power/_compute.py:68-119)
 *   jfli_lpt_adjoint       <- VJP of jaxpm lpt (pm/lpt.py:119)
 *   jfli_ic_filter_tangent <- derivative of initial.py:167-182 with respect to the P(k) table
 */
#ifndef JFLI_B200_H
#define JFLI_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JFLI_OK 0
#define JFLI_EINVAL 1      /* bad argument (null pointer, bad shape, short workspace) */
#define JFLI_ECUDA 2       /* a CUDA call or kernel launch failed */
#define JFLI_EUNSUPPORTED 3 /* valid but unsupported configuration */

#define JFLI_STEP_KICK 1   /* v += F(x) * kick, F the CIC readout of the force meshes */
#define JFLI_STEP_DRIFT 2  /* x += v * drift */
#define JFLI_STEP_PAINT 4  /* CIC deposit at the new position */
#define JFLI_STEP_FORCE 8  /* (jfli_pm_step) solve the Poisson equation for the new positions */
#define JFLI_STEP_CORRECT 16 /* x += F(x) * kick instead of a kick (PGD position correction) */
#define JFLI_STEP_CLEAR 32 /* (jfli_kick_drift_paint) clear rho right before the pass paints into it */

#define JFLI_HEALPIX_NGP 0
#define JFLI_HEALPIX_BILINEAR 1

/* Library identification and device checks. */
const char* jfli_version(void);
/* Number of kernels this library has launched in the calling process. */
long long jfli_launch_count(void);
/* JFLI_OK if the current device is sm_100 (B200). */
int jfli_device_check(char* err, size_t errlen);
/* 1 if an FFT over an (nx, ny, nz) mesh is supported. */
int jfli_mesh_supported(int nx, int ny, int nz);
/* Complex elements of one half spectrum: nx * ny * (nz/2 + 1). */
long long jfli_spectrum_elems(int nx, int ny, int nz);

/* Forward real-to-complex 3D FFT (unnormalised, numpy.fft.rfftn convention). */
int jfli_rfft3d(void* stream, const float* mesh, void* spec, int nx, int ny, int nz, int batch, char* err,
                size_t errlen);
/* Inverse complex-to-real 3D FFT, normalised by 1/(nx ny nz) (numpy.fft.irfftn).
 * The spectrum is used as scratch and is overwritten. */
int jfli_irfft3d(void* stream, void* spec, float* mesh, int nx, int ny, int nz, int batch, char* err, size_t errlen);

/* CIC deposit of weight `weight` (times weights[p] when weights != NULL) per particle.
 * accumulate = 0 clears the mesh first. */
int jfli_paint_cic(void* stream, const float* pos, int absolute, const float* weights, float weight, float* mesh,
                   int accumulate, int nx, int ny, int nz, int batch, char* err, size_t errlen);
/* CIC interpolation of a scalar mesh at the particle positions, out[batch][nx][ny][nz]. */
int jfli_readout_cic(void* stream, const float* pos, int absolute, const float* mesh, float* out, int nx, int ny,
                     int nz, int batch, char* err, size_t errlen);

/* pot = irfft(rfft(rho - rho_mean) * (-1/k^2)), k in radians per cell, k = 0 -> 0. */
size_t jfli_poisson_workspace_bytes(int nx, int ny, int nz, int batch);
int jfli_poisson_potential(void* stream, const float* rho, float rho_mean, float* pot, void* workspace,
                           size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen);
/* PGD potential: as jfli_poisson_potential with the extra filter exp(-kl^2/k^2) exp(-k^4/ks^4)
 * (kl, ks in radians per cell). Replaces pm/correction.py:170-189 (PGDKernel.apply). */
int jfli_pgd_potential(void* stream, const float* rho, float rho_mean, float kl, float ks, float* pot, void* workspace,
                       size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen);
/* The reversible step's kick and SharpeningKernel's velocity boost as one potential:
 * pot = irfft(rfft(rho - rho_mean) (-1/k^2) (kick + boost exp(-kl^2/k^2) exp(-k^4/ks^4))),
 * so that the CIC readout of its force mesh with factor 1 is kick F + boost F_pgd at the
 * same positions. Replaces ReversibleDoubleKickDrift.step's kick and
 * SharpeningKernel.apply (pm/solvers.py:292-318, pm/correction.py:248-333; boost =
 * alpha / the full drift factor) and EfficientDriftDoubleKick.step's boost and kick at the
 * drifted positions (pm/solvers.py:174-195; boost = alpha / the bare drift factor).
 * Workspace as jfli_pgd_potential. */
int jfli_sharpen_potential(void* stream, const float* rho, float rho_mean, float kick, float boost, float kl, float ks,
                           float* pot, void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch,
                           char* err, size_t errlen);
/* Adjoint of the PGD correction x' = x + alpha F_pgd(x) (the `jfli_pgd` entries' `_bwd`;
 * F_pgd the CIC readout of the FD force mesh of jfli_pgd_potential's potential of the
 * particles' own density, reference pm/correction.py:157-202): lam_x += alpha J^T u with J
 * = dF_pgd/dx at the relative positions disp and u the cotangent of x' (pass lam_x = u to
 * get the full cotangent of x). J^T u = grad_x R_x[sum_a u_a F_a] + grad_x R_x[rho_bar],
 * rho_bar = P_pgd(div_FD paint(u)), the PGD filter being symmetric. Workspace:
 * jfli_pgd_adjoint_workspace_bytes. */
size_t jfli_pgd_adjoint_workspace_bytes(int nx, int ny, int nz, int batch);
int jfli_pgd_adjoint(void* stream, const float* disp, const float* u, float alpha, float kl, float ks, float* lam_x,
                     void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                     size_t errlen);
/* The same VJP for the PM force itself: lam_x += scale J^T u, J = dF/dx for F the CIC
 * readout of the FD force mesh of the Poisson potential of the particles' own density at
 * the relative positions disp (the force the KDK and KKD steps kick with, unscaled).
 * Workspace: jfli_pgd_adjoint_workspace_bytes. */
int jfli_force_adjoint(void* stream, const float* disp, const float* u, float scale, float* lam_x, void* workspace,
                       size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen);
/* forces[p] = scale * CIC readout of -grad_FD(pot) at the particle positions. */
int jfli_readout_gradient(void* stream, const float* pos, int absolute, const float* pot, float scale, float* forces,
                          int nx, int ny, int nz, int batch, char* err, size_t errlen);
/* forces = scale * (paint -> Poisson -> -grad_FD -> readout); jax-fli's _forces uses scale = 1.5 Omega_m. */
size_t jfli_pm_forces_workspace_bytes(int nx, int ny, int nz, int batch);
int jfli_pm_forces(void* stream, const float* pos, int absolute, float scale, float* forces, void* workspace,
                   size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen);

/* Force meshes: force = scale * (-D pot), AoS float4 [batch][nx][ny][nz][4] =
 * (Fx, Fy, Fz, 0) (16-byte aligned; one aligned load per CIC corner), D the 4-point
 * finite difference whose Fourier eigenvalue is JaxPM's gradient_kernel. Its CIC readout is
 * the force of jaxpm pm_forces (pm/solvers.py:19-32). */
int jfli_force_mesh(void* stream, const float* pot, float scale, float* force, int nx, int ny, int nz, int batch,
                    char* err, size_t errlen);
/* Force meshes of a density: pot = jfli_poisson_potential(rho, rho_mean), then
 * force = jfli_force_mesh(pot, scale), in one call (the Poisson solve and gradient of
 * pm/solvers.py:19-32 _forces, jaxpm pm_forces, before the readout). With clear_rho != 0
 * the density mesh is set to 0 as the forward FFT reads it, ready for a later paint; pot
 * must not alias rho then. (A step loop does better with JFLI_STEP_CLEAR on the paint: the
 * zeroed lines are then still in L2 when the deposits arrive.) Workspace:
 * jfli_poisson_workspace_bytes. */
int jfli_poisson_force(void* stream, float* rho, float rho_mean, int clear_rho, float scale, float* pot, float* force,
                       void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                       size_t errlen);
/* Fused particle pass: [kick, or with CORRECT a position shift, by kick * the CIC readout
 * of `force` (jfli_force_mesh layout) at the current position] -> [drift] -> [paint into
 * rho (accumulating)]. Positions are relative (displacements). */
int jfli_kick_drift_paint(void* stream, float* disp, float* vel, const float* force, float kick, float drift,
                          int flags, float weight, float* rho, int nx, int ny, int nz, int batch, char* err,
                          size_t errlen);
/* One PM step: clear rho, kick/drift/paint (flags KICK|DRIFT), then with FORCE solve the
 * Poisson equation for the new positions and write the new force meshes into `force`. */
size_t jfli_pm_step_workspace_bytes(int nx, int ny, int nz, int batch);
int jfli_pm_step(void* stream, float* disp, float* vel, float kick, float drift, int flags, float* rho, float* force,
                 void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                 size_t errlen);

/* One PM step over `batch` independent simulations of the same mesh size, each with its
 * own schedule: slot b is kicked by kicks[b], drifted by drifts[b] with slot_flags[b]
 * (JFLI_STEP_* bits; 0 leaves the slot untouched), painted, and gets new force meshes.
 * kicks, drifts, slot_flags are device arrays of length batch, so the launches can be
 * recorded once and replayed with new per-slot factors. Replaces a vmapped step() over a
 * batch of forward-model evaluations (probabilistic_models/forward_model.py:24-79). */
int jfli_pm_step_slots(void* stream, float* disp, float* vel, const float* kicks, const float* drifts,
                       const int* slot_flags, float* rho, float* force, void* workspace, size_t workspace_bytes, int nx,
                       int ny, int nz, int batch, char* err, size_t errlen);

/* out = irfft(rfft(noise) * sqrt(P(|k|) * M / V)), P by linear interpolation (with end
 * extrapolation) of the device tables ktab/ptab (h/Mpc, (Mpc/h)^3). zero_mode_one sets
 * P(k=0) to 1. Workspace: jfli_poisson_workspace_bytes. */
int jfli_ic_filter(void* stream, const float* noise, float* out, const float* ktab, const float* ptab, int ntab,
                   float lx, float ly, float lz, int zero_mode_one, void* workspace, size_t workspace_bytes, int nx,
                   int ny, int nz, int batch, char* err, size_t errlen);

/* LPT at the grid points: F1 = -grad_FD laplace^-1 ic, and for order 2 the same from the
 * second-order source; dx = c1x F1 + c2x F2, p = c1p (c1x F1) + c2p (c2x F2). */
size_t jfli_lpt_workspace_bytes(int nx, int ny, int nz, int batch);
int jfli_lpt(void* stream, const float* ic, int order, float c1x, float c2x, float c1p, float c2p, float* dx, float* p,
             void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen);
/* Light-cone-mode LPT (reference pm/lpt.py:110-130, the per-particle scale factors of
 * utils.py:234-244 compute_particle_scale_factors): each particle takes
 * a = a_of_chi(|x - observer|), x its Lagrangian grid point in Mpc/h ((i, j, k) L / N), and
 *   dx = D1(a) F1 + 3/7 D2(a) F2,   p = a^2 E(a) (f1(a) D1(a) F1 + f2(a) 3/7 D2(a) F2)
 * with F1, F2 the LPT forces at the grid points (as jfli_lpt). FP64 arithmetic from
 * `tables` (device, FP64): [chi | a(chi)] of n_chi points, chi ascending, then
 * [a | D1 | f1 | D2 | f2] of n_g points (linear interpolation with end extrapolation, D1
 * clipped to [0, 1]); `background` (host, 5 doubles): Omega_m, Omega_k, Omega_de, w0, wa
 * for E(a). a_out (optional, [batch][nx][ny][nz]) receives each particle's a.
 * Workspace: jfli_lpt_lightcone_workspace_bytes. */
size_t jfli_lpt_lightcone_workspace_bytes(int nx, int ny, int nz, int batch);
int jfli_lpt_lightcone(void* stream, const float* ic, int order, const double* tables, int n_chi, int n_g,
                       const double* background, float lx, float ly, float lz, float ox, float oy, float oz, float* dx,
                       float* p, float* a_out, void* workspace, size_t workspace_bytes, int nx, int ny, int nz,
                       int batch, char* err, size_t errlen);

/* P(k) sums over the full Fourier grid of `mesh` (ortho normalisation), binned with
 * numpy.digitize(|k|, kedges). out[batch][3][nedges+1] (FP64): sum |delta_k|^2, mode
 * count, sum |k|; bin 0 and bin nedges are the under/overflow bins. */
size_t jfli_power_spectrum_workspace_bytes(int nx, int ny, int nz, int batch, int nedges);
int jfli_power_spectrum(void* stream, const float* mesh, const float* kedges, int nedges, float lx, float ly,
                        float lz, double* out, void* workspace, size_t workspace_bytes, int nx, int ny, int nz,
                        int batch, char* err, size_t errlen);

/* Cross spectra and multipoles: FP64 sums over the full Fourier grid of `mesh` (and
 * `mesh2`, or mesh itself when NULL), ortho normalisation, binned by numpy.digitize(|k|,
 * kedges). For each multipole l = ells[e] (host array, nell <= 8, l <= 16):
 *   out[batch][2e][bin], out[batch][2e+1][bin] = sums of Re, Im of (2l + 1) L_l(mu) F1 conj(F2)
 * with mu = (k . los) / |k| (0 at k = 0); then out[batch][2 nell] = mode count and
 * out[batch][2 nell + 1] = sum of |k|. nedges <= 512. The caller forms |sum| (cross) or the
 * real sum (auto), divides by the count, drops bins 0 and nedges and multiplies by
 * prod(L/N). Workspace: jfli_power_poles_workspace_bytes (cross = mesh2 != NULL). */
size_t jfli_power_poles_workspace_bytes(int nx, int ny, int nz, int batch, int nedges, int nell, int cross);
int jfli_power_poles(void* stream, const float* mesh, const float* mesh2, const float* kedges, int nedges, float lx,
                     float ly, float lz, float losx, float losy, float losz, const int* ells, int nell, double* out,
                     void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                     size_t errlen);

/* HEALPix RING-ordered shell map of the particles with rmin < |x - observer| <= rmax
 * (Mpc/h), deposited by `scheme` (JFLI_HEALPIX_NGP or JFLI_HEALPIX_BILINEAR).
 * map[batch][12 nside^2]; accumulate = 0 clears it first. Raw weight sums. */
int jfli_healpix_paint(void* stream, const float* disp, int absolute, const float* weights, float weight, float lx,
                       float ly, float lz, float ox, float oy, float oz, float rmin, float rmax, int nside, int scheme,
                       float* map, int accumulate, int nx, int ny, int nz, int batch, char* err, size_t errlen);
/* Several shells of one particle set (batch 1) in one pass over the particles: shell s
 * keeps rmin[s] < |x - observer| <= rmax[s] and receives weight * scale[s] per particle
 * (weights[p] * weight * scale[s] with per-particle weights) into maps[s][12 nside^2];
 * shells may overlap. rmin, rmax, scale: host arrays of nshells. scheme 0 (ngp), 1
 * (bilinear) or 2 (rbf_neighbor, with sigma as jfli_healpix_paint_rbf). accumulate = 0
 * clears the nshells maps first. The same maps as one jfli_healpix_paint per shell, with
 * the particle set read once instead of nshells times. */
int jfli_healpix_paint_shells(void* stream, const float* disp, int absolute, const float* weights, float weight,
                              float lx, float ly, float lz, float ox, float oy, float oz, int nshells,
                              const double* rmin, const double* rmax, const float* scale, int nside, int scheme,
                              float sigma, float* maps, int accumulate, int nx, int ny, int nz, int batch, char* err,
                              size_t errlen);
/* Adjoint of jfli_healpix_paint_shells (ngp or bilinear), the shell painter's `_bwd`: with
 * maps_bar[s][12 nside^2] the cotangent of shell s's map, adds to disp_bar (particle grid
 * layout) each particle's weight_p scale_s sum_q maps_bar[s][pix_q] d w_q / d disp (zero
 * for ngp), and, when weights_bar is not NULL, weight scale_s sum_q maps_bar[s][pix_q] w_q
 * to weights_bar. Shell membership (a step in the distance) contributes nothing. The other
 * arguments as jfli_healpix_paint_shells; batch 1. */
int jfli_healpix_paint_shells_adjoint(void* stream, const float* disp, int absolute, const float* weights,
                                      float weight, float lx, float ly, float lz, float ox, float oy, float oz,
                                      int nshells, const double* rmin, const double* rmax, const float* scale,
                                      int nside, int scheme, const float* maps_bar, float* disp_bar,
                                      float* weights_bar, int nx, int ny, int nz, int batch, char* err,
                                      size_t errlen);
/* HEALPix shell painting with the "rbf_neighbor" scheme (reference
 * _src/fields/_painting.py:18,291; its arithmetic lives in the absent jaxpm fork, so this
 * is the library's own definition): each particle in rmin < r <= rmax deposits onto the 4
 * pixels around its direction (those of the bilinear scheme), weighted by
 * exp(-d^2 / (2 sigma^2)) of the angle d to each pixel centre and normalised to sum 1;
 * sigma in radians, 0 < sigma < pi. Otherwise as jfli_healpix_paint. */
int jfli_healpix_paint_rbf(void* stream, const float* disp, int absolute, const float* weights, float weight,
                           float lx, float ly, float lz, float ox, float oy, float oz, float rmin, float rmax, int nside,
                           float sigma, float* map, int accumulate, int nx, int ny, int nz, int batch, char* err,
                           size_t errlen);

/* HEALPix shell map of `ntiles` (<= 27) replicas of the particles, in one pass. For
 * replica i, with c = x - observer (x in Mpc/h from the grid index and disp):
 *   q = R_i c + s_i      R_i = rotations[9i..9i+8] (host, row-major; signed permutation
 *                        matrices only), s_i = shifts[3i..3i+2] (host, Mpc/h)
 * Without vel, q + observer is painted. With vel (the momenta) each replica is drifted to
 * its light-cone crossing with the rotated momentum R_i v, as jfli_lightcone_drift does:
 *   telephoto = 0: x' = q + observer, a_t from |x' - observer|, x' += D R_i v
 *   telephoto = 1: a_t from |q - observer|, q += D R_i v, x' = q + observer
 * D = (interp(a_t; ga, g) - gp_t) / interp(sqrt(t a_t); da, dgfa). dbound must bound |D|
 * over the distance table; replicas farther than dbound |v| from the shell are skipped.
 * Painting as jfli_healpix_paint (rmin < r <= rmax, scheme, weights * weight). */
int jfli_healpix_paint_tiled(void* stream, const float* disp, int absolute, const float* vel, const float* weights,
                             float weight, float lx, float ly, float lz, float ox, float oy, float oz, int ntiles,
                             const signed char* rotations, const float* shifts, int telephoto, float rmin, float rmax,
                             float t, float gp_t, float dbound, const float* chi, const float* a_chi, int n_chi,
                             const float* ga, const float* g, int n_g, const float* da, const float* dgfa, int n_d,
                             int nside, int scheme, float* map, int accumulate, int nx, int ny, int nz, int batch,
                             char* err, size_t errlen);
/* Adjoint of jfli_healpix_paint_tiled (its `_bwd`; ngp or bilinear): for the cotangent
 * map_bar[batch][12 nside^2] of the shell, each painted copy q' = q + D(r) M v (q = M c + s,
 * r = |q| or, telephoto, |q - o|) passes back the painter's g = dL/dq' (as
 * jfli_healpix_paint_shells_adjoint) as dL/dc += M^T (g + D'(r) (M v . g) dr/dq) and
 * dL/dv += D M^T g, D' the derivative of the interpolated drift tables (zero where the
 * growth is clipped). Adds to disp_bar (particle grid layout), vel_bar (with vel) and
 * weights_bar (when not NULL). The other arguments as jfli_healpix_paint_tiled. */
int jfli_healpix_paint_tiled_adjoint(void* stream, const float* disp, int absolute, const float* vel,
                                     const float* weights, float weight, float lx, float ly, float lz, float ox,
                                     float oy, float oz, int ntiles, const signed char* rotations, const float* shifts,
                                     int telephoto, float rmin, float rmax, float t, float gp_t, float dbound,
                                     const float* chi, const float* a_chi, int n_chi, const float* ga, const float* g,
                                     int n_g, const float* da, const float* dgfa, int n_d, int nside, int scheme,
                                     const float* map_bar, float* disp_bar, float* vel_bar, float* weights_bar,
                                     int nx, int ny, int nz, int batch, char* err, size_t errlen);

/* Positions (Mpc/h, particle layout) of one replica of the particles: rotation (host,
 * row-major signed permutation matrix) and shift (host, Mpc/h) applied to x - observer, and
 * with vel the light-cone drift, exactly as one replica of jfli_healpix_paint_tiled (same
 * telephoto convention). Feeds the flat-sky painter for TelephotoInterp planes beyond the box. */
int jfli_replica_positions(void* stream, const float* disp, int absolute, const float* vel, float lx, float ly,
                           float lz, float ox, float oy, float oz, const signed char* rotation, const float* shift,
                           int telephoto, float t, float gp_t, const float* chi, const float* a_chi, int n_chi,
                           const float* ga, const float* g, int n_g, const float* da, const float* dgfa, int n_d,
                           float* out, int nx, int ny, int nz, int batch, char* err, size_t errlen);

/* Flat-sky plane of the particles with zlo < z <= zhi (absolute grid units along z, from
 * the box origin): x and y scaled to the map (npx / nx, npy / ny), wrapped, deposited with
 * 2D CIC weights on map[batch][npx][npy]; weights * weight per particle (raw sums: divide by
 * the pixel volume for DENSITY units). accumulate = 0 clears the map first. */
int jfli_paint_flat(void* stream, const float* disp, int absolute, const float* weights, float weight, float zlo,
                    float zhi, int npx, int npy, float* map, int accumulate, int nx, int ny, int nz, int batch,
                    char* err, size_t errlen);
/* Adjoint of jfli_paint_flat with a scalar weight (the VJP of paint_2d; reference
 * _src/fields/_painting.py:117-202): pos_bar[p] += the gradient in the particle's x and y
 * (grid units) of <map_bar, plane>, the slab edges in z passing none. map_bar has the
 * planes' shape (batch, npx, npy); pos_bar the particles'. */
int jfli_paint_flat_adjoint(void* stream, const float* disp, int absolute, float weight, float zlo, float zhi, int npx,
                            int npy, const float* map_bar, float* pos_bar, int nx, int ny, int nz, int batch, char* err,
                            size_t errlen);

/* Flat-sky angular power sums of maps [batch][npx][npy] (auto, or cross with map2):
 * Re(F1 conj F2) of the full 2D FFT grid binned by ell = |2 pi fftfreq(n, d)| with
 * numpy.digitize on ell_edges (FP32 ascending, nedges <= 1024); dnx = npx * d_x and
 * dny = npy * d_y (radians). out[batch][3][nedges+1] (FP64): sum of power, mode count, sum
 * of ell; bins 0 and nedges are the under/overflow bins. The normalisation
 * (d_x d_y) / (npx npy) is the caller's. Workspace: jfli_flat_cl_workspace_bytes. */
size_t jfli_flat_cl_workspace_bytes(int npx, int npy, int batch, int nedges, int cross);
int jfli_flat_cl(void* stream, const float* map1, const float* map2, int npx, int npy, int batch, float dnx,
                 float dny, const float* ell_edges, int nedges, double* out, void* workspace, size_t workspace_bytes,
                 char* err, size_t errlen);

/* Positions (Mpc/h) of the particles drifted to their light-cone crossing:
 *   x = (grid index + disp) / N * L;  a_t = interp(|x - observer|; chi, a_chi);
 *   x += v * (interp(a_t; ga, g) - gp_t) / interp(sqrt(t a_t); da, dgfa)
 * with jax_cosmo's linear interpolation (end extrapolation) on ascending tables;
 * gp_t = Gp(t). out has the particle layout. */
int jfli_lightcone_drift(void* stream, const float* disp, const float* vel, float* out, float lx, float ly, float lz,
                         float ox, float oy, float oz, float t, float gp_t, const float* chi, const float* a_chi,
                         int n_chi, const float* ga, const float* g, int n_g, const float* da, const float* dgfa,
                         int n_d, int nx, int ny, int nz, int batch, char* err, size_t errlen);

/* Born convergence of nplanes HEALPix shell maps [nplanes][npix]:
 *   out[k][pix] = sum_p weights[k][p] (maps[p][pix] / mean_p - 1),  k < nsrc,
 * mean_p the pixel mean of map p (FP64 sum; 0 -> FP32 eps). The weights carry the lensing
 * efficiency, the plane factor and any n(z) quadrature. nplanes <= 256, nsrc <= 32.
 * Workspace: jfli_born_workspace_bytes. */
size_t jfli_born_workspace_bytes(int nplanes, long long npix);
int jfli_born(void* stream, const float* maps, int nplanes, long long npix, const float* weights, int nsrc,
              float* out, void* workspace, size_t workspace_bytes, char* err, size_t errlen);
/* Adjoint of jfli_born (its `_bwd`): maps_bar[p][pix] = u_p / mean_p - sum_pix' u_p m_p /
 * (mean_p^2 npix) with u_p = sum_k weights[k][p] kappa_bar[k][pix], the maps' cotangent
 * from the convergence maps' (the second term is the share through each plane's mean).
 * Workspace: jfli_born_adjoint_workspace_bytes. */
size_t jfli_born_adjoint_workspace_bytes(int nplanes, long long npix);
int jfli_born_adjoint(void* stream, const float* maps, int nplanes, long long npix, const float* weights, int nsrc,
                      const float* kappa_bar, float* maps_bar, void* workspace, size_t workspace_bytes, char* err,
                      size_t errlen);

/* Born convergence of nplanes flat-sky planes [nplanes][n0][n1]: out[k][i0][i1] =
 * sum_p weights[k][p] (v_p / mean_p - 1), v_p the periodic bilinear sample of plane p at
 * axis-0 coordinate i1 s0[p] - 0.5 and axis-1 coordinate i0 s1[p] - 0.5 (s0, s1 device
 * arrays: pixel angle x chi_p / pixel size). Workspace: jfli_born_workspace_bytes. */
int jfli_born_flat(void* stream, const float* maps, int nplanes, int n0, int n1, const float* weights, int nsrc,
                   const float* s0, const float* s1, float* out, void* workspace, size_t workspace_bytes, char* err,
                   size_t errlen);

/* Legendre stages of the spherical harmonic transform of a HEALPix RING map (FP64).
 * F and G are [nrings][lmax + 1] complex (interleaved doubles): per ring r the Fourier
 * coefficients of the ring along phi for m = 0..lmax, with the ring's e^{-i m phi_0}
 * applied; z[r] = cos theta_r. alm is packed by m, a[m][l - m] at offset
 * m (lmax + 1) - m (m - 1) / 2, (lmax + 1)(lmax + 2) / 2 complex values.
 *   jfli_sht_map2alm: alm = weight * sum_r lambda_lm(theta_r) F[r][m]  (alm cleared first)
 *   jfli_sht_alm2map: G[r][m] = sum_l alm[l][m] lambda_lm(theta_r)
 * lambda_lm: orthonormal associated Legendre functions with the Condon-Shortley phase.
 * lmax <= 8191, nrings <= 65535. */
/* Ring transforms along phi of a RING-ordered map [12 nside^2] (FP64), rings north to south
 * (4 nside - 1 of them), phi_j = phi_0 + 2 pi j / n_r:
 *   jfli_sht_ring_analysis:  F[r][m] = sum_j map_j e^{-i m phi_j},  m = 0..lmax
 *   jfli_sht_ring_synthesis: map_j = Re G[r][0] + 2 sum_{m=1..lmax} Re(G[r][m] e^{i m phi_j})
 * Direct FP64 sums (phases exact every 64 terms). nside <= 4096, lmax <= 8191. */
int jfli_sht_ring_analysis(void* stream, const double* map, int nside, int lmax, double* F, char* err,
                           size_t errlen);
int jfli_sht_ring_synthesis(void* stream, const double* G, int nside, int lmax, double* map, char* err,
                            size_t errlen);

int jfli_sht_map2alm(void* stream, const double* F, const double* z, int nrings, int lmax, double weight,
                     double* alm, char* err, size_t errlen);
int jfli_sht_alm2map(void* stream, const double* alm, const double* z, int nrings, int lmax, double* G, char* err,
                     size_t errlen);
/* Variant of the x pass of the Poisson, PGD and initial-condition filter chains (the
 * forward x FFT, k-space operator and inverse x FFT in one read and write of the half
 * spectrum): 0 (default) loads each pencil tile from global memory into registers; 1
 * stages the tile in shared memory with a TMA bulk tensor load and writes it back with a
 * bulk tensor store (meshes whose x-plane stride is a multiple of 16 bytes; others keep
 * mode 0). Both give the same spectrum to FP32 rounding. Process-wide. */
int jfli_set_fft_x_pass(int mode, char* err, size_t errlen);
/* Set n floats to zero (the library's own kernel: 16-byte stores where aligned). A step
 * loop clears its density mesh with it, or with JFLI_STEP_CLEAR, right before the paint. */
int jfli_zero(void* stream, float* data, long long n, char* err, size_t errlen);
/* Status word of the library's bounded device waits: bit 0 is set when a kernel's wait on
 * an mbarrier ran out of its bound (the kernel then left its output untouched). Read
 * synchronously; reset != 0 clears it. */
int jfli_device_status(unsigned* status, int reset, char* err, size_t errlen);

/* Angular power spectrum of packed a_lm (healpy alm2cl, reference
 * _src/power/_compute.py:175-191 via anafast): cl[l] = (Re a_l0 b_l0* + 2 sum_{m=1..l}
 * Re a_lm b_lm*) / (2l + 1), l = 0..lmax; alm2 NULL gives the auto spectrum of alm1.
 * FP64, summed in increasing m. */
int jfli_sht_alm2cl(void* stream, const double* alm1, const double* alm2, int lmax, double* cl, char* err,
                    size_t errlen);

/* ---- adjoints ------------------------------------------------------------------
 * Reverse sweep of one reversible KKD step  v' = v + kick F(x);  x' = x + drift v'
 * (F the CIC readout of the three force meshes), after the caller has un-drifted the
 * positions (x = x' - drift v') and rebuilt the force meshes at x:
 *   jfli_adjoint_unkick_paint: per particle u = lam_v + drift lam_x; v = v' - kick F(x);
 *     lam_v = u; ubar_a = CIC paint of u_a (three meshes [batch][3][nx][ny][nz], cleared
 *     first); partials[batch][nctas][2] = per-CTA sums of <u, F> (dL/dkick) and
 *     <lam_x, v'> (dL/ddrift), nctas = jfli_adjoint_partials_count / (2 batch).
 *   jfli_poisson_divergence: out = scale * P(sum_a D_a (alpha u_a + beta w_a)), P the
 *     Poisson operator -1/k^2 (k = 0 -> 0), D_a the 4-point finite difference; u and w
 *     are three meshes (aos = 0) or particle grids (aos = 1); w may be NULL. With
 *     u = ubar it gives the density cotangent rho_bar of the force readout.
 *   jfli_adjoint_position: lam_x += scale * grad_x R_x[rho_bar + sum_a u_a force_a] at
 *     the relative positions disp (R the CIC readout; rho_bar or u/force may be NULL).
 *     With scale = kick, u = lam_v it completes the step VJP; with force = NULL it is
 *     the adjoint of the CIC paint. */
size_t jfli_adjoint_partials_count(int nx, int ny, int nz, int batch);
int jfli_adjoint_unkick_paint(void* stream, const float* disp, float* vel, const float* lam_x, float* lam_v,
                              const float* force, float kick, float drift, float* ubar, double* partials,
                              size_t partials_count, int nx, int ny, int nz, int batch, char* err, size_t errlen);
size_t jfli_poisson_divergence_workspace_bytes(int nx, int ny, int nz, int batch);
int jfli_poisson_divergence(void* stream, const float* u, float alpha, const float* w, float beta, int aos, float scale,
                            float* out, void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch,
                            char* err, size_t errlen);
int jfli_adjoint_position(void* stream, const float* disp, const float* u, const float* rho_bar, const float* force,
                          float scale, float* lam_x, int nx, int ny, int nz, int batch, char* err, size_t errlen);

/* The reversible KKD loop and its reverse sweep as single calls, for callers that would
 * otherwise issue several launches per step (the gradient of a forward model):
 *   jfli_kkd_run: from positions disp and momenta vel, paint, solve and take the steps
 *     v += kicks[i] F(x); x += drifts[i] v for i < nsteps (F from the current positions);
 *     rho receives the CIC density of the final positions.
 *   jfli_kkd_adjoint: the reverse sweep from the final state (disp, vel) with cotangents
 *     (lam_x, lam_v), all updated in place to the initial state and its cotangents;
 *     sens[i][2] (device, FP64) = (dL/dkicks[i], dL/ddrifts[i]).
 * kicks and drifts are host arrays of nsteps floats. Workspace: jfli_kkd_workspace_bytes
 * (the same buffer serves both). */
size_t jfli_kkd_workspace_bytes(int nx, int ny, int nz, int batch);
int jfli_kkd_run(void* stream, float* disp, float* vel, const float* kicks, const float* drifts, int nsteps,
                 float* rho, void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                 size_t errlen);
int jfli_kkd_adjoint(void* stream, float* disp, float* vel, float* lam_x, float* lam_v, const float* kicks,
                     const float* drifts, int nsteps, double* sens, void* workspace, size_t workspace_bytes, int nx,
                     int ny, int nz, int batch, char* err, size_t errlen);

/* The same pair trading memory for work: jfli_kkd_run_stored writes the potential whose
 * force kicks step i to pots[i] (device, nsteps x batch x nx ny nz floats, [step][batch]
 * [cells]); jfli_kkd_adjoint_stored then rebuilds each step's force mesh from pots[i]
 * instead of un-drifting, painting and solving for it, and un-drifts the positions inside
 * the cotangent paint. The forward results are those of jfli_kkd_run; the reverse sweep
 * uses the forward pass's own forces (the recomputing sweep uses forces at the
 * reconstructed positions, equal up to FP32 rounding). Same workspace. */
int jfli_kkd_run_stored(void* stream, float* disp, float* vel, const float* kicks, const float* drifts, int nsteps,
                        float* rho, float* pots, void* workspace, size_t workspace_bytes, int nx, int ny, int nz,
                        int batch, char* err, size_t errlen);
int jfli_kkd_adjoint_stored(void* stream, float* disp, float* vel, float* lam_x, float* lam_v, const float* kicks,
                            const float* drifts, int nsteps, const float* pots, double* sens, void* workspace,
                            size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen);

/* The pair with SharpeningKernel (pm/correction.py:214-333 in pm/solvers.py:258-411): the
 * force of step i is jfli_sharpen_potential's combined force with (kicks[i], boosts[i]),
 * host arrays, boosts[i] = alpha / drift factor of step i, applied with factor 1; the reverse
 * sweep un-drifts, takes the boost and the kick off together and solves the adjoint with the
 * same (symmetric) combined operator. pots may be null (recompute) or as the stored pair.
 * sens[i][b][0] is then dL/d(the combined force's factor), not dL/dk. Same workspace. */
int jfli_kkd_run_sharpened(void* stream, float* disp, float* vel, const float* kicks, const float* drifts,
                           const float* boosts, float kl, float ks, int nsteps, float* rho, float* pots, void* workspace,
                           size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen);
int jfli_kkd_adjoint_sharpened(void* stream, float* disp, float* vel, float* lam_x, float* lam_v, const float* kicks,
                               const float* drifts, const float* boosts, float kl, float ks, int nsteps,
                               const float* pots, double* sens, void* workspace, size_t workspace_bytes, int nx,
                               int ny, int nz, int batch, char* err, size_t errlen);

/* dL/dmesh of P(k): out = irfft(rfft(mesh) * weights[digitize(|k|, kedges)] / M), with
 * weights[b] = 2 (dL/dP_b) prod(L/N) / count_b for the kept bins and 0 for bin 0 and
 * bin nedges. Workspace: jfli_poisson_workspace_bytes. */
int jfli_power_spectrum_adjoint(void* stream, const float* mesh, const float* kedges, const float* weights,
                                int nedges, float lx, float ly, float lz, float* out, void* workspace,
                                size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err, size_t errlen);
/* The same for Legendre multipoles of an auto spectrum (the VJP of jfli_power_poles
 * without mesh2; reference _src/power/_compute.py:68-119 with multipoles): out =
 * irfft(rfft(mesh) * w(k) / M), w(k) the mean over the mode and its conjugate partner of
 * sum_e weights[e][bin] (2 l_e + 1) L_l_e(mu), mu = (k . los) / |k| with los = (losx, losy,
 * losz) normalised (the partner's frequencies negated except on Nyquist planes), weights
 * nell x (nedges + 1) (2 dL/dP_e,b prod(L/N) / count_b, 0 outside the kept bins). ells:
 * nell <= 8 values in [0, 16]. For the cross spectrum |S_e,b| of meshes 1 and 2 (mesh2),
 * complex_weights = 1 and weights holds the real then the imaginary parts of c_e,b = u_e,b
 * dL/dP_e,b prod(L/N) / count_b, u = S / |S|: called on mesh 2 with c it gives dL/dmesh1,
 * on mesh 1 with conj(c) dL/dmesh2; the multiplier is then the Hermitian part of c w(k).
 * nedges + (1 + complex_weights) nell (nedges + 1) <= 4097. Workspace:
 * jfli_poisson_workspace_bytes. */
int jfli_power_poles_adjoint(void* stream, const float* mesh, const float* kedges, const float* weights, int nedges,
                             const int* ells, int nell, int complex_weights, float lx, float ly, float lz, float losx,
                             float losy, float losz, float* out, void* workspace, size_t workspace_bytes, int nx,
                             int ny, int nz, int batch, char* err, size_t errlen);

/* dL/d ic of jfli_lpt given dL/ddx (lam_x) and dL/dp (lam_v). Workspace:
 * jfli_lpt_adjoint_workspace_bytes. */
size_t jfli_lpt_adjoint_workspace_bytes(int nx, int ny, int nz, int batch);
int jfli_lpt_adjoint(void* stream, const float* ic, int order, float c1x, float c2x, float c1p, float c2p,
                     const float* lam_x, const float* lam_v, float* out, void* workspace, size_t workspace_bytes,
                     int nx, int ny, int nz, int batch, char* err, size_t errlen);

/* Tangent of jfli_ic_filter along a change dptab of the P(k) table:
 * out = irfft(rfft(noise) * interp(dptab) M/V / (2 sqrt(P M/V))), 0 where P <= 0.
 * Workspace: jfli_poisson_workspace_bytes. */
int jfli_ic_filter_tangent(void* stream, const float* noise, float* out, const float* ktab, const float* ptab,
                           const float* dptab, int ntab, float lx, float ly, float lz, int zero_mode_one,
                           void* workspace, size_t workspace_bytes, int nx, int ny, int nz, int batch, char* err,
                           size_t errlen);

/* P(k) that allocates nothing. This entry point has no counterpart in the reference.
 *
 * Some callers cannot allocate device memory when they need P(k): a JAX/XLA custom-call
 * handler runs in a process where XLA has already reserved most of the GPU memory for its
 * own pool, so a cudaMalloc from inside the handler can fail or break XLA's accounting,
 * and the handler has no workspace of its own unless XLA hands it one. This variant takes the same inputs and writes the same out[batch][3][nedges+1]
 * sums as jfli_power_spectrum, but needs no workspace: its scratch (the half spectrum and
 * the histogram partials) is an 11 MiB array compiled into the library, which every GPU
 * that loads the library holds until the process exits. That bounds the mesh: up to
 * 128^3 cells (with up to 128 bin edges); larger requests return JFLI_EUNSUPPORTED.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress;
 * again after the device's context has been re-created), so make that first call before
 * any stream capture. Every call overwrites the array, so
 * two calls that run on the GPU at the same time (other streams, other host threads)
 * corrupt each other's results; serialise them. */
int jfli_power_spectrum_noalloc(void* stream, const float* mesh, const float* kedges, int nedges, float lx, float ly,
                                float lz, double* out, int nx, int ny, int nz, int batch, char* err, size_t errlen);

#ifdef __cplusplus
}
#endif

#endif /* JFLI_B200_H */
