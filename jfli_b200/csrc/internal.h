// Internal C++ interface between the kernel files and the C-ABI layer (api.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace jfli {

// Counts kernel launches issued by this library (reported by jfli_launch_count).
void note_launch();

struct MeshDims {
  int nx, ny, nz, batch;
  __host__ __device__ long long cells() const { return (long long)nx * ny * nz; }
  __host__ __device__ int hz() const { return nz / 2 + 1; }
  __host__ __device__ long long spec_elems() const { return (long long)nx * ny * (nz / 2 + 1); }
};

// ---- fft.cu ----
bool fft_axis_supported(int n);
bool mesh_fft_supported(int nx, int ny, int nz);
int x_pass_ctas(const MeshDims& d);
cudaError_t rfft3d_forward(const float* in, float2* spec, const MeshDims& d, float sub, cudaStream_t s);
cudaError_t rfft3d_inverse(float2* spec, float* out, const MeshDims& d, float scale, cudaStream_t s);
cudaError_t rfft2d_forward(const float* in, float2* spec, const MeshDims& d, cudaStream_t s);  // d.nx == 1
// clear: the density mesh (rho itself), set to 0 by the r2c pass once read, so the next
// paint needs no memset; nullptr leaves rho as it is.
cudaError_t poisson_potential(const float* rho, float2* spec, float* pot, const MeshDims& d, float rho_mean,
                              float scale, cudaStream_t s, float* clear = nullptr);
cudaError_t pgd_potential(const float* rho, float2* spec, float* pot, const MeshDims& d, float rho_mean, float kl,
                          float ks, float scale, cudaStream_t s);
// pot_k = delta_k (-1/k^2) (c0 + c1 PGD filter) * scale: (0, 1) is pgd_potential, (kick, boost)
// the reversible step's kick plus the sharpening boost as one potential.
cudaError_t mixed_pgd_potential(const float* rho, float2* spec, float* pot, const MeshDims& d, float rho_mean,
                                float kl, float ks, float c0, float c1, float scale, cudaStream_t s);
// dptab != null: the tangent of the filter along a change dptab of the P(k) table.
cudaError_t ic_filter(const float* noise, float2* spec, float* out, const MeshDims& d, const float* ktab,
                      const float* ptab, int ntab, const float* box, int zero_mode_one, cudaStream_t s,
                      const float* dptab = nullptr);
cudaError_t power_adjoint(const float* mesh, float2* spec, float* out, const MeshDims& d, const float* kedges,
                          const float* weights, int nedges, const float* box, cudaStream_t s);
// The same for multipoles: weights nell x (nedges + 1) (with cplx, real then imaginary parts
// of a complex factor per bin), each mode weighted by sum_e weights[e][bin] (2l_e + 1)
// L_l_e(mu), mu along the unit vector los, averaged with its conjugate partner.
cudaError_t power_poles_adjoint(const float* mesh, float2* spec, float* out, const MeshDims& d, const float* kedges,
                                const float* weights, int nedges, const int* ells, int nell, const float* box,
                                const float* los, int cplx, cudaStream_t s);
cudaError_t power_partials(const float* mesh, float2* spec, double* partials, const MeshDims& d, const float* kedges,
                           int nedges, const float* box, float norm, cudaStream_t s);

// ---- cic.cu ----
// Particle update program flags for kick_drift_paint.
enum StepFlags {
  kStepKick = 1,   // v += F(x) * kick, F the CIC readout of the force meshes
  kStepDrift = 2,  // x += v * drift
  kStepPaint = 4,  // CIC deposit of weight `weight` at the (new) position into rho
  kStepCorrect = 16,  // x += F(x) * kick (position correction, PGD); exclusive with kStepKick
};
cudaError_t cic_paint(const float* pos, int absolute, const float* weights, float weight, float* mesh,
                      const MeshDims& d, cudaStream_t s);
cudaError_t cic_readout(const float* pos, int absolute, const float* mesh, float* out, const MeshDims& d,
                        cudaStream_t s);
cudaError_t cic_readout_gradient(const float* pos, int absolute, const float* pot, float* out, float scale,
                                 const MeshDims& d, cudaStream_t s);
cudaError_t kick_drift_paint(float* disp, float* vel, const float* force, float kick, float drift, int flags,
                             float weight, float* rho, const MeshDims& d, cudaStream_t s);
cudaError_t force_mesh(const float* pot, float* force, float scale, const MeshDims& d, cudaStream_t s);
cudaError_t kick_drift_paint_slots(float* disp, float* vel, const float* force, const float* kicks,
                                   const float* drifts, const int* slot_flags, float weight, float* rho,
                                   const MeshDims& d, cudaStream_t s);
cudaError_t grid_gradient(const float* pot, float* out, float scale, int accumulate, const MeshDims& d,
                          cudaStream_t s);
// 2LPT source from the first-order field F = -D phi1 (AoS, k_grid_gradient's layout)
cudaError_t lpt2_source(const float* grad, float* out, const MeshDims& d, cudaStream_t s);
cudaError_t lpt_combine(const float* f1, const float* f2, float c1x, float c2x, float c1p, float c2p, float* dx,
                        float* p, const MeshDims& d, cudaStream_t s);
cudaError_t axpy_particles(float* y, const float* x, float a, const MeshDims& d, cudaStream_t s);
// q: six scratch meshes; out (+)= dL/dphi1 for sbar = dL/d delta2.
cudaError_t lpt2_source_adjoint(const float* pot, const float* sbar, float* q, float* out, int accumulate,
                                const MeshDims& d, cudaStream_t s);

// ---- lightcone.cu ----
// tables of the light-cone drift (chi -> a, growth D1, dGfa), all ascending
struct DriftTables {
  const float* chi;  // comoving distance (Mpc/h)
  const float* a_chi;
  int n_chi;
  const float* ga;  // growth table scale factors
  const float* g;   // D1 at ga
  int n_g;
  const float* da;  // dense scale-factor grid
  const float* dgfa;
  int n_d;
};

// Light-cone-mode LPT: FP64 tables packed as [chi | a_chi] (n_chi each; chi ascending)
// then [ga | D1 | f1 | D2 | f2] (n_g each), and the background for E(a).
struct LptLightcone {
  const double* tables;
  int n_chi, n_g;
  double box[3], obs[3];
  double om, ok, ode, w0, wa;
};
cudaError_t lpt_combine_lightcone(const float* f1, const float* f2, float* dx, float* p, float* a_out,
                                  const LptLightcone& lc, const MeshDims& d, cudaStream_t s);

constexpr int kMaxTiles = 27;

cudaError_t lightcone_drift(const float* disp, const float* vel, float* out, const float* box, const float* observer,
                            float t, float gp_t, const float* chi, const float* a_chi, int n_chi, const float* ga,
                            const float* gtab, int n_g, const float* da, const float* dgfa, int n_d, const MeshDims& d,
                            cudaStream_t s);

// ---- born.cu ----
int born_ctas(long long npix);
cudaError_t born_convergence(const float* maps, int nplanes, long long npix, const float* weights, int nsrc,
                             float* out, double* partials, float* mean, cudaStream_t s);
// Adjoint of born_convergence: maps_bar[p][pix] from kappa_bar[k][pix] (partials: nplanes x
// born_ctas doubles; mean, c: nplanes floats of scratch).
cudaError_t born_convergence_adjoint(const float* maps, int nplanes, long long npix, const float* weights, int nsrc,
                                     const float* kappa_bar, float* maps_bar, double* partials, float* mean,
                                     float* c, cudaStream_t s);
cudaError_t born_flat(const float* maps, int nplanes, int n0, int n1, const float* weights, int nsrc, const float* s0,
                      const float* s1, float* out, double* partials, float* mean, cudaStream_t s);

// ---- sht.cu ----
cudaError_t sht_analysis(const double* F, const double* z, int nrings, int lmax, double weight, double* alm,
                         cudaStream_t s);
cudaError_t sht_synthesis(const double* alm, const double* z, int nrings, int lmax, double* G, cudaStream_t s);
cudaError_t sht_ring_analysis(const double* map, int nside, int lmax, double* F, cudaStream_t s);
cudaError_t sht_ring_synthesis(const double* G, int nside, int lmax, double* map, cudaStream_t s);
cudaError_t sht_alm2cl(const double* alm1, const double* alm2, int lmax, double* cl, cudaStream_t s);
cudaError_t zero_floats(float* y, long long n, cudaStream_t s);
// x pass of the Poisson / PGD / IC filter chains: 0 register pass, 1 TMA-staged pass
void set_x_pass_mode(int mode);
int x_pass_mode();
// status word of bounded device waits (bit 0: an mbarrier wait ran out); read, optionally cleared
cudaError_t device_status(unsigned* out, bool reset);

// ---- adjoint.cu ----
size_t adjoint_partials_count(const MeshDims& d);
// ubar: three meshes [batch][3][cells], or with vec4 one float4 mesh [batch][cells] (x, y, z, 0).
// undrift_disp (== disp, or null): un-drift the positions first (x = x' - drift v') and
// write them back.
cudaError_t adjoint_unkick_paint(const float* disp, float* vel, const float* lam_x, float* lam_v, const float* force,
                                 float kick, float drift, float* ubar, double* partials, const MeshDims& d,
                                 cudaStream_t s, bool vec4 = false, float* undrift_disp = nullptr);
cudaError_t sum_adjoint_partials(const double* partials, const MeshDims& d, double* out, cudaStream_t s);
cudaError_t divergence_fd(const float* u, float alpha, const float* w, float beta, int aos, int accumulate,
                          float* out, const MeshDims& d, cudaStream_t s);
// CIC paint of u (3 per particle) onto a float4 mesh (x, y, z, 0) cleared by the caller
cudaError_t paint_vec4(const float* disp, const float* u, float* ubar, const MeshDims& d, cudaStream_t s);
cudaError_t adjoint_position(const float* disp, const float* u, const float* rho_bar, const float* force, float scale,
                             float* lam_x, const MeshDims& d, cudaStream_t s);

// P(k) whose scratch is a file-scope device array (no allocation).
cudaError_t noalloc_scratch(void** out);
size_t noalloc_scratch_bytes();
int noalloc_pk_ctas(const MeshDims& d);
cudaError_t power_partials_noalloc(const float* mesh, float2* spec, double* partials, const MeshDims& d,
                                   const float* kedges, int nedges, const float* box, float norm, cudaStream_t s);

// ---- spectra.cu ----
cudaError_t power_finalize(const double* partials, int nctas, int nbins, double* out, int batch, cudaStream_t s);
cudaError_t sums_finalize(const double* partials, int nctas, int nvals, double* out, int batch, cudaStream_t s);
// ---- poles.cu ----
int power_poles_ctas(const MeshDims& d);
cudaError_t power_poles(const float* mesh1, const float* mesh2, const MeshDims& d, const float* kedges, int nedges,
                        const float* box, const float* los, const int* ells, int nell, float2* spec1, float2* spec2,
                        double* partials, double* out, cudaStream_t s);

// ---- healpix.cu ----
cudaError_t healpix_paint(const float* disp, int absolute, const float* weights, float weight, const MeshDims& d,
                          const float* box, const float* observer, float rmin, float rmax, int nside, int scheme,
                          float* map, cudaStream_t s, float sigma = 0.f);
// Up to kMaxShellsPerPass shells per launch (more are painted in further launches);
// shell s: rmin[s] < r <= rmax[s], weight * scale[s], into maps + s * 12 nside^2.
constexpr int kMaxShellsPerPass = 64;
// Adjoint of healpix_paint_shells (scheme 0 or 1): accumulates the position cotangent
// into disp_bar and, when non-null, the weight cotangent into weights_bar.
cudaError_t healpix_paint_shells_adjoint(const float* disp, int absolute, const float* weights, float weight,
                                         const MeshDims& d, const float* box, const float* observer, int nshells,
                                         const double* rmin, const double* rmax, const float* scale, int nside,
                                         int scheme, const float* maps_bar, float* disp_bar, float* weights_bar,
                                         cudaStream_t s);
cudaError_t healpix_paint_shells(const float* disp, int absolute, const float* weights, float weight,
                                 const MeshDims& d, const float* box, const float* observer, int nshells,
                                 const double* rmin, const double* rmax, const float* scale, int nside, int scheme,
                                 float* maps, cudaStream_t s, float sigma = 0.f);
cudaError_t replica_positions(const float* disp, int absolute, const float* vel, const MeshDims& d, const float* box,
                              const float* observer, const signed char* rotation, const float* shift, int telephoto,
                              float t, float gp_t, const DriftTables& tb, float* out, cudaStream_t s);
cudaError_t healpix_paint_tiled(const float* disp, int absolute, const float* vel, const float* weights, float weight,
                                const MeshDims& d, const float* box, const float* observer, int ntiles,
                                const signed char* rotations, const float* shifts, int telephoto, float rmin,
                                float rmax, float t, float gp_t, float dbound, const DriftTables& tb, int nside,
                                int scheme, float* map, cudaStream_t s);
// Adjoint of healpix_paint_tiled (one shell's map cotangent): accumulates into disp_bar and,
// when non-null, vel_bar and weights_bar.
cudaError_t healpix_paint_tiled_adjoint(const float* disp, int absolute, const float* vel, const float* weights,
                                        float weight, const MeshDims& d, const float* box, const float* observer,
                                        int ntiles, const signed char* rotations, const float* shifts, int telephoto,
                                        float rmin, float rmax, float t, float gp_t, float dbound,
                                        const DriftTables& tb, int nside, int scheme, const float* map_bar,
                                        float* disp_bar, float* vel_bar, float* weights_bar, cudaStream_t s);

// ---- flat.cu ----
cudaError_t paint_flat(const float* disp, int absolute, const float* weights, float weight, const MeshDims& d, int npx,
                       int npy, float zlo, float zhi, float* map, cudaStream_t s);
// Adjoint of paint_flat with a scalar weight: pos_bar[p] += d<map_bar, plane>/d(x, y) (in place).
cudaError_t paint_flat_adjoint(const float* disp, int absolute, float weight, const MeshDims& d, int npx, int npy,
                               float zlo, float zhi, const float* map_bar, float* pos_bar, cudaStream_t s);
int flat_cl_ctas(int n0, int n1);
cudaError_t flat_cl(const float* map1, const float* map2, int n0, int n1, int batch, float dn0, float dn1,
                    const float* edges, int nedges, float2* spec1, float2* spec2, double* partials, double* out,
                    cudaStream_t s);

}  // namespace jfli
