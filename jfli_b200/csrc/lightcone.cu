// Drift of every particle to its light-cone crossing (reference pm/interp.py:110-121,
// used by DriftInterp.paint, pm/interp.py:254-318):
//   x  = position in Mpc/h ((grid index + displacement) / N * L, PositionUnit.MPC_H)
//   r  = |x - observer|,  a_t = a_of_chi(r),  a_c = sqrt(t a_t)
//   x += v * (Gp(a_t) - Gp(t)) / dGfa(a_c)
// with v the momentum array as stored (the reference adds it to the Mpc/h positions
// unconverted). a_of_chi and Gp interpolate the host's FP64 tables (chi -> a on the
// 256-point distance table, D1 on the 128-point growth table) with jax_cosmo's linear
// interpolation and end extrapolation; dGfa is read from a dense table of the host's FP64
// dGfa. Output: drifted positions in Mpc/h, same layout as the input.
#include "cic.cuh"
#include "common.cuh"
#include "internal.h"
#include "kspace_ops.cuh"

namespace jfli {

__global__ void k_lightcone_drift(const float* __restrict__ disp, const float* __restrict__ vel,
                                  float* __restrict__ out, float lx, float ly, float lz, float ox, float oy,
                                  float oz, float t, float gp_t, DriftTables tb, PGrid g) {
  const long long b = blockIdx.y;
  disp += b * g.np * 3;
  vel += b * g.np * 3;
  out += b * g.np * 3;
  const float nx = (float)g.nx, ny = (float)g.ny, nz = (float)g.nz;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int i, j, k;
    particle_ijk(g, p, i, j, k);
    const float x = ((float)i + disp[3 * p + 0]) / nx * lx;
    const float y = ((float)j + disp[3 * p + 1]) / ny * ly;
    const float z = ((float)k + disp[3 * p + 2]) / nz * lz;
    const float dx = x - ox, dy = y - oy, dz = z - oz;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz);
    const float at = interp_table(r, tb.chi, tb.a_chi, tb.n_chi);
    const float ac = sqrtf(t * at);
    const float gp_at = fminf(fmaxf(interp_table(at, tb.ga, tb.g, tb.n_g), 0.f), 1.f);  // Gp is clipped to [0, 1]
    const float drift = (gp_at - gp_t) / interp_table(ac, tb.da, tb.dgfa, tb.n_d);
    out[3 * p + 0] = x + drift * vel[3 * p + 0];
    out[3 * p + 1] = y + drift * vel[3 * p + 1];
    out[3 * p + 2] = z + drift * vel[3 * p + 2];
  }
}

cudaError_t lightcone_drift(const float* disp, const float* vel, float* out, const float* box, const float* observer,
                            float t, float gp_t, const float* chi, const float* a_chi, int n_chi, const float* ga,
                            const float* gtab, int n_g, const float* da, const float* dgfa, int n_d, const MeshDims& d,
                            cudaStream_t s) {
  const DriftTables tb{chi, a_chi, n_chi, ga, gtab, n_g, da, dgfa, n_d};
  k_lightcone_drift<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(
      disp, vel, out, box[0], box[1], box[2], observer[0], observer[1], observer[2], t, gp_t, tb, make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// Light-cone-mode LPT (reference pm/lpt.py:110-130 with utils.py:234-244): every particle
// takes the scale factor of its own light-cone crossing, a = a_of_chi(|x - observer|) with
// x its Lagrangian grid point in Mpc/h, and the LPT growth coefficients at that a:
//   dx = D1(a) F1 + 3/7 D2(a) F2,  p = a^2 E(a) (f1(a) D1(a) F1 + f2(a) 3/7 D2(a) F2)
// (jaxpm lpt with an array of scale factors). F1, F2 are the first- and second-order LPT
// forces at the grid points. All of it in FP64 from the host's FP64 tables, interpolated
// as the host functions do (a_of_chi on the 256-point distance table; D1 clipped to
// [0, 1], f1, D2, f2 on the 128-point growth table; E(a) in closed form).
__device__ __forceinline__ double interp_table_f64(double x, const double* xp, const double* fp, int n) {
  int lo = 0, hi = n;  // first index with xp[i] >= x (searchsorted, side="left")
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (xp[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  int i = lo - 1;
  i = i < 0 ? 0 : (i > n - 2 ? n - 2 : i);
  return fp[i] + (x - xp[i]) * ((fp[i + 1] - fp[i]) / (xp[i + 1] - xp[i]));
}

__global__ void k_lpt_combine_lightcone(const float* __restrict__ f1, const float* __restrict__ f2,
                                        float* __restrict__ dx, float* __restrict__ pv, float* __restrict__ a_out,
                                        LptLightcone lc, PGrid g) {
  const long long b = blockIdx.y;
  f1 += b * g.np * 3;
  if (f2) f2 += b * g.np * 3;
  dx += b * g.np * 3;
  pv += b * g.np * 3;
  if (a_out) a_out += b * g.np;
  const int nc = lc.n_chi, ng = lc.n_g;
  const double* chi = lc.tables;
  const double* a_chi = chi + nc;
  const double* ga = a_chi + nc;
  const double* gg = ga + ng;
  const double* gf = gg + ng;
  const double* g2 = gf + ng;
  const double* f2t = g2 + ng;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int i, j, k;
    particle_ijk(g, p, i, j, k);
    const double x = (double)i / g.nx * lc.box[0] - lc.obs[0];
    const double y = (double)j / g.ny * lc.box[1] - lc.obs[1];
    const double z = (double)k / g.nz * lc.box[2] - lc.obs[2];
    const double r = sqrt(x * x + y * y + z * z);
    const double a = interp_table_f64(r, chi, a_chi, nc);
    const double d1 = fmin(fmax(interp_table_f64(a, ga, gg, ng), 0.0), 1.0);
    const double rate1 = interp_table_f64(a, ga, gf, ng);
    const double d2 = interp_table_f64(a, ga, g2, ng);
    const double rate2 = interp_table_f64(a, ga, f2t, ng);
    double de;
    if (lc.wa == 0.0)
      de = lc.ode * pow(a, -3.0 * (1.0 + lc.w0));
    else
      de = lc.ode * pow(a, -3.0 * (1.0 + lc.w0 + lc.wa) + 3.0 * lc.wa * (a - 1.0) / log(a));
    const double e = sqrt(lc.om / (a * a * a) + lc.ok / (a * a) + de);
    const double c1x = d1, c2x = 3.0 / 7.0 * d2, c1p = a * a * rate1 * e, c2p = a * a * rate2 * e;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double u = f1[3ull * p + c];
      double xv = c1x * u;
      double vv = c1p * xv;
      if (f2) {
        const double x2 = c2x * (double)f2[3ull * p + c];
        xv += x2;
        vv += c2p * x2;
      }
      dx[3ull * p + c] = (float)xv;
      pv[3ull * p + c] = (float)vv;
    }
    if (a_out) a_out[p] = (float)a;
  }
}

cudaError_t lpt_combine_lightcone(const float* f1, const float* f2, float* dx, float* p, float* a_out,
                                  const LptLightcone& lc, const MeshDims& d, cudaStream_t s) {
  k_lpt_combine_lightcone<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(f1, f2, dx, p, a_out, lc,
                                                                                          make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

}  // namespace jfli
