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

}  // namespace jfli
