// Flat-sky painting and the flat-sky angular power spectrum.
//
// Painting (reference _src/fields/_painting.py:117-202, _single_paint_2d, with jaxpm's
// cic_paint_2d): particles in absolute grid coordinates; x and y are scaled to the map's
// pixels (npx / nx, npy / ny) and wrapped periodically; a particle belongs to the plane when
// zlo < z <= zhi (grid units along z, measured from the box origin as the reference does);
// it is deposited on the 4 surrounding pixels with weights (1 - |x - n_x|)(1 - |y - n_y|),
// n the floor of the position and floor + 1, wrapped. map[npx][npy].
//
// Flat C_ell (reference _src/power/_compute.py:122-172, _flat_cl): the 2D FFT of each map
// (this library's own r2c passes, run on a 1 x npx x npy mesh), Re(F1 conj F2) of every
// mode of the full grid binned by ell = |2 pi fftfreq| with numpy.digitize on the edges;
// the half spectrum stands for the full grid (modes with 0 < ky < npy / 2 count twice, as
// their conjugate partners carry the same power and |ell|). ell is formed in FP32 the way
// the reference's float32 grid is (k / (n d), times 2 pi, squares summed, square root),
// without fused multiply-adds, so that modes on a bin edge fall on the same side.
#include "cic.cuh"
#include "common.cuh"
#include "internal.h"

namespace jfli {

__global__ void k_paint_flat(const float* __restrict__ disp, int absolute, const float* __restrict__ weights,
                             float weight, PGrid g, float sx, float sy, float zlo, float zhi, int npx, int npy,
                             float* __restrict__ map) {
  const long long b = blockIdx.y;
  disp += b * g.np * 3;
  if (weights) weights += b * g.np;
  map += b * (long long)npx * npy;
  const float fnx = (float)npx, fny = (float)npy;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    float gx = disp[3 * p + 0], gy = disp[3 * p + 1], gz = disp[3 * p + 2];
    if (!absolute) {
      int i, j, k;
      particle_ijk(g, p, i, j, k);
      gx += (float)i;
      gy += (float)j;
      gz += (float)k;
    }
    if (!(gz > zlo && gz <= zhi)) continue;
    float x = __fmul_rn(gx, sx), y = __fmul_rn(gy, sy);
    x = fmodf(x, fnx);  // periodic wrap as jnp.mod does it: exact remainder, then + n when negative
    y = fmodf(y, fny);
    if (x < 0.f) x += fnx;
    if (y < 0.f) y += fny;
    const float fx0 = floorf(x), fy0 = floorf(y);
    const float wx[2] = {1.f - fabsf(x - fx0), 1.f - fabsf(x - (fx0 + 1.f))};
    const float wy[2] = {1.f - fabsf(y - fy0), 1.f - fabsf(y - (fy0 + 1.f))};
    int ix0 = (int)fx0 % npx, iy0 = (int)fy0 % npy;
    if (ix0 < 0) ix0 += npx;
    if (iy0 < 0) iy0 += npy;
    const int ix[2] = {ix0, ix0 + 1 == npx ? 0 : ix0 + 1};
    const int iy[2] = {iy0, iy0 + 1 == npy ? 0 : iy0 + 1};
    const float w = weights ? weights[p] * weight : weight;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int c = 0; c < 2; ++c) atomicAdd(map + (long long)ix[a] * npy + iy[c], wx[a] * wy[c] * w);
  }
}

cudaError_t paint_flat(const float* disp, int absolute, const float* weights, float weight, const MeshDims& d, int npx,
                       int npy, float zlo, float zhi, float* map, cudaStream_t s) {
  const float sx = (float)((double)npx / d.nx), sy = (float)((double)npy / d.ny);
  k_paint_flat<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(disp, absolute, weights, weight,
                                                                             make_pgrid(d), sx, sy, zlo, zhi, npx,
                                                                             npy, map);
  note_launch();
  return cudaGetLastError();
}

// Adjoint of k_paint_flat with a scalar weight: for the plane cotangent map_bar, each
// particle in the slab adds weight * sum over its 4 cells of map_bar times the gradient of
// the 2D CIC weights to its x and y (the scaling to the plane grid and the periodic wrap
// have derivative s_x, s_y and 1; the slab edges pass no gradient), placed as the forward
// places it.
__global__ void k_paint_flat_adjoint(const float* __restrict__ disp, int absolute, float weight, PGrid g, float sx,
                                     float sy, float zlo, float zhi, int npx, int npy,
                                     const float* __restrict__ map_bar, float* __restrict__ pos_bar) {
  const long long b = blockIdx.y;
  disp += b * g.np * 3;
  pos_bar += b * g.np * 3;
  map_bar += b * (long long)npx * npy;
  const float fnx = (float)npx, fny = (float)npy;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    float gx = disp[3 * p + 0], gy = disp[3 * p + 1], gz = disp[3 * p + 2];
    if (!absolute) {
      int i, j, k;
      particle_ijk(g, p, i, j, k);
      gx += (float)i;
      gy += (float)j;
      gz += (float)k;
    }
    if (!(gz > zlo && gz <= zhi)) continue;
    float x = __fmul_rn(gx, sx), y = __fmul_rn(gy, sy);
    x = fmodf(x, fnx);
    y = fmodf(y, fny);
    if (x < 0.f) x += fnx;
    if (y < 0.f) y += fny;
    const float fx0 = floorf(x), fy0 = floorf(y);
    const float wx[2] = {1.f - fabsf(x - fx0), 1.f - fabsf(x - (fx0 + 1.f))};
    const float wy[2] = {1.f - fabsf(y - fy0), 1.f - fabsf(y - (fy0 + 1.f))};
    const float dx[2] = {-1.f, 1.f}, dy[2] = {-1.f, 1.f};  // d w / d x of the two cells
    int ix0 = (int)fx0 % npx, iy0 = (int)fy0 % npy;
    if (ix0 < 0) ix0 += npx;
    if (iy0 < 0) iy0 += npy;
    const int ix[2] = {ix0, ix0 + 1 == npx ? 0 : ix0 + 1};
    const int iy[2] = {iy0, iy0 + 1 == npy ? 0 : iy0 + 1};
    float ax = 0.f, ay = 0.f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const float m = map_bar[(long long)ix[a] * npy + iy[c]];
        ax += m * dx[a] * wy[c];
        ay += m * wx[a] * dy[c];
      }
    pos_bar[3 * p + 0] += weight * sx * ax;
    pos_bar[3 * p + 1] += weight * sy * ay;
  }
}

cudaError_t paint_flat_adjoint(const float* disp, int absolute, float weight, const MeshDims& d, int npx, int npy,
                               float zlo, float zhi, const float* map_bar, float* pos_bar, cudaStream_t s) {
  const float sx = (float)((double)npx / d.nx), sy = (float)((double)npy / d.ny);
  k_paint_flat_adjoint<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(
      disp, absolute, weight, make_pgrid(d), sx, sy, zlo, zhi, npx, npy, map_bar, pos_bar);
  note_launch();
  return cudaGetLastError();
}

constexpr int kFlatThreads = 256;

__device__ __forceinline__ float ell_component(int i, int n, float dn) {
  const int k = i < (n + 1) / 2 ? i : i - n;  // numpy fftfreq order
  const float f = __fdiv_rn((float)k, dn);
  return __fmul_rn(6.2831854820251465f, f);  // float32(2 pi) * f
}

// Per-CTA sums over the modes of the half spectrum: [3][nb] = (sum Re(F1 conj F2), modes,
// sum ell), nb = nedges + 1 bins (0 and nedges the under/overflow bins).
__global__ void __launch_bounds__(kFlatThreads) k_flat_cl_partials(const float2* __restrict__ spec1,
                                                                   const float2* __restrict__ spec2, int n0, int n1,
                                                                   float dn0, float dn1, const float* __restrict__ edges,
                                                                   int nedges, double* __restrict__ partials) {
  extern __shared__ double sums[];  // [3][nb]
  const int nb = nedges + 1;
  const int hz = n1 / 2 + 1;
  const long long nmodes = (long long)n0 * hz;
  const long long b = blockIdx.y;
  spec1 += b * nmodes;
  spec2 += b * nmodes;
  for (int i = threadIdx.x; i < 3 * nb; i += blockDim.x) sums[i] = 0.0;
  __syncthreads();
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < nmodes;
       m += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(m / hz), i1 = (int)(m - (long long)i0 * hz);
    const float lx = ell_component(i0, n0, dn0), ly = ell_component(i1, n1, dn1);
    const float ell = sqrtf(__fadd_rn(__fmul_rn(lx, lx), __fmul_rn(ly, ly)));
    int lo = 0, hi = nedges;  // digitize: number of edges <= ell
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (edges[mid] <= ell)
        lo = mid + 1;
      else
        hi = mid;
    }
    const float2 a = spec1[m], c = spec2[m];
    const double pw = (double)a.x * (double)c.x + (double)a.y * (double)c.y;
    const double w = (i1 == 0 || (n1 % 2 == 0 && i1 == n1 / 2)) ? 1.0 : 2.0;
    atomicAdd(&sums[lo], w * pw);
    atomicAdd(&sums[nb + lo], w);
    atomicAdd(&sums[2 * nb + lo], w * (double)ell);
  }
  __syncthreads();
  double* out = partials + (b * gridDim.x + blockIdx.x) * 3 * nb;
  for (int i = threadIdx.x; i < 3 * nb; i += blockDim.x) out[i] = sums[i];
}

int flat_cl_ctas(int n0, int n1) {
  const long long nmodes = (long long)n0 * (n1 / 2 + 1);
  long long c = (nmodes + kFlatThreads - 1) / kFlatThreads;
  const long long cap = (long long)sm_count() * 4;
  return (int)(c < cap ? (c < 1 ? 1 : c) : cap);
}

cudaError_t flat_cl(const float* map1, const float* map2, int n0, int n1, int batch, float dn0, float dn1,
                    const float* edges, int nedges, float2* spec1, float2* spec2, double* partials, double* out,
                    cudaStream_t s) {
  const MeshDims d{1, n0, n1, batch};
  cudaError_t e = rfft2d_forward(map1, spec1, d, s);
  if (e == cudaSuccess && map2) e = rfft2d_forward(map2, spec2, d, s);
  if (e != cudaSuccess) return e;
  const int ctas = flat_cl_ctas(n0, n1);
  const size_t smem = sizeof(double) * 3 * (nedges + 1);
  k_flat_cl_partials<<<dim3(ctas, batch), kFlatThreads, smem, s>>>(spec1, map2 ? spec2 : spec1, n0, n1, dn0, dn1,
                                                                   edges, nedges, partials);
  note_launch();
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return power_finalize(partials, ctas, nedges + 1, out, batch, s);
}

}  // namespace jfli
