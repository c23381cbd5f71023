// Cross spectra and Legendre multipoles of P(k) (reference _src/power/_compute.py:68-119,
// _power with mesh2 and/or multipoles != 0).
//
// The reference bins the full complex grid: w_l = (2l + 1) L_l(mu) with mu = (k . los) / |k|
// (0 at k = 0), and sums Re and Im of w_l F1 conj(F2) per bin (|F|^2 for an auto spectrum).
// Here the meshes go through this library's r2c (the half spectrum, [nx][ny][nz/2 + 1]) and
// every element with 0 < kz < nz/2 also adds its conjugate partner (-k; for real meshes
// F(-k) = conj F(k)) with the partner's own wavevector, so the sums are those of the full
// grid, odd multipoles and imaginary parts included. |k| and the bin are formed as the
// monopole kernel forms them (kspace_ops.cuh PkOp); mu with the reference's float32 order
// (x, y, z products summed, then divided by |k|); L_l by the reference's recurrence in FP32.
// Per-CTA FP64 sums: [2 nell + 2][nedges + 1] = for each l (Re, Im), then mode count, sum |k|.
#include "common.cuh"
#include "internal.h"
#include "kspace_ops.cuh"

namespace jfli {

constexpr int kPolesThreads = 256;
constexpr int kMaxPoles = 8;

struct PolesArgs {
  int nx, ny, nz, nedges, nell;
  float cx, cy, cz, lx, ly, lz, norm;
  int ells[kMaxPoles];
};

// adds mode (ix, iy, iz) with the value c = F1 conj F2 (norm applied) to the CTA's sums
__device__ __forceinline__ void add_mode(const PolesArgs& a, int ix, int iy, int iz, double cre, double cim,
                                         const float* edges, double* sums) {
  const int nb = a.nedges + 1;
  const float ax = __fmul_rn(a.cx, (float)signed_freq(ix, a.nx));
  const float ay = __fmul_rn(a.cy, (float)signed_freq(iy, a.ny));
  const float az = __fmul_rn(a.cz, (float)signed_freq(iz, a.nz));
  const float kmag = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ax, ax), __fmul_rn(ay, ay)), __fmul_rn(az, az)));
  int lo = 0, hi = a.nedges;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (edges[mid] <= kmag)
      lo = mid + 1;
    else
      hi = mid;
  }
  const float dot = __fadd_rn(__fadd_rn(__fmul_rn(ax, a.lx), __fmul_rn(ay, a.ly)), __fmul_rn(az, a.lz));
  const float mu = kmag == 0.f ? 0.f : __fdiv_rn(dot, kmag);
  for (int e = 0; e < a.nell; ++e) {
    const int ell = a.ells[e];
    const double w = (double)__fmul_rn((float)(2 * ell + 1), legendre_f32(ell, mu));
    atomicAdd(&sums[(2 * e) * nb + lo], w * cre);
    atomicAdd(&sums[(2 * e + 1) * nb + lo], w * cim);
  }
  atomicAdd(&sums[(2 * a.nell) * nb + lo], 1.0);
  atomicAdd(&sums[(2 * a.nell + 1) * nb + lo], (double)kmag);
}

__global__ void __launch_bounds__(kPolesThreads) k_power_poles(const float2* __restrict__ spec1,
                                                               const float2* __restrict__ spec2, PolesArgs a,
                                                               const float* __restrict__ kedges,
                                                               double* __restrict__ partials) {
  extern __shared__ double sums[];  // [2 nell + 2][nb], then the edges as float
  const int nb = a.nedges + 1;
  const int nq = 2 * a.nell + 2;
  float* edges = reinterpret_cast<float*>(sums + nq * nb);
  for (int i = threadIdx.x; i < nq * nb; i += blockDim.x) sums[i] = 0.0;
  for (int i = threadIdx.x; i < a.nedges; i += blockDim.x) edges[i] = kedges[i];
  __syncthreads();
  const int hz = a.nz / 2 + 1;
  const long long nel = (long long)a.nx * a.ny * hz;
  const long long b = blockIdx.y;
  spec1 += b * nel;
  spec2 += b * nel;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(e % hz);
    const long long r = e / hz;
    const int iy = (int)(r % a.ny), ix = (int)(r / a.ny);
    const float2 f = spec1[e], g = spec2[e];
    // F1 conj(F2) * norm
    const double cre = ((double)f.x * g.x + (double)f.y * g.y) * (double)a.norm;
    const double cim = ((double)f.y * g.x - (double)f.x * g.y) * (double)a.norm;
    add_mode(a, ix, iy, iz, cre, cim, edges, sums);
    if (iz > 0 && 2 * iz < a.nz)  // the partner -k lies in the other half: conj(F1 conj F2)
      add_mode(a, (a.nx - ix) % a.nx, (a.ny - iy) % a.ny, a.nz - iz, cre, -cim, edges, sums);
  }
  __syncthreads();
  double* out = partials + (b * gridDim.x + blockIdx.x) * (long long)nq * nb;
  for (int i = threadIdx.x; i < nq * nb; i += blockDim.x) out[i] = sums[i];
}

int power_poles_ctas(const MeshDims& d) {
  const long long nel = d.spec_elems();
  long long c = (nel + kPolesThreads - 1) / kPolesThreads;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long cap = (long long)nsm * 2;
  return (int)(c < cap ? (c < 1 ? 1 : c) : cap);
}

cudaError_t power_poles(const float* mesh1, const float* mesh2, const MeshDims& d, const float* kedges, int nedges,
                        const float* box, const float* los, const int* ells, int nell, float2* spec1, float2* spec2,
                        double* partials, double* out, cudaStream_t s) {
  cudaError_t e = rfft3d_forward(mesh1, spec1, d, 0.0f, s);
  if (e == cudaSuccess && mesh2) e = rfft3d_forward(mesh2, spec2, d, 0.0f, s);
  if (e != cudaSuccess) return e;
  PolesArgs a;
  a.nx = d.nx;
  a.ny = d.ny;
  a.nz = d.nz;
  a.nedges = nedges;
  a.nell = nell;
  a.cx = (float)(2.0 * M_PI / (double)box[0]);
  a.cy = (float)(2.0 * M_PI / (double)box[1]);
  a.cz = (float)(2.0 * M_PI / (double)box[2]);
  a.lx = los[0];
  a.ly = los[1];
  a.lz = los[2];
  a.norm = 1.0f / ((float)d.nx * (float)d.ny * (float)d.nz);
  for (int i = 0; i < kMaxPoles; ++i) a.ells[i] = i < nell ? ells[i] : 0;
  const int ctas = power_poles_ctas(d);
  const int nq = 2 * nell + 2;
  const size_t smem = sizeof(double) * nq * (nedges + 1) + sizeof(float) * nedges;
  e = cudaFuncSetAttribute(k_power_poles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_power_poles<<<dim3(ctas, d.batch), kPolesThreads, smem, s>>>(spec1, mesh2 ? spec2 : spec1, a, kedges, partials);
  note_launch();
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return sums_finalize(partials, ctas, nq * (nedges + 1), out, d.batch, s);
}

}  // namespace jfli
