// Born convergence of spherical shell maps (reference _src/lensing/_born.py:29-130):
//   delta_p(pix) = map_p(pix) / mean_p - 1                     (mean 0 -> FP32 eps)
//   kappa_k(pix) = sum_p W[k][p] delta_p(pix)
// W folds the lensing efficiency clip(1 - r_p / chi_s, 0, 1000), the plane factor
// 3/2 Omega_m (H0/c)^2 dr r_p / a_p and, for n(z) sources, the Simpson weights of the
// source integral (computed on the host in FP64). The per-plane means are FP64 sums over
// the pixels, per-CTA partials reduced in a fixed order.
#include "cic.cuh"
#include "common.cuh"
#include "internal.h"

namespace jfli {

constexpr int kBornThreads = 256;

__global__ void __launch_bounds__(kBornThreads) k_plane_partials(const float* __restrict__ maps, long long npix,
                                                                double* __restrict__ partials) {
  const long long p = blockIdx.y;
  const float* m = maps + p * npix;
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (long long)gridDim.x * blockDim.x)
    acc += (double)m[i];
  __shared__ double sh[kBornThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kBornThreads / 32; ++w) s += sh[w];
    partials[p * gridDim.x + blockIdx.x] = s;
  }
}

// One thread per plane: mean = (sum of the partials in CTA order) / npix.
__global__ void k_plane_means(const double* __restrict__ partials, int nctas, int nplanes, long long npix,
                              float* __restrict__ mean) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nplanes) return;
  double s = 0.0;
  for (int c = 0; c < nctas; ++c) s += partials[(long long)p * nctas + c];
  const float m = (float)(s / (double)npix);
  mean[p] = (m == 0.f) ? 1.1920929e-07f : m;  // FP32 eps, as the reference's safe mean
}

__global__ void k_born_combine(const float* __restrict__ maps, int nplanes, long long npix,
                               const float* __restrict__ mean, const float* __restrict__ w, int nsrc,
                               float* __restrict__ out) {
  extern __shared__ float sm[];  // mean[nplanes], w[nsrc][nplanes]
  for (int i = threadIdx.x; i < nplanes; i += blockDim.x) sm[i] = mean[i];
  for (int i = threadIdx.x; i < nsrc * nplanes; i += blockDim.x) sm[nplanes + i] = w[i];
  __syncthreads();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (long long)gridDim.x * blockDim.x) {
    float acc[8];
    for (int k0 = 0; k0 < nsrc; k0 += 8) {
      const int kn = (nsrc - k0) < 8 ? (nsrc - k0) : 8;
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[k] = 0.f;
      for (int p = 0; p < nplanes; ++p) {
        const float d = maps[(long long)p * npix + i] / sm[p] - 1.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (k < kn) acc[k] += sm[nplanes + (k0 + k) * nplanes + p] * d;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (k < kn) out[(long long)(k0 + k) * npix + i] = acc[k];
    }
  }
}

// Adjoint of k_born_combine, the maps' cotangent from kappa's (kbar):
//   u_p = sum_k W[k][p] kbar_k,   mbar_p = u_p / mean_p - c_p,
//   c_p = sum_pix u_p m_p / (mean_p^2 npix)   (the share through the plane's mean).
// First pass, one CTA row per plane: mbar_p = u_p / mean_p and per-CTA FP64 partials of
// sum u_p m_p.
__global__ void __launch_bounds__(kBornThreads) k_born_adj_u(const float* __restrict__ maps, long long npix,
                                                            const float* __restrict__ mean,
                                                            const float* __restrict__ w, int nsrc, int nplanes,
                                                            const float* __restrict__ kbar,
                                                            float* __restrict__ maps_bar,
                                                            double* __restrict__ dots) {
  const int p = blockIdx.y;
  const float* m = maps + p * npix;
  float* mb = maps_bar + p * npix;
  const float inv_mean = 1.0f / mean[p];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (long long)gridDim.x * blockDim.x) {
    float u = 0.f;
    for (int k = 0; k < nsrc; ++k) u += __ldg(w + k * nplanes + p) * kbar[k * npix + i];
    mb[i] = u * inv_mean;
    acc += (double)u * (double)m[i];
  }
  __shared__ double sh[kBornThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < kBornThreads / 32; ++i) s += sh[i];
    dots[p * gridDim.x + blockIdx.x] = s;
  }
}

// One thread per plane: c_p from the partials in CTA order.
__global__ void k_born_adj_c(const double* __restrict__ dots, int nctas, int nplanes, long long npix,
                             const float* __restrict__ mean, float* __restrict__ c) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nplanes) return;
  double s = 0.0;
  for (int i = 0; i < nctas; ++i) s += dots[(long long)p * nctas + i];
  const double mu = (double)mean[p];
  c[p] = (float)(s / (mu * mu * (double)npix));
}

__global__ void k_born_adj_sub(float* __restrict__ maps_bar, long long npix, const float* __restrict__ c) {
  const int p = blockIdx.y;
  const float cp = c[p];
  float* mb = maps_bar + p * npix;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (long long)gridDim.x * blockDim.x)
    mb[i] -= cp;
}

cudaError_t born_convergence_adjoint(const float* maps, int nplanes, long long npix, const float* weights, int nsrc,
                                     const float* kappa_bar, float* maps_bar, double* partials, float* mean,
                                     float* c, cudaStream_t s) {
  const int nctas = born_ctas(npix);
  k_plane_partials<<<dim3(nctas, nplanes), kBornThreads, 0, s>>>(maps, npix, partials);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_plane_means<<<(nplanes + 127) / 128, 128, 0, s>>>(partials, nctas, nplanes, npix, mean);
  note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_born_adj_u<<<dim3(nctas, nplanes), kBornThreads, 0, s>>>(maps, npix, mean, weights, nsrc, nplanes, kappa_bar,
                                                            maps_bar, partials);
  note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_born_adj_c<<<(nplanes + 127) / 128, 128, 0, s>>>(partials, nctas, nplanes, npix, mean, c);
  note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_born_adj_sub<<<dim3(nctas, nplanes), kBornThreads, 0, s>>>(maps_bar, npix, c);
  note_launch();
  return cudaGetLastError();
}

// Flat-sky planes (reference _src/lensing/_born.py:29-97 with coords, and _born_flat,
// 133-186): each output pixel (i0, i1) samples plane p by periodic bilinear interpolation
// (jax map_coordinates, order 1, mode "wrap") at axis-0 coordinate i1 s0_p - 0.5 and axis-1
// coordinate i0 s1_p - 0.5, where s0_p, s1_p (host) are the pixel angle times chi_p over the
// plane's pixel size, in the reference's pairing of grid axes; then delta = v / mean_p - 1
// and kappa_k = sum_p W[k][p] delta.
__global__ void k_born_flat(const float* __restrict__ maps, int nplanes, int n0, int n1,
                            const float* __restrict__ mean, const float* __restrict__ w, int nsrc,
                            const float* __restrict__ s0, const float* __restrict__ s1, float* __restrict__ out) {
  extern __shared__ float sm[];  // mean[nplanes], s0[nplanes], s1[nplanes], w[nsrc][nplanes]
  for (int i = threadIdx.x; i < nplanes; i += blockDim.x) {
    sm[i] = mean[i];
    sm[nplanes + i] = s0[i];
    sm[2 * nplanes + i] = s1[i];
  }
  for (int i = threadIdx.x; i < nsrc * nplanes; i += blockDim.x) sm[3 * nplanes + i] = w[i];
  __syncthreads();
  const long long npix = (long long)n0 * n1;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(q / n1), i1 = (int)(q - (long long)i0 * n1);
    float acc[8];
    for (int k0 = 0; k0 < nsrc; k0 += 8) {
      const int kn = (nsrc - k0) < 8 ? (nsrc - k0) : 8;
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[k] = 0.f;
      for (int p = 0; p < nplanes; ++p) {
        const float u = (float)i1 * sm[nplanes + p] - 0.5f;  // along axis 0 of the plane
        const float v = (float)i0 * sm[2 * nplanes + p] - 0.5f;  // along axis 1
        const float fu = floorf(u), fv = floorf(v);
        const float wu = u - fu, wv = v - fv;
        int a0 = (int)fu % n0, b0 = (int)fv % n1;
        if (a0 < 0) a0 += n0;
        if (b0 < 0) b0 += n1;
        const int a1 = a0 + 1 == n0 ? 0 : a0 + 1, b1 = b0 + 1 == n1 ? 0 : b0 + 1;
        const float* m = maps + (long long)p * npix;
        const float val = (1.f - wu) * ((1.f - wv) * m[(long long)a0 * n1 + b0] + wv * m[(long long)a0 * n1 + b1]) +
                          wu * ((1.f - wv) * m[(long long)a1 * n1 + b0] + wv * m[(long long)a1 * n1 + b1]);
        const float d = val / sm[p] - 1.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (k < kn) acc[k] += sm[3 * nplanes + (k0 + k) * nplanes + p] * d;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (k < kn) out[(long long)(k0 + k) * npix + q] = acc[k];
    }
  }
}

int born_ctas(long long npix) {
  long long b = (npix + kBornThreads - 1) / kBornThreads;
  const long long cap = (long long)sm_count() * 4;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

cudaError_t born_convergence(const float* maps, int nplanes, long long npix, const float* weights, int nsrc,
                             float* out, double* partials, float* mean, cudaStream_t s) {
  const int nctas = born_ctas(npix);
  k_plane_partials<<<dim3(nctas, nplanes), kBornThreads, 0, s>>>(maps, npix, partials);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_plane_means<<<(nplanes + 127) / 128, 128, 0, s>>>(partials, nctas, nplanes, npix, mean);
  note_launch();
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t smem = sizeof(float) * (size_t)nplanes * (1 + nsrc);
  k_born_combine<<<born_ctas(npix), kBornThreads, smem, s>>>(maps, nplanes, npix, mean, weights, nsrc, out);
  note_launch();
  return cudaGetLastError();
}

cudaError_t born_flat(const float* maps, int nplanes, int n0, int n1, const float* weights, int nsrc, const float* s0,
                      const float* s1, float* out, double* partials, float* mean, cudaStream_t s) {
  const long long npix = (long long)n0 * n1;
  const int nctas = born_ctas(npix);
  k_plane_partials<<<dim3(nctas, nplanes), kBornThreads, 0, s>>>(maps, npix, partials);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_plane_means<<<(nplanes + 127) / 128, 128, 0, s>>>(partials, nctas, nplanes, npix, mean);
  note_launch();
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t smem = sizeof(float) * (size_t)nplanes * (3 + nsrc);
  k_born_flat<<<born_ctas(npix), kBornThreads, smem, s>>>(maps, nplanes, n0, n1, mean, weights, nsrc, s0, s1, out);
  note_launch();
  return cudaGetLastError();
}

}  // namespace jfli
