// Shared-memory Stockham FFT engine used by every FFT pass of the library.
//
// A CTA holds a tile of `ncol` (a power of two) independent transforms of length n
// in shared memory, element (e, c) at buf[e * P + c] (P >= ncol; P odd when the tile
// was filled with a transposing store). Each Stockham stage reads its radix-R
// butterfly inputs from one buffer and writes the autosorted outputs to the other, so
// a thread holds only one butterfly in registers. Threads are mapped column-fastest,
// which keeps every stage free of shared-memory bank conflicts for 8-byte elements.
//
// Twiddles: tw[m] = exp(-2*pi*i*m/n) for m in [0, n) (the forward table); inverse
// transforms conjugate on the fly. No normalisation is applied.
#pragma once

#include "common.cuh"

namespace jfli {

template <int R, int SIGN>
__device__ __forceinline__ void small_dft(float2* v);

template <>
__device__ __forceinline__ void small_dft<2, -1>(float2* v) {
  float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}
template <>
__device__ __forceinline__ void small_dft<2, 1>(float2* v) {
  small_dft<2, -1>(v);
}

template <int SIGN>
__device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3) {
  float2 a0 = cadd(v0, v2), a1 = csub(v0, v2);
  float2 a2 = cadd(v1, v3), a3 = mul_si<SIGN>(csub(v1, v3));
  v0 = cadd(a0, a2);
  v2 = csub(a0, a2);
  v1 = cadd(a1, a3);
  v3 = csub(a1, a3);
}

template <>
__device__ __forceinline__ void small_dft<4, -1>(float2* v) {
  dft4<-1>(v[0], v[1], v[2], v[3]);
}
template <>
__device__ __forceinline__ void small_dft<4, 1>(float2* v) {
  dft4<1>(v[0], v[1], v[2], v[3]);
}

template <int SIGN>
__device__ __forceinline__ void dft3(float2* v) {
  const float h = 0.86602540378443864676f;  // sqrt(3)/2
  float2 s = cadd(v[1], v[2]);
  float2 d = csub(v[1], v[2]);
  float2 t = make_float2(v[0].x - 0.5f * s.x, v[0].y - 0.5f * s.y);
  float2 r = mul_si<SIGN>(cscale(d, h));
  v[0] = cadd(v[0], s);
  v[1] = cadd(t, r);
  v[2] = csub(t, r);
}
template <>
__device__ __forceinline__ void small_dft<3, -1>(float2* v) {
  dft3<-1>(v);
}
template <>
__device__ __forceinline__ void small_dft<3, 1>(float2* v) {
  dft3<1>(v);
}

template <int SIGN>
__device__ __forceinline__ void dft8(float2* v) {
  const float r2 = 0.70710678118654752440f;
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<SIGN>(e0, e1, e2, e3);
  dft4<SIGN>(o0, o1, o2, o3);
  // o_k *= w8^k, w8 = exp(SIGN * i * pi / 4)
  o1 = make_float2(r2 * (o1.x - SIGN * o1.y), r2 * (o1.y + SIGN * o1.x));
  o2 = mul_si<SIGN>(o2);
  o3 = make_float2(r2 * (-o3.x - SIGN * o3.y), r2 * (-o3.y + SIGN * o3.x));
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}
template <>
__device__ __forceinline__ void small_dft<8, -1>(float2* v) {
  dft8<-1>(v);
}
template <>
__device__ __forceinline__ void small_dft<8, 1>(float2* v) {
  dft8<1>(v);
}

// One radix-R Stockham stage, src -> dst (ping-pong). Ns = product of radices so far.
template <int R, int SIGN>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ src, float2* __restrict__ dst, int P, int n,
                                          int ncol_log2, int Ns, const float2* tw) {
  const int nb = n / R;
  const int ncol = 1 << ncol_log2;
  const int total = nb << ncol_log2;
  const int twstep = n / (Ns * R);
  for (int w = threadIdx.x; w < total; w += blockDim.x) {
    const int j = w >> ncol_log2;
    const int c = w & (ncol - 1);
    const int k = j % Ns;
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = src[(j + t * nb) * P + c];
    if (Ns > 1) {
#pragma unroll
      for (int t = 1; t < R; ++t) {
        float2 wt = tw[k * t * twstep];
        if (SIGN > 0) wt.y = -wt.y;
        v[t] = cmul(v[t], wt);
      }
    }
    small_dft<R, SIGN>(v);
    const int base = ((j - k) * R + k) * P + c;
#pragma unroll
    for (int t = 0; t < R; ++t) dst[base + t * Ns * P] = v[t];
  }
  __syncthreads();
}

// Full transform of a tile held in `a` (loaded and synchronised on entry), using `b`
// as the second buffer. Returns the buffer that holds the result. ncol = 2^ncol_log2.
template <int SIGN>
__device__ __forceinline__ float2* tile_fft(float2* a, float2* b, int P, int ncol_log2, const FftPlan& pl,
                                            const float2* tw) {
  float2* src = a;
  float2* dst = b;
  int Ns = 1;
  for (int s = 0; s < pl.nst; ++s) {
    const int R = pl.radix[s];
    if (R == 8)
      fft_stage<8, SIGN>(src, dst, P, pl.n, ncol_log2, Ns, tw);
    else if (R == 4)
      fft_stage<4, SIGN>(src, dst, P, pl.n, ncol_log2, Ns, tw);
    else if (R == 2)
      fft_stage<2, SIGN>(src, dst, P, pl.n, ncol_log2, Ns, tw);
    else
      fft_stage<3, SIGN>(src, dst, P, pl.n, ncol_log2, Ns, tw);
    Ns *= R;
    float2* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

// tw[m] = exp(-2 pi i m / n), m in [0, n), computed in double then rounded.
__device__ __forceinline__ void fill_twiddles(float2* tw, int n) {
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)m / (double)n, &s, &c);
    tw[m] = make_float2((float)c, (float)-s);
  }
}

}  // namespace jfli
