// Shared device helpers for the jfli-b200 kernels (sm_100a).
//
// Layout conventions used by every kernel in this library:
//   * a mesh is float32 [nx][ny][nz], C order (z fastest), batch-major when batched;
//   * particles live on the Lagrangian grid of the same shape: particle (i,j,k) is
//     row (i*ny + j)*nz + k of an AoS float32 [.., 3] array (dx, dy, dz);
//   * a half spectrum (real-to-complex along z) is float2 [nx][ny][nz/2+1].
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace jfli {

constexpr int kFftThreads = 256;     // threads per FFT CTA
constexpr int kFftTileElems = 4096;  // complex elements held per FFT CTA (32 KB)
constexpr int kMaxRadixStages = 16;

// Factorisation of one FFT axis (n = 2^a 3^b) into radix-8/4/2/3 Stockham stages.
struct FftPlan {
  int n;
  int nst;
  int radix[kMaxRadixStages];
};

// A set of independent 1D transforms ("columns") over a half spectrum.
// Column c, element e lives at  (c / hz) * outer_stride + (c % hz) + e * stride.
struct ColGeom {
  int n;                  // transform length
  int ncols;              // number of columns
  int hz;                 // inner column count (nz/2+1)
  int w;                  // columns per CTA tile
  long long stride;       // element stride along the transform axis
  long long outer_stride; // stride of the outer column index
};

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by (sign * i)
template <int SIGN>
__device__ __forceinline__ float2 mul_si(float2 a) {
  return SIGN > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

__device__ __forceinline__ int wrap_index(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}

// Signed frequency index of bin i for an axis of length n (numpy fftfreq * n).
__device__ __forceinline__ int signed_freq(int i, int n) { return (i < (n + 1) / 2) ? i : i - n; }

// Division of 32-bit unsigned numerators by a fixed divisor d with a multiply-high and
// shifts (round-up magic number, Granlund & Montgomery 1994).
struct FastDiv {
  unsigned d, m, s;
  static FastDiv make(unsigned d) {
    FastDiv f;
    f.d = d;
    if (d <= 1) {
      f.m = 0;
      f.s = 0;
      return f;
    }
    unsigned l = 0;
    while ((1ull << l) < d) ++l;
    f.m = (unsigned)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
    f.s = l;
    return f;
  }
  __device__ __forceinline__ unsigned div(unsigned x) const {
    if (d <= 1) return x;
    const unsigned t = __umulhi(x, m);
    return (t + ((x - t) >> 1)) >> (s - 1);
  }
};

// Index of one periodic axis shifted by a small offset (|offset| <= n).
__device__ __forceinline__ int wrap1(int v, int n) {
  v += (v < 0) ? n : 0;
  v -= (v >= n) ? n : 0;
  return v;
}

}  // namespace jfli
