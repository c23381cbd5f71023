// Register-resident FFT building blocks for the specialised transform lengths.
//
// A length-N transform is split N = P * Q. Stage 1: P "lanes" per transform each hold Q
// elements x[t + P m] (m < Q) in registers, run a Q-point DFT, multiply by
// w_N^(t kb) and write the result to shared memory. Stage 2: Q lanes per transform each
// read the P values Y[kb][t] (t < P), run a P-point DFT and hold X[kb + Q ka] (ka < P).
// Small DFTs of composite size are themselves split (R = A * B) with their twiddles
// taken from the same table of w_N^m, so every twiddle is a table read.
#pragma once

#include "common.cuh"

namespace jfli {

template <int SIGN>
__device__ __forceinline__ float2 twid(const float2* __restrict__ tw, int m) {
  float2 w = tw[m];
  if (SIGN > 0) w.y = -w.y;
  return w;
}

// In-place DFT of size R on v[0..R), natural-order output. TS = N / R: stride into the
// w_N table that gives w_R.
template <int R, int SIGN, int TS>
struct RegDFT;

template <int SIGN, int TS>
struct RegDFT<1, SIGN, TS> {
  static __device__ __forceinline__ void run(float2*, const float2*) {}
};

template <int SIGN, int TS>
struct RegDFT<2, SIGN, TS> {
  static __device__ __forceinline__ void run(float2* v, const float2*) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int SIGN, int TS>
struct RegDFT<3, SIGN, TS> {
  static __device__ __forceinline__ void run(float2* v, const float2*) {
    const float h = 0.86602540378443864676f;  // sqrt(3)/2
    const float2 s = cadd(v[1], v[2]);
    const float2 d = csub(v[1], v[2]);
    const float2 t = make_float2(v[0].x - 0.5f * s.x, v[0].y - 0.5f * s.y);
    const float2 r = mul_si<SIGN>(cscale(d, h));
    v[0] = cadd(v[0], s);
    v[1] = cadd(t, r);
    v[2] = csub(t, r);
  }
};

template <int SIGN, int TS>
struct RegDFT<4, SIGN, TS> {
  static __device__ __forceinline__ void run(float2* v, const float2*) {
    const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const float2 a2 = cadd(v[1], v[3]), a3 = mul_si<SIGN>(csub(v[1], v[3]));
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3);
    v[3] = csub(a1, a3);
  }
};

template <int SIGN, int TS>
struct RegDFT<8, SIGN, TS> {
  static __device__ __forceinline__ void run(float2* v, const float2* tw) {
    const float r2 = 0.70710678118654752440f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    RegDFT<4, SIGN, TS>::run(e, tw);
    RegDFT<4, SIGN, TS>::run(o, tw);
    o[1] = make_float2(r2 * (o[1].x - SIGN * o[1].y), r2 * (o[1].y + SIGN * o[1].x));
    o[2] = mul_si<SIGN>(o[2]);
    o[3] = make_float2(r2 * (-o[3].x - SIGN * o[3].y), r2 * (-o[3].y + SIGN * o[3].x));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = cadd(e[k], o[k]);
      v[k + 4] = csub(e[k], o[k]);
    }
  }
};

// R = A * B: x[a + A b] -> X[kb + B ka].
template <int A, int B, int SIGN, int TS>
__device__ __forceinline__ void rdft_ab(float2* v, const float2* tw) {
  float2 y[A * B];
#pragma unroll
  for (int a = 0; a < A; ++a) {
    float2 u[B];
#pragma unroll
    for (int b = 0; b < B; ++b) u[b] = v[a + A * b];
    RegDFT<B, SIGN, TS * A>::run(u, tw);
#pragma unroll
    for (int kb = 0; kb < B; ++kb) y[a * B + kb] = (a * kb == 0) ? u[kb] : cmul(u[kb], twid<SIGN>(tw, a * kb * TS));
  }
#pragma unroll
  for (int kb = 0; kb < B; ++kb) {
    float2 u[A];
#pragma unroll
    for (int a = 0; a < A; ++a) u[a] = y[a * B + kb];
    RegDFT<A, SIGN, TS * B>::run(u, tw);
#pragma unroll
    for (int ka = 0; ka < A; ++ka) v[kb + B * ka] = u[ka];
  }
}

template <int SIGN, int TS>
struct RegDFT<6, SIGN, TS> {
  static __device__ __forceinline__ void run(float2* v, const float2* tw) { rdft_ab<2, 3, SIGN, TS>(v, tw); }
};
template <int SIGN, int TS>
struct RegDFT<12, SIGN, TS> {
  static __device__ __forceinline__ void run(float2* v, const float2* tw) { rdft_ab<4, 3, SIGN, TS>(v, tw); }
};
template <int SIGN, int TS>
struct RegDFT<16, SIGN, TS> {
  static __device__ __forceinline__ void run(float2* v, const float2* tw) { rdft_ab<4, 4, SIGN, TS>(v, tw); }
};
template <int SIGN, int TS>
struct RegDFT<24, SIGN, TS> {
  static __device__ __forceinline__ void run(float2* v, const float2* tw) { rdft_ab<8, 3, SIGN, TS>(v, tw); }
};
template <int SIGN, int TS>
struct RegDFT<32, SIGN, TS> {
  static __device__ __forceinline__ void run(float2* v, const float2* tw) { rdft_ab<8, 4, SIGN, TS>(v, tw); }
};

// Split of each specialised length into P x Q (P lanes of Q elements in stage 1).
template <int N>
struct Split;
#define JFLI_SPLIT(N_, P_, Q_)        \
  template <>                         \
  struct Split<N_> {                  \
    static constexpr int P = P_;      \
    static constexpr int Q = Q_;      \
  };
JFLI_SPLIT(8, 4, 2)
JFLI_SPLIT(12, 4, 3)
JFLI_SPLIT(16, 4, 4)
JFLI_SPLIT(24, 8, 3)
JFLI_SPLIT(32, 8, 4)
JFLI_SPLIT(48, 8, 6)
JFLI_SPLIT(64, 8, 8)
JFLI_SPLIT(96, 12, 8)
JFLI_SPLIT(128, 16, 8)
JFLI_SPLIT(192, 16, 12)
JFLI_SPLIT(256, 16, 16)
JFLI_SPLIT(384, 24, 16)
JFLI_SPLIT(512, 32, 16)
JFLI_SPLIT(768, 32, 24)
JFLI_SPLIT(1024, 32, 32)
#undef JFLI_SPLIT

// Columns per CTA of a strided column pass of length N.
template <int N>
struct ColCfg {
  static constexpr int W = N <= 128 ? 32 : (N <= 512 ? 16 : 8);
  static constexpr int T = W * Split<N>::Q;  // threads: one stage-2 item each
};

constexpr int pow2_floor_c(int v) { return v < 2 ? 1 : 2 * pow2_floor_c(v / 2); }

// Rows per CTA of a contiguous (z) pass whose complex length is N.
template <int N>
struct RowCfg {
  static constexpr int Q = Split<N>::Q;
  static constexpr int R0 = 4096 / N;
  static constexpr int RT = 512 / Q;
  static constexpr int R = pow2_floor_c(R0 < RT ? R0 : RT);
  static constexpr int T = R * Q;
};

}  // namespace jfli
