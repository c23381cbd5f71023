// 3D real FFT passes for sm_100a: r2c along z, complex column passes along y and x,
// and c2r along z. The x pass carries a k-space operator so that
//   forward x FFT -> operator -> inverse x FFT
// happens in one read and one write of the half spectrum (Poisson solve, initial
// condition filter), or so that the forward x FFT feeds the P(k) histogram without
// writing the spectrum back at all.
//
// Pass structure of a Poisson solve on an [nx][ny][nz] mesh (M = nx*ny*nz cells):
//   rfft_z   : read 4M B real,     write 8(M/2+...) B half spectrum
//   cols(y)  : read+write the half spectrum
//   x_op     : read+write the half spectrum (forward x, multiply, inverse x)
//   cols(y)^-1
//   irfft_z  : read the half spectrum, write 4M B real
#include <atomic>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"
#include "fft_engine.cuh"
#include "fft_reg.cuh"
#include "fft_tma.cuh"
#include "internal.h"
#include "kspace_ops.cuh"

namespace jfli {

static __device__ __forceinline__ int ilog2(int v) { return 31 - __clz(v); }

// ---------------------------------------------------------------------------------
// r2c along z: a CTA owns `rows` (a power of two) consecutive z-rows. Each row of nz
// reals is read as nh = nz/2 complex pairs (x[2j] + i x[2j+1]), transformed with an
// nh-point FFT and untangled into the nh+1 non-redundant outputs. `sub` is subtracted
// from every input (it only changes the k = 0 mode and keeps FP32 headroom for the
// fluctuations of a density of mean `sub`).
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(kFftThreads) k_rfft_z(const float* __restrict__ in, float2* __restrict__ out,
                                                        int nrows, int nz, int rows, FftPlan pl, float sub,
                                                        long long in_bstride, long long out_bstride) {
  extern __shared__ float2 sm[];
  const int nh = nz >> 1;
  const int hz = nh + 1;
  const int P = rows + 1;
  float2* bufa = sm;
  float2* bufb = bufa + (size_t)hz * P;
  float2* tw = bufb + (size_t)hz * P;
  float2* tw2 = tw + nh;
  in += (long long)blockIdx.y * in_bstride;
  out += (long long)blockIdx.y * out_bstride;
  const int row0 = blockIdx.x * rows;

  fill_twiddles(tw, nh);
  for (int m = threadIdx.x; m <= nh; m += blockDim.x) {
    double s, c;
    sincospi((double)m / (double)nh, &s, &c);
    tw2[m] = make_float2((float)c, (float)-s);  // exp(-2 pi i m / nz)
  }
  const float2* in2 = reinterpret_cast<const float2*>(in);
  const int E = rows * nh;
  for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
    const int r = idx / nh;
    const int j = idx - r * nh;
    const int row = row0 + r;
    float2 z = make_float2(0.f, 0.f);
    if (row < nrows) {
      z = in2[(long long)row * nh + j];
      z.x -= sub;
      z.y -= sub;
    }
    bufa[j * P + r] = z;
  }
  __syncthreads();
  const float2* res = tile_fft<-1>(bufa, bufb, P, ilog2(rows), pl, tw);
  const int E2 = rows * hz;
  for (int idx = threadIdx.x; idx < E2; idx += blockDim.x) {
    const int r = idx / hz;
    const int k = idx - r * hz;
    const int row = row0 + r;
    if (row >= nrows) continue;
    const float2 zk = res[(k == nh ? 0 : k) * P + r];
    const float2 zm = res[(k == 0 ? 0 : nh - k) * P + r];
    const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);  // zk - conj(zm)
    const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);   // d / (2i)
    out[(long long)row * hz + k] = cadd(e, cmul(tw2[k], o));
  }
}

// ---------------------------------------------------------------------------------
// c2r along z (unnormalised; callers fold 1/M into the k-space operator or pass
// `scale`). Reads nh+1 half-spectrum entries per row, re-tangles them into nh complex
// values, inverse-transforms and writes nz reals.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(kFftThreads) k_irfft_z(const float2* __restrict__ in, float* __restrict__ out,
                                                         int nrows, int nz, int rows, FftPlan pl, float scale,
                                                         long long in_bstride, long long out_bstride) {
  extern __shared__ float2 sm[];
  const int nh = nz >> 1;
  const int hz = nh + 1;
  const int P = rows + 1;
  float2* bufa = sm;
  float2* bufb = bufa + (size_t)hz * P;
  float2* tw = bufb + (size_t)hz * P;
  float2* tw2 = tw + nh;
  in += (long long)blockIdx.y * in_bstride;
  out += (long long)blockIdx.y * out_bstride;
  const int row0 = blockIdx.x * rows;

  fill_twiddles(tw, nh);
  for (int m = threadIdx.x; m <= nh; m += blockDim.x) {
    double s, c;
    sincospi((double)m / (double)nh, &s, &c);
    tw2[m] = make_float2((float)c, (float)s);  // exp(+2 pi i m / nz)
  }
  const int E2 = rows * hz;
  for (int idx = threadIdx.x; idx < E2; idx += blockDim.x) {
    const int r = idx / hz;
    const int k = idx - r * hz;
    const int row = row0 + r;
    bufb[k * P + r] = (row < nrows) ? in[(long long)row * hz + k] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  // Z[k] = (X[k] + conj X[nh-k]) + i (X[k] - conj X[nh-k]) exp(+2 pi i k / nz)
  const int E = rows * nh;
  for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
    const int k = idx / rows;
    const int r = idx - k * rows;
    const float2 xk = bufb[k * P + r];
    const float2 xm = bufb[(nh - k) * P + r];
    const float2 e = make_float2(xk.x + xm.x, xk.y - xm.y);
    const float2 d = cmul(make_float2(xk.x - xm.x, xk.y + xm.y), tw2[k]);
    bufa[k * P + r] = make_float2(e.x - d.y, e.y + d.x);
  }
  __syncthreads();
  const float2* res = tile_fft<1>(bufa, bufb, P, ilog2(rows), pl, tw);
  float2* out2 = reinterpret_cast<float2*>(out);
  for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
    const int r = idx / nh;
    const int j = idx - r * nh;
    const int row = row0 + r;
    if (row < nrows) out2[(long long)row * nh + j] = cscale(res[j * P + r], scale);
  }
}

// ---------------------------------------------------------------------------------
// Column pass (used for y, and for x without an operator).
// ---------------------------------------------------------------------------------
__device__ __forceinline__ long long col_addr(const ColGeom& g, int c, int e) {
  const int o = c / g.hz;
  return (long long)o * g.outer_stride + (c - o * g.hz) + (long long)e * g.stride;
}

template <int SIGN>
__global__ void __launch_bounds__(kFftThreads) k_fft_cols(float2* __restrict__ data, ColGeom g, FftPlan pl,
                                                          long long bstride) {
  extern __shared__ float2 sm[];
  float2* bufa = sm;
  float2* bufb = bufa + (size_t)g.n * g.w;
  float2* tw = bufb + (size_t)g.n * g.w;
  data += (long long)blockIdx.y * bstride;
  const int c0 = blockIdx.x * g.w;
  const int wl = ilog2(g.w);
  fill_twiddles(tw, g.n);
  const int E = g.n * g.w;
  for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
    const int e = idx >> wl;
    const int c = c0 + (idx & (g.w - 1));
    bufa[idx] = (c < g.ncols) ? data[col_addr(g, c, e)] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = tile_fft<SIGN>(bufa, bufb, g.w, wl, pl, tw);
  for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
    const int e = idx >> wl;
    const int c = c0 + (idx & (g.w - 1));
    if (c < g.ncols) data[col_addr(g, c, e)] = res[idx];
  }
}

// ---------------------------------------------------------------------------------
// x pass with a k-space operator. Columns are (ky, kz) pairs, c = ky*hz + kz, and the
// transform runs over kx with stride ny*hz. Op decides what happens between the
// forward and the (optional) inverse transform.
// ---------------------------------------------------------------------------------
template <class Op>
__global__ void __launch_bounds__(kFftThreads) k_fft_x_op(float2* __restrict__ data, ColGeom g, FftPlan pl, Op op,
                                                          long long bstride) {
  extern __shared__ float2 sm[];
  float2* bufa = sm;
  float2* bufb = bufa + (size_t)g.n * g.w;
  float2* tw = bufb + (size_t)g.n * g.w;
  float* opsm = reinterpret_cast<float*>(tw + g.n);
  const int batch = blockIdx.y;
  data += (long long)batch * bstride;
  const int c0 = blockIdx.x * g.w;
  const int wl = ilog2(g.w);
  fill_twiddles(tw, g.n);
  op.prologue(opsm, batch);
  const int E = g.n * g.w;
  for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
    const int e = idx >> wl;
    const int c = c0 + (idx & (g.w - 1));
    bufa[idx] = (c < g.ncols) ? data[(long long)c + (long long)e * g.stride] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* res = tile_fft<-1>(bufa, bufb, g.w, wl, pl, tw);
  for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
    const int e = idx >> wl;
    const int c = c0 + (idx & (g.w - 1));
    if (c < g.ncols) {
      const int ky = c / g.hz;
      res[idx] = op.apply(res[idx], e, ky, c - ky * g.hz, opsm, batch);
    }
  }
  __syncthreads();
  op.epilogue(opsm, batch, blockIdx.x, gridDim.x);
  if (Op::kInverse) res = tile_fft<1>(res, res == bufa ? bufb : bufa, g.w, wl, pl, tw);
  if (Op::kStore) {
    for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
      const int e = idx >> wl;
      const int c = c0 + (idx & (g.w - 1));
      if (c < g.ncols) data[(long long)c + (long long)e * g.stride] = res[idx];
    }
  }
}

// =================================================================================
// Register-resident passes for the specialised lengths (fft_reg.cuh). Dynamic shared
// memory: the w_N table, the stage exchange buffer, and (x pass) the operator's space.
// =================================================================================
__device__ __forceinline__ long long col_base(const ColGeom& g, int c) {
  const int o = c / g.hz;
  return (long long)o * g.outer_stride + (c - o * g.hz);
}

template <int N, int SIGN>
__global__ void __launch_bounds__(ColCfg<N>::T) k_cols_reg(float2* __restrict__ data, ColGeom g,
                                                           const float2* __restrict__ twg, long long bstride) {
  constexpr int P = Split<N>::P, Q = Split<N>::Q, W = ColCfg<N>::W, T = ColCfg<N>::T;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* ybuf = sm + N;
  data += (long long)blockIdx.y * bstride;
  const int tid = threadIdx.x;
  for (int m = tid; m < N; m += T) tw[m] = twg[m];
  __syncthreads();
  const int c0 = blockIdx.x * W;
  for (int w = tid; w < W * P; w += T) {
    const int c = w % W, t = w / W;
    const int col = c0 + c;
    float2 u[Q];
    if (col < g.ncols) {
      const float2* src = data + col_base(g, col) + (long long)t * g.stride;
#pragma unroll
      for (int m = 0; m < Q; ++m) u[m] = src[(long long)(P * m) * g.stride];
    } else {
#pragma unroll
      for (int m = 0; m < Q; ++m) u[m] = make_float2(0.f, 0.f);
    }
    RegDFT<Q, SIGN, P>::run(u, tw);
#pragma unroll
    for (int kb = 0; kb < Q; ++kb)
      ybuf[(kb * P + t) * W + c] = (kb == 0) ? u[0] : cmul(u[kb], twid<SIGN>(tw, t * kb));
  }
  __syncthreads();
  const int c = tid % W, kb = tid / W;
  float2 u[P];
#pragma unroll
  for (int t = 0; t < P; ++t) u[t] = ybuf[(kb * P + t) * W + c];
  RegDFT<P, SIGN, Q>::run(u, tw);
  const int col = c0 + c;
  if (col < g.ncols) {
    float2* dst = data + col_base(g, col) + (long long)kb * g.stride;
#pragma unroll
    for (int ka = 0; ka < P; ++ka) dst[(long long)(Q * ka) * g.stride] = u[ka];
  }
}

template <int N, class Op>
__global__ void __launch_bounds__(ColCfg<N>::T) k_x_op_reg(float2* __restrict__ data, ColGeom g,
                                                           const float2* __restrict__ twg, Op op, long long bstride) {
  constexpr int P = Split<N>::P, Q = Split<N>::Q, W = ColCfg<N>::W, T = ColCfg<N>::T;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* ybuf = sm + N;
  float* opsm = reinterpret_cast<float*>(ybuf + N * W);
  const int batch = blockIdx.y;
  data += (long long)batch * bstride;
  const int tid = threadIdx.x;
  for (int m = tid; m < N; m += T) tw[m] = twg[m];
  op.prologue(opsm, batch);  // ends with __syncthreads()
  const int c0 = blockIdx.x * W;
  // forward stage 1
  for (int w = tid; w < W * P; w += T) {
    const int c = w % W, t = w / W;
    const int col = c0 + c;
    float2 u[Q];
    if (col < g.ncols) {
      const float2* src = data + col + (long long)t * g.stride;
#pragma unroll
      for (int m = 0; m < Q; ++m) u[m] = src[(long long)(P * m) * g.stride];
    } else {
#pragma unroll
      for (int m = 0; m < Q; ++m) u[m] = make_float2(0.f, 0.f);
    }
    RegDFT<Q, -1, P>::run(u, tw);
#pragma unroll
    for (int kb = 0; kb < Q; ++kb)
      ybuf[(kb * P + t) * W + c] = (kb == 0) ? u[0] : cmul(u[kb], twid<-1>(tw, t * kb));
  }
  __syncthreads();
  // forward stage 2: this thread holds X[kb + Q ka], ka < P
  const int c = tid % W, kb = tid / W;
  const int col = c0 + c;
  float2 u[P];
#pragma unroll
  for (int t = 0; t < P; ++t) u[t] = ybuf[(kb * P + t) * W + c];
  RegDFT<P, -1, Q>::run(u, tw);
  if (col < g.ncols) {
    const int ky = col / g.hz;
    const int kz = col - ky * g.hz;
#pragma unroll
    for (int ka = 0; ka < P; ++ka) u[ka] = op.apply(u[ka], kb + Q * ka, ky, kz, opsm, batch);
  }
  __syncthreads();
  op.epilogue(opsm, batch, blockIdx.x, gridDim.x);
  if (Op::kInverse) {
    // inverse stage 1': t' = kb holds x'[t' + Q m'] = u[m'], m' < P
    RegDFT<P, 1, Q>::run(u, tw);
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1)
      ybuf[(k1 * Q + kb) * W + c] = (k1 == 0) ? u[0] : cmul(u[k1], twid<1>(tw, kb * k1));
    __syncthreads();
    // inverse stage 2': items (c, k1), k1 < P
    for (int w = tid; w < W * P; w += T) {
      const int cc = w % W, k1 = w / W;
      const int col2 = c0 + cc;
      float2 v[Q];
#pragma unroll
      for (int t = 0; t < Q; ++t) v[t] = ybuf[(k1 * Q + t) * W + cc];
      RegDFT<Q, 1, P>::run(v, tw);
      if (col2 < g.ncols) {
        float2* dst = data + col2 + (long long)k1 * g.stride;
#pragma unroll
        for (int k2 = 0; k2 < Q; ++k2) dst[(long long)(P * k2) * g.stride] = v[k2];
      }
    }
  } else if (Op::kStore) {
    if (col < g.ncols) {
      float2* dst = data + col + (long long)kb * g.stride;
#pragma unroll
      for (int ka = 0; ka < P; ++ka) dst[(long long)(Q * ka) * g.stride] = u[ka];
    }
  }
}

// r2c along z, nh = nz/2 = N complex per row, R rows per CTA.
// With `clear` (the input mesh itself) each input value is overwritten with 0 by the thread
// that read it, so a density mesh comes out cleared for the next paint.
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::T) k_rfft_z_reg(const float* in, float2* __restrict__ out,
                                                             int nrows, float sub, const float2* __restrict__ twg,
                                                             const float2* __restrict__ twg2, long long in_b,
                                                             long long out_b, float* clear) {
  constexpr int P = Split<N>::P, Q = Split<N>::Q, R = RowCfg<N>::R, T = RowCfg<N>::T;
  constexpr int S = P * (Q + 1);
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tw2 = tw + N;        // N+1 entries: exp(-2 pi i k / (2N))
  float2* ybuf = tw2 + N + 1;  // R*S; reused for the Z rows (stride N+1 <= S)
  in += (long long)blockIdx.y * in_b;
  out += (long long)blockIdx.y * out_b;
  if (clear) clear += (long long)blockIdx.y * in_b;
  const int tid = threadIdx.x;
  for (int m = tid; m < N; m += T) tw[m] = twg[m];
  for (int m = tid; m <= N; m += T) tw2[m] = twg2[m];
  __syncthreads();
  const int row0 = blockIdx.x * R;
  const float2* in2 = reinterpret_cast<const float2*>(in);
  for (int w = tid; w < R * P; w += T) {
    const int t = w % P, r = w / P;
    const int row = row0 + r;
    float2 u[Q];
    if (row < nrows) {
      const float2* src = in2 + (long long)row * N + t;
#pragma unroll
      for (int m = 0; m < Q; ++m) {
        const float2 z = src[P * m];
        u[m] = make_float2(z.x - sub, z.y - sub);
      }
      if (clear) {
        float2* dst = reinterpret_cast<float2*>(clear) + (long long)row * N + t;
#pragma unroll
        for (int m = 0; m < Q; ++m) dst[P * m] = make_float2(0.f, 0.f);
      }
    } else {
#pragma unroll
      for (int m = 0; m < Q; ++m) u[m] = make_float2(0.f, 0.f);
    }
    RegDFT<Q, -1, P>::run(u, tw);
#pragma unroll
    for (int kb = 0; kb < Q; ++kb)
      ybuf[r * S + t * (Q + 1) + kb] = (kb == 0) ? u[0] : cmul(u[kb], twid<-1>(tw, t * kb));
  }
  __syncthreads();
  const int kb = tid % Q, r = tid / Q;
  float2 u[P];
#pragma unroll
  for (int t = 0; t < P; ++t) u[t] = ybuf[r * S + t * (Q + 1) + kb];
  RegDFT<P, -1, Q>::run(u, tw);
  __syncthreads();
#pragma unroll
  for (int ka = 0; ka < P; ++ka) ybuf[r * (N + 1) + kb + Q * ka] = u[ka];
  __syncthreads();
  for (int w = tid; w < R * (N + 1); w += T) {
    const int rr = w / (N + 1);
    const int k = w - rr * (N + 1);
    const int row = row0 + rr;
    if (row >= nrows) continue;
    const float2 zk = ybuf[rr * (N + 1) + (k == N ? 0 : k)];
    const float2 zm = ybuf[rr * (N + 1) + (k == 0 ? 0 : N - k)];
    const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);
    const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
    out[(long long)row * (N + 1) + k] = cadd(e, cmul(tw2[k], o));
  }
}

// c2r along z (unnormalised times `scale`).
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::T) k_irfft_z_reg(const float2* __restrict__ in, float* __restrict__ out,
                                                              int nrows, float scale, const float2* __restrict__ twg,
                                                              const float2* __restrict__ twg2, long long in_b,
                                                              long long out_b) {
  constexpr int P = Split<N>::P, Q = Split<N>::Q, R = RowCfg<N>::R, T = RowCfg<N>::T;
  constexpr int S = P * (Q + 1);
  constexpr int IT = (R * P + T - 1) / T;  // stage-1 items per thread
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* tw2 = tw + N;
  float2* xbuf = tw2 + N + 1;  // R*(N+1) input rows, then (aliased) the R*S exchange buffer
  float2* ybuf = xbuf;
  in += (long long)blockIdx.y * in_b;
  out += (long long)blockIdx.y * out_b;
  const int tid = threadIdx.x;
  for (int m = tid; m < N; m += T) tw[m] = twg[m];
  for (int m = tid; m <= N; m += T) tw2[m] = twg2[m];
  const int row0 = blockIdx.x * R;
  for (int w = tid; w < R * (N + 1); w += T) {
    const int rr = w / (N + 1);
    const int k = w - rr * (N + 1);
    const int row = row0 + rr;
    xbuf[w] = (row < nrows) ? in[(long long)row * (N + 1) + k] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2 u1[IT][Q];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int w = tid + it * T;
    if (w >= R * P) continue;
    const int t = w % P, r = w / P;
#pragma unroll
    for (int m = 0; m < Q; ++m) {
      const int e = t + P * m;
      const float2 xk = xbuf[r * (N + 1) + e];
      const float2 xm = xbuf[r * (N + 1) + N - e];
      const float2 ee = make_float2(xk.x + xm.x, xk.y - xm.y);
      const float2 dd = cmul(make_float2(xk.x - xm.x, xk.y + xm.y), conjf2(tw2[e]));
      u1[it][m] = make_float2(ee.x - dd.y, ee.y + dd.x);
    }
    RegDFT<Q, 1, P>::run(u1[it], tw);
  }
  __syncthreads();  // every input row has been read; the exchange buffer may overwrite it
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int w = tid + it * T;
    if (w >= R * P) continue;
    const int t = w % P, r = w / P;
#pragma unroll
    for (int kb = 0; kb < Q; ++kb)
      ybuf[r * S + t * (Q + 1) + kb] = (kb == 0) ? u1[it][0] : cmul(u1[it][kb], twid<1>(tw, t * kb));
  }
  __syncthreads();
  const int kb = tid % Q, r = tid / Q;
  const int row = row0 + r;
  float2 u[P];
#pragma unroll
  for (int t = 0; t < P; ++t) u[t] = ybuf[r * S + t * (Q + 1) + kb];
  RegDFT<P, 1, Q>::run(u, tw);
  if (row < nrows) {
    float2* dst = reinterpret_cast<float2*>(out) + (long long)row * N + kb;
#pragma unroll
    for (int ka = 0; ka < P; ++ka) dst[Q * ka] = cscale(u[ka], scale);
  }
}

// ---------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------
bool make_fft_plan(int n, FftPlan* p) {
  if (n < 2) return false;
  int m = n, a = 0, b = 0;
  while (m % 2 == 0) {
    m /= 2;
    ++a;
  }
  while (m % 3 == 0) {
    m /= 3;
    ++b;
  }
  if (m != 1) return false;
  p->n = n;
  p->nst = 0;
  while (a >= 3) {
    p->radix[p->nst++] = 8;
    a -= 3;
  }
  if (a == 2) p->radix[p->nst++] = 4;
  if (a == 1) p->radix[p->nst++] = 2;
  for (int i = 0; i < b; ++i) p->radix[p->nst++] = 3;
  return p->nst <= kMaxRadixStages;
}

bool fft_axis_supported(int n) {
  FftPlan p;
  return n >= 2 && n <= kFftTileElems && make_fft_plan(n, &p);
}

bool mesh_fft_supported(int nx, int ny, int nz) {
  return nz % 2 == 0 && nz >= 4 && fft_axis_supported(nx) && fft_axis_supported(ny) && fft_axis_supported(nz / 2);
}

static int pow2_floor(int v) {
  int p = 1;
  while (p * 2 <= v) p *= 2;
  return p;
}

static int z_rows_per_cta(int nz) { return pow2_floor(kFftTileElems / (nz / 2)) > 0 ? pow2_floor(kFftTileElems / (nz / 2)) : 1; }

static int col_tile_width(int n) {
  int w = kFftTileElems / n;
  if (w > 16) w = 16;
  return w < 1 ? 1 : pow2_floor(w);
}

// ---- twiddle tables w_n^m = exp(-2 pi i m / n), one per (device, n), built once on the host
static std::mutex g_tw_mutex;
static std::map<std::pair<int, int>, float2*> g_tw_tables;

const float2* twiddle_table(int n) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_tw_mutex);
  auto key = std::make_pair(dev, n);
  auto it = g_tw_tables.find(key);
  if (it != g_tw_tables.end()) return it->second;
  std::vector<float2> h(n);
  for (int m = 0; m < n; ++m) {
    const double ang = 2.0 * M_PI * (double)m / (double)n;
    h[m] = make_float2((float)std::cos(ang), (float)-std::sin(ang));
  }
  float2* d = nullptr;
  if (cudaMalloc(&d, sizeof(float2) * n) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, h.data(), sizeof(float2) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  g_tw_tables[key] = d;
  return d;
}

#define JFLI_REG_SIZES(X) \
  X(8) X(12) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024)

static bool reg_size(int n) {
  switch (n) {
#define JFLI_CASE(N_) case N_:
    JFLI_REG_SIZES(JFLI_CASE)
#undef JFLI_CASE
    return true;
    default:
      return false;
  }
}

static int reg_col_w(int n) {
  switch (n) {
#define JFLI_CASE(N_) \
  case N_:            \
    return ColCfg<N_>::W;
    JFLI_REG_SIZES(JFLI_CASE)
#undef JFLI_CASE
    default:
      return 0;
  }
}

template <int N>
static cudaError_t rfft_z_reg(const float* in, float2* out, const MeshDims& d, float sub, cudaStream_t s,
                              float* clear) {
  constexpr int R = RowCfg<N>::R, T = RowCfg<N>::T, P = Split<N>::P, Q = Split<N>::Q;
  const float2* tw = twiddle_table(N);
  const float2* tw2 = twiddle_table(2 * N);
  if (!tw || !tw2) return cudaErrorMemoryAllocation;
  const int nrows = d.nx * d.ny;
  const size_t smem = ((size_t)N + N + 1 + (size_t)R * P * (Q + 1)) * sizeof(float2);
  cudaFuncSetAttribute(k_rfft_z_reg<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_rfft_z_reg<N><<<dim3((nrows + R - 1) / R, d.batch), T, smem, s>>>(in, out, nrows, sub, tw, tw2, d.cells(),
                                                                       d.spec_elems(), clear);
  note_launch();
  return cudaGetLastError();
}

template <int N>
static cudaError_t irfft_z_reg(const float2* in, float* out, const MeshDims& d, float scale, cudaStream_t s) {
  constexpr int R = RowCfg<N>::R, T = RowCfg<N>::T, P = Split<N>::P, Q = Split<N>::Q;
  const float2* tw = twiddle_table(N);
  const float2* tw2 = twiddle_table(2 * N);
  if (!tw || !tw2) return cudaErrorMemoryAllocation;
  const int nrows = d.nx * d.ny;
  const size_t rows_buf = (size_t)R * P * (Q + 1) > (size_t)R * (N + 1) ? (size_t)R * P * (Q + 1) : (size_t)R * (N + 1);
  const size_t smem = ((size_t)N + N + 1 + rows_buf) * sizeof(float2);
  cudaFuncSetAttribute(k_irfft_z_reg<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_irfft_z_reg<N><<<dim3((nrows + R - 1) / R, d.batch), T, smem, s>>>(in, out, nrows, scale, tw, tw2,
                                                                        d.spec_elems(), d.cells());
  note_launch();
  return cudaGetLastError();
}

template <int N, int SIGN>
static cudaError_t cols_reg(float2* data, const ColGeom& g, long long bstride, int batch, cudaStream_t s) {
  constexpr int W = ColCfg<N>::W, T = ColCfg<N>::T;
  const float2* tw = twiddle_table(N);
  if (!tw) return cudaErrorMemoryAllocation;
  const size_t smem = ((size_t)N + (size_t)N * W) * sizeof(float2);
  cudaFuncSetAttribute(k_cols_reg<N, SIGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_cols_reg<N, SIGN><<<dim3((g.ncols + W - 1) / W, batch), T, smem, s>>>(data, g, tw, bstride);
  note_launch();
  return cudaGetLastError();
}

template <int N, class Op>
static cudaError_t x_op_reg(float2* data, const ColGeom& g, const Op& op, long long bstride, int batch,
                            cudaStream_t s) {
  constexpr int W = ColCfg<N>::W, T = ColCfg<N>::T;
  const float2* tw = twiddle_table(N);
  if (!tw) return cudaErrorMemoryAllocation;
  const size_t smem = ((size_t)N + (size_t)N * W) * sizeof(float2) + Op::smem_bytes(op);
  cudaFuncSetAttribute(k_x_op_reg<N, Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_x_op_reg<N, Op><<<dim3((g.ncols + W - 1) / W, batch), T, smem, s>>>(data, g, tw, op, bstride);
  note_launch();
  return cudaGetLastError();
}

// ---- generic (shared-memory Stockham) launchers for the remaining lengths
// `clear`: the input mesh, set to 0 once it has been read (nullptr: left as it is).
static cudaError_t launch_rfft_z(const float* in, float2* out, const MeshDims& d, float sub, cudaStream_t s,
                                 float* clear = nullptr) {
  switch (d.nz / 2) {
#define JFLI_CASE(N_) \
  case N_:            \
    return rfft_z_reg<N_>(in, out, d, sub, s, clear);
    JFLI_REG_SIZES(JFLI_CASE)
#undef JFLI_CASE
    default:
      break;
  }
  FftPlan pl;
  make_fft_plan(d.nz / 2, &pl);
  const int nrows = d.nx * d.ny;
  const int rows = z_rows_per_cta(d.nz);
  const int nh = d.nz / 2;
  const size_t smem = ((size_t)2 * (nh + 1) * (rows + 1) + nh + nh + 1) * sizeof(float2);
  dim3 grid((nrows + rows - 1) / rows, d.batch);
  cudaFuncSetAttribute(k_rfft_z, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_rfft_z<<<grid, kFftThreads, smem, s>>>(in, out, nrows, d.nz, rows, pl, sub, d.cells(), d.spec_elems());
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && clear) e = cudaMemsetAsync(clear, 0, sizeof(float) * (size_t)d.cells() * d.batch, s);
  return e;
}

static cudaError_t launch_irfft_z(const float2* in, float* out, const MeshDims& d, float scale, cudaStream_t s) {
  switch (d.nz / 2) {
#define JFLI_CASE(N_) \
  case N_:            \
    return irfft_z_reg<N_>(in, out, d, scale, s);
    JFLI_REG_SIZES(JFLI_CASE)
#undef JFLI_CASE
    default:
      break;
  }
  FftPlan pl;
  make_fft_plan(d.nz / 2, &pl);
  const int nrows = d.nx * d.ny;
  const int rows = z_rows_per_cta(d.nz);
  const int nh = d.nz / 2;
  const size_t smem = ((size_t)2 * (nh + 1) * (rows + 1) + nh + nh + 1) * sizeof(float2);
  dim3 grid((nrows + rows - 1) / rows, d.batch);
  cudaFuncSetAttribute(k_irfft_z, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_irfft_z<<<grid, kFftThreads, smem, s>>>(in, out, nrows, d.nz, rows, pl, scale, d.spec_elems(), d.cells());
  note_launch();
  return cudaGetLastError();
}

static ColGeom y_geom(const MeshDims& d) {
  ColGeom g;
  g.n = d.ny;
  g.hz = d.hz();
  g.ncols = d.nx * g.hz;
  g.w = col_tile_width(g.n);
  g.stride = g.hz;
  g.outer_stride = (long long)d.ny * g.hz;
  return g;
}

static ColGeom x_geom(const MeshDims& d) {
  ColGeom g;
  g.n = d.nx;
  g.hz = d.hz();
  g.ncols = d.ny * g.hz;
  g.w = col_tile_width(g.n);
  g.stride = (long long)d.ny * g.hz;
  g.outer_stride = g.hz;
  return g;
}

template <int SIGN>
static cudaError_t launch_cols(float2* data, const ColGeom& g, long long bstride, int batch, cudaStream_t s) {
  switch (g.n) {
#define JFLI_CASE(N_) \
  case N_:            \
    return cols_reg<N_, SIGN>(data, g, bstride, batch, s);
    JFLI_REG_SIZES(JFLI_CASE)
#undef JFLI_CASE
    default:
      break;
  }
  FftPlan pl;
  make_fft_plan(g.n, &pl);
  const size_t smem = ((size_t)2 * g.n * g.w + g.n) * sizeof(float2);
  dim3 grid((g.ncols + g.w - 1) / g.w, batch);
  cudaFuncSetAttribute(k_fft_cols<SIGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_fft_cols<SIGN><<<grid, kFftThreads, smem, s>>>(data, g, pl, bstride);
  note_launch();
  return cudaGetLastError();
}

// ---- TMA-staged x pass
static std::atomic<int> g_x_pass_mode{1};  // 0 register pass, 1 TMA-staged pass (default)

void set_x_pass_mode(int mode) { g_x_pass_mode.store(mode); }
int x_pass_mode() { return g_x_pass_mode.load(); }

cudaError_t device_status(unsigned* out, bool reset) {
  cudaError_t e = cudaMemcpyFromSymbol(out, g_jfli_status, sizeof(unsigned));
  if (e == cudaSuccess && reset) {
    const unsigned zero = 0;
    e = cudaMemcpyToSymbol(g_jfli_status, &zero, sizeof(unsigned));
  }
  return e;
}

bool x_pass_tensor_map(CUtensorMap* map, const float2* spec, const MeshDims& d, int w) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode encode = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<Encode>(f);
  }();
  if (encode == nullptr || ((uintptr_t)spec % 16) != 0) return false;
  const cuuint64_t inner = 2ull * (cuuint64_t)d.ny * (cuuint64_t)d.hz();  // floats of one x plane
  const cuuint64_t plane_bytes = inner * sizeof(float);
  const cuuint64_t batch_bytes = (cuuint64_t)d.spec_elems() * sizeof(float2);
  if (plane_bytes % 16 != 0 || batch_bytes % 16 != 0 || (2 * w * sizeof(float)) % 16 != 0) return false;
  const cuuint64_t dims[3] = {inner, (cuuint64_t)d.nx, (cuuint64_t)d.batch};
  const cuuint64_t strides[2] = {plane_bytes, batch_bytes};
  const cuuint32_t box[3] = {(cuuint32_t)(2 * w), (cuuint32_t)(d.nx > kTmaBoxRows ? kTmaBoxRows : d.nx), 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float2*>(spec), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int N, class Op>
static cudaError_t x_op_tma(float2* data, const MeshDims& d, const Op& op, bool* done, cudaStream_t s) {
  *done = false;
  constexpr int W = ColCfg<N>::W, T = ColCfg<N>::T;
  if (N % TmaCfg<N>::ROWS != 0) return cudaSuccess;
  CUtensorMap map;
  if (!x_pass_tensor_map(&map, data, d, W)) return cudaSuccess;
  const float2* tw = twiddle_table(N);
  if (!tw) return cudaErrorMemoryAllocation;
  const ColGeom g = x_geom(d);
  const size_t smem = TmaCfg<N>::tile_bytes * 2 + sizeof(float2) * (size_t)N + Op::smem_bytes(op);
  cudaError_t e = cudaFuncSetAttribute(k_x_op_tma<N, Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_x_op_tma<N, Op><<<dim3((g.ncols + W - 1) / W, d.batch), T, smem, s>>>(map, g, tw, op);
  note_launch();
  *done = true;
  return cudaGetLastError();
}

template <class Op>
static cudaError_t launch_x_op(float2* data, const MeshDims& d, const Op& op, cudaStream_t s) {
  const ColGeom g = x_geom(d);
  if constexpr (Op::kInverse) {
    if (x_pass_mode() == 1) {
      bool done = false;
      cudaError_t e = cudaSuccess;
      switch (g.n) {
#define JFLI_CASE(N_)                              \
  case N_:                                         \
    e = x_op_tma<N_, Op>(data, d, op, &done, s);   \
    break;
        JFLI_REG_SIZES(JFLI_CASE)
#undef JFLI_CASE
        default:
          break;
      }
      if (e != cudaSuccess || done) return e;
    }
  }
  switch (g.n) {
#define JFLI_CASE(N_) \
  case N_:            \
    return x_op_reg<N_, Op>(data, g, op, d.spec_elems(), d.batch, s);
    JFLI_REG_SIZES(JFLI_CASE)
#undef JFLI_CASE
    default:
      break;
  }
  FftPlan pl;
  make_fft_plan(g.n, &pl);
  const size_t smem = ((size_t)2 * g.n * g.w + g.n) * sizeof(float2) + Op::smem_bytes(op);
  dim3 grid((g.ncols + g.w - 1) / g.w, d.batch);
  cudaFuncSetAttribute(k_fft_x_op<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_fft_x_op<Op><<<grid, kFftThreads, smem, s>>>(data, g, pl, op, d.spec_elems());
  note_launch();
  return cudaGetLastError();
}

int x_pass_ctas(const MeshDims& d) {
  const ColGeom g = x_geom(d);
  const int w = reg_size(g.n) ? reg_col_w(g.n) : g.w;
  return (g.ncols + w - 1) / w;
}

cudaError_t rfft3d_forward(const float* in, float2* spec, const MeshDims& d, float sub, cudaStream_t s) {
  cudaError_t e = launch_rfft_z(in, spec, d, sub, s);
  if (e != cudaSuccess) return e;
  e = launch_cols<-1>(spec, y_geom(d), d.spec_elems(), d.batch, s);
  if (e != cudaSuccess) return e;
  return launch_cols<-1>(spec, x_geom(d), d.spec_elems(), d.batch, s);
}

// 2D r2c of (ny, nz) maps: the z and y passes of rfft3d_forward on a mesh with nx = 1
cudaError_t rfft2d_forward(const float* in, float2* spec, const MeshDims& d, cudaStream_t s) {
  cudaError_t e = launch_rfft_z(in, spec, d, 0.0f, s);
  if (e != cudaSuccess) return e;
  return launch_cols<-1>(spec, y_geom(d), d.spec_elems(), d.batch, s);
}

cudaError_t rfft3d_inverse(float2* spec, float* out, const MeshDims& d, float scale, cudaStream_t s) {
  cudaError_t e = launch_cols<1>(spec, x_geom(d), d.spec_elems(), d.batch, s);
  if (e != cudaSuccess) return e;
  e = launch_cols<1>(spec, y_geom(d), d.spec_elems(), d.batch, s);
  if (e != cudaSuccess) return e;
  return launch_irfft_z(spec, out, d, scale, s);
}

// real mesh -> (forward 3D FFT, k-space op, inverse 3D FFT) -> real mesh.
template <class Op>
static cudaError_t filter_chain(const float* in, float2* spec, float* out, const MeshDims& d, float sub, const Op& op,
                                cudaStream_t s, float* clear = nullptr) {
  cudaError_t e = launch_rfft_z(in, spec, d, sub, s, clear);
  if (e != cudaSuccess) return e;
  e = launch_cols<-1>(spec, y_geom(d), d.spec_elems(), d.batch, s);
  if (e != cudaSuccess) return e;
  e = launch_x_op(spec, d, op, s);
  if (e != cudaSuccess) return e;
  e = launch_cols<1>(spec, y_geom(d), d.spec_elems(), d.batch, s);
  if (e != cudaSuccess) return e;
  return launch_irfft_z(spec, out, d, 1.0f, s);
}

cudaError_t poisson_potential(const float* rho, float2* spec, float* pot, const MeshDims& d, float rho_mean,
                              float scale, cudaStream_t s, float* clear) {
  PoissonOp op;
  op.nx = d.nx;
  op.ny = d.ny;
  op.nz = d.nz;
  op.norm = scale / ((float)d.nx * (float)d.ny * (float)d.nz);
  return filter_chain(rho, spec, pot, d, rho_mean, op, s, clear);
}

cudaError_t pgd_potential(const float* rho, float2* spec, float* pot, const MeshDims& d, float rho_mean, float kl,
                          float ks, float scale, cudaStream_t s) {
  return mixed_pgd_potential(rho, spec, pot, d, rho_mean, kl, ks, 0.f, 1.f, scale, s);
}

cudaError_t mixed_pgd_potential(const float* rho, float2* spec, float* pot, const MeshDims& d, float rho_mean,
                                float kl, float ks, float c0, float c1, float scale, cudaStream_t s) {
  PgdOp op;
  op.nx = d.nx;
  op.ny = d.ny;
  op.nz = d.nz;
  op.norm = scale / ((float)d.nx * (float)d.ny * (float)d.nz);
  op.kl2 = kl * kl;
  op.ks4 = ks * ks * ks * ks;
  op.c0 = c0;
  op.c1 = c1;
  return filter_chain(rho, spec, pot, d, rho_mean, op, s);
}

cudaError_t ic_filter(const float* noise, float2* spec, float* out, const MeshDims& d, const float* ktab,
                      const float* ptab, int ntab, const float* box, int zero_mode_one, cudaStream_t s,
                      const float* dptab) {
  IcOp op;
  op.dptab = dptab;
  op.nx = d.nx;
  op.ny = d.ny;
  op.nz = d.nz;
  op.ktab = ktab;
  op.ptab = ptab;
  op.ntab = ntab;
  op.lx = box[0];
  op.ly = box[1];
  op.lz = box[2];
  op.factor = (float)(((double)d.nx * d.ny * d.nz) / ((double)box[0] * box[1] * box[2]));
  op.norm = 1.0f / ((float)d.nx * (float)d.ny * (float)d.nz);
  op.zero_mode_one = zero_mode_one;
  return filter_chain(noise, spec, out, d, 0.0f, op, s);
}

cudaError_t power_adjoint(const float* mesh, float2* spec, float* out, const MeshDims& d, const float* kedges,
                          const float* weights, int nedges, const float* box, cudaStream_t s) {
  PkAdjOp op;
  op.nx = d.nx;
  op.ny = d.ny;
  op.nz = d.nz;
  op.kedges = kedges;
  op.weights = weights;
  op.nedges = nedges;
  op.cx = (float)(2.0 * M_PI / (double)box[0]);
  op.cy = (float)(2.0 * M_PI / (double)box[1]);
  op.cz = (float)(2.0 * M_PI / (double)box[2]);
  op.norm = 1.0f / ((float)d.nx * (float)d.ny * (float)d.nz);
  return filter_chain(mesh, spec, out, d, 0.0f, op, s);
}

cudaError_t power_poles_adjoint(const float* mesh, float2* spec, float* out, const MeshDims& d, const float* kedges,
                                const float* weights, int nedges, const int* ells, int nell, const float* box,
                                const float* los, int cplx, cudaStream_t s) {
  PkAdjOp op;
  op.nx = d.nx;
  op.ny = d.ny;
  op.nz = d.nz;
  op.kedges = kedges;
  op.weights = weights;
  op.nedges = nedges;
  op.cx = (float)(2.0 * M_PI / (double)box[0]);
  op.cy = (float)(2.0 * M_PI / (double)box[1]);
  op.cz = (float)(2.0 * M_PI / (double)box[2]);
  op.norm = 1.0f / ((float)d.nx * (float)d.ny * (float)d.nz);
  op.nell = nell;
  op.cplx = cplx;
  for (int e = 0; e < nell && e < kMaxAdjPoles; ++e) op.ells[e] = ells[e];
  op.lx = los[0];
  op.ly = los[1];
  op.lz = los[2];
  return filter_chain(mesh, spec, out, d, 0.0f, op, s);
}

cudaError_t power_partials(const float* mesh, float2* spec, double* partials, const MeshDims& d, const float* kedges,
                           int nedges, const float* box, float norm, cudaStream_t s) {
  cudaError_t e = launch_rfft_z(mesh, spec, d, 0.0f, s);
  if (e != cudaSuccess) return e;
  e = launch_cols<-1>(spec, y_geom(d), d.spec_elems(), d.batch, s);
  if (e != cudaSuccess) return e;
  PkOp op;
  op.nx = d.nx;
  op.ny = d.ny;
  op.nz = d.nz;
  op.kedges = kedges;
  op.nedges = nedges;
  op.cx = (float)(2.0 * M_PI / (double)box[0]);
  op.cy = (float)(2.0 * M_PI / (double)box[1]);
  op.cz = (float)(2.0 * M_PI / (double)box[2]);
  op.norm = norm;
  op.partials = partials;
  return launch_x_op(spec, d, op, s);
}

// ---------------------------------------------------------------------------------
// P(k) without any allocation, for callers that cannot allocate device memory.
//
// The half spectrum and the per-CTA histogram partials live in one file-scope device
// array of kNoAllocScratchBytes. The transforms use the shared-memory Stockham kernels,
// which build their twiddles in the kernel, so no twiddle table is created either.
// ---------------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = 11u << 20;  // 11 MiB: a 128^3 spectrum plus its partials
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mutex;
static void* g_noalloc_ptr[kNoAllocMaxDevices];  // device -> address of g_noalloc_scratch on it
static void* g_noalloc_ctx[kNoAllocMaxDevices];  // the context that address belongs to

// The calling thread's current driver context (cuCtxGetCurrent through the runtime's
// driver entry point, so the library needs no link to libcuda), or nullptr.
static void* current_context() {
  using GetCurrent = int (*)(void**);
  static GetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetCurrent>(f);
  }();
  void* ctx = nullptr;
  if (fn == nullptr || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// Device address of the scratch array on the current device. The first call on a device
// looks it up with cudaGetSymbolAddress (with that device current); later calls reuse it.
// The address is tied to the device's context: a new context on the device (after
// cudaDeviceReset, for instance) gets a new lookup, so no call uses a stale address.
cudaError_t noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  void* ctx = g_noalloc_ptr[dev] ? current_context() : nullptr;
  if (g_noalloc_ptr[dev] == nullptr || ctx == nullptr || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // makes the device's primary context current
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = p;
    g_noalloc_ctx[dev] = current_context();
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

size_t noalloc_scratch_bytes() { return kNoAllocScratchBytes; }

int noalloc_pk_ctas(const MeshDims& d) {
  const ColGeom g = x_geom(d);
  return (g.ncols + g.w - 1) / g.w;
}

cudaError_t power_partials_noalloc(const float* mesh, float2* spec, double* partials, const MeshDims& d,
                                   const float* kedges, int nedges, const float* box, float norm, cudaStream_t s) {
  // r2c along z (Stockham, twiddles built in the kernel)
  {
    FftPlan pl;
    make_fft_plan(d.nz / 2, &pl);
    const int nrows = d.nx * d.ny;
    const int rows = z_rows_per_cta(d.nz);
    const int nh = d.nz / 2;
    const size_t smem = ((size_t)2 * (nh + 1) * (rows + 1) + nh + nh + 1) * sizeof(float2);
    cudaFuncSetAttribute(k_rfft_z, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_rfft_z<<<dim3((nrows + rows - 1) / rows, d.batch), kFftThreads, smem, s>>>(mesh, spec, nrows, d.nz, rows, pl,
                                                                               0.0f, d.cells(), d.spec_elems());
    note_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  // forward y
  {
    const ColGeom g = y_geom(d);
    FftPlan pl;
    make_fft_plan(g.n, &pl);
    const size_t smem = ((size_t)2 * g.n * g.w + g.n) * sizeof(float2);
    cudaFuncSetAttribute(k_fft_cols<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_fft_cols<-1><<<dim3((g.ncols + g.w - 1) / g.w, d.batch), kFftThreads, smem, s>>>(spec, g, pl, d.spec_elems());
    note_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  // forward x feeding the histogram
  PkOp op;
  op.nx = d.nx;
  op.ny = d.ny;
  op.nz = d.nz;
  op.kedges = kedges;
  op.nedges = nedges;
  op.cx = (float)(2.0 * M_PI / (double)box[0]);
  op.cy = (float)(2.0 * M_PI / (double)box[1]);
  op.cz = (float)(2.0 * M_PI / (double)box[2]);
  op.norm = norm;
  op.partials = partials;
  const ColGeom g = x_geom(d);
  FftPlan pl;
  make_fft_plan(g.n, &pl);
  const size_t smem = ((size_t)2 * g.n * g.w + g.n) * sizeof(float2) + PkOp::smem_bytes(op);
  cudaFuncSetAttribute(k_fft_x_op<PkOp>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_fft_x_op<PkOp><<<dim3((g.ncols + g.w - 1) / g.w, d.batch), kFftThreads, smem, s>>>(spec, g, pl, op,
                                                                                     d.spec_elems());
  note_launch();
  return cudaGetLastError();
}

}  // namespace jfli
