// TMA-staged variant of the fused x pass (forward x FFT -> k-space operator -> inverse x
// FFT) for sm_100a.
//
// The x pass of a half spectrum [batch][nx][ny][nz/2+1] transforms columns along x whose
// elements lie ny (nz/2+1) complex values apart. Viewed as a 3D tensor of FP32 values
// (inner: the 2 ny (nz/2+1) floats of one x plane; then the nx planes; then the batch),
// a CTA's pencil tile -- W neighbouring columns over all N planes -- is one box of
// 2W x N x 1 floats (N <= 256; longer transforms take N / 256 boxes). One elected thread
// moves it into shared memory with cp.async.bulk.tensor (completion on an mbarrier), the
// CTA computes from shared memory, writes its results back into the same tile and the
// elected thread stores it with one bulk tensor store. Loads and stores touch only this
// GPU's own buffer and use no cluster multicast.
//
// The tensor map needs the plane stride ny (nz/2+1) 8 bytes to be a multiple of 16 (ny
// even, or nz/2+1 even) and a 16-byte aligned spectrum; other shapes keep the register
// pass. A tile's inner coordinate 2 c0 floats = 8 c0 bytes is a multiple of 16 because W
// is even. Columns past the last one read as zeros (the box's out-of-bounds fill) and are
// not stored (the bulk store clips them).
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "fft_reg.cuh"
#include "internal.h"

namespace jfli {

// Set (bit 0) by a kernel whose wait on an mbarrier ran out of its bound; read and cleared
// by jfli_device_status. (This header is included by fft.cu alone, which owns the word.)
__device__ unsigned g_jfli_status = 0;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait (about 2 s at the SM clock): true when the phase completed; false after the
// bound, with bit 0 of g_jfli_status set.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > 4000000000ll) {
      atomicOr(&g_jfli_status, 1u);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(smem_dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* smem_src, int x, int y, int z) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];"
               ::"l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(smem_src)), "r"(x), "r"(y), "r"(z)
               : "memory");
}

__device__ __forceinline__ void tma_store_commit_and_drain() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

constexpr int kTmaBoxRows = 256;  // a box dimension holds at most 256 elements

template <int N>
struct TmaCfg {
  static constexpr int W = ColCfg<N>::W;
  static constexpr int BOXES = N > kTmaBoxRows ? N / kTmaBoxRows : 1;
  static constexpr int ROWS = N > kTmaBoxRows ? kTmaBoxRows : N;
  static constexpr size_t tile_bytes = sizeof(float2) * (size_t)N * W;
};

// Shared memory: tile[N][W] (128-byte aligned, TMA destination and source), ybuf[N*W],
// tw[N], then the operator's table.
template <int N, class Op>
__global__ void __launch_bounds__(ColCfg<N>::T) k_x_op_tma(const __grid_constant__ CUtensorMap map, ColGeom g,
                                                           const float2* __restrict__ twg, Op op) {
  constexpr int P = Split<N>::P, Q = Split<N>::Q, W = ColCfg<N>::W, T = ColCfg<N>::T;
  static_assert(Op::kInverse, "the TMA x pass writes the inverse-transformed tile back");
  extern __shared__ __align__(128) unsigned char smraw[];
  float2* tile = reinterpret_cast<float2*>(smraw);
  float2* ybuf = tile + N * W;
  float2* tw = ybuf + N * W;
  float* opsm = reinterpret_cast<float*>(tw + N);
  __shared__ __align__(8) uint64_t bar;
  const int batch = blockIdx.y;
  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * W;
  if (tid == 0) {
    mbar_init(&bar, 1);
    mbar_expect_tx(&bar, (unsigned)TmaCfg<N>::tile_bytes);
#pragma unroll
    for (int b = 0; b < TmaCfg<N>::BOXES; ++b)
      tma_load_3d(tile + (size_t)b * TmaCfg<N>::ROWS * W, &map, 2 * c0, b * TmaCfg<N>::ROWS, batch, &bar);
  }
  for (int m = tid; m < N; m += T) tw[m] = twg[m];
  op.prologue(opsm, batch);  // ends with __syncthreads(): the barrier's init is visible to all
  if (!mbar_wait_bounded(&bar, 0)) {
    // the tile never arrived: leave the spectrum as it is; wait (bounded) so that no copy
    // is still writing this CTA's shared memory when it exits
    mbar_wait_bounded(&bar, 0);
    return;
  }
  // forward stage 1 from the tile
  for (int w = tid; w < W * P; w += T) {
    const int c = w % W, t = w / W;
    float2 u[Q];
#pragma unroll
    for (int m = 0; m < Q; ++m) u[m] = tile[(t + P * m) * W + c];
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
  // inverse stage 1': t' = kb holds x'[t' + Q m'] = u[m'], m' < P
  RegDFT<P, 1, Q>::run(u, tw);
#pragma unroll
  for (int k1 = 0; k1 < P; ++k1) ybuf[(k1 * Q + kb) * W + c] = (k1 == 0) ? u[0] : cmul(u[k1], twid<1>(tw, kb * k1));
  __syncthreads();
  // inverse stage 2' into the tile
  for (int w = tid; w < W * P; w += T) {
    const int cc = w % W, k1 = w / W;
    float2 v[Q];
#pragma unroll
    for (int t = 0; t < Q; ++t) v[t] = ybuf[(k1 * Q + t) * W + cc];
    RegDFT<Q, 1, P>::run(v, tw);
#pragma unroll
    for (int k2 = 0; k2 < Q; ++k2) tile[(k1 + P * k2) * W + cc] = v[k2];
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic-proxy writes -> bulk store
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int b = 0; b < TmaCfg<N>::BOXES; ++b)
      tma_store_3d(&map, tile + (size_t)b * TmaCfg<N>::ROWS * W, 2 * c0, b * TmaCfg<N>::ROWS, batch);
    tma_store_commit_and_drain();
  }
}

// Tensor map of the x pass over a half spectrum: FP32, dims (2 ny hz, nx, batch), box
// (2W, min(N, 256), 1). false when the layout does not meet the TMA rules (the caller
// then keeps the register pass) or the driver entry point is unavailable.
bool x_pass_tensor_map(CUtensorMap* map, const float2* spec, const MeshDims& d, int w);

}  // namespace jfli
