// Deterministic reduction of the per-CTA P(k) histogram partials written by the x pass
// (kspace_ops.cuh PkOp): one thread per (batch, bin, quantity), CTAs summed in a fixed
// order with Kahan-compensated FP64 accumulation.
#include "common.cuh"
#include "internal.h"

namespace jfli {

__global__ void k_power_finalize(const double* __restrict__ partials, int nctas, int nvals, double* __restrict__ out,
                                 int batch) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nvals * batch) return;
  const int b = t / nvals;
  const int v = t - b * nvals;
  const double* src = partials + (long long)b * nctas * nvals + v;
  double s = 0.0, c = 0.0;
  for (int i = 0; i < nctas; ++i) {
    const double y = src[(long long)i * nvals] - c;
    const double t2 = s + y;
    c = (t2 - s) - y;
    s = t2;
  }
  out[(long long)b * nvals + v] = s;
}

// The same fixed-order reduction for nvals values per CTA (layout [batch][nctas][nvals]).
cudaError_t sums_finalize(const double* partials, int nctas, int nvals, double* out, int batch, cudaStream_t s) {
  const int total = nvals * batch;
  k_power_finalize<<<(total + 127) / 128, 128, 0, s>>>(partials, nctas, nvals, out, batch);
  note_launch();
  return cudaGetLastError();
}

cudaError_t power_finalize(const double* partials, int nctas, int nbins, double* out, int batch, cudaStream_t s) {
  const int nvals = 3 * nbins;
  const int total = nvals * batch;
  k_power_finalize<<<(total + 127) / 128, 128, 0, s>>>(partials, nctas, nvals, out, batch);
  note_launch();
  return cudaGetLastError();
}

}  // namespace jfli
