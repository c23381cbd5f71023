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
#include <cmath>

#include "common.cuh"
#include "fft_engine.cuh"
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

static cudaError_t launch_rfft_z(const float* in, float2* out, const MeshDims& d, float sub, cudaStream_t s) {
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
  return cudaGetLastError();
}

static cudaError_t launch_irfft_z(const float2* in, float* out, const MeshDims& d, float scale, cudaStream_t s) {
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
  FftPlan pl;
  make_fft_plan(g.n, &pl);
  const size_t smem = ((size_t)2 * g.n * g.w + g.n) * sizeof(float2);
  dim3 grid((g.ncols + g.w - 1) / g.w, batch);
  cudaFuncSetAttribute(k_fft_cols<SIGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_fft_cols<SIGN><<<grid, kFftThreads, smem, s>>>(data, g, pl, bstride);
  note_launch();
  return cudaGetLastError();
}

template <class Op>
static cudaError_t launch_x_op(float2* data, const MeshDims& d, const Op& op, cudaStream_t s) {
  const ColGeom g = x_geom(d);
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
  return (g.ncols + g.w - 1) / g.w;
}

cudaError_t rfft3d_forward(const float* in, float2* spec, const MeshDims& d, float sub, cudaStream_t s) {
  cudaError_t e = launch_rfft_z(in, spec, d, sub, s);
  if (e != cudaSuccess) return e;
  e = launch_cols<-1>(spec, y_geom(d), d.spec_elems(), d.batch, s);
  if (e != cudaSuccess) return e;
  return launch_cols<-1>(spec, x_geom(d), d.spec_elems(), d.batch, s);
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
                                cudaStream_t s) {
  cudaError_t e = launch_rfft_z(in, spec, d, sub, s);
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
                              float scale, cudaStream_t s) {
  PoissonOp op;
  op.nx = d.nx;
  op.ny = d.ny;
  op.nz = d.nz;
  op.norm = scale / ((float)d.nx * (float)d.ny * (float)d.nz);
  return filter_chain(rho, spec, pot, d, rho_mean, op, s);
}

cudaError_t pgd_potential(const float* rho, float2* spec, float* pot, const MeshDims& d, float rho_mean, float kl,
                          float ks, float scale, cudaStream_t s) {
  PgdOp op;
  op.nx = d.nx;
  op.ny = d.ny;
  op.nz = d.nz;
  op.norm = scale / ((float)d.nx * (float)d.ny * (float)d.nz);
  op.kl2 = kl * kl;
  op.ks4 = ks * ks * ks * ks;
  return filter_chain(rho, spec, pot, d, rho_mean, op, s);
}

cudaError_t ic_filter(const float* noise, float2* spec, float* out, const MeshDims& d, const float* ktab,
                      const float* ptab, int ntab, const float* box, int zero_mode_one, cudaStream_t s) {
  IcOp op;
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

}  // namespace jfli
