// Particle <-> mesh kernels: CIC paint, CIC readout, the fused particle update of one
// PM step (FD-gradient readout + kick + drift + paint), and the grid-point kernels of LPT.
//
// CIC follows JaxPM `cic_paint_dx` / `cic_read_dx` (reference call sites
// _src/fields/_painting.py:67 and fields/particles.py:203): a particle at grid point
// (i,j,k) with displacement d deposits onto the 8 cells around (i,j,k)+d with weights
// prod_a (1 - |pos_a - cell_a|), periodic wrap. The integer and fractional parts of
// the displacement are split before they are added to the grid index, so the weights
// keep full FP32 precision at any mesh size.
//
// The force is F = -D(pot), D the 4-point finite difference
//   D f(c) = [8 (f(c+1) - f(c-1)) - (f(c+2) - f(c-2))] / 12,
// whose Fourier eigenvalue i (8 sin k - sin 2k) / 6 is JaxPM's `gradient_kernel`;
// applying it in real space at the 8 CIC corners equals the k-space gradient followed
// by an inverse FFT per component (reference pm/solvers.py:19-32 -> pm_forces).
#include "common.cuh"
#include "internal.h"

namespace jfli {

struct Cic1 {
  int i0, i1;
  float w0, w1;
};

// Relative mode: grid index g plus displacement d.
__device__ __forceinline__ Cic1 cic_rel(int g, float d, int n) {
  const float f = floorf(d);
  const float t = d - f;
  Cic1 c;
  c.w0 = 1.0f - t;
  c.w1 = t;
  c.i0 = wrap_index(g + (int)f, n);
  c.i1 = (c.i0 + 1 == n) ? 0 : c.i0 + 1;
  return c;
}

// Absolute mode: position in grid units.
__device__ __forceinline__ Cic1 cic_abs(float p, int n) {
  const float f = floorf(p);
  const float t = p - f;
  Cic1 c;
  c.w0 = 1.0f - t;
  c.w1 = t;
  c.i0 = wrap_index((int)f, n);
  c.i1 = (c.i0 + 1 == n) ? 0 : c.i0 + 1;
  return c;
}

__device__ __forceinline__ void particle_grid(long long p, int ny, int nz, int& i, int& j, int& k) {
  const long long yz = (long long)ny * nz;
  i = (int)(p / yz);
  const long long r = p - (long long)i * yz;
  j = (int)(r / nz);
  k = (int)(r - (long long)j * nz);
}

__device__ __forceinline__ void cic_setup(const float* pos3, long long p, int absolute, const MeshDims& d, Cic1& cx,
                                          Cic1& cy, Cic1& cz) {
  const float px = pos3[0], py = pos3[1], pz = pos3[2];
  if (absolute) {
    cx = cic_abs(px, d.nx);
    cy = cic_abs(py, d.ny);
    cz = cic_abs(pz, d.nz);
  } else {
    int i, j, k;
    particle_grid(p, d.ny, d.nz, i, j, k);
    cx = cic_rel(i, px, d.nx);
    cy = cic_rel(j, py, d.ny);
    cz = cic_rel(k, pz, d.nz);
  }
}

__device__ __forceinline__ long long cell(const MeshDims& d, int x, int y, int z) {
  return ((long long)x * d.ny + y) * d.nz + z;
}

__device__ __forceinline__ void deposit(float* mesh, const MeshDims& d, const Cic1& cx, const Cic1& cy,
                                        const Cic1& cz, float w) {
  const float wx[2] = {cx.w0, cx.w1}, wy[2] = {cy.w0, cy.w1}, wz[2] = {cz.w0, cz.w1};
  const int ix[2] = {cx.i0, cx.i1}, iy[2] = {cy.i0, cy.i1}, iz[2] = {cz.i0, cz.i1};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int c = 0; c < 2; ++c) atomicAdd(mesh + cell(d, ix[a], iy[b], iz[c]), wx[a] * wy[b] * wz[c] * w);
}

__device__ __forceinline__ float gather(const float* __restrict__ mesh, const MeshDims& d, const Cic1& cx,
                                        const Cic1& cy, const Cic1& cz) {
  const float wx[2] = {cx.w0, cx.w1}, wy[2] = {cy.w0, cy.w1}, wz[2] = {cz.w0, cz.w1};
  const int ix[2] = {cx.i0, cx.i1}, iy[2] = {cy.i0, cy.i1}, iz[2] = {cz.i0, cz.i1};
  float acc = 0.f;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int c = 0; c < 2; ++c) acc += mesh[cell(d, ix[a], iy[b], iz[c])] * (wx[a] * wy[b] * wz[c]);
  return acc;
}

// -F = D(pot) at both CIC corners of one line: values v[0..5] = pot at i0-2 .. i0+3.
__device__ __forceinline__ void fd_pair(const float* v, float& g0, float& g1) {
  const float s = 1.0f / 12.0f;
  g0 = (8.0f * (v[3] - v[1]) - (v[4] - v[0])) * s;
  g1 = (8.0f * (v[4] - v[2]) - (v[5] - v[1])) * s;
}

// F = -grad_FD(pot) read out with CIC weights at one particle (56 distinct loads).
__device__ __forceinline__ void gather_force(const float* __restrict__ pot, const MeshDims& d, const Cic1& cx,
                                             const Cic1& cy, const Cic1& cz, float& fx, float& fy, float& fz) {
  const int x[6] = {wrap_index(cx.i0 - 2, d.nx), wrap_index(cx.i0 - 1, d.nx), cx.i0, cx.i1,
                    wrap_index(cx.i0 + 2, d.nx), wrap_index(cx.i0 + 3, d.nx)};
  const int y[6] = {wrap_index(cy.i0 - 2, d.ny), wrap_index(cy.i0 - 1, d.ny), cy.i0, cy.i1,
                    wrap_index(cy.i0 + 2, d.ny), wrap_index(cy.i0 + 3, d.ny)};
  const int z[6] = {wrap_index(cz.i0 - 2, d.nz), wrap_index(cz.i0 - 1, d.nz), cz.i0, cz.i1,
                    wrap_index(cz.i0 + 2, d.nz), wrap_index(cz.i0 + 3, d.nz)};
  const float wx[2] = {cx.w0, cx.w1}, wy[2] = {cy.w0, cy.w1}, wz[2] = {cz.w0, cz.w1};
  float c[2][2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) c[a][b][e] = __ldg(pot + cell(d, x[2 + a], y[2 + b], z[2 + e]));
  float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int e = 0; e < 2; ++e) {  // x lines
      float v[6];
      v[0] = __ldg(pot + cell(d, x[0], y[2 + b], z[2 + e]));
      v[1] = __ldg(pot + cell(d, x[1], y[2 + b], z[2 + e]));
      v[2] = c[0][b][e];
      v[3] = c[1][b][e];
      v[4] = __ldg(pot + cell(d, x[4], y[2 + b], z[2 + e]));
      v[5] = __ldg(pot + cell(d, x[5], y[2 + b], z[2 + e]));
      float g0, g1;
      fd_pair(v, g0, g1);
      gx += wy[b] * wz[e] * (wx[0] * g0 + wx[1] * g1);
    }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int e = 0; e < 2; ++e) {  // y lines
      float v[6];
      v[0] = __ldg(pot + cell(d, x[2 + a], y[0], z[2 + e]));
      v[1] = __ldg(pot + cell(d, x[2 + a], y[1], z[2 + e]));
      v[2] = c[a][0][e];
      v[3] = c[a][1][e];
      v[4] = __ldg(pot + cell(d, x[2 + a], y[4], z[2 + e]));
      v[5] = __ldg(pot + cell(d, x[2 + a], y[5], z[2 + e]));
      float g0, g1;
      fd_pair(v, g0, g1);
      gy += wx[a] * wz[e] * (wy[0] * g0 + wy[1] * g1);
    }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {  // z lines
      float v[6];
      v[0] = __ldg(pot + cell(d, x[2 + a], y[2 + b], z[0]));
      v[1] = __ldg(pot + cell(d, x[2 + a], y[2 + b], z[1]));
      v[2] = c[a][b][0];
      v[3] = c[a][b][1];
      v[4] = __ldg(pot + cell(d, x[2 + a], y[2 + b], z[4]));
      v[5] = __ldg(pot + cell(d, x[2 + a], y[2 + b], z[5]));
      float g0, g1;
      fd_pair(v, g0, g1);
      gz += wx[a] * wy[b] * (wz[0] * g0 + wz[1] * g1);
    }
  fx = -gx;
  fy = -gy;
  fz = -gz;
}

// ----------------------------------------------------------------------------------
__global__ void k_paint(const float* __restrict__ pos, int absolute, const float* __restrict__ weights, float weight,
                        float* __restrict__ mesh, MeshDims d) {
  const long long np = d.cells();
  const int b = blockIdx.y;
  pos += (long long)b * np * 3;
  mesh += (long long)b * np;
  if (weights) weights += (long long)b * np;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    Cic1 cx, cy, cz;
    cic_setup(pos + 3 * p, p, absolute, d, cx, cy, cz);
    const float w = weights ? weights[p] * weight : weight;
    deposit(mesh, d, cx, cy, cz, w);
  }
}

__global__ void k_readout(const float* __restrict__ pos, int absolute, const float* __restrict__ mesh,
                          float* __restrict__ out, MeshDims d) {
  const long long np = d.cells();
  const int b = blockIdx.y;
  pos += (long long)b * np * 3;
  mesh += (long long)b * np;
  out += (long long)b * np;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    Cic1 cx, cy, cz;
    cic_setup(pos + 3 * p, p, absolute, d, cx, cy, cz);
    out[p] = gather(mesh, d, cx, cy, cz);
  }
}

__global__ void k_readout_gradient(const float* __restrict__ pos, int absolute, const float* __restrict__ pot,
                                   float* __restrict__ out, float scale, MeshDims d) {
  const long long np = d.cells();
  const int b = blockIdx.y;
  pos += (long long)b * np * 3;
  pot += (long long)b * np;
  out += (long long)b * np * 3;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    Cic1 cx, cy, cz;
    cic_setup(pos + 3 * p, p, absolute, d, cx, cy, cz);
    float fx, fy, fz;
    gather_force(pot, d, cx, cy, cz, fx, fy, fz);
    out[3 * p + 0] = fx * scale;
    out[3 * p + 1] = fy * scale;
    out[3 * p + 2] = fz * scale;
  }
}

// One fused particle pass of a PM step. Order inside: kick (with the force at the
// current position) -> drift (with the kicked velocity) -> paint (at the new position).
__global__ void k_kick_drift_paint(float* __restrict__ disp, float* __restrict__ vel, const float* __restrict__ pot,
                                   float kick, float drift, int flags, float weight, float* __restrict__ rho,
                                   MeshDims d) {
  const long long np = d.cells();
  const int b = blockIdx.y;
  disp += (long long)b * np * 3;
  vel += (long long)b * np * 3;
  if (pot) pot += (long long)b * np;
  if (rho) rho += (long long)b * np;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    particle_grid(p, d.ny, d.nz, i, j, k);
    float x0 = disp[3 * p + 0], x1 = disp[3 * p + 1], x2 = disp[3 * p + 2];
    if (flags & (kStepKick | kStepCorrect)) {
      const Cic1 cx = cic_rel(i, x0, d.nx), cy = cic_rel(j, x1, d.ny), cz = cic_rel(k, x2, d.nz);
      float fx, fy, fz;
      gather_force(pot, d, cx, cy, cz, fx, fy, fz);
      if (flags & kStepKick) {
        vel[3 * p + 0] += fx * kick;
        vel[3 * p + 1] += fy * kick;
        vel[3 * p + 2] += fz * kick;
      } else {
        x0 += fx * kick;
        x1 += fy * kick;
        x2 += fz * kick;
      }
    }
    if (flags & kStepDrift) {
      x0 += vel[3 * p + 0] * drift;
      x1 += vel[3 * p + 1] * drift;
      x2 += vel[3 * p + 2] * drift;
    }
    if (flags & (kStepDrift | kStepCorrect)) {
      disp[3 * p + 0] = x0;
      disp[3 * p + 1] = x1;
      disp[3 * p + 2] = x2;
    }
    if (flags & kStepPaint) {
      const Cic1 cx = cic_rel(i, x0, d.nx), cy = cic_rel(j, x1, d.ny), cz = cic_rel(k, x2, d.nz);
      deposit(rho, d, cx, cy, cz, weight);
    }
  }
}

// F = scale * (-D pot) at every grid point (particles exactly on the grid), optionally
// accumulated into `out` (AoS [..,3]).
__global__ void k_grid_gradient(const float* __restrict__ pot, float* __restrict__ out, float scale, int accumulate,
                                MeshDims d) {
  const long long np = d.cells();
  const int b = blockIdx.y;
  pot += (long long)b * np;
  out += (long long)b * np * 3;
  const float s = 1.0f / 12.0f;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    particle_grid(p, d.ny, d.nz, i, j, k);
    float g[3];
    {
      const float a = pot[cell(d, wrap_index(i + 1, d.nx), j, k)], bm = pot[cell(d, wrap_index(i - 1, d.nx), j, k)];
      const float c = pot[cell(d, wrap_index(i + 2, d.nx), j, k)], e = pot[cell(d, wrap_index(i - 2, d.nx), j, k)];
      g[0] = -(8.0f * (a - bm) - (c - e)) * s;
    }
    {
      const float a = pot[cell(d, i, wrap_index(j + 1, d.ny), k)], bm = pot[cell(d, i, wrap_index(j - 1, d.ny), k)];
      const float c = pot[cell(d, i, wrap_index(j + 2, d.ny), k)], e = pot[cell(d, i, wrap_index(j - 2, d.ny), k)];
      g[1] = -(8.0f * (a - bm) - (c - e)) * s;
    }
    {
      const float a = pot[cell(d, i, j, wrap_index(k + 1, d.nz))], bm = pot[cell(d, i, j, wrap_index(k - 1, d.nz))];
      const float c = pot[cell(d, i, j, wrap_index(k + 2, d.nz))], e = pot[cell(d, i, j, wrap_index(k - 2, d.nz))];
      g[2] = -(8.0f * (a - bm) - (c - e)) * s;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float v = g[a] * scale;
      out[3 * p + a] = accumulate ? out[3 * p + a] + v : v;
    }
  }
}

// Second-order LPT source from the first-order potential (JaxPM `lpt`, order 2):
//   delta2 = sum_{i<j} phi_ii phi_jj - phi_ij^2,  phi_ij = D_i D_j phi,
// with D the same 4-point finite difference (its square is the k-space product
// gradient_kernel_i * gradient_kernel_j used by the reference).
__constant__ float c_d5[5] = {1.0f / 12.0f, -8.0f / 12.0f, 0.0f, 8.0f / 12.0f, -1.0f / 12.0f};

__global__ void k_lpt2_source(const float* __restrict__ pot, float* __restrict__ out, MeshDims d) {
  const long long np = d.cells();
  const int b = blockIdx.y;
  pot += (long long)b * np;
  out += (long long)b * np;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    particle_grid(p, d.ny, d.nz, i, j, k);
    float h[3][3];
    // diagonal: D_a D_a
    for (int a = 0; a < 3; ++a) {
      float acc = 0.f;
      for (int s = 0; s < 5; ++s) {
        if (s == 2) continue;
        for (int t = 0; t < 5; ++t) {
          if (t == 2) continue;
          const int off = (s - 2) + (t - 2);
          const int ii = a == 0 ? wrap_index(i + off, d.nx) : i;
          const int jj = a == 1 ? wrap_index(j + off, d.ny) : j;
          const int kk = a == 2 ? wrap_index(k + off, d.nz) : k;
          acc += c_d5[s] * c_d5[t] * pot[cell(d, ii, jj, kk)];
        }
      }
      h[a][a] = acc;
    }
    // off-diagonal: D_a D_b
    for (int a = 0; a < 3; ++a)
      for (int bb = a + 1; bb < 3; ++bb) {
        float acc = 0.f;
        for (int s = 0; s < 5; ++s) {
          if (s == 2) continue;
          for (int t = 0; t < 5; ++t) {
            if (t == 2) continue;
            int o[3] = {0, 0, 0};
            o[a] = s - 2;
            o[bb] = t - 2;
            acc += c_d5[s] * c_d5[t] *
                   pot[cell(d, wrap_index(i + o[0], d.nx), wrap_index(j + o[1], d.ny), wrap_index(k + o[2], d.nz))];
          }
        }
        h[a][bb] = acc;
      }
    // accumulate in the reference's loop order
    float delta2 = 0.f, acc_diag = 0.f;
    for (int a = 0; a < 3; ++a) {
      delta2 += h[a][a] * acc_diag;
      acc_diag += h[a][a];
      for (int bb = a + 1; bb < 3; ++bb) delta2 -= h[a][bb] * h[a][bb];
    }
    out[p] = delta2;
  }
}

__global__ void k_lpt_combine(const float* __restrict__ f1, const float* __restrict__ f2, float c1x, float c2x,
                              float c1p, float c2p, float* __restrict__ dx, float* __restrict__ pv, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const float a = f1[q];
    const float b = f2 ? f2[q] : 0.f;
    float x = c1x * a;
    float v = c1p * x;
    if (f2) {
      const float x2 = c2x * b;
      x += x2;
      v += c2p * x2;
    }
    dx[q] = x;
    pv[q] = v;
  }
}

__global__ void k_axpy(float* __restrict__ y, const float* __restrict__ x, float a, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    y[q] += a * x[q];
}

// ----------------------------------------------------------------------------------
static int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

static dim3 particle_grid_dims(long long np, int batch, int threads, int per_sm) {
  long long blocks = (np + threads - 1) / threads;
  const long long cap = (long long)sm_count() * per_sm;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return dim3((unsigned)blocks, batch);
}

cudaError_t cic_paint(const float* pos, int absolute, const float* weights, float weight, float* mesh,
                      const MeshDims& d, cudaStream_t s) {
  k_paint<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pos, absolute, weights, weight, mesh, d);
  note_launch();
  return cudaGetLastError();
}

cudaError_t cic_readout(const float* pos, int absolute, const float* mesh, float* out, const MeshDims& d,
                        cudaStream_t s) {
  k_readout<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pos, absolute, mesh, out, d);
  note_launch();
  return cudaGetLastError();
}

cudaError_t cic_readout_gradient(const float* pos, int absolute, const float* pot, float* out, float scale,
                                 const MeshDims& d, cudaStream_t s) {
  k_readout_gradient<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pos, absolute, pot, out, scale,
                                                                                     d);
  note_launch();
  return cudaGetLastError();
}

cudaError_t kick_drift_paint(float* disp, float* vel, const float* pot, float kick, float drift, int flags,
                             float weight, float* rho, const MeshDims& d, cudaStream_t s) {
  k_kick_drift_paint<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(disp, vel, pot, kick, drift,
                                                                                     flags, weight, rho, d);
  note_launch();
  return cudaGetLastError();
}

cudaError_t grid_gradient(const float* pot, float* out, float scale, int accumulate, const MeshDims& d,
                          cudaStream_t s) {
  k_grid_gradient<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pot, out, scale, accumulate, d);
  note_launch();
  return cudaGetLastError();
}

cudaError_t lpt2_source(const float* pot, float* out, const MeshDims& d, cudaStream_t s) {
  k_lpt2_source<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pot, out, d);
  note_launch();
  return cudaGetLastError();
}

cudaError_t lpt_combine(const float* f1, const float* f2, float c1x, float c2x, float c1p, float c2p, float* dx,
                        float* p, const MeshDims& d, cudaStream_t s) {
  const long long n = d.cells() * 3 * d.batch;
  k_lpt_combine<<<particle_grid_dims(n, 1, 256, 16), 256, 0, s>>>(f1, f2, c1x, c2x, c1p, c2p, dx, p, n);
  note_launch();
  return cudaGetLastError();
}

cudaError_t axpy_particles(float* y, const float* x, float a, const MeshDims& d, cudaStream_t s) {
  const long long n = d.cells() * 3 * d.batch;
  k_axpy<<<particle_grid_dims(n, 1, 256, 16), 256, 0, s>>>(y, x, a, n);
  note_launch();
  return cudaGetLastError();
}

}  // namespace jfli
