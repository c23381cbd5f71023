// CIC building blocks shared by the particle kernels (cic.cu) and their adjoints
// (adjoint.cu): per-axis cell/weight pairs, the particle grid with fast index
// decomposition, deposit (paint) and gather (readout) of one particle, and the launch
// shape of the grid-stride particle loops.
#pragma once

#include "common.cuh"
#include "internal.h"

namespace jfli {

struct Cic1 {
  int i0, i1;
  float w0, w1;
};

// Particle grid with fast index decomposition; cells < 2^31 so offsets are 32-bit.
struct PGrid {
  int nx, ny, nz, yz;
  unsigned np;
  FastDiv dyz, dz;
};

inline PGrid make_pgrid(const MeshDims& d) {
  PGrid g;
  g.nx = d.nx;
  g.ny = d.ny;
  g.nz = d.nz;
  g.yz = d.ny * d.nz;
  g.np = (unsigned)d.cells();
  g.dyz = FastDiv::make((unsigned)g.yz);
  g.dz = FastDiv::make((unsigned)d.nz);
  return g;
}

__device__ __forceinline__ void particle_ijk(const PGrid& g, unsigned p, int& i, int& j, int& k) {
  const unsigned ii = g.dyz.div(p);
  const unsigned r = p - ii * (unsigned)g.yz;
  const unsigned jj = g.dz.div(r);
  i = (int)ii;
  j = (int)jj;
  k = (int)(r - jj * (unsigned)g.nz);
}

// Relative mode: grid index g plus displacement d (integer part split off first).
__device__ __forceinline__ Cic1 cic_rel(int gidx, float d, int n) {
  const float f = floorf(d);
  Cic1 c;
  c.w1 = d - f;
  c.w0 = 1.0f - c.w1;
  int i = gidx + (int)f;
  if ((unsigned)i >= (unsigned)n) i = wrap_index(i, n);
  c.i0 = i;
  c.i1 = (i + 1 == n) ? 0 : i + 1;
  return c;
}

// Absolute mode: position in grid units.
__device__ __forceinline__ Cic1 cic_abs(float p, int n) {
  const float f = floorf(p);
  Cic1 c;
  c.w1 = p - f;
  c.w0 = 1.0f - c.w1;
  int i = (int)f;
  if ((unsigned)i >= (unsigned)n) i = wrap_index(i, n);
  c.i0 = i;
  c.i1 = (i + 1 == n) ? 0 : i + 1;
  return c;
}

__device__ __forceinline__ void cic_setup(const float* pos3, unsigned p, int absolute, const PGrid& g, Cic1& cx,
                                          Cic1& cy, Cic1& cz) {
  const float px = pos3[0], py = pos3[1], pz = pos3[2];
  if (absolute) {
    cx = cic_abs(px, g.nx);
    cy = cic_abs(py, g.ny);
    cz = cic_abs(pz, g.nz);
  } else {
    int i, j, k;
    particle_ijk(g, p, i, j, k);
    cx = cic_rel(i, px, g.nx);
    cy = cic_rel(j, py, g.ny);
    cz = cic_rel(k, pz, g.nz);
  }
}

__device__ __forceinline__ void deposit(float* mesh, const PGrid& g, const Cic1& cx, const Cic1& cy, const Cic1& cz,
                                        float w) {
  const int xo[2] = {cx.i0 * g.yz, cx.i1 * g.yz}, yo[2] = {cy.i0 * g.nz, cy.i1 * g.nz}, zo[2] = {cz.i0, cz.i1};
  const float wx[2] = {cx.w0 * w, cx.w1 * w}, wy[2] = {cy.w0, cy.w1}, wz[2] = {cz.w0, cz.w1};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const float wab = wx[a] * wy[b];
#pragma unroll
      for (int c = 0; c < 2; ++c) atomicAdd(mesh + (xo[a] + yo[b] + zo[c]), wab * wz[c]);
    }
}

// CIC deposit for lanes that hold consecutive particles of one z row (the grid-stride
// particle loops: lane L has particle p, lane L+1 particle p+1). When lane L's upper-z
// corners are lane L+1's lower-z corners (same x and y cells, next z cell: neighbouring
// particles that moved together), lane L hands its four upper-z weights to lane L+1 with
// a shuffle and lane L+1 adds them to its own lower-z deposits, so that pair of cells
// takes one atomic instead of two. The sums reaching each cell are the same as with
// deposit(); only the FP32 addition order differs. The active lanes of a warp must be a
// prefix of it, which holds for the grid-stride loops (the last iteration drops lanes
// from the top).
__device__ __forceinline__ void deposit_lane_merged(float* mesh, const PGrid& g, const Cic1& cx, const Cic1& cy,
                                                    const Cic1& cz, float w) {
  const unsigned mask = __activemask();
  const int lane = threadIdx.x & 31;
  const int xy0 = cx.i0 * g.yz + cy.i0 * g.nz;
  const int lo = xy0 + cz.i0;  // my lower-z corner at (x0, y0)
  const int hi = xy0 + cz.i1;  // my upper-z corner at (x0, y0)
  const int next_lo = __shfl_down_sync(mask, lo, 1);
  const int prev_hi = __shfl_up_sync(mask, hi, 1);
  const bool give = lane < 31 && ((mask >> (lane + 1)) & 1u) && next_lo == hi;
  const bool take = lane > 0 && ((mask >> (lane - 1)) & 1u) && prev_hi == lo;
  const int xo[2] = {cx.i0 * g.yz, cx.i1 * g.yz}, yo[2] = {cy.i0 * g.nz, cy.i1 * g.nz};
  const float wx[2] = {cx.w0 * w, cx.w1 * w}, wy[2] = {cy.w0, cy.w1};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const float wab = wx[a] * wy[b];
      const float up = wab * cz.w1;
      const float recv = __shfl_up_sync(mask, up, 1);
      const float low = wab * cz.w0 + (take ? recv : 0.f);
      atomicAdd(mesh + (xo[a] + yo[b] + cz.i0), low);
      if (!give) atomicAdd(mesh + (xo[a] + yo[b] + cz.i1), up);
    }
}

__device__ __forceinline__ float gather(const float* __restrict__ mesh, const PGrid& g, const Cic1& cx,
                                        const Cic1& cy, const Cic1& cz) {
  const int xo[2] = {cx.i0 * g.yz, cx.i1 * g.yz}, yo[2] = {cy.i0 * g.nz, cy.i1 * g.nz}, zo[2] = {cz.i0, cz.i1};
  const float wx[2] = {cx.w0, cx.w1}, wy[2] = {cy.w0, cy.w1}, wz[2] = {cz.w0, cz.w1};
  float acc = 0.f;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int c = 0; c < 2; ++c) acc += __ldg(mesh + (xo[a] + yo[b] + zo[c])) * (wx[a] * wy[b] * wz[c]);
  return acc;
}

// CIC readout of the force mesh at one particle. The force mesh is AoS float4
// [nx][ny][nz] = (Fx, Fy, Fz, 0): one 16-byte load per CIC corner.
__device__ __forceinline__ void gather_force_mesh(const float* __restrict__ F, const PGrid& g, const Cic1& cx,
                                                  const Cic1& cy, const Cic1& cz, float& fx, float& fy, float& fz) {
  const float4* F4 = reinterpret_cast<const float4*>(F);
  const int xo[2] = {cx.i0 * g.yz, cx.i1 * g.yz}, yo[2] = {cy.i0 * g.nz, cy.i1 * g.nz}, zo[2] = {cz.i0, cz.i1};
  const float wx[2] = {cx.w0, cx.w1}, wy[2] = {cy.w0, cy.w1}, wz[2] = {cz.w0, cz.w1};
  float ax = 0.f, ay = 0.f, az = 0.f;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const float wab = wx[a] * wy[b];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const float4 f = __ldg(F4 + (xo[a] + yo[b] + zo[c]));
        const float w = wab * wz[c];
        ax += f.x * w;
        ay += f.y * w;
        az += f.z * w;
      }
    }
  fx = ax;
  fy = ay;
  fz = az;
}

inline int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Depth (x planes per chunk) of the 8 (y) x 32 (z) brick walks of the particle kernels: the
// deepest of 16, 8, 4, 2, 1 planes that still gives `min_ctas` bricks over the batch, so
// that a small mesh run alone still spreads over the GPU (64^3 at 16 planes is 64 bricks).
inline int brick_xdepth(int nx, int ny, int nz, int batch, long long min_ctas) {
  const long long rows = (long long)(ny / 8) * (nz / 32) * batch;
  int depth = 16;
  while (depth > 1 && rows * ((nx + depth - 1) / depth) < min_ctas) depth >>= 1;
  return depth;
}

inline dim3 particle_grid_dims(long long np, int batch, int threads, int per_sm) {
  long long blocks = (np + threads - 1) / threads;
  const long long cap = (long long)sm_count() * per_sm;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return dim3((unsigned)blocks, batch);
}

}  // namespace jfli
