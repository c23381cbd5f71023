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
#include "cic.cuh"
#include "common.cuh"
#include "internal.h"

namespace jfli {

// -F = D(pot) at both CIC corners of one line: values v[0..5] = pot at i0-2 .. i0+3.
__device__ __forceinline__ void fd_pair(const float* v, float& g0, float& g1) {
  const float s = 1.0f / 12.0f;
  g0 = (8.0f * (v[3] - v[1]) - (v[4] - v[0])) * s;
  g1 = (8.0f * (v[4] - v[2]) - (v[5] - v[1])) * s;
}

// F = -grad_FD(pot) read out with CIC weights at one particle (56 distinct loads).
// Needs every axis >= 4 cells (offsets -2..+3 wrap at most once).
__device__ __forceinline__ void gather_force(const float* __restrict__ pot, const PGrid& g, const Cic1& cx,
                                             const Cic1& cy, const Cic1& cz, float& fx, float& fy, float& fz) {
  int x[6], y[6], z[6];
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    x[s] = wrap1(cx.i0 + s - 2, g.nx) * g.yz;
    y[s] = wrap1(cy.i0 + s - 2, g.ny) * g.nz;
    z[s] = wrap1(cz.i0 + s - 2, g.nz);
  }
  const float wx[2] = {cx.w0, cx.w1}, wy[2] = {cy.w0, cy.w1}, wz[2] = {cz.w0, cz.w1};
  float c[2][2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) c[a][b][e] = __ldg(pot + (x[2 + a] + y[2 + b] + z[2 + e]));
  float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int e = 0; e < 2; ++e) {  // x lines
      const int o = y[2 + b] + z[2 + e];
      float v[6];
      v[0] = __ldg(pot + (x[0] + o));
      v[1] = __ldg(pot + (x[1] + o));
      v[2] = c[0][b][e];
      v[3] = c[1][b][e];
      v[4] = __ldg(pot + (x[4] + o));
      v[5] = __ldg(pot + (x[5] + o));
      float g0, g1;
      fd_pair(v, g0, g1);
      gx += wy[b] * wz[e] * (wx[0] * g0 + wx[1] * g1);
    }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int e = 0; e < 2; ++e) {  // y lines
      const int o = x[2 + a] + z[2 + e];
      float v[6];
      v[0] = __ldg(pot + (y[0] + o));
      v[1] = __ldg(pot + (y[1] + o));
      v[2] = c[a][0][e];
      v[3] = c[a][1][e];
      v[4] = __ldg(pot + (y[4] + o));
      v[5] = __ldg(pot + (y[5] + o));
      float g0, g1;
      fd_pair(v, g0, g1);
      gy += wx[a] * wz[e] * (wy[0] * g0 + wy[1] * g1);
    }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {  // z lines
      const int o = x[2 + a] + y[2 + b];
      float v[6];
      v[0] = __ldg(pot + (z[0] + o));
      v[1] = __ldg(pot + (z[1] + o));
      v[2] = c[a][b][0];
      v[3] = c[a][b][1];
      v[4] = __ldg(pot + (z[4] + o));
      v[5] = __ldg(pot + (z[5] + o));
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
                        float* __restrict__ mesh, PGrid g) {
  const long long b = blockIdx.y;
  pos += b * g.np * 3;
  mesh += b * g.np;
  if (weights) weights += b * g.np;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    Cic1 cx, cy, cz;
    cic_setup(pos + 3ull * p, p, absolute, g, cx, cy, cz);
    const float w = weights ? weights[p] * weight : weight;
    deposit_lane_merged(mesh, g, cx, cy, cz, w);
  }
}

__global__ void k_readout(const float* __restrict__ pos, int absolute, const float* __restrict__ mesh,
                          float* __restrict__ out, PGrid g) {
  const long long b = blockIdx.y;
  pos += b * g.np * 3;
  mesh += b * g.np;
  out += b * g.np;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    Cic1 cx, cy, cz;
    cic_setup(pos + 3ull * p, p, absolute, g, cx, cy, cz);
    out[p] = gather(mesh, g, cx, cy, cz);
  }
}

__global__ void k_readout_gradient(const float* __restrict__ pos, int absolute, const float* __restrict__ pot,
                                   float* __restrict__ out, float scale, PGrid g) {
  const long long b = blockIdx.y;
  pos += b * g.np * 3;
  pot += b * g.np;
  out += b * g.np * 3;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    Cic1 cx, cy, cz;
    cic_setup(pos + 3ull * p, p, absolute, g, cx, cy, cz);
    float fx, fy, fz;
    gather_force(pot, g, cx, cy, cz, fx, fy, fz);
    out[3 * p + 0] = fx * scale;
    out[3 * p + 1] = fy * scale;
    out[3 * p + 2] = fz * scale;
  }
}

// The upper-x corners (x plane cx.i1) of a lane's previous particle in the brick walk,
// held back in registers: when the lane's next particle, one Lagrangian plane further in
// x, has its lower-x corners in the same four cells (neighbours that moved together), the
// two deposits are added before one atomic each, so a plane of cells takes one set of
// atomics instead of two.
struct XCarry {
  int xo, yo0, yo1, z0, z1;  // cell offsets of the 2 (y) x 2 (z) corners: x ny nz, y nz, z
  float w00, w01, w10, w11;  // weights [y][z]
  bool valid;
};

// Deposit, for every lane of a full warp, the 2 (y) x 2 (z) corners of one x plane, with
// the z lane merge of deposit_lane_merged: when lane L's upper-z pair of cells is lane
// L+1's lower-z pair (same x and y cells, next z cell), lane L hands its two upper-z
// weights to lane L+1, which adds them to its own lower-z deposits. Lanes with `on` false
// deposit nothing and take part in no merge. Cell offsets are unique per cell, so equal
// offsets mean equal cells.
__device__ __forceinline__ void deposit_plane_merged(float* rho, bool on, int xo, int yo0, int yo1, int z0, int z1,
                                                     float w00, float w01, float w10, float w11) {
  const int lane = threadIdx.x & 31;
  const int lo = on ? xo + yo0 + z0 : -1;
  const int hi = on ? xo + yo0 + z1 : -2;
  const int next_lo = __shfl_down_sync(0xffffffffu, lo, 1);
  const int prev_hi = __shfl_up_sync(0xffffffffu, hi, 1);
  const bool give = on && lane < 31 && next_lo == hi;
  const bool take = on && lane > 0 && prev_hi == lo;
  const float r0 = __shfl_up_sync(0xffffffffu, w01, 1);
  const float r1 = __shfl_up_sync(0xffffffffu, w11, 1);
  if (on) {
    atomicAdd(rho + (xo + yo0 + z0), take ? w00 + r0 : w00);
    atomicAdd(rho + (xo + yo1 + z0), take ? w10 + r1 : w10);
    if (!give) {
      atomicAdd(rho + (xo + yo0 + z1), w01);
      atomicAdd(rho + (xo + yo1 + z1), w11);
    }
  }
}

__device__ __forceinline__ void carry_flush(float* rho, XCarry& c) {
  atomicAdd(rho + (c.xo + c.yo0 + c.z0), c.w00);
  atomicAdd(rho + (c.xo + c.yo0 + c.z1), c.w01);
  atomicAdd(rho + (c.xo + c.yo1 + c.z0), c.w10);
  atomicAdd(rho + (c.xo + c.yo1 + c.z1), c.w11);
  c.valid = false;
}

// CIC deposit of one particle in the brick walk (full warps, lanes on consecutive z
// particles of one row, successive calls of a lane on successive x planes): the lower-x
// plane is deposited now, with the carried upper-x plane of the lane's previous particle
// added when the cells are the same (otherwise the carry is deposited on its own first),
// and the upper-x plane becomes the new carry. The sums reaching each cell are those of
// deposit(); only the FP32 addition order differs.
__device__ __forceinline__ void deposit_carried(float* rho, const PGrid& g, const Cic1& cx, const Cic1& cy,
                                                const Cic1& cz, float w, XCarry& c) {
  const float wx0 = cx.w0 * w, wx1 = cx.w1 * w;
  const int xo0 = cx.i0 * g.yz, yo0 = cy.i0 * g.nz, yo1 = cy.i1 * g.nz;
  float a00 = (wx0 * cy.w0) * cz.w0, a01 = (wx0 * cy.w0) * cz.w1;
  float a10 = (wx0 * cy.w1) * cz.w0, a11 = (wx0 * cy.w1) * cz.w1;
  if (c.valid) {
    if (c.xo == xo0 && c.yo0 == yo0 && c.z0 == cz.i0) {
      a00 += c.w00;
      a01 += c.w01;
      a10 += c.w10;
      a11 += c.w11;
    } else {
      carry_flush(rho, c);
    }
  }
  deposit_plane_merged(rho, true, xo0, yo0, yo1, cz.i0, cz.i1, a00, a01, a10, a11);
  c.xo = cx.i1 * g.yz;
  c.yo0 = yo0;
  c.yo1 = yo1;
  c.z0 = cz.i0;
  c.z1 = cz.i1;
  c.w00 = (wx1 * cy.w0) * cz.w0;
  c.w01 = (wx1 * cy.w0) * cz.w1;
  c.w10 = (wx1 * cy.w1) * cz.w0;
  c.w11 = (wx1 * cy.w1) * cz.w1;
  c.valid = true;
}

// Kick (with the CIC readout of the force mesh at the current position), drift (with the
// kicked velocity) of one particle held in registers; `flags` as for the fused pass.
__device__ __forceinline__ void kdp_update(const float* __restrict__ force, float kick, float drift, int flags,
                                           const PGrid& g, int i, int j, int k, float& x0, float& x1, float& x2,
                                           float& v0, float& v1, float& v2) {
  if (flags & (kStepKick | kStepCorrect)) {
    const Cic1 cx = cic_rel(i, x0, g.nx), cy = cic_rel(j, x1, g.ny), cz = cic_rel(k, x2, g.nz);
    float fx, fy, fz;
    gather_force_mesh(force, g, cx, cy, cz, fx, fy, fz);
    if (flags & kStepKick) {
      v0 += fx * kick;
      v1 += fy * kick;
      v2 += fz * kick;
    } else {
      x0 += fx * kick;
      x1 += fy * kick;
      x2 += fz * kick;
    }
  }
  if (flags & kStepDrift) {
    x0 += v0 * drift;
    x1 += v1 * drift;
    x2 += v2 * drift;
  }
}

// One particle of the fused pass in the grid-stride walk. Order inside: kick -> drift ->
// paint (at the new position). Positions and velocities stream through once per pass:
// streaming (evict-first) loads and stores, so that they do not push the force and
// density meshes out of L2.
__device__ __forceinline__ void kdp_particle(float* __restrict__ disp, float* __restrict__ vel,
                                             const float* __restrict__ force, float kick, float drift, int flags,
                                             float weight, float* __restrict__ rho, const PGrid& g, unsigned p, int i,
                                             int j, int k) {
  float x0 = __ldcs(disp + 3 * p + 0), x1 = __ldcs(disp + 3 * p + 1), x2 = __ldcs(disp + 3 * p + 2);
  const bool use_v = flags & (kStepKick | kStepDrift);
  float v0 = 0.f, v1 = 0.f, v2 = 0.f;
  if (use_v) {
    v0 = __ldcs(vel + 3 * p + 0);
    v1 = __ldcs(vel + 3 * p + 1);
    v2 = __ldcs(vel + 3 * p + 2);
  }
  kdp_update(force, kick, drift, flags, g, i, j, k, x0, x1, x2, v0, v1, v2);
  if (flags & kStepKick) {
    __stcs(vel + 3 * p + 0, v0);
    __stcs(vel + 3 * p + 1, v1);
    __stcs(vel + 3 * p + 2, v2);
  }
  if (flags & (kStepDrift | kStepCorrect)) {
    __stcs(disp + 3 * p + 0, x0);
    __stcs(disp + 3 * p + 1, x1);
    __stcs(disp + 3 * p + 2, x2);
  }
  if (flags & kStepPaint) {
    const Cic1 cx = cic_rel(i, x0, g.nx), cy = cic_rel(j, x1, g.ny), cz = cic_rel(k, x2, g.nz);
    deposit_lane_merged(rho, g, cx, cy, cz, weight);
  }
}

// The 32 particles of one z row of the brick walk: their positions (and velocities) are
// 384 contiguous, 16-byte aligned bytes per array. Lanes 0..23 move them as float4 with
// streaming loads and stores through the warp's shared buffers (24 float4 per array), and
// every lane reads or writes its own 3 floats there (stride 3: no bank conflicts). A warp
// thus issues one 16-byte load and one store per array and row instead of three 4-byte
// ones, each touching 12 sectors. The row is loaded one iteration ahead (xa, va hold it
// when the call starts; the next row's loads are issued before this row's force gathers),
// so the gathers, not the row loads, are the latency of an iteration. The deposit holds
// back the upper-x plane for the lane's next particle (deposit_carried).
__device__ __forceinline__ void kdp_brick_row(float* __restrict__ disp, float* __restrict__ vel,
                                              const float* __restrict__ force, float kick, float drift, int flags,
                                              float weight, float* __restrict__ rho, const PGrid& g, unsigned p0, int i,
                                              int j, int k, int lane, float4* bx, float4* bv, XCarry& carry,
                                              float4& xa, float4& va, bool prefetch, unsigned p_next) {
  const bool use_v = flags & (kStepKick | kStepDrift);
  if (lane < 24) {
    bx[lane] = xa;
    bv[lane] = va;
  }
  __syncwarp();
  const float* fx = reinterpret_cast<const float*>(bx);
  const float* fv = reinterpret_cast<const float*>(bv);
  float x0 = fx[3 * lane], x1 = fx[3 * lane + 1], x2 = fx[3 * lane + 2];
  float v0 = fv[3 * lane], v1 = fv[3 * lane + 1], v2 = fv[3 * lane + 2];
  __syncwarp();
  if (prefetch && lane < 24) {
    xa = __ldcs(reinterpret_cast<const float4*>(disp + 3ull * p_next) + lane);
    if (use_v) va = __ldcs(reinterpret_cast<const float4*>(vel + 3ull * p_next) + lane);
  }
  kdp_update(force, kick, drift, flags, g, i, j, k, x0, x1, x2, v0, v1, v2);
  const bool store_v = flags & kStepKick, store_x = flags & (kStepDrift | kStepCorrect);
  if (store_v || store_x) {
    float* wx = reinterpret_cast<float*>(bx);
    float* wv = reinterpret_cast<float*>(bv);
    wx[3 * lane] = x0;
    wx[3 * lane + 1] = x1;
    wx[3 * lane + 2] = x2;
    wv[3 * lane] = v0;
    wv[3 * lane + 1] = v1;
    wv[3 * lane + 2] = v2;
    __syncwarp();
    if (lane < 24) {
      if (store_x) __stcs(reinterpret_cast<float4*>(disp + 3ull * p0) + lane, bx[lane]);
      if (store_v) __stcs(reinterpret_cast<float4*>(vel + 3ull * p0) + lane, bv[lane]);
    }
    __syncwarp();
  }
  if (flags & kStepPaint) {
    const Cic1 cx = cic_rel(i, x0, g.nx), cy = cic_rel(j, x1, g.ny), cz = cic_rel(k, x2, g.nz);
    deposit_carried(rho, g, cx, cy, cz, weight, carry);
  }
}

constexpr int kBrickY = 8, kBrickZ = 32;  // CTA of 256 = 8 warps; x walked in chunks of xdepth planes

// One fused particle pass of a PM step over all particles. With per-slot arrays (kicks !=
// nullptr) every batch entry b takes its own kick, drift and flags from kicks[b],
// drifts[b], slot_flags[b]; flags 0 leaves the slot untouched.
// Work order: when nz is a multiple of 32 and ny of 8 (and the CTA has 256 threads), a CTA
// takes an 8 (y) x 32 (z) brick of Lagrangian cells and walks it along x in chunks of
// xdepth planes (brick_xdepth: 16, fewer for a small mesh); warps stay on z rows (the lane-merged deposit needs them), but the rows and
// planes whose particles share CIC corners are gathered on one SM close in time, so the
// force-mesh lines they share are served by L1. Other shapes use a grid-stride walk.
template <int xdepth>
__global__ void __launch_bounds__(256, 4) k_kick_drift_paint(float* __restrict__ disp, float* __restrict__ vel, const float* __restrict__ force,
                                   float kick, float drift, int flags, float weight, float* __restrict__ rho,
                                   PGrid g, const float* __restrict__ kicks, const float* __restrict__ drifts,
                                   const int* __restrict__ slot_flags) {
  const long long b = blockIdx.y;
  if (kicks) {
    kick = kicks[b];
    drift = drifts[b];
    flags = slot_flags[b];
    if (flags == 0) return;
  }
  disp += b * g.np * 3;
  vel += b * g.np * 3;
  if (force) force += b * g.np * 4;
  if (rho) rho += b * g.np;
  __shared__ float4 rowbuf[kBrickY][2][24];  // per warp: positions, velocities of one z row
  if (blockDim.x == kBrickY * kBrickZ && g.nz % kBrickZ == 0 && g.ny % kBrickY == 0 &&
      ((reinterpret_cast<uintptr_t>(disp) | reinterpret_cast<uintptr_t>(vel)) & 15) == 0) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int tz = g.nz / kBrickZ, ty = g.ny / kBrickY, txc = (g.nx + xdepth - 1) / xdepth;
    const long long items = (long long)tz * ty * txc;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
      const int iz = (int)(it % tz);
      const long long rest = it / tz;
      const int iy = (int)(rest % ty), xc = (int)(rest / ty);
      const int j = iy * kBrickY + w, k = iz * kBrickZ + lane;
      const int i1 = min(g.nx, (xc + 1) * xdepth);
      XCarry carry;
      carry.valid = false;
      const unsigned row_stride = (unsigned)g.ny * (unsigned)g.nz;  // one x plane
      const bool use_v = flags & (kStepKick | kStepDrift);
      unsigned p0 = ((unsigned)(xc * xdepth) * (unsigned)g.ny + (unsigned)j) * (unsigned)g.nz + (unsigned)(k - lane);
      float4 xa = make_float4(0.f, 0.f, 0.f, 0.f), va = xa;
      if (lane < 24) {
        xa = __ldcs(reinterpret_cast<const float4*>(disp + 3ull * p0) + lane);
        if (use_v) va = __ldcs(reinterpret_cast<const float4*>(vel + 3ull * p0) + lane);
      }
      for (int i = xc * xdepth; i < i1; ++i, p0 += row_stride)
        kdp_brick_row(disp, vel, force, kick, drift, flags, weight, rho, g, p0, i, j, k, lane, rowbuf[w][0],
                      rowbuf[w][1], carry, xa, va, i + 1 < i1, p0 + row_stride);
      // every lane of the warp ran the same planes: the carries go out together, z-merged
      deposit_plane_merged(rho, carry.valid, carry.xo, carry.yo0, carry.yo1, carry.z0, carry.z1, carry.w00,
                           carry.w01, carry.w10, carry.w11);
    }
    return;
  }
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int i, j, k;
    particle_ijk(g, p, i, j, k);
    kdp_particle(disp, vel, force, kick, drift, flags, weight, rho, g, p, i, j, k);
  }
}

// ----------------------------------------------------------------------------------
// Force mesh: F = scale * (-D pot) at every cell, AoS float4 [nx][ny][nz] = (Fx, Fy, Fz, 0).
// The particle pass then reads one 16-byte value per CIC corner (8 loads) instead of the
// 56-point FD stencil of the potential; the CIC readout of F equals the stencil readout
// of pot. The fourth lane is padding that makes every corner a single aligned load.
// ----------------------------------------------------------------------------------
__global__ void k_force_mesh(const float* __restrict__ pot, float* __restrict__ F, float scale, PGrid g) {
  const long long b = blockIdx.y;
  pot += b * g.np;
  F += b * g.np * 4;
  const float s = scale / 12.0f;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int i, j, k;
    particle_ijk(g, p, i, j, k);
    const int xo = i * g.yz, yo = j * g.nz;
    const float* r = pot + xo + yo;
    const float fz = (8.0f * (__ldg(r + wrap1(k + 1, g.nz)) - __ldg(r + wrap1(k - 1, g.nz))) -
                      (__ldg(r + wrap1(k + 2, g.nz)) - __ldg(r + wrap1(k - 2, g.nz))));
    const float* cy = pot + xo + k;
    const float fy = (8.0f * (__ldg(cy + wrap1(j + 1, g.ny) * g.nz) - __ldg(cy + wrap1(j - 1, g.ny) * g.nz)) -
                      (__ldg(cy + wrap1(j + 2, g.ny) * g.nz) - __ldg(cy + wrap1(j - 2, g.ny) * g.nz)));
    const float* cx = pot + yo + k;
    const float fx = (8.0f * (__ldg(cx + wrap1(i + 1, g.nx) * g.yz) - __ldg(cx + wrap1(i - 1, g.nx) * g.yz)) -
                      (__ldg(cx + wrap1(i + 2, g.nx) * g.yz) - __ldg(cx + wrap1(i - 2, g.nx) * g.yz)));
    reinterpret_cast<float4*>(F)[p] = make_float4(-fx * s, -fy * s, -fz * s, 0.f);
  }
}

// The same stencil for four consecutive z cells per thread (nz % 4 == 0): 11 aligned
// 16-byte loads and 4 16-byte stores per 4 cells, row offsets and wraps shared.
constexpr int kForceMeshThreads = 256;

__global__ void __launch_bounds__(kForceMeshThreads) k_force_mesh4(const float* __restrict__ pot,
                                                                   float* __restrict__ F, float scale, PGrid g) {
  const long long b = blockIdx.y;
  pot += b * g.np;
  F += b * g.np * 4;
  const float s = scale / 12.0f;
  const unsigned nq = g.np >> 2;  // groups of 4 cells
  const int nz4 = g.nz >> 2;
  // A warp's 32 groups are 128 consecutive cells: their float4 results go through shared
  // memory so that each store instruction writes 512 contiguous bytes (a thread's own four
  // cells would make every store half-fill 32 sectors).
  __shared__ float4 stage[kForceMeshThreads / 32][128];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // the mesh is written tail first: its head, which the next particle pass (Lagrangian
  // order, head first) gathers from first, is then the part still in L2
  for (unsigned q0 = blockIdx.x * blockDim.x + threadIdx.x; q0 < nq; q0 += gridDim.x * blockDim.x) {
    const unsigned q = nq - 1 - q0;
    const unsigned row = q / (unsigned)nz4;  // i * ny + j
    const int k0 = (int)(q - row * (unsigned)nz4) << 2;
    const int i = (int)(row / (unsigned)g.ny);
    const int j = (int)row - i * g.ny;
    const int xo = i * g.yz, yo = j * g.nz;
    const float4* r = reinterpret_cast<const float4*>(pot + xo + yo);
    const float4 zm = __ldg(r + (wrap1(k0 - 4, g.nz) >> 2));
    const float4 z0 = __ldg(r + (k0 >> 2));
    const float4 zp = __ldg(r + (wrap1(k0 + 4, g.nz) >> 2));
    const float w[12] = {zm.x, zm.y, zm.z, zm.w, z0.x, z0.y, z0.z, z0.w, zp.x, zp.y, zp.z, zp.w};
    const float* cx = pot + yo + k0;
    const float4 xp1 = __ldg(reinterpret_cast<const float4*>(cx + wrap1(i + 1, g.nx) * g.yz));
    const float4 xm1 = __ldg(reinterpret_cast<const float4*>(cx + wrap1(i - 1, g.nx) * g.yz));
    const float4 xp2 = __ldg(reinterpret_cast<const float4*>(cx + wrap1(i + 2, g.nx) * g.yz));
    const float4 xm2 = __ldg(reinterpret_cast<const float4*>(cx + wrap1(i - 2, g.nx) * g.yz));
    const float* cy = pot + xo + k0;
    const float4 yp1 = __ldg(reinterpret_cast<const float4*>(cy + wrap1(j + 1, g.ny) * g.nz));
    const float4 ym1 = __ldg(reinterpret_cast<const float4*>(cy + wrap1(j - 1, g.ny) * g.nz));
    const float4 yp2 = __ldg(reinterpret_cast<const float4*>(cy + wrap1(j + 2, g.ny) * g.nz));
    const float4 ym2 = __ldg(reinterpret_cast<const float4*>(cy + wrap1(j - 2, g.ny) * g.nz));
    const float fx[4] = {xp1.x - xm1.x, xp1.y - xm1.y, xp1.z - xm1.z, xp1.w - xm1.w};
    const float fx2[4] = {xp2.x - xm2.x, xp2.y - xm2.y, xp2.z - xm2.z, xp2.w - xm2.w};
    const float fy[4] = {yp1.x - ym1.x, yp1.y - ym1.y, yp1.z - ym1.z, yp1.w - ym1.w};
    const float fy2[4] = {yp2.x - ym2.x, yp2.y - ym2.y, yp2.z - ym2.z, yp2.w - ym2.w};
    float4 res[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const float gz = -(8.0f * (w[5 + t] - w[3 + t]) - (w[6 + t] - w[2 + t])) * s;
      res[t] = make_float4(-(8.0f * fx[t] - fx2[t]) * s, -(8.0f * fy[t] - fy2[t]) * s, gz, 0.f);
    }
    // the whole warp is in this iteration when its last lane's group exists (q0 of lane L
    // is the warp's first q0 plus L: block size and grid stride are multiples of 32)
    const unsigned q0_first = q0 - lane;
    if (q0_first + 31 < nq) {
      const unsigned q_min = nq - 1 - (q0_first + 31);  // group of lane 31; lane L holds q_min + 31 - L
#pragma unroll
      for (int t = 0; t < 4; ++t) stage[warp][4 * (31 - lane) + t] = res[t];
      __syncwarp();
      float4* base = reinterpret_cast<float4*>(F) + 4ull * q_min;
#pragma unroll
      for (int t = 0; t < 4; ++t) base[32 * t + lane] = stage[warp][32 * t + lane];
      __syncwarp();
    } else {
      float4* out = reinterpret_cast<float4*>(F) + (xo + yo + k0);
#pragma unroll
      for (int t = 0; t < 4; ++t) out[t] = res[t];
    }
  }
}

// F = scale * (-D pot) at every grid point (particles exactly on the grid), optionally
// accumulated into `out` (AoS [..,3]).
__global__ void k_grid_gradient(const float* __restrict__ pot, float* __restrict__ out, float scale, int accumulate,
                                PGrid g) {
  const long long b = blockIdx.y;
  pot += b * g.np;
  out += b * g.np * 3;
  const float s = 1.0f / 12.0f;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int i, j, k;
    particle_ijk(g, p, i, j, k);
    const int xo = i * g.yz, yo = j * g.nz;
    float gr[3];
    {
      const float a = pot[wrap1(i + 1, g.nx) * g.yz + yo + k], bm = pot[wrap1(i - 1, g.nx) * g.yz + yo + k];
      const float c = pot[wrap1(i + 2, g.nx) * g.yz + yo + k], e = pot[wrap1(i - 2, g.nx) * g.yz + yo + k];
      gr[0] = -(8.0f * (a - bm) - (c - e)) * s;
    }
    {
      const float a = pot[xo + wrap1(j + 1, g.ny) * g.nz + k], bm = pot[xo + wrap1(j - 1, g.ny) * g.nz + k];
      const float c = pot[xo + wrap1(j + 2, g.ny) * g.nz + k], e = pot[xo + wrap1(j - 2, g.ny) * g.nz + k];
      gr[1] = -(8.0f * (a - bm) - (c - e)) * s;
    }
    {
      const float a = pot[xo + yo + wrap1(k + 1, g.nz)], bm = pot[xo + yo + wrap1(k - 1, g.nz)];
      const float c = pot[xo + yo + wrap1(k + 2, g.nz)], e = pot[xo + yo + wrap1(k - 2, g.nz)];
      gr[2] = -(8.0f * (a - bm) - (c - e)) * s;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float v = gr[a] * scale;
      out[3ull * p + a] = accumulate ? out[3ull * p + a] + v : v;
    }
  }
}

// Second-order LPT source from the first-order potential (JaxPM `lpt`, order 2):
//   delta2 = sum_{i<j} phi_ii phi_jj - phi_ij^2,  phi_ij = D_i D_j phi,
// with D the same 4-point finite difference (its square is the k-space product
// gradient_kernel_i * gradient_kernel_j used by the reference). Needs axes >= 4 cells.
__constant__ float c_d5[5] = {1.0f / 12.0f, -8.0f / 12.0f, 0.0f, 8.0f / 12.0f, -1.0f / 12.0f};

// (D_a D_b f)(c) for the 4-point finite difference D (5-point stencil c_d5 per axis):
// offsets -4..4 along a for a == b, a 4x4 cross for a != b. The stencil is symmetric
// under (s, t) -> (-s, -t), so the operator is its own transpose.
__device__ __forceinline__ float hess_component(const float* __restrict__ f, const int* c3, const int* n3,
                                                const int* st, int base, int a, int bb) {
  float acc = 0.f;
  if (a == bb) {
    const int rest = base - c3[a] * st[a];
    for (int s = 0; s < 5; ++s) {
      if (s == 2) continue;
      for (int t = 0; t < 5; ++t) {
        if (t == 2) continue;
        const int off = (s - 2) + (t - 2);
        acc += c_d5[s] * c_d5[t] * f[rest + wrap1(c3[a] + off, n3[a]) * st[a]];
      }
    }
  } else {
    const int rest = base - c3[a] * st[a] - c3[bb] * st[bb];
    for (int s = 0; s < 5; ++s) {
      if (s == 2) continue;
      const int oa = wrap1(c3[a] + s - 2, n3[a]) * st[a];
      for (int t = 0; t < 5; ++t) {
        if (t == 2) continue;
        acc += c_d5[s] * c_d5[t] * f[rest + oa + wrap1(c3[bb] + t - 2, n3[bb]) * st[bb]];
      }
    }
  }
  return acc;
}

// The 2LPT source (reference call site pm/lpt.py:119), from the first-order field
// F = -D phi (AoS, as k_grid_gradient writes it, which the LPT has just computed):
// phi_ab = D_b D_a phi = -D_b F_a, since the FD operators are convolutions and commute.
// Four loads per component instead of the 16 of hess_component's two-stencil product;
// the same operator, with F rounded to FP32 in between.
__global__ void k_lpt2_source_grad(const float* __restrict__ F, float* __restrict__ out, PGrid g) {
  const long long b = blockIdx.y;
  F += b * g.np * 3;
  out += b * g.np;
  const int n3[3] = {g.nx, g.ny, g.nz};
  const int st[3] = {g.yz, g.nz, 1};
  const float inv12 = 1.0f / 12.0f;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int c3[3];
    particle_ijk(g, p, c3[0], c3[1], c3[2]);
    float h[3][3];
#pragma unroll
    for (int bb = 0; bb < 3; ++bb) {
      const int rest = (int)p - c3[bb] * st[bb];
      const int m2 = 3 * (rest + wrap1(c3[bb] - 2, n3[bb]) * st[bb]);
      const int m1 = 3 * (rest + wrap1(c3[bb] - 1, n3[bb]) * st[bb]);
      const int p1 = 3 * (rest + wrap1(c3[bb] + 1, n3[bb]) * st[bb]);
      const int p2 = 3 * (rest + wrap1(c3[bb] + 2, n3[bb]) * st[bb]);
#pragma unroll
      for (int a = 0; a <= bb; ++a)
        h[a][bb] = -(8.0f * (__ldg(F + p1 + a) - __ldg(F + m1 + a)) - (__ldg(F + p2 + a) - __ldg(F + m2 + a))) * inv12;
    }
    // accumulate in the reference's loop order
    float delta2 = 0.f, acc_diag = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      delta2 += h[a][a] * acc_diag;
      acc_diag += h[a][a];
#pragma unroll
      for (int bb = a + 1; bb < 3; ++bb) delta2 -= h[a][bb] * h[a][bb];
    }
    out[p] = delta2;
  }
}

// Adjoint of the 2LPT source, first half: with s = dL/d delta2 at a cell,
//   q_aa = s * sum_{b != a} phi_bb  (a = 0, 1, 2)   and   q_ab = -2 s phi_ab  (01, 02, 12),
// written as six meshes [6][cells].
__global__ void k_lpt2_source_adj_products(const float* __restrict__ pot, const float* __restrict__ sbar,
                                           float* __restrict__ q, PGrid g) {
  const long long b = blockIdx.y;
  pot += b * g.np;
  sbar += b * g.np;
  q += b * g.np * 6;
  const int n3[3] = {g.nx, g.ny, g.nz};
  const int st[3] = {g.yz, g.nz, 1};
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int c3[3];
    particle_ijk(g, p, c3[0], c3[1], c3[2]);
    const int base = c3[0] * g.yz + c3[1] * g.nz + c3[2];
    float h[3][3];
    for (int a = 0; a < 3; ++a)
      for (int bb = a; bb < 3; ++bb) h[a][bb] = hess_component(pot, c3, n3, st, base, a, bb);
    const float sv = sbar[p];
    q[p] = sv * (h[1][1] + h[2][2]);
    q[g.np + p] = sv * (h[0][0] + h[2][2]);
    q[2ull * g.np + p] = sv * (h[0][0] + h[1][1]);
    q[3ull * g.np + p] = -2.0f * sv * h[0][1];
    q[4ull * g.np + p] = -2.0f * sv * h[0][2];
    q[5ull * g.np + p] = -2.0f * sv * h[1][2];
  }
}

// Second half: dL/d phi1 = sum_a D_a D_a q_aa + sum_{a<b} D_a D_b q_ab (each operator is
// its own transpose), optionally accumulated into out.
__global__ void k_lpt2_source_adj_apply(const float* __restrict__ q, float* __restrict__ out, int accumulate,
                                        PGrid g) {
  const long long b = blockIdx.y;
  q += b * g.np * 6;
  out += b * g.np;
  const int n3[3] = {g.nx, g.ny, g.nz};
  const int st[3] = {g.yz, g.nz, 1};
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int c3[3];
    particle_ijk(g, p, c3[0], c3[1], c3[2]);
    const int base = c3[0] * g.yz + c3[1] * g.nz + c3[2];
    float acc = 0.f;
    for (int m = 0; m < 6; ++m) acc += hess_component(q + (size_t)m * g.np, c3, n3, st, base, pa[m], pb[m]);
    out[p] = accumulate ? out[p] + acc : acc;
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

// Zero n floats (16-byte stores where the pointer allows; the tail element by element).
__global__ void k_zero(float* __restrict__ y, long long n) {
  const long long n4 = ((reinterpret_cast<uintptr_t>(y) & 15) == 0) ? n / 4 : 0;
  float4* y4 = reinterpret_cast<float4*>(y);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride)
    y4[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (long long q = 4 * n4 + (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) y[q] = 0.f;
}

cudaError_t zero_floats(float* y, long long n, cudaStream_t s) {
  k_zero<<<particle_grid_dims((n + 3) / 4, 1, 256, 16), 256, 0, s>>>(y, n);
  note_launch();
  return cudaGetLastError();
}

__global__ void k_axpy(float* __restrict__ y, const float* __restrict__ x, float a, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    y[q] += a * x[q];
}

// ----------------------------------------------------------------------------------
cudaError_t cic_paint(const float* pos, int absolute, const float* weights, float weight, float* mesh,
                      const MeshDims& d, cudaStream_t s) {
  k_paint<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pos, absolute, weights, weight, mesh, make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

cudaError_t cic_readout(const float* pos, int absolute, const float* mesh, float* out, const MeshDims& d,
                        cudaStream_t s) {
  k_readout<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pos, absolute, mesh, out, make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

cudaError_t cic_readout_gradient(const float* pos, int absolute, const float* pot, float* out, float scale,
                                 const MeshDims& d, cudaStream_t s) {
  k_readout_gradient<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pos, absolute, pot, out, scale,
                                                                                     make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

// The brick depth is a template argument: a runtime depth costs the kernel registers (it
// spilled at the 64-register bound).
static void launch_kdp(float* disp, float* vel, const float* force, float kick, float drift, int flags, float weight,
                       float* rho, const MeshDims& d, const float* kicks, const float* drifts, const int* slot_flags,
                       cudaStream_t s) {
  const dim3 grid = particle_grid_dims(d.cells(), d.batch, 256, 16);
  const PGrid g = make_pgrid(d);
  switch (brick_xdepth(d.nx, d.ny, d.nz, d.batch, 4ll * sm_count())) {
    case 16:
      k_kick_drift_paint<16><<<grid, 256, 0, s>>>(disp, vel, force, kick, drift, flags, weight, rho, g, kicks, drifts,
                                                  slot_flags);
      break;
    case 8:
      k_kick_drift_paint<8><<<grid, 256, 0, s>>>(disp, vel, force, kick, drift, flags, weight, rho, g, kicks, drifts,
                                                 slot_flags);
      break;
    case 4:
      k_kick_drift_paint<4><<<grid, 256, 0, s>>>(disp, vel, force, kick, drift, flags, weight, rho, g, kicks, drifts,
                                                 slot_flags);
      break;
    case 2:
      k_kick_drift_paint<2><<<grid, 256, 0, s>>>(disp, vel, force, kick, drift, flags, weight, rho, g, kicks, drifts,
                                                 slot_flags);
      break;
    default:
      k_kick_drift_paint<1><<<grid, 256, 0, s>>>(disp, vel, force, kick, drift, flags, weight, rho, g, kicks, drifts,
                                                 slot_flags);
  }
  note_launch();
}

cudaError_t kick_drift_paint(float* disp, float* vel, const float* force, float kick, float drift, int flags,
                             float weight, float* rho, const MeshDims& d, cudaStream_t s) {
  launch_kdp(disp, vel, force, kick, drift, flags, weight, rho, d, nullptr, nullptr, nullptr, s);
  return cudaGetLastError();
}

cudaError_t kick_drift_paint_slots(float* disp, float* vel, const float* force, const float* kicks,
                                   const float* drifts, const int* slot_flags, float weight, float* rho,
                                   const MeshDims& d, cudaStream_t s) {
  launch_kdp(disp, vel, force, 0.f, 0.f, 0, weight, rho, d, kicks, drifts, slot_flags, s);
  return cudaGetLastError();
}

cudaError_t force_mesh(const float* pot, float* force, float scale, const MeshDims& d, cudaStream_t s) {
  const bool vec4 = d.nz % 4 == 0 && d.nz >= 8 && ((uintptr_t)pot % 16) == 0 && ((uintptr_t)force % 16) == 0;
  if (vec4)
    k_force_mesh4<<<particle_grid_dims(d.cells() / 4, d.batch, kForceMeshThreads, 16), kForceMeshThreads, 0, s>>>(
        pot, force, scale, make_pgrid(d));
  else
    k_force_mesh<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pot, force, scale, make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

cudaError_t grid_gradient(const float* pot, float* out, float scale, int accumulate, const MeshDims& d,
                          cudaStream_t s) {
  k_grid_gradient<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pot, out, scale, accumulate, make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

cudaError_t lpt2_source(const float* grad, float* out, const MeshDims& d, cudaStream_t s) {
  k_lpt2_source_grad<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(grad, out, make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

cudaError_t lpt2_source_adjoint(const float* pot, const float* sbar, float* q, float* out, int accumulate,
                                const MeshDims& d, cudaStream_t s) {
  k_lpt2_source_adj_products<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(pot, sbar, q,
                                                                                            make_pgrid(d));
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_lpt2_source_adj_apply<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(q, out, accumulate,
                                                                                         make_pgrid(d));
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
