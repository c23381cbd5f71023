// Adjoint (vector-Jacobian) kernels of the PM force step and the reversible KKD update.
//
// The force on a particle at x is F_a(x) = R_x[M_a], the CIC readout R of the force mesh
// M_a = -D_a P (rho - mean), rho = sum_q W(x_q - .) the CIC density, P the Poisson
// operator (-1/k^2, k = 0 -> 0) and D_a the 4-point finite difference. For a cotangent u
// per particle the transpose J^T u of dF/dx has two parts:
//   * readout: u . grad_x R_x[M] = grad_x R_x[sum_a u_a M_a]    (corners combined first)
//   * density: grad_x R_x[rho_bar], rho_bar = sum_a (-D_a P)^T Ubar_a = P(div_FD Ubar),
//     Ubar_a = CIC paint of the particles with weights u_a (D_a^T = -D_a, P^T = P).
// The reversible step (reference pm/solvers.py:258-411, backward loop
// pm/integrate.py:288-535) is  v' = v + k F(x);  x' = x + d v'.  Its reverse recomputes
// x = x' - d v', F(x), v = v' - k F(x); its VJP is
//   lambda_v_total = lambda_v' + d lambda_x',   dL/dd = <lambda_x', v'>,
//   dL/dk = <lambda_v_total, F(x)>,   lambda_x = lambda_x' + k J^T lambda_v_total.
#include "cic.cuh"
#include "common.cuh"
#include "internal.h"

namespace jfli {

constexpr int kAdjThreads = 256;
constexpr int kAdjCtasPerSm = 8;

// Block-wide sum of two doubles; thread 0 returns the result.
__device__ __forceinline__ void block_sum2(double& a, double& b) {
  __shared__ double sa[kAdjThreads / 32], sb[kAdjThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = 0.0;
    b = 0.0;
    for (int i = 0; i < kAdjThreads / 32; ++i) {  // fixed order
      a += sa[i];
      b += sb[i];
    }
  }
}

// CIC deposit of the vector u on a float4 mesh [cell] = (u0, u1, u2, 0), one 16-byte vector
// atomic per corner where three meshes take three scalar ones. The lanes hold consecutive
// particles of one z row (the grid-stride loop; the active lanes a prefix of the warp),
// with deposit_lane_merged's z merge: when lane L's
// upper-z corners are lane L+1's lower-z corners, lane L+1 receives lane L's vector and its
// four upper-z weights and adds them to its own lower-z deposits (one vector atomic per
// shared cell instead of two).
__device__ __forceinline__ void deposit_vec4_lane_merged(float4* mesh, const PGrid& g, const Cic1& cx, const Cic1& cy,
                                                         const Cic1& cz, const float u[3]) {
  const unsigned mask = __activemask();
  const int lane = threadIdx.x & 31;
  const int xy0 = cx.i0 * g.yz + cy.i0 * g.nz;
  const int lo = xy0 + cz.i0, hi = xy0 + cz.i1;
  const int next_lo = __shfl_down_sync(mask, lo, 1);
  const int prev_hi = __shfl_up_sync(mask, hi, 1);
  const bool give = lane < 31 && ((mask >> (lane + 1)) & 1u) && next_lo == hi;
  const bool take = lane > 0 && ((mask >> (lane - 1)) & 1u) && prev_hi == lo;
  const float p0 = __shfl_up_sync(mask, u[0], 1), p1 = __shfl_up_sync(mask, u[1], 1),
              p2 = __shfl_up_sync(mask, u[2], 1);
  const int xo[2] = {cx.i0 * g.yz, cx.i1 * g.yz}, yo[2] = {cy.i0 * g.nz, cy.i1 * g.nz};
  const float wx[2] = {cx.w0, cx.w1}, wy[2] = {cy.w0, cy.w1};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const float wab = wx[a] * wy[b];
      const float up = wab * cz.w1;
      const float recv = __shfl_up_sync(mask, up, 1);
      const float wl = wab * cz.w0;
      float4 low = make_float4(wl * u[0], wl * u[1], wl * u[2], 0.f);
      if (take) {
        low.x += recv * p0;
        low.y += recv * p1;
        low.z += recv * p2;
      }
      atomicAdd(mesh + (xo[a] + yo[b] + cz.i0), low);
      if (!give) atomicAdd(mesh + (xo[a] + yo[b] + cz.i1), make_float4(up * u[0], up * u[1], up * u[2], 0.f));
    }
}

// Reverse kick + first half of the VJP of one reversible step, at the un-drifted
// positions x (relative displacements). Per particle:
//   F = R_x[force];  <lambda_x, v'> -> partial[1];  u = lambda_v + drift * lambda_x;
//   <u, F> -> partial[0];  v = v' - kick F;  lambda_v = u;  ubar_a += W * u_a.
// partials holds 2 doubles per CTA and batch entry, summed in a fixed order later.
// ubar: three meshes [3][cells] (kVec4 false) or one float4 mesh [cells] (kVec4 true).
// The arithmetic of one particle, on its values in registers: x, v, lx (lambda_x), lv
// (lambda_v) in; x (un-drifted when undrift), v (un-kicked) and lv (= u) out.
template <bool kVec4>
__device__ __forceinline__ void unkick_core(float x[3], float v[3], const float lx[3], float lv[3], bool undrift,
                                            const float* __restrict__ force, float kick, float drift,
                                            float* __restrict__ ubar, const PGrid& g, int i, int j, int k, double& sk,
                                            double& sd) {
  if (undrift) {
#pragma unroll
    for (int a = 0; a < 3; ++a) x[a] += v[a] * -drift;
  }
  const Cic1 cx = cic_rel(i, x[0], g.nx), cy = cic_rel(j, x[1], g.ny), cz = cic_rel(k, x[2], g.nz);
  float f[3];
  gather_force_mesh(force, g, cx, cy, cz, f[0], f[1], f[2]);
  float u[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    sd += (double)lx[a] * (double)v[a];
    u[a] = lv[a] + drift * lx[a];
    sk += (double)u[a] * (double)f[a];
    v[a] = v[a] - f[a] * kick;
    lv[a] = u[a];
  }
  if (kVec4) {
    deposit_vec4_lane_merged(reinterpret_cast<float4*>(ubar), g, cx, cy, cz, u);
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) deposit(ubar + (size_t)a * g.np, g, cx, cy, cz, u[a]);
  }
}

// One particle with its own 4-byte loads and stores. With undrift (the float4 form of the
// reverse sweep over stored potentials), disp holds x' on entry: the particle is first
// un-drifted, x = x' - drift v', and x is written back.
template <bool kVec4>
__device__ __forceinline__ void unkick_particle(float* __restrict__ disp, bool undrift, float* __restrict__ vel,
                                                const float* __restrict__ lam_x, float* __restrict__ lam_v,
                                                const float* __restrict__ force, float kick, float drift,
                                                float* __restrict__ ubar, const PGrid& g, unsigned p, int i, int j,
                                                int k, double& sk, double& sd) {
  float x[3], v[3], lx[3], lv[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    x[a] = disp[3 * p + a];
    v[a] = vel[3 * p + a];
    lx[a] = lam_x[3 * p + a];
    lv[a] = lam_v[3 * p + a];
  }
  unkick_core<kVec4>(x, v, lx, lv, undrift, force, kick, drift, ubar, g, i, j, k, sk, sd);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (undrift) disp[3 * p + a] = x[a];
    vel[3 * p + a] = v[a];
    lam_v[3 * p + a] = lv[a];
  }
}

// The 32 particles of one z row (lane = z offset; the row's arrays start 16-byte aligned):
// lanes 0..23 move each array's 384 bytes as float4 with streaming loads and stores
// through the warp's shared buffers (4 x 24 float4), and every lane reads and writes its
// own 3 floats there (stride 3, no bank conflicts): one 16-byte instruction per array and
// row where the lanes' own accesses take three 4-byte ones.
template <bool kVec4>
__device__ __forceinline__ void unkick_row(float* __restrict__ disp, bool undrift, float* __restrict__ vel,
                                           const float* __restrict__ lam_x, float* __restrict__ lam_v,
                                           const float* __restrict__ force, float kick, float drift,
                                           float* __restrict__ ubar, const PGrid& g, unsigned p0, int i, int j, int k,
                                           int lane, float4 (*buf)[24], double& sk, double& sd) {
  float4* d4 = reinterpret_cast<float4*>(disp + 3ull * p0);
  float4* v4 = reinterpret_cast<float4*>(vel + 3ull * p0);
  const float4* x4 = reinterpret_cast<const float4*>(lam_x + 3ull * p0);
  float4* l4 = reinterpret_cast<float4*>(lam_v + 3ull * p0);
  if (lane < 24) {
    buf[0][lane] = __ldcs(d4 + lane);
    buf[1][lane] = __ldcs(v4 + lane);
    buf[2][lane] = __ldcs(x4 + lane);
    buf[3][lane] = __ldcs(l4 + lane);
  }
  __syncwarp();
  float x[3], v[3], lx[3], lv[3];
  const float* f0 = reinterpret_cast<const float*>(buf[0]);
  const float* f1 = reinterpret_cast<const float*>(buf[1]);
  const float* f2 = reinterpret_cast<const float*>(buf[2]);
  const float* f3 = reinterpret_cast<const float*>(buf[3]);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    x[a] = f0[3 * lane + a];
    v[a] = f1[3 * lane + a];
    lx[a] = f2[3 * lane + a];
    lv[a] = f3[3 * lane + a];
  }
  __syncwarp();
  unkick_core<kVec4>(x, v, lx, lv, undrift, force, kick, drift, ubar, g, i, j, k, sk, sd);
  float* w0 = reinterpret_cast<float*>(buf[0]);
  float* w1 = reinterpret_cast<float*>(buf[1]);
  float* w3 = reinterpret_cast<float*>(buf[3]);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    w0[3 * lane + a] = x[a];
    w1[3 * lane + a] = v[a];
    w3[3 * lane + a] = lv[a];
  }
  __syncwarp();
  if (lane < 24) {
    if (undrift) __stcs(d4 + lane, buf[0][lane]);
    __stcs(v4 + lane, buf[1][lane]);
    __stcs(l4 + lane, buf[3][lane]);
  }
  __syncwarp();
}

constexpr int kAdjBrickY = 8, kAdjBrickZ = 32;

// Work order of the float4 form: when nz is a multiple of 32 and ny of 8, a CTA of 8 warps
// takes an 8 (y) x 32 (z) brick of Lagrangian cells and walks it along x in chunks of
// xdepth planes (brick_xdepth), each warp on one z row (the z merge of the deposit needs consecutive z in a
// warp), so that the rows and planes whose particles share CIC corners gather and deposit
// on one SM close in time (as the forward particle pass). Otherwise a grid-stride walk.
template <bool kVec4>
__global__ void __launch_bounds__(kAdjThreads, 3) k_adj_unkick_paint(
    float* __restrict__ disp, int undrift, float* __restrict__ vel, const float* __restrict__ lam_x,
    float* __restrict__ lam_v, const float* __restrict__ force, float kick, float drift, float* __restrict__ ubar,
    double* __restrict__ partials, PGrid g, int xdepth) {
  const long long b = blockIdx.y;
  disp += b * g.np * 3;
  vel += b * g.np * 3;
  lam_x += b * g.np * 3;
  lam_v += b * g.np * 3;
  force += b * g.np * 4;
  ubar += b * g.np * (kVec4 ? 4 : 3);
  double sk = 0.0, sd = 0.0;
  __shared__ float4 rowbuf[kVec4 ? kAdjBrickY : 1][4][24];  // per warp: disp, vel, lam_x, lam_v of one z row
  if (kVec4 && blockDim.x == kAdjBrickY * kAdjBrickZ && g.nz % kAdjBrickZ == 0 && g.ny % kAdjBrickY == 0) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool staged = ((reinterpret_cast<uintptr_t>(disp) | reinterpret_cast<uintptr_t>(vel) |
                          reinterpret_cast<uintptr_t>(lam_x) | reinterpret_cast<uintptr_t>(lam_v)) & 15) == 0;
    const int tz = g.nz / kAdjBrickZ, ty = g.ny / kAdjBrickY, txc = (g.nx + xdepth - 1) / xdepth;
    const long long items = (long long)tz * ty * txc;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
      const int iz = (int)(it % tz);
      const long long rest = it / tz;
      const int iy = (int)(rest % ty), xc = (int)(rest / ty);
      const int j = iy * kAdjBrickY + w, k = iz * kAdjBrickZ + lane;
      const int i1 = min(g.nx, (xc + 1) * xdepth);
      for (int i = xc * xdepth; i < i1; ++i) {
        const unsigned p = ((unsigned)i * (unsigned)g.ny + (unsigned)j) * (unsigned)g.nz + (unsigned)k;
        if (staged)
          unkick_row<kVec4>(disp, undrift != 0, vel, lam_x, lam_v, force, kick, drift, ubar, g, p - (unsigned)lane,
                            i, j, k, lane, rowbuf[kVec4 ? w : 0], sk, sd);
        else
          unkick_particle<kVec4>(disp, undrift != 0, vel, lam_x, lam_v, force, kick, drift, ubar, g, p, i, j, k, sk,
                                 sd);
      }
    }
  } else {
    for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
      int i, j, k;
      particle_ijk(g, p, i, j, k);
      unkick_particle<kVec4>(disp, undrift != 0, vel, lam_x, lam_v, force, kick, drift, ubar, g, p, i, j, k, sk, sd);
    }
  }
  block_sum2(sk, sd);
  if (threadIdx.x == 0) {
    double* dst = partials + 2 * (b * gridDim.x + blockIdx.x);
    dst[0] = sk;
    dst[1] = sd;
  }
}

// CIC paint of a vector per particle (u, 3 floats, particle grid layout) onto a float4
// mesh, cleared by the caller: the cotangent paint of the PGD correction's adjoint.
__global__ void k_paint_vec4(const float* __restrict__ disp, const float* __restrict__ u, float* __restrict__ ubar,
                             PGrid g) {
  const long long b = blockIdx.y;
  disp += b * g.np * 3;
  u += b * g.np * 3;
  ubar += b * g.np * 4;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int i, j, k;
    particle_ijk(g, p, i, j, k);
    const Cic1 cx = cic_rel(i, disp[3 * p + 0], g.nx), cy = cic_rel(j, disp[3 * p + 1], g.ny),
               cz = cic_rel(k, disp[3 * p + 2], g.nz);
    const float uu[3] = {u[3 * p + 0], u[3 * p + 1], u[3 * p + 2]};
    deposit_vec4_lane_merged(reinterpret_cast<float4*>(ubar), g, cx, cy, cz, uu);
  }
}

cudaError_t paint_vec4(const float* disp, const float* u, float* ubar, const MeshDims& d, cudaStream_t s) {
  k_paint_vec4<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(disp, u, ubar, make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

// out(c) = [accumulate ? out(c) : 0] + sum_a D_a (alpha u_a + beta w_a)(c), with
// D_a f(c) = [8 (f(c+e_a) - f(c-e_a)) - (f(c+2e_a) - f(c-2e_a))] / 12. Component a of
// cell c is at index c * cell_stride + a * comp_stride (SoA meshes: 1, cells; AoS
// particle grids: 3, 1). w may be null.
__global__ void k_div_fd(const float* __restrict__ u, float alpha, const float* __restrict__ w, float beta,
                         long long cell_stride, long long comp_stride, int accumulate, float* __restrict__ out,
                         PGrid g) {
  const long long b = blockIdx.y;
  u += b * g.np * 3;
  if (w) w += b * g.np * 3;
  out += b * g.np;
  const float s = 1.0f / 12.0f;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int c3[3];
    particle_ijk(g, p, c3[0], c3[1], c3[2]);
    const int n3[3] = {g.nx, g.ny, g.nz};
    const int st[3] = {g.yz, g.nz, 1};
    const int base = c3[0] * g.yz + c3[1] * g.nz + c3[2];
    float acc = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int rest = base - c3[a] * st[a];
      float v[4];
      const int off[4] = {-2, -1, 1, 2};
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const long long q = (long long)(rest + wrap1(c3[a] + off[t], n3[a]) * st[a]);
        float val = alpha * u[q * cell_stride + a * comp_stride];
        if (w) val += beta * w[q * cell_stride + a * comp_stride];
        v[t] = val;
      }
      acc += (8.0f * (v[2] - v[1]) - (v[3] - v[0])) * s;
    }
    out[p] = accumulate ? out[p] + acc : acc;
  }
}

// lam_x += scale * grad_x R_x[h], h(corner) = rho_bar(corner) + sum_a u_a force_a(corner)
// (force AoS float4 per cell, as written by the force-mesh kernels),
// at relative positions disp. Either of rho_bar or (u, force) may be null. The gradient
// of the trilinear weights is one-sided at cell faces, like the derivative of the
// floor-based weights.
// The gradient of R_x[h] at one particle from its position x and vector u in registers:
// (gx, gy, gz) = grad_x R_x[rho_bar + sum_a u_a force_a].
__device__ __forceinline__ void adj_position_core(const float x[3], const float ua[3], bool use_u,
                                                  const float* __restrict__ rho_bar,
                                                  const float* __restrict__ force, const PGrid& g, int i, int j, int k,
                                                  float& gx, float& gy, float& gz) {
  const Cic1 cx = cic_rel(i, x[0], g.nx), cy = cic_rel(j, x[1], g.ny), cz = cic_rel(k, x[2], g.nz);
  const int xo[2] = {cx.i0 * g.yz, cx.i1 * g.yz}, yo[2] = {cy.i0 * g.nz, cy.i1 * g.nz}, zo[2] = {cz.i0, cz.i1};
  float h[2][2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int bb = 0; bb < 2; ++bb)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int o = xo[a] + yo[bb] + zo[c];
        float v = rho_bar ? __ldg(rho_bar + o) : 0.f;
        if (use_u) {
          const float4 f = __ldg(reinterpret_cast<const float4*>(force) + o);
          v += ua[0] * f.x + ua[1] * f.y + ua[2] * f.z;
        }
        h[a][bb][c] = v;
      }
  const float wx[2] = {cx.w0, cx.w1}, wy[2] = {cy.w0, cy.w1}, wz[2] = {cz.w0, cz.w1};
  gx = 0.f;
  gy = 0.f;
  gz = 0.f;
#pragma unroll
  for (int bb = 0; bb < 2; ++bb)
#pragma unroll
    for (int c = 0; c < 2; ++c) gx += wy[bb] * wz[c] * (h[1][bb][c] - h[0][bb][c]);
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int c = 0; c < 2; ++c) gy += wx[a] * wz[c] * (h[a][1][c] - h[a][0][c]);
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int bb = 0; bb < 2; ++bb) gz += wx[a] * wy[bb] * (h[a][bb][1] - h[a][bb][0]);
}

__device__ __forceinline__ void adj_position_particle(const float* __restrict__ disp, const float* __restrict__ u,
                                                      const float* __restrict__ rho_bar,
                                                      const float* __restrict__ force, float scale,
                                                      float* __restrict__ lam_x, const PGrid& g, unsigned p, int i,
                                                      int j, int k) {
  const float x[3] = {disp[3 * p + 0], disp[3 * p + 1], disp[3 * p + 2]};
  const bool use_u = u && force;
  float ua[3] = {0.f, 0.f, 0.f};
  if (use_u) {
    ua[0] = u[3 * p + 0];
    ua[1] = u[3 * p + 1];
    ua[2] = u[3 * p + 2];
  }
  float gx, gy, gz;
  adj_position_core(x, ua, use_u, rho_bar, force, g, i, j, k, gx, gy, gz);
  lam_x[3 * p + 0] += scale * gx;
  lam_x[3 * p + 1] += scale * gy;
  lam_x[3 * p + 2] += scale * gz;
}

__global__ void __launch_bounds__(256) k_adj_position(const float* __restrict__ disp, const float* __restrict__ u,
                                                      const float* __restrict__ rho_bar,
                                                      const float* __restrict__ force, float scale,
                                                      float* __restrict__ lam_x, PGrid g) {
  const long long b = blockIdx.y;
  disp += b * g.np * 3;
  lam_x += b * g.np * 3;
  if (u) u += b * g.np * 3;
  if (force) force += b * g.np * 4;
  if (rho_bar) rho_bar += b * g.np;
  // (staging its rows through shared memory, as the un-kick does, measured 10% slower)
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    int i, j, k;
    particle_ijk(g, p, i, j, k);
    adj_position_particle(disp, u, rho_bar, force, scale, lam_x, g, p, i, j, k);
  }
}

// ----------------------------------------------------------------------------------
static dim3 adj_grid(const MeshDims& d) { return particle_grid_dims(d.cells(), d.batch, kAdjThreads, kAdjCtasPerSm); }

size_t adjoint_partials_count(const MeshDims& d) { return (size_t)2 * adj_grid(d).x * d.batch; }

// out[b][2] = sums of the per-CTA partials of batch entry b: each thread adds a strided
// slice, then a shared-memory tree in a fixed order (deterministic).
__global__ void __launch_bounds__(256) k_sum_partials(const double* __restrict__ partials, int nctas,
                                                      double* __restrict__ out) {
  __shared__ double sk[256], sd[256];
  const double* p = partials + 2ll * nctas * blockIdx.x;
  double a = 0.0, c = 0.0;
  for (int i = threadIdx.x; i < nctas; i += 256) {
    a += p[2 * i];
    c += p[2 * i + 1];
  }
  sk[threadIdx.x] = a;
  sd[threadIdx.x] = c;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sk[threadIdx.x] += sk[threadIdx.x + w];
      sd[threadIdx.x] += sd[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = sk[0];
    out[2 * blockIdx.x + 1] = sd[0];
  }
}

cudaError_t sum_adjoint_partials(const double* partials, const MeshDims& d, double* out, cudaStream_t s) {
  k_sum_partials<<<d.batch, 256, 0, s>>>(partials, (int)adj_grid(d).x, out);
  note_launch();
  return cudaGetLastError();
}

cudaError_t adjoint_unkick_paint(const float* disp, float* vel, const float* lam_x, float* lam_v, const float* force,
                                 float kick, float drift, float* ubar, double* partials, const MeshDims& d,
                                 cudaStream_t s, bool vec4, float* undrift_disp) {
  // without undrift_disp the kernel only reads the positions
  float* dp = undrift_disp ? undrift_disp : const_cast<float*>(disp);
  const int undrift = undrift_disp != nullptr;
  cudaError_t e = cudaMemsetAsync(ubar, 0, sizeof(float) * (vec4 ? 4 : 3) * (size_t)d.cells() * d.batch, s);
  if (e != cudaSuccess) return e;
  if (vec4)
    k_adj_unkick_paint<true><<<adj_grid(d), kAdjThreads, 0, s>>>(dp, undrift, vel, lam_x, lam_v, force, kick, drift, ubar,
                                                                 partials, make_pgrid(d),
                                                                 brick_xdepth(d.nx, d.ny, d.nz, d.batch, 4ll * sm_count()));
  else
    k_adj_unkick_paint<false><<<adj_grid(d), kAdjThreads, 0, s>>>(dp, undrift, vel, lam_x, lam_v, force, kick, drift, ubar,
                                                                  partials, make_pgrid(d), 16);
  note_launch();
  return cudaGetLastError();
}

cudaError_t divergence_fd(const float* u, float alpha, const float* w, float beta, int aos, int accumulate,
                          float* out, const MeshDims& d, cudaStream_t s) {
  // aos 0: three meshes; 1: particle grids (3 floats per cell); 2: float4 meshes
  const long long cell_stride = aos == 2 ? 4 : (aos ? 3 : 1);
  const long long comp_stride = aos ? 1 : d.cells();
  k_div_fd<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(u, alpha, w, beta, cell_stride, comp_stride,
                                                                          accumulate, out, make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

cudaError_t adjoint_position(const float* disp, const float* u, const float* rho_bar, const float* force, float scale,
                             float* lam_x, const MeshDims& d, cudaStream_t s) {
  k_adj_position<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(disp, u, rho_bar, force, scale,
                                                                                lam_x, make_pgrid(d));
  note_launch();
  return cudaGetLastError();
}

}  // namespace jfli
