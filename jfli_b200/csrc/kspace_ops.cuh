// k-space operators applied inside the x pass of the 3D FFT (see fft.cu).
//
// Wavenumbers follow the particle-mesh convention of JaxPM's `fftk`
// (k_i = 2*pi*fftfreq(n_i), radians per cell) for the Poisson/PGD kernels, and the
// physical convention of jax-fli's `_initialize_pk` (k_i = 2*pi*fftfreq(n_i)*n_i/L_i,
// h/Mpc) for P(k) and initial conditions.
#pragma once

#include "common.cuh"

namespace jfli {

// k_i^2 for bin i of an axis of length n, rounded to float like fftk's float32 table.
__device__ __forceinline__ float k_rad_per_cell(int i, int n) {
  return (float)(6.283185307179586476925 * (double)signed_freq(i, n) / (double)n);
}

// Poisson potential: pot_k = delta_k * (-1/k^2) * norm, k = 0 -> 0.
// Follows JaxPM `invlaplace_kernel` (reference call site pm/solvers.py:22 via pm_forces).
struct PoissonOp {
  static constexpr bool kInverse = true;
  static constexpr bool kStore = true;
  int nx, ny, nz;
  float norm;
  static size_t smem_bytes(const PoissonOp& op) { return sizeof(float) * op.nx; }
  __device__ void prologue(float* sm, int) const {
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
      const float k = k_rad_per_cell(i, nx);
      sm[i] = k * k;
    }
    __syncthreads();
  }
  __device__ float2 apply(float2 v, int kx, int ky, int kz, float* sm, int) const {
    const float k1 = k_rad_per_cell(ky, ny);
    const float k2 = k_rad_per_cell(kz, nz);
    const float kk = sm[kx] + k1 * k1 + k2 * k2;
    const float g = (kk == 0.f) ? 0.f : -1.f / kk;
    return cscale(v, g * norm);
  }
  __device__ void epilogue(float*, int, int, int) const {}
};

// PGD short-range potential (reference pm/correction.py:177-189), optionally mixed with the
// Poisson potential:
// pot_k = delta_k * (-1/k^2) * (c0 + c1 exp(-kl^2/k^2) exp(-k^4/ks^4)) * norm, k = 0 -> 0.
// (c0, c1) = (0, 1) is the PGD potential; (kick, boost) the combined potential whose force
// is a reversible step's kick plus SharpeningKernel's velocity boost at the same positions
// (reference pm/solvers.py:292-318, pm/correction.py:214-333).
struct PgdOp {
  static constexpr bool kInverse = true;
  static constexpr bool kStore = true;
  int nx, ny, nz;
  float norm, kl2, ks4;
  float c0 = 0.f, c1 = 1.f;
  static size_t smem_bytes(const PgdOp& op) { return sizeof(float) * op.nx; }
  __device__ void prologue(float* sm, int) const {
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
      const float k = k_rad_per_cell(i, nx);
      sm[i] = k * k;
    }
    __syncthreads();
  }
  __device__ float2 apply(float2 v, int kx, int ky, int kz, float* sm, int) const {
    const float k1 = k_rad_per_cell(ky, ny);
    const float k2 = k_rad_per_cell(kz, nz);
    const float kk = sm[kx] + k1 * k1 + k2 * k2;
    if (kk == 0.f) return make_float2(0.f, 0.f);
    const float range = expf(-kl2 / kk) * expf(-(kk * kk) / ks4);
    return cscale(v, (-1.f / kk) * (c0 + c1 * range) * norm);
  }
  __device__ void epilogue(float*, int, int, int) const {}
};

// Linear interpolation with end extrapolation on a tabulated P(k), the behaviour of
// jax_cosmo's `interp` used by JaxPM `interpolate_power_spectrum`
// (reference call site initial.py:171-173; infer/dist.py:50-53).
__device__ __forceinline__ float interp_table(float x, const float* xp, const float* fp, int n) {
  // first index with xp[i] >= x (searchsorted, side="left")
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (xp[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  int i = lo - 1;
  i = i < 0 ? 0 : (i > n - 2 ? n - 2 : i);
  const float slope = (fp[i + 1] - fp[i]) / (xp[i + 1] - xp[i]);
  return fp[i] + (x - xp[i]) * slope;
}

// interp_table with the slope of the segment it used (the derivative of the linear
// interpolation, end segments extrapolated as in the value).
__device__ __forceinline__ float interp_table_d(float x, const float* xp, const float* fp, int n, float& slope) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (xp[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  int i = lo - 1;
  i = i < 0 ? 0 : (i > n - 2 ? n - 2 : i);
  slope = (fp[i + 1] - fp[i]) / (xp[i + 1] - xp[i]);
  return fp[i] + (x - xp[i]) * slope;
}

// Gaussian initial conditions (reference initial.py:175-182):
// field_k *= sqrt(P(|k|) * M / V) * norm, |k| in h/Mpc. `zero_mode_one` reproduces the
// k = 0 guard of infer/dist.py:68.
struct IcOp {
  static constexpr bool kInverse = true;
  static constexpr bool kStore = true;
  int nx, ny, nz;
  const float* ktab;
  const float* ptab;
  int ntab;
  float lx, ly, lz;  // box side lengths L_i
  float factor;      // M / V
  float norm;        // 1 / M
  int zero_mode_one;
  // Tangent mode (dptab != null): the derivative of the multiplier along a change dptab
  // of the table, interp(dptab) * factor / (2 sqrt(P)) (0 where P <= 0 and at the
  // k = 0 guard), used for gradients with respect to the cosmology behind P(k).
  const float* dptab = nullptr;
  static size_t smem_bytes(const IcOp& op) { return sizeof(float) * (op.nx + 3 * op.ntab); }
  __device__ void prologue(float* sm, int) const {
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
      sm[i] = k_rad_per_cell(i, nx) / lx * (float)nx;
    }
    for (int i = threadIdx.x; i < ntab; i += blockDim.x) {
      sm[nx + i] = ktab[i];
      sm[nx + ntab + i] = ptab[i];
      if (dptab) sm[nx + 2 * ntab + i] = dptab[i];
    }
    __syncthreads();
  }
  __device__ float2 apply(float2 v, int kx, int ky, int kz, float* sm, int) const {
    const float ax = sm[kx];
    const float ay = k_rad_per_cell(ky, ny) / ly * (float)ny;
    const float az = k_rad_per_cell(kz, nz) / lz * (float)nz;
    const float kmag = sqrtf(ax * ax + ay * ay + az * az);
    float pk = interp_table(kmag, sm + nx, sm + nx + ntab, ntab) * factor;
    if (dptab) {
      const float dpk = interp_table(kmag, sm + nx, sm + nx + 2 * ntab, ntab) * factor;
      float m = pk > 0.f ? dpk / (2.0f * sqrtf(pk)) : 0.f;
      if (zero_mode_one && kmag == 0.f) m = 0.f;
      return cscale(v, m * norm);
    }
    if (zero_mode_one && kmag == 0.f) pk = 1.f;
    return cscale(v, sqrtf(pk) * norm);
  }
  __device__ void epilogue(float*, int, int, int) const {}
};

// Power spectrum histogram (reference _src/power/_compute.py:23-119): |delta_k|^2 with
// ortho normalisation binned by digitize(|k|, kedges) over the full grid. The half
// spectrum stores each mode with 0 < kz < nz/2 once for itself and its conjugate
// partner, so those modes count twice. Sums are kept in FP64.
struct PkOp {
  static constexpr bool kInverse = false;
  static constexpr bool kStore = false;
  int nx, ny, nz;
  const float* kedges;
  int nedges;
  float cx, cy, cz;  // 2*pi / L_i
  float norm;        // 1 / M for norm="ortho"
  double* partials;  // [batch][nctas][3][nedges+1]
  static size_t smem_bytes(const PkOp& op) {
    return sizeof(double) * 3 * (op.nedges + 1) + sizeof(float) * (op.nedges + 1);
  }
  __device__ void prologue(float* smf, int) const {
    double* bins = reinterpret_cast<double*>(smf);
    float* edges = reinterpret_cast<float*>(bins + 3 * (nedges + 1));
    for (int i = threadIdx.x; i < 3 * (nedges + 1); i += blockDim.x) bins[i] = 0.0;
    for (int i = threadIdx.x; i < nedges; i += blockDim.x) edges[i] = kedges[i];
    __syncthreads();
  }
  __device__ float2 apply(float2 v, int kx, int ky, int kz, float* smf, int) const {
    double* bins = reinterpret_cast<double*>(smf);
    const float* edges = reinterpret_cast<const float*>(bins + 3 * (nedges + 1));
    // |k| with the rounding of the reference's float32 grid: no FMA contraction, sum in
    // x, y, z order, correctly rounded sqrt (decides the bin of modes on an edge)
    const float ax = __fmul_rn(cx, (float)signed_freq(kx, nx));
    const float ay = __fmul_rn(cy, (float)signed_freq(ky, ny));
    const float az = __fmul_rn(cz, (float)signed_freq(kz, nz));
    const float kmag = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ax, ax), __fmul_rn(ay, ay)), __fmul_rn(az, az)));
    // digitize(right=False): number of edges <= kmag
    int lo = 0, hi = nedges;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (edges[mid] <= kmag)
        lo = mid + 1;
      else
        hi = mid;
    }
    const int bin = lo;
    const double w = (kz == 0 || 2 * kz == nz) ? 1.0 : 2.0;
    const double p = w * ((double)v.x * v.x + (double)v.y * v.y) * (double)norm;
    const double kw = w * (double)kmag;
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, bin);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    double sp = 0.0, sw = 0.0, sk = 0.0;
    unsigned m = peers;
    while (m) {
      const int l = __ffs(m) - 1;
      sp += __shfl_sync(peers, p, l);
      sw += __shfl_sync(peers, w, l);
      sk += __shfl_sync(peers, kw, l);
      m &= m - 1;
    }
    if (lane == leader) {
      atomicAdd(&bins[bin], sp);
      atomicAdd(&bins[(nedges + 1) + bin], sw);
      atomicAdd(&bins[2 * (nedges + 1) + bin], sk);
    }
    return v;
  }
  __device__ void epilogue(float* smf, int batch, int cta, int nctas) const {
    const double* bins = reinterpret_cast<const double*>(smf);
    const int nb = 3 * (nedges + 1);
    double* dst = partials + ((long long)batch * nctas + cta) * nb;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) dst[i] = bins[i];
  }
};

// Adjoint of P(k) with respect to the mesh: mode k is scaled by weights[bin(k)] * norm,
// bin(k) = digitize(|k|, kedges) with the same |k| rounding as PkOp, so that the inverse
// transform gives dL/dmesh = sum over bins of dL/dP_b * dP_b/dmesh when
// weights[b] = 2 * dL/dP_b * prod(L/N) / count_b (0 for the dropped under/overflow bins).
// L_l(mu) by the reference's recurrence, in FP32 (the multipole weights (2l + 1) L_l(mu) of
// the reference's _power, _src/power/_compute.py:96-103)
__device__ __forceinline__ float legendre_f32(int ell, float mu) {
  if (ell == 0) return 1.f;
  if (ell == 1) return mu;
  float p0 = 1.f, p1 = mu;
  for (int n = 2; n <= ell; ++n) {
    const float pn = __fdiv_rn(__fsub_rn(__fmul_rn(__fmul_rn((float)(2 * n - 1), mu), p1), __fmul_rn((float)(n - 1), p0)),
                               (float)n);
    p0 = p1;
    p1 = pn;
  }
  return p1;
}

constexpr int kMaxAdjPoles = 8;

// Adjoint of the binned P(k) sums: out = irfft(rfft(mesh) * w(k) / M). Monopole (nell = 0):
// w(k) = weights[bin(|k|)]. Multipoles of an auto spectrum (nell > 0): the mode's weight is
// sum over the multipoles e of weights[e][bin] (2l_e + 1) L_l_e(mu), mu = (k . los) / |k|,
// and w(k) its mean over the mode and its conjugate partner (a real mesh's gradient sees
// only that Hermitian part). The partner's signed frequencies are the mode's negated, except
// along an axis where the mode sits on the Nyquist plane (index n/2, frequency -n/2 for
// both): there mu is not -mu, and odd multipoles of an auto spectrum do not vanish.
// Cross spectra (cplx = 1): weights holds the real then the imaginary parts, nell x (nedges +
// 1) each, of a complex per-bin factor c; the Hermitian part of c w(k) is the multiplier:
// Re(c) (w(k) + w(partner)) / 2 + i Im(c) (w(k) - w(partner)) / 2.
struct PkAdjOp {
  static constexpr bool kInverse = true;
  static constexpr bool kStore = true;
  int nx, ny, nz;
  const float* kedges;
  const float* weights;  // nedges + 1
  int nedges;
  float cx, cy, cz;  // 2*pi / L_i
  float norm;        // 1 / M (inverse transform)
  int nell = 0;      // multipoles: weights holds nell x (nedges + 1) (twice that when cplx)
  int cplx = 0;
  int ells[kMaxAdjPoles] = {};
  float lx = 0.f, ly = 0.f, lz = 1.f;  // unit line of sight
  static size_t smem_bytes(const PkAdjOp& op) {
    return sizeof(float) * (op.nedges + (op.cplx ? 2 : 1) * (op.nell > 0 ? op.nell : 1) * (op.nedges + 1));
  }
  __device__ void prologue(float* sm, int) const {
    const int nw = (cplx ? 2 : 1) * (nell > 0 ? nell : 1) * (nedges + 1);
    for (int i = threadIdx.x; i < nedges; i += blockDim.x) sm[i] = kedges[i];
    for (int i = threadIdx.x; i < nw; i += blockDim.x) sm[nedges + i] = weights[i];
    __syncthreads();
  }
  __device__ float2 apply(float2 v, int kx, int ky, int kz, float* sm, int) const {
    const float ax = __fmul_rn(cx, (float)signed_freq(kx, nx));
    const float ay = __fmul_rn(cy, (float)signed_freq(ky, ny));
    const float az = __fmul_rn(cz, (float)signed_freq(kz, nz));
    const float kmag = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ax, ax), __fmul_rn(ay, ay)), __fmul_rn(az, az)));
    int lo = 0, hi = nedges;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (sm[mid] <= kmag)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (nell == 0) return cscale(v, sm[nedges + lo] * norm);
    const float dot = __fadd_rn(__fadd_rn(__fmul_rn(ax, lx), __fmul_rn(ay, ly)), __fmul_rn(az, lz));
    const float mu = kmag == 0.f ? 0.f : __fdiv_rn(dot, kmag);
    const float px = 2 * kx == nx ? ax : -ax, py = 2 * ky == ny ? ay : -ay, pz = 2 * kz == nz ? az : -az;
    const float dotp = __fadd_rn(__fadd_rn(__fmul_rn(px, lx), __fmul_rn(py, ly)), __fmul_rn(pz, lz));
    const float mup = kmag == 0.f ? 0.f : __fdiv_rn(dotp, kmag);
    float w = 0.f, wo = 0.f;
    const int im0 = nedges + nell * (nedges + 1);
    for (int e = 0; e < nell; ++e) {
      const float f = (float)(2 * ells[e] + 1);
      const float a = __fmul_rn(f, legendre_f32(ells[e], mu)), b = __fmul_rn(f, legendre_f32(ells[e], mup));
      w += sm[nedges + e * (nedges + 1) + lo] * (0.5f * (a + b));
      if (cplx) wo += sm[im0 + e * (nedges + 1) + lo] * (0.5f * (a - b));
    }
    if (!cplx) return cscale(v, w * norm);
    return make_float2((v.x * w - v.y * wo) * norm, (v.x * wo + v.y * w) * norm);
  }
  __device__ void epilogue(float*, int, int, int) const {}
};

}  // namespace jfli
