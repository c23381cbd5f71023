// Legendre stages of the spherical harmonic transform of HEALPix ring maps (FP64), the
// O(lmax^2 x rings) part of healpy's anafast (reference _src/power/_compute.py:175-191).
// The ring FFTs along phi run on the host; these kernels take and return per-ring Fourier
// coefficients F[r][m] (m = 0..lmax, phase e^{-i m phi_0} applied).
//
//   analysis:  a_lm  = w * sum_r lambda_lm(theta_r) F[r][m]
//   synthesis: G[r][m] = sum_l a_lm lambda_lm(theta_r)
//
// lambda_lm are the orthonormal associated Legendre functions with the Condon-Shortley
// phase: lambda_mm = (-1)^m sqrt((2m+1)/(4 pi) (2m)!/(4^m (m!)^2)) sin^m theta, then the
// three-term recursion in l. lambda_mm is formed in log space; where it is below FP64
// range the recursion runs on values scaled by e^s and drops the scale as they grow
// (factor 1e100 at a time), so that rings where lambda_lm becomes significant before lmax
// are not lost to underflow. a_lm is packed by m: a[m][l - m], offset m (lmax + 1) - m (m - 1) / 2.
#include "common.cuh"
#include "internal.h"

namespace jfli {

constexpr int kShtThreads = 128;
constexpr int kShtLTile = 16;
// row stride of the per-tile contributions (one row per l): one element of padding so that
// the reduction's lanes, which read one element per row, fall in different banks
constexpr int kShtRow = kShtThreads + 1;

__host__ __device__ __forceinline__ long long alm_offset(int m, int lmax) {
  return (long long)m * (lmax + 1) - (long long)m * (m - 1) / 2;
}

struct LegendreState {
  double prev, cur, scale, escale;
};

// lambda_mm for one ring (scaled), and e^-scale.
__device__ __forceinline__ LegendreState legendre_start(int m, double z) {
  const double logc = 0.5 * log((2.0 * m + 1.0) / (4.0 * 3.14159265358979323846)) +
                      0.5 * (lgamma(2.0 * m + 1.0) - 2.0 * lgamma(m + 1.0) - m * log(4.0));
  const double s2 = 1.0 - z * z;
  LegendreState st;
  const double logv = (m == 0) ? logc : logc + 0.5 * m * log(s2);
  st.scale = (logv < -600.0) ? (-300.0 - logv) : 0.0;
  const double sign = (m & 1) ? -1.0 : 1.0;
  st.cur = sign * exp(logv + st.scale);
  st.prev = 0.0;
  st.escale = (st.scale == 0.0) ? 1.0 : (st.scale < 745.0 ? exp(-st.scale) : 0.0);
  return st;
}

// Advance to l (>= m + 1) with the recursion coefficients of (l, m); returns lambda_lm.
__device__ __forceinline__ double legendre_step(LegendreState& st, double z, double a, double b) {
  double nxt = a * (z * st.cur - b * st.prev);
  if (st.scale > 0.0 && fabs(nxt) > 1e100) {
    nxt *= 1e-100;
    st.cur *= 1e-100;
    st.scale -= 230.25850929940458;  // ln 1e100
    st.escale = (st.scale < 745.0) ? exp(-st.scale) : 0.0;
  }
  st.prev = st.cur;
  st.cur = nxt;
  return nxt * st.escale;
}

// recursion coefficients for l of a tile (a_l, b_l; l = m + 1 uses a = sqrt(2m+3), b = 0)
__device__ __forceinline__ void legendre_coeffs(int l, int m, double& a, double& b) {
  if (l == m + 1) {
    a = sqrt(2.0 * m + 3.0);
    b = 0.0;
  } else {
    const double ll = (double)l, mm = (double)m;
    a = sqrt((4.0 * ll * ll - 1.0) / (ll * ll - mm * mm));
    b = sqrt(((ll - 1.0) * (ll - 1.0) - mm * mm) / (4.0 * (ll - 1.0) * (ll - 1.0) - 1.0));
  }
}

__global__ void __launch_bounds__(kShtThreads) k_sht_analysis(const double2* __restrict__ F, const double* __restrict__ z,
                                                               int nrings, int lmax, double w, double2* __restrict__ alm) {
  extern __shared__ double2 contrib[];  // [kShtLTile][kShtRow]
  __shared__ double coef[2][kShtLTile];
  __shared__ double2 part[kShtThreads / kShtLTile][kShtLTile];
  const int m = blockIdx.y;
  const int r = blockIdx.x * kShtThreads + threadIdx.x;
  const bool active = r < nrings;
  const double zr = active ? z[r] : 0.0;
  const double2 f = active ? F[(long long)r * (lmax + 1) + m] : make_double2(0.0, 0.0);
  LegendreState st = legendre_start(m, active ? zr : 0.0);
  const long long off = alm_offset(m, lmax);
  for (int l0 = m; l0 <= lmax; l0 += kShtLTile) {
    if (threadIdx.x < kShtLTile) {
      const int l = l0 + threadIdx.x;
      double a = 0.0, b = 0.0;
      if (l > m && l <= lmax) legendre_coeffs(l, m, a, b);
      coef[0][threadIdx.x] = a;
      coef[1][threadIdx.x] = b;
    }
    __syncthreads();
    for (int t = 0; t < kShtLTile; ++t) {
      const int l = l0 + t;
      double lam = 0.0;
      if (l == m)
        lam = st.cur * st.escale;
      else if (l <= lmax)
        lam = legendre_step(st, zr, coef[0][t], coef[1][t]);
      contrib[t * kShtRow + threadIdx.x] = active ? make_double2(lam * f.x, lam * f.y) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    {  // thread (q, row): sum of kShtLTile rings of one l
      const int row = threadIdx.x & (kShtLTile - 1), q = threadIdx.x / kShtLTile;
      double sx = 0.0, sy = 0.0;
      for (int i = 0; i < kShtLTile; ++i) {
        const double2 c = contrib[row * kShtRow + q * kShtLTile + i];
        sx += c.x;
        sy += c.y;
      }
      part[q][row] = make_double2(sx, sy);
    }
    __syncthreads();
    if (threadIdx.x < kShtLTile) {
      const int l = l0 + threadIdx.x;
      if (l <= lmax) {
        double sx = 0.0, sy = 0.0;
        for (int q = 0; q < kShtThreads / kShtLTile; ++q) {
          sx += part[q][threadIdx.x].x;
          sy += part[q][threadIdx.x].y;
        }
        atomicAdd(&alm[off + (l - m)].x, w * sx);
        atomicAdd(&alm[off + (l - m)].y, w * sy);
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kShtThreads) k_sht_synthesis(const double2* __restrict__ alm,
                                                                const double* __restrict__ z, int nrings, int lmax,
                                                                double2* __restrict__ G) {
  __shared__ double coef[2][kShtLTile];
  __shared__ double2 a_tile[kShtLTile];
  const int m = blockIdx.y;
  const int r = blockIdx.x * kShtThreads + threadIdx.x;
  const bool active = r < nrings;
  const double zr = active ? z[r] : 0.0;
  LegendreState st = legendre_start(m, zr);
  const long long off = alm_offset(m, lmax);
  double gx = 0.0, gy = 0.0;
  for (int l0 = m; l0 <= lmax; l0 += kShtLTile) {
    if (threadIdx.x < kShtLTile) {
      const int l = l0 + threadIdx.x;
      double a = 0.0, b = 0.0;
      if (l > m && l <= lmax) legendre_coeffs(l, m, a, b);
      coef[0][threadIdx.x] = a;
      coef[1][threadIdx.x] = b;
      a_tile[threadIdx.x] = (l <= lmax) ? alm[off + (l - m)] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int t = 0; t < kShtLTile; ++t) {
      const int l = l0 + t;
      if (l > lmax) break;
      const double lam = (l == m) ? st.cur * st.escale : legendre_step(st, zr, coef[0][t], coef[1][t]);
      gx += lam * a_tile[t].x;
      gy += lam * a_tile[t].y;
    }
    __syncthreads();
  }
  if (active) G[(long long)r * (lmax + 1) + m] = make_double2(gx, gy);
}

// ---- ring transforms along phi ------------------------------------------------------
// RING geometry of ring r (0 = northernmost, i = r + 1): pixel count, first pixel, and the
// longitude of the first pixel centre (Gorski et al. 2005).
struct RingPhi {
  long long start;
  int n;
  double phi0;
};

__device__ __forceinline__ RingPhi ring_phi(int r, int nside) {
  const int i = r + 1;
  const long long npix = 12LL * nside * nside;
  RingPhi g;
  if (i < nside) {
    g.n = 4 * i;
    g.start = 2LL * i * (i - 1);
    g.phi0 = 3.14159265358979323846 / (4.0 * i);
  } else if (i <= 3 * nside) {
    g.n = 4 * nside;
    g.start = 2LL * nside * (nside - 1) + (long long)(i - nside) * 4 * nside;
    g.phi0 = ((i - nside + 1) % 2 == 1) ? 0.0 : 3.14159265358979323846 / (4.0 * nside);
  } else {
    const int j = 4 * nside - i;
    g.n = 4 * j;
    g.start = npix - 2LL * j * (j + 1);
    g.phi0 = 3.14159265358979323846 / (4.0 * j);
  }
  return g;
}

constexpr int kRingThreads = 128;
constexpr int kReseed = 64;  // exact phase every 64 terms; rotations in between

// e^{-i m phi_j}, phi_j = phi0 + 2 pi j / n, with the angle reduced exactly: (m j) mod n.
__device__ __forceinline__ double2 phase(int m, int j, int n, double phi0, double sign) {
  const long long q = ((long long)m * j) % n;
  const double ang = (double)m * phi0 + 6.283185307179586476925 * (double)q / (double)n;
  double sn, cs;
  sincos(ang, &sn, &cs);
  return make_double2(cs, sign * sn);
}

// F[r][m] = sum_j f_j e^{-i m phi_j}, m = 0..lmax (aliasing for m >= n is the DFT's own).
// One block per (ring, 128 m); the ring's values staged in shared memory.
__global__ void __launch_bounds__(kRingThreads) k_ring_analysis(const double* __restrict__ map, int nside, int lmax,
                                                                double2* __restrict__ F) {
  extern __shared__ double ring[];
  const int r = blockIdx.y;
  const RingPhi g = ring_phi(r, nside);
  for (int j = threadIdx.x; j < g.n; j += blockDim.x) ring[j] = map[g.start + j];
  __syncthreads();
  const int m = blockIdx.x * kRingThreads + threadIdx.x;
  if (m > lmax) return;
  double2 step;  // e^{-i 2 pi m / n}
  {
    const double ang = 6.283185307179586476925 * (double)(m % g.n) / (double)g.n;
    double sn, cs;
    sincos(ang, &sn, &cs);
    step = make_double2(cs, -sn);
  }
  double sx = 0.0, sy = 0.0;
  for (int j0 = 0; j0 < g.n; j0 += kReseed) {
    double2 w = phase(m, j0, g.n, g.phi0, -1.0);
    const int j1 = min(j0 + kReseed, g.n);
    for (int j = j0; j < j1; ++j) {
      const double f = ring[j];
      sx += f * w.x;
      sy += f * w.y;
      w = make_double2(w.x * step.x - w.y * step.y, w.x * step.y + w.y * step.x);
    }
  }
  F[(long long)r * (lmax + 1) + m] = make_double2(sx, sy);
}

// f_j = Re G[r][0] + 2 sum_{m >= 1} Re(G[r][m] e^{i m phi_j}). One block per (ring, 128
// pixels); the ring's coefficients staged in shared memory.
__global__ void __launch_bounds__(kRingThreads) k_ring_synthesis(const double2* __restrict__ G, int nside, int lmax,
                                                                 double* __restrict__ map) {
  extern __shared__ double2 coef[];
  const int r = blockIdx.y;
  const RingPhi g = ring_phi(r, nside);
  for (int m = threadIdx.x; m <= lmax; m += blockDim.x) coef[m] = G[(long long)r * (lmax + 1) + m];
  __syncthreads();
  const int j = blockIdx.x * kRingThreads + threadIdx.x;
  if (j >= g.n) return;
  const double phij = g.phi0 + 6.283185307179586476925 * (double)j / (double)g.n;
  double2 step;  // e^{i phi_j}
  {
    double sn, cs;
    sincos(phij, &sn, &cs);
    step = make_double2(cs, sn);
  }
  double acc = 0.0;
  for (int m0 = 1; m0 <= lmax; m0 += kReseed) {
    double2 w = phase(m0, j, g.n, g.phi0, 1.0);
    const int m1 = min(m0 + kReseed, lmax + 1);
    for (int m = m0; m < m1; ++m) {
      acc += coef[m].x * w.x - coef[m].y * w.y;
      w = make_double2(w.x * step.x - w.y * step.y, w.x * step.y + w.y * step.x);
    }
  }
  map[g.start + j] = coef[0].x + 2.0 * acc;
}

cudaError_t sht_ring_analysis(const double* map, int nside, int lmax, double* F, cudaStream_t s) {
  const int nrings = 4 * nside - 1;
  const size_t smem = sizeof(double) * 4 * (size_t)nside;
  cudaError_t e = cudaFuncSetAttribute(k_ring_analysis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((lmax + kRingThreads) / kRingThreads, nrings);
  k_ring_analysis<<<grid, kRingThreads, smem, s>>>(map, nside, lmax, reinterpret_cast<double2*>(F));
  note_launch();
  return cudaGetLastError();
}

cudaError_t sht_ring_synthesis(const double* G, int nside, int lmax, double* map, cudaStream_t s) {
  const int nrings = 4 * nside - 1;
  const size_t smem = sizeof(double2) * (size_t)(lmax + 1);
  cudaError_t e = cudaFuncSetAttribute(k_ring_synthesis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((4 * nside + kRingThreads - 1) / kRingThreads, nrings);
  k_ring_synthesis<<<grid, kRingThreads, smem, s>>>(reinterpret_cast<const double2*>(G), nside, lmax, map);
  note_launch();
  return cudaGetLastError();
}

cudaError_t sht_analysis(const double* F, const double* z, int nrings, int lmax, double weight, double* alm,
                         cudaStream_t s) {
  const long long nalm = alm_offset(lmax + 1, lmax);
  cudaError_t e = cudaMemsetAsync(alm, 0, sizeof(double2) * (size_t)nalm, s);
  if (e != cudaSuccess) return e;
  const size_t smem = sizeof(double2) * kShtLTile * kShtRow;
  e = cudaFuncSetAttribute(k_sht_analysis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((nrings + kShtThreads - 1) / kShtThreads, lmax + 1);
  k_sht_analysis<<<grid, kShtThreads, smem, s>>>(reinterpret_cast<const double2*>(F), z, nrings, lmax, weight,
                                                  reinterpret_cast<double2*>(alm));
  note_launch();
  return cudaGetLastError();
}

cudaError_t sht_synthesis(const double* alm, const double* z, int nrings, int lmax, double* G, cudaStream_t s) {
  const dim3 grid((nrings + kShtThreads - 1) / kShtThreads, lmax + 1);
  k_sht_synthesis<<<grid, kShtThreads, 0, s>>>(reinterpret_cast<const double2*>(alm), z, nrings, lmax,
                                                reinterpret_cast<double2*>(G));
  note_launch();
  return cudaGetLastError();
}

// C_l = (Re a_l0 b_l0* + 2 sum_{m=1..l} Re a_lm b_lm*) / (2l + 1) (healpy alm2cl), one
// thread per l, FP64 sums in increasing m (a fixed order: the result is deterministic).
__global__ void k_sht_alm2cl(const double2* __restrict__ a, const double2* __restrict__ b, int lmax,
                             double* __restrict__ cl) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l > lmax) return;
  double acc = 0.0;
  for (int m = 1; m <= l; ++m) {
    const long long o = alm_offset(m, lmax) + (l - m);
    const double2 x = a[o], y = b[o];
    acc += x.x * y.x + x.y * y.y;
  }
  const double2 x0 = a[l], y0 = b[l];
  cl[l] = (x0.x * y0.x + x0.y * y0.y + 2.0 * acc) / (2.0 * l + 1.0);
}

cudaError_t sht_alm2cl(const double* alm1, const double* alm2, int lmax, double* cl, cudaStream_t s) {
  const int threads = 128;
  k_sht_alm2cl<<<(lmax + threads) / threads, threads, 0, s>>>(reinterpret_cast<const double2*>(alm1),
                                                            reinterpret_cast<const double2*>(alm2 ? alm2 : alm1),
                                                            lmax, cl);
  note_launch();
  return cudaGetLastError();
}

}  // namespace jfli
