// HEALPix lightcone shell painting (reference pm/interp.py:161-209 ->
// fields/particles.py:326-442 -> _src/fields/_painting.py:249-348 -> JaxPM
// `paint_particles_spherical`).
//
// Each particle is placed in comoving Mpc/h, its distance r to the observer selects the
// shell R_min < r <= R_max, and its direction is deposited on the RING-ordered HEALPix
// map either on one pixel ("ngp", ang2pix) or on the 4 pixels of the bilinear
// interpolation ("bilinear", the default scheme). Pixel geometry follows the published
// HEALPix construction (Gorski et al. 2005, ApJ 622:759): ring index, ring start pixel,
// ring length, ring colatitude and the half-pixel shift of alternate equatorial rings.
// Angles are computed in FP64 from the FP32 positions.
#include <math.h>

#include <cmath>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "cic.cuh"
#include "common.cuh"
#include "internal.h"
#include "kspace_ops.cuh"

namespace jfli {

struct RingInfo {
  long long start;
  int npix;
  double theta;
  int shifted;
};

// Ring geometry: start pixel, pixel count and half-pixel shift from integer arithmetic;
// the colatitude from the table of the rings' FP64 colatitudes (ring_theta_table).
__device__ __forceinline__ RingInfo ring_info_tab(int ring, int nside, const double* __restrict__ theta_tab) {
  const long long npix = 12LL * nside * nside;
  const long long ncap = 2LL * nside * (nside - 1);
  const int north = ring > 2 * nside ? 4 * nside - ring : ring;
  RingInfo r;
  if (north < nside) {
    r.npix = 4 * north;
    r.shifted = 1;
    r.start = 2LL * north * (north - 1);
  } else {
    r.npix = 4 * nside;
    r.shifted = ((north - nside) & 1) == 0;
    r.start = ncap + (long long)(north - nside) * 4 * nside;
  }
  if (north != ring) r.start = npix - r.start - r.npix;
  r.theta = __ldg(theta_tab + ring);
  return r;
}

// Number of the ring at or above colatitude with cos(theta) = z (0 = north pole).
__device__ __forceinline__ int ring_above(double z, int nside) {
  const double az = fabs(z);
  if (az <= 2.0 / 3.0) return (int)(nside * (2.0 - 1.5 * z));
  const int ir = (int)(nside * sqrt(3.0 * (1.0 - az)));
  return z > 0 ? ir : 4 * nside - ir - 1;
}

__device__ __forceinline__ long long ang2pix_ring(double z, double phi, int nside) {
  const double twopi = 2.0 * M_PI;
  double ph = fmod(phi, twopi);
  if (ph < 0) ph += twopi;
  const double tt = ph / (0.5 * M_PI);  // in [0, 4)
  const double za = fabs(z);
  const long long npix = 12LL * nside * nside;
  const long long ncap = 2LL * nside * (nside - 1);
  if (za <= 2.0 / 3.0) {
    const double t1 = nside * (0.5 + tt);
    const double t2 = nside * z * 0.75;
    const long long jp = (long long)(t1 - t2);
    const long long jm = (long long)(t1 + t2);
    const long long ir = nside + 1 + jp - jm;
    const long long kshift = 1 - (ir & 1);
    long long ip = (jp + jm - nside + kshift + 1) / 2;
    ip %= 4LL * nside;
    if (ip < 0) ip += 4LL * nside;
    return ncap + (ir - 1) * 4LL * nside + ip;
  }
  const double tp = tt - (double)(int)tt;
  const double tmp = nside * sqrt(3.0 * (1.0 - za));
  const long long jp = (long long)(tp * tmp);
  const long long jm = (long long)((1.0 - tp) * tmp);
  const long long ir = jp + jm + 1;
  long long ip = (long long)(tt * ir);
  ip %= 4 * ir;
  if (ip < 0) ip += 4 * ir;
  return z > 0 ? 2 * ir * (ir - 1) + ip : npix - 2 * ir * (ir + 1) + ip;
}

// Bilinear interpolation pixels and weights (the 4-neighbour scheme of HEALPix
// get_interpol / healpy get_interp_weights, RING ordering).
__device__ __forceinline__ void interp_weights(double theta, double phi, int nside, const double* __restrict__ theta_tab,
                                               long long pix[4], double w[4]) {
  const double twopi = 2.0 * M_PI;
  double ph = fmod(phi, twopi);
  if (ph < 0) ph += twopi;
  const long long npix = 12LL * nside * nside;
  const double z = cos(theta);
  const int ir1 = ring_above(z, nside);
  const int ir2 = ir1 + 1;
  double theta1 = 0.0, theta2 = 0.0;
  if (ir1 > 0) {
    const RingInfo r = ring_info_tab(ir1, nside, theta_tab);
    theta1 = r.theta;
    const double dphi = twopi / r.npix;
    const double tmp = ph / dphi - 0.5 * r.shifted;
    long long i1 = tmp < 0 ? (long long)tmp - 1 : (long long)tmp;
    const double wp = (ph - (i1 + 0.5 * r.shifted) * dphi) / dphi;
    long long i2 = i1 + 1;
    if (i1 < 0) i1 += r.npix;
    if (i2 >= r.npix) i2 -= r.npix;
    pix[0] = r.start + i1;
    pix[1] = r.start + i2;
    w[0] = 1.0 - wp;
    w[1] = wp;
  }
  if (ir2 < 4 * nside) {
    const RingInfo r = ring_info_tab(ir2, nside, theta_tab);
    theta2 = r.theta;
    const double dphi = twopi / r.npix;
    const double tmp = ph / dphi - 0.5 * r.shifted;
    long long i1 = tmp < 0 ? (long long)tmp - 1 : (long long)tmp;
    const double wp = (ph - (i1 + 0.5 * r.shifted) * dphi) / dphi;
    long long i2 = i1 + 1;
    if (i1 < 0) i1 += r.npix;
    if (i2 >= r.npix) i2 -= r.npix;
    pix[2] = r.start + i1;
    pix[3] = r.start + i2;
    w[2] = 1.0 - wp;
    w[3] = wp;
  }
  if (ir1 == 0) {
    const double wt = theta / theta2;
    w[2] *= wt;
    w[3] *= wt;
    const double fac = (1.0 - wt) * 0.25;
    w[0] = fac;
    w[1] = fac;
    w[2] += fac;
    w[3] += fac;
    pix[0] = (pix[2] + 2) & 3;
    pix[1] = (pix[3] + 2) & 3;
  } else if (ir2 == 4 * nside) {
    const double wt = (theta - theta1) / (M_PI - theta1);
    w[0] *= (1.0 - wt);
    w[1] *= (1.0 - wt);
    const double fac = wt * 0.25;
    w[0] += fac;
    w[1] += fac;
    w[2] = fac;
    w[3] = fac;
    pix[2] = ((pix[0] + 2) & 3) + npix - 4;
    pix[3] = ((pix[1] + 2) & 3) + npix - 4;
  } else {
    const double wt = (theta - theta1) / (theta2 - theta1);
    w[0] *= (1.0 - wt);
    w[1] *= (1.0 - wt);
    w[2] *= wt;
    w[3] *= wt;
  }
}

// interp_weights with the weights' derivatives along theta and phi (the adjoint of the
// bilinear deposit). Inside a ring pair the weights are products of the ring weight
// (linear in theta between the two rings' thetas) and the in-ring weights (linear in phi
// between the two bracketing pixel centres); the polar caps add the quarter weights of
// the four polar pixels, linear in theta. A weight's jump where the bracket changes is
// continuous in the map, so the piecewise derivatives are the map's.
__device__ __forceinline__ void interp_weights_grad(double theta, double phi, int nside,
                                                    const double* __restrict__ theta_tab, long long pix[4],
                                                    double w[4], double dth[4], double dph[4]) {
  interp_weights(theta, phi, nside, theta_tab, pix, w);
  const double twopi = 2.0 * M_PI;
  const double z = cos(theta);
  const int ir1 = ring_above(z, nside);
  const int ir2 = ir1 + 1;
  double theta1 = 0.0, theta2 = 0.0, a[4] = {0.0, 0.0, 0.0, 0.0}, da[4] = {0.0, 0.0, 0.0, 0.0};
  double ph = fmod(phi, twopi);
  if (ph < 0) ph += twopi;
  if (ir1 > 0) {
    const RingInfo r = ring_info_tab(ir1, nside, theta_tab);
    theta1 = r.theta;
    const double dphi = twopi / r.npix;
    const double tmp = ph / dphi - 0.5 * r.shifted;
    const long long i1 = tmp < 0 ? (long long)tmp - 1 : (long long)tmp;
    const double wp = (ph - (i1 + 0.5 * r.shifted) * dphi) / dphi;
    a[0] = 1.0 - wp;
    a[1] = wp;
    da[0] = -1.0 / dphi;
    da[1] = 1.0 / dphi;
  }
  if (ir2 < 4 * nside) {
    const RingInfo r = ring_info_tab(ir2, nside, theta_tab);
    theta2 = r.theta;
    const double dphi = twopi / r.npix;
    const double tmp = ph / dphi - 0.5 * r.shifted;
    const long long i1 = tmp < 0 ? (long long)tmp - 1 : (long long)tmp;
    const double wp = (ph - (i1 + 0.5 * r.shifted) * dphi) / dphi;
    a[2] = 1.0 - wp;
    a[3] = wp;
    da[2] = -1.0 / dphi;
    da[3] = 1.0 / dphi;
  }
  if (ir1 == 0) {
    const double wt = theta / theta2, dwt = 1.0 / theta2;
    dth[0] = dth[1] = -0.25 * dwt;
    dth[2] = a[2] * dwt - 0.25 * dwt;
    dth[3] = a[3] * dwt - 0.25 * dwt;
    dph[0] = dph[1] = 0.0;
    dph[2] = da[2] * wt;
    dph[3] = da[3] * wt;
  } else if (ir2 == 4 * nside) {
    const double wt = (theta - theta1) / (M_PI - theta1), dwt = 1.0 / (M_PI - theta1);
    dth[0] = -a[0] * dwt + 0.25 * dwt;
    dth[1] = -a[1] * dwt + 0.25 * dwt;
    dth[2] = dth[3] = 0.25 * dwt;
    dph[0] = da[0] * (1.0 - wt);
    dph[1] = da[1] * (1.0 - wt);
    dph[2] = dph[3] = 0.0;
  } else {
    const double wt = (theta - theta1) / (theta2 - theta1), dwt = 1.0 / (theta2 - theta1);
    dth[0] = -a[0] * dwt;
    dth[1] = -a[1] * dwt;
    dth[2] = a[2] * dwt;
    dth[3] = a[3] * dwt;
    dph[0] = da[0] * (1.0 - wt);
    dph[1] = da[1] * (1.0 - wt);
    dph[2] = da[2] * wt;
    dph[3] = da[3] * wt;
  }
}

// Centre (theta, phi) of RING pixel pix: its ring found by bisection on the rings' start
// pixels, phi = (index in ring + shift / 2) 2 pi / pixels in ring.
__device__ __forceinline__ void pix_centre_ring(long long pix, int nside, const double* __restrict__ theta_tab,
                                                double& theta, double& phi) {
  int lo = 1, hi = 4 * nside - 1;  // last ring whose start <= pix
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ring_info_tab(mid, nside, theta_tab).start <= pix)
      lo = mid;
    else
      hi = mid - 1;
  }
  const RingInfo r = ring_info_tab(lo, nside, theta_tab);
  theta = r.theta;
  phi = ((double)(pix - r.start) + 0.5 * r.shifted) * (2.0 * M_PI / r.npix);
}

// Deposit of weight w at direction (vx, vy, vz) (length rr > 0, FP64) on the RING map.
// scheme 0: nearest pixel; 1: bilinear weights of the 4 surrounding pixel centres; 2 (the
// "rbf_neighbor" scheme): the same 4 pixels weighted by a Gaussian radial basis function of
// the angle d between the direction and each pixel centre, exp(-d^2 / (2 sigma^2)),
// normalised to sum 1 (sigma in radians; taken relative to the nearest centre, so the
// weights never all underflow).
__device__ __forceinline__ void deposit_direction(double vx, double vy, double vz, double rr, float w, int nside,
                                                  int scheme, const double* __restrict__ theta_tab,
                                                  float* __restrict__ map, float sigma = 0.f) {
  const long long npix = 12LL * nside * nside;
  const double dr = rr;
  const double zc = vz / dr;
  const double phi = atan2(vy, vx);
  if (scheme == 0) {
    const long long pix = ang2pix_ring(zc, phi, nside);
    if (pix >= 0 && pix < npix) atomicAdd(map + pix, w);
  } else if (scheme == 2) {
    long long pix[4];
    double wt[4];
    interp_weights(acos(fmin(1.0, fmax(-1.0, zc))), phi, nside, theta_tab, pix, wt);
    const double ux = vx / dr, uy = vy / dr, uz = zc;
    double d2[4], dmin = 1e300;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double th, ph;
      pix_centre_ring(pix[q], nside, theta_tab, th, ph);
      const double st = sin(th);
      const double cx = st * cos(ph) - ux, cy = st * sin(ph) - uy, cz = cos(th) - uz;
      const double d = 2.0 * asin(fmin(1.0, 0.5 * sqrt(cx * cx + cy * cy + cz * cz)));
      d2[q] = d * d;
      dmin = fmin(dmin, d2[q]);
    }
    const double inv = 1.0 / (2.0 * (double)sigma * (double)sigma);
    double sum = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      wt[q] = exp(-(d2[q] - dmin) * inv);
      sum += wt[q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (pix[q] >= 0 && pix[q] < npix) atomicAdd(map + pix[q], (float)(wt[q] / sum * (double)w));
  } else {
    long long pix[4];
    double wt[4];
    interp_weights(acos(fmin(1.0, fmax(-1.0, zc))), phi, nside, theta_tab, pix, wt);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (pix[q] >= 0 && pix[q] < npix) atomicAdd(map + pix[q], (float)(wt[q] * (double)w));
  }
}

// The observer-centred position, its length and the shell test are FP64 (from the FP32
// positions): an FP32 |x - o| at a few hundred Mpc/h carries ~1e-5 Mpc/h of rounding, which
// moves particles within that distance of an edge across it.
__global__ void k_healpix_paint(const float* __restrict__ disp, int absolute, const float* __restrict__ weights,
                                float weight, MeshDims d, double3 cell, double3 obs, double rmin, double rmax,
                                int nside, int scheme, const double* __restrict__ theta_tab, float* __restrict__ map,
                                float sigma) {
  const long long np = d.cells();
  const long long npix = 12LL * nside * nside;
  const int b = blockIdx.y;
  disp += (long long)b * np * 3;
  map += (long long)b * npix;
  if (weights) weights += (long long)b * np;
  const long long yz = (long long)d.ny * d.nz;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    double gx = disp[3 * p + 0], gy = disp[3 * p + 1], gz = disp[3 * p + 2];
    if (!absolute) {
      const int i = (int)(p / yz);
      const long long r = p - (long long)i * yz;
      const int j = (int)(r / d.nz);
      const int k = (int)(r - (long long)j * d.nz);
      gx += (double)i;
      gy += (double)j;
      gz += (double)k;
    }
    const double vx = gx * cell.x - obs.x, vy = gy * cell.y - obs.y, vz = gz * cell.z - obs.z;
    const double rr = sqrt(vx * vx + vy * vy + vz * vz);
    if (!(rr > rmin && rr <= rmax)) continue;
    deposit_direction(vx, vy, vz, rr, weights ? weights[p] * weight : weight, nside, scheme, theta_tab, map, sigma);
  }
}

// Several shells of one particle set in one pass (paint_spherical with an array of
// centres, light-cone LPT painted straight to its shells): each particle's FP64 distance
// is tested against every shell (overlapping shells each get their deposit), and the
// particle set is read once instead of once per shell. Shell s deposits weight * scale[s]
// into maps[s].
struct ShellSet {
  int n;
  double rmin[kMaxShellsPerPass], rmax[kMaxShellsPerPass];
  float scale[kMaxShellsPerPass];
};

__global__ void k_healpix_paint_shells(const float* __restrict__ disp, int absolute, const float* __restrict__ weights,
                                       float weight, MeshDims d, double3 cell, double3 obs, ShellSet shells,
                                       int nside, int scheme, const double* __restrict__ theta_tab,
                                       float* __restrict__ maps, float sigma) {
  const long long np = d.cells();
  const long long npix = 12LL * nside * nside;
  const long long yz = (long long)d.ny * d.nz;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    double gx = disp[3 * p + 0], gy = disp[3 * p + 1], gz = disp[3 * p + 2];
    if (!absolute) {
      const int i = (int)(p / yz);
      const long long r = p - (long long)i * yz;
      const int j = (int)(r / d.nz);
      const int k = (int)(r - (long long)j * d.nz);
      gx += (double)i;
      gy += (double)j;
      gz += (double)k;
    }
    const double vx = gx * cell.x - obs.x, vy = gy * cell.y - obs.y, vz = gz * cell.z - obs.z;
    const double rr = sqrt(vx * vx + vy * vy + vz * vz);
    const float w = weights ? weights[p] * weight : weight;
    for (int sh = 0; sh < shells.n; ++sh)
      if (rr > shells.rmin[sh] && rr <= shells.rmax[sh])
        deposit_direction(vx, vy, vz, rr, w * shells.scale[sh], nside, scheme, theta_tab, maps + sh * npix, sigma);
  }
}

// Adjoint of k_healpix_paint_shells for the bilinear and ngp schemes. With maps_bar[s] the
// cotangent of shell s's map, a particle of shell s deposited weight_p scale_s w_q at
// pixels pix_q, so it adds
//   to its position cotangent:  weight_p scale_s sum_q maps_bar[s][pix_q] d w_q / d disp
//   to its weight cotangent:    weight scale_s sum_q maps_bar[s][pix_q] w_q
// (ngp: w = 1 at one pixel, no position term). Shell membership is a step in the distance
// and contributes nothing (as the derivative of a mask). d w / d disp chains the weights'
// theta and phi derivatives with theta = acos(v_z / r), phi = atan2(v_y, v_x),
// v = (grid + disp) cell - observer. Accumulates into disp_bar (and weights_bar).
__global__ void k_healpix_paint_shells_adjoint(const float* __restrict__ disp, int absolute,
                                               const float* __restrict__ weights, float weight, MeshDims d,
                                               double3 cell, double3 obs, ShellSet shells, int nside, int scheme,
                                               const double* __restrict__ theta_tab,
                                               const float* __restrict__ maps_bar, float* __restrict__ disp_bar,
                                               float* __restrict__ weights_bar) {
  const long long np = d.cells();
  const long long npix = 12LL * nside * nside;
  const long long yz = (long long)d.ny * d.nz;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    double gx = disp[3 * p + 0], gy = disp[3 * p + 1], gz = disp[3 * p + 2];
    if (!absolute) {
      const int i = (int)(p / yz);
      const long long r = p - (long long)i * yz;
      const int j = (int)(r / d.nz);
      const int k = (int)(r - (long long)j * d.nz);
      gx += (double)i;
      gy += (double)j;
      gz += (double)k;
    }
    const double vx = gx * cell.x - obs.x, vy = gy * cell.y - obs.y, vz = gz * cell.z - obs.z;
    const double rr = sqrt(vx * vx + vy * vy + vz * vz);
    bool any = false;
    long long pix[4] = {-1, -1, -1, -1};
    double w[4] = {0.0, 0.0, 0.0, 0.0}, dth[4] = {0.0, 0.0, 0.0, 0.0}, dph[4] = {0.0, 0.0, 0.0, 0.0};
    double g_th = 0.0, g_ph = 0.0, g_w = 0.0;
    for (int sh = 0; sh < shells.n; ++sh) {
      if (!(rr > shells.rmin[sh] && rr <= shells.rmax[sh])) continue;
      if (!any) {
        any = true;
        const double zc = vz / rr;
        const double phi = atan2(vy, vx);
        if (scheme == 0) {
          pix[0] = ang2pix_ring(zc, phi, nside);
          w[0] = 1.0;
        } else {
          interp_weights_grad(acos(fmin(1.0, fmax(-1.0, zc))), phi, nside, theta_tab, pix, w, dth, dph);
        }
      }
      const float* mb = maps_bar + sh * npix;
      double gt = 0.0, gp = 0.0, gs = 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (pix[q] < 0 || pix[q] >= npix) continue;
        const double m = (double)__ldg(mb + pix[q]);
        gt += m * dth[q];
        gp += m * dph[q];
        gs += m * w[q];
      }
      const double sc = (double)shells.scale[sh];
      g_th += sc * gt;
      g_ph += sc * gp;
      g_w += sc * gs;
    }
    if (!any) continue;
    if (weights_bar) weights_bar[p] += (float)((double)weight * g_w);
    if (scheme == 0) continue;
    const double wp = weights ? (double)weights[p] * (double)weight : (double)weight;
    const double s2 = vx * vx + vy * vy;
    if (!(s2 > 0.0)) continue;  // on the polar axis: phi is undefined (measure zero)
    const double sxy = sqrt(s2), r2 = rr * rr;
    const double gvx = wp * (g_th * vz * vx / (r2 * sxy) - g_ph * vy / s2);
    const double gvy = wp * (g_th * vz * vy / (r2 * sxy) + g_ph * vx / s2);
    const double gvz = wp * (-g_th * sxy / r2);
    disp_bar[3 * p + 0] += (float)(gvx * cell.x);
    disp_bar[3 * p + 1] += (float)(gvy * cell.y);
    disp_bar[3 * p + 2] += (float)(gvz * cell.z);
  }
}

// Tiled shell painting (OnionTiler._paint_tiled_27, pm/interp.py:418-504, and
// TelephotoInterp._paint_telephoto, pm/interp.py:643-699). Every particle is read once and
// placed in each of the tiles in turn: its observer-centred position c = x - o (x in
// Mpc/h) becomes q = M c + s with M a signed permutation matrix (exact in FP32) and s the
// tile's shift. With the light-cone drift on, q is drifted with the rotated momentum
// M v by (Gp(a_t) - Gp(t)) / dGfa(sqrt(t a_t)), a_t = a_of_chi(distance):
//   onion:     x' = q + o, distance |x' - o|, x' += D M v
//   telephoto: distance |q - o| (the reference measures it from the observer-centred q),
//              q += D M v, x' = q + o
// and x' is painted on the shell rmin < |x' - o| <= rmax. The cull below runs in FP32 with
// margins; a copy that passes it is placed again in FP64 (c, q and q + D M v, whose length
// is x' - o without the FP32 rounding of adding and removing o), and the shell test and the
// direction use that.
//
// Copies that cannot reach the shell are skipped before the drift. With D bounded by
// dbound (the host's bound on |D| over the distance table: the Gp difference is at most
// max(Gp(t), 1 - Gp(t)) after the clip to [0, 1], and dGfa is at least its smallest table
// value over the scale factors sqrt(t a) reachable), the painted distance lies within
// dbound |v| of |q|. A copy whose drift distance is beyond the table (extrapolated) is
// always evaluated in full.
struct TileSet {
  int n;
  signed char m[kMaxTiles][9];
  float shift[kMaxTiles][3];
};

__global__ void __launch_bounds__(256, 4)
    k_healpix_paint_tiled(const float* __restrict__ disp, int absolute, const float* __restrict__ vel,
                          const float* __restrict__ weights, float weight, PGrid g, float3 box, float3 obs, TileSet ts,
                          int telephoto, float rmin, float rmax, float t, float gp_t, float dbound, DriftTables tb,
                          int nside, int scheme, const double* __restrict__ theta_tab, float* __restrict__ map) {
  const long long b = blockIdx.y;
  const long long npix = 12LL * nside * nside;
  disp += b * g.np * 3;
  if (vel) vel += b * g.np * 3;
  if (weights) weights += b * g.np;
  map += b * npix;
  const float nx = (float)g.nx, ny = (float)g.ny, nz = (float)g.nz;
  // |q| below which the drift distance is inside the table: |q| itself (onion), or up to
  // |q| + |observer| (telephoto's distance from the observer-centred replica)
  float cm2 = 0.f;
  if (vel) {
    const float onorm = sqrtf(obs.x * obs.x + obs.y * obs.y + obs.z * obs.z);
    const float cm = tb.chi[tb.n_chi - 1] * (1.f - 1e-5f) - 0.01f - (telephoto ? onorm : 0.f);
    cm2 = cm > 0.f ? cm * cm * (1.f - 1e-6f) : -1.f;
  }
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    const float d0 = disp[3 * p + 0], d1 = disp[3 * p + 1], d2 = disp[3 * p + 2];  // grid units
    int i = 0, j = 0, k = 0;
    if (!absolute) particle_ijk(g, p, i, j, k);
    const float c[3] = {((float)i + d0) / nx * box.x - obs.x, ((float)j + d1) / ny * box.y - obs.y,
                        ((float)k + d2) / nz * box.z - obs.z};
    float v[3] = {0.f, 0.f, 0.f}, vmag = 0.f;
    if (vel) {
      v[0] = vel[3 * p + 0];
      v[1] = vel[3 * p + 1];
      v[2] = vel[3 * p + 2];
      vmag = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
    const float w = weights ? weights[p] * weight : weight;
    // skip bounds on the squared undrifted distance: a replica with |q| <= lo or |q| > hi
    // cannot land in the shell (margin = dbound |v| + FP32 slack 4e-3 + 4e-6 |q|, solved
    // for |q|; the squares widened by 1e-6 against rounding)
    const float dv = dbound * vmag;
    const float lo = (rmin - dv - 4e-3f) / (1.f + 4e-6f), hi = (rmax + dv + 4e-3f) / (1.f - 4e-6f);
    const float lo2 = lo > 0.f ? lo * lo * (1.f - 1e-6f) : -1.f, hi2 = hi * hi * (1.f + 1e-6f);
    for (int tile = 0; tile < ts.n; ++tile) {
      const signed char* M = ts.m[tile];
      float q[3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
        q[r] = (float)M[3 * r + 0] * c[0] + (float)M[3 * r + 1] * c[1] + (float)M[3 * r + 2] * c[2] + ts.shift[tile][r];
      const float qn2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
      // the bounds hold while the drift distance lies inside the distance table
      if ((!vel || qn2 <= cm2) && (qn2 <= lo2 || qn2 > hi2)) continue;
      // the copy in FP64: cd = x - o, qd = M cd + s (M a signed permutation)
      const double cd[3] = {((double)i + (double)d0) / nx * box.x - obs.x, ((double)j + (double)d1) / ny * box.y - obs.y,
                            ((double)k + (double)d2) / nz * box.z - obs.z};
      double qd[3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
        qd[r] = (double)M[3 * r + 0] * cd[0] + (double)M[3 * r + 1] * cd[1] + (double)M[3 * r + 2] * cd[2] +
                (double)ts.shift[tile][r];
      if (vel) {
        double dist;
        if (telephoto) {
          const double ex = qd[0] - obs.x, ey = qd[1] - obs.y, ez = qd[2] - obs.z;
          dist = sqrt(ex * ex + ey * ey + ez * ez);
        } else {
          dist = sqrt(qd[0] * qd[0] + qd[1] * qd[1] + qd[2] * qd[2]);
        }
        const float at = interp_table((float)dist, tb.chi, tb.a_chi, tb.n_chi);
        const float ac = sqrtf(t * at);
        const float gp_at = fminf(fmaxf(interp_table(at, tb.ga, tb.g, tb.n_g), 0.f), 1.f);
        const float drift = (gp_at - gp_t) / interp_table(ac, tb.da, tb.dgfa, tb.n_d);
#pragma unroll
        for (int r = 0; r < 3; ++r)
          qd[r] += (double)(drift * ((float)M[3 * r + 0] * v[0] + (float)M[3 * r + 1] * v[1] +
                                     (float)M[3 * r + 2] * v[2]));
      }
      const double rr = sqrt(qd[0] * qd[0] + qd[1] * qd[1] + qd[2] * qd[2]);
      if (!(rr > (double)rmin && rr <= (double)rmax)) continue;
      deposit_direction(qd[0], qd[1], qd[2], rr, w, nside, scheme, theta_tab, map);
    }
  }
}

// Adjoint of k_healpix_paint_tiled (ngp or bilinear) for one shell's map cotangent
// map_bar. Each painted copy q' = q + D(r) u (q = M c + s, u = M v, r = |q| onion or
// |q - o| telephoto, D the light-cone drift factor of interpolated tables) passes back
// g = dL/dq' from the painter (as k_healpix_paint_shells_adjoint), and
//   dL/dq = g + D'(r) (u . g) dr/dq,   dL/dc += M^T dL/dq,   dL/dv += D M^T g,
// D'(r) chaining the slopes of the tables' segments (a(chi), Gp(a) unless clipped,
// dGfa(sqrt(t a))). The cull and the FP64 placement are the forward's; shell edges pass
// nothing back. Accumulates into disp_bar, vel_bar and weights_bar (each may be null but
// disp_bar).
__global__ void k_healpix_paint_tiled_adjoint(const float* __restrict__ disp, int absolute,
                                              const float* __restrict__ vel, const float* __restrict__ weights,
                                              float weight, PGrid g, float3 box, float3 obs, TileSet ts,
                                              int telephoto, float rmin, float rmax, float t, float gp_t,
                                              float dbound, DriftTables tb, int nside, int scheme,
                                              const double* __restrict__ theta_tab,
                                              const float* __restrict__ map_bar, float* __restrict__ disp_bar,
                                              float* __restrict__ vel_bar, float* __restrict__ weights_bar) {
  const long long b = blockIdx.y;
  const long long npix = 12LL * nside * nside;
  disp += b * g.np * 3;
  disp_bar += b * g.np * 3;
  if (vel) vel += b * g.np * 3;
  if (vel_bar) vel_bar += b * g.np * 3;
  if (weights) weights += b * g.np;
  if (weights_bar) weights_bar += b * g.np;
  map_bar += b * npix;
  const float nx = (float)g.nx, ny = (float)g.ny, nz = (float)g.nz;
  float cm2 = 0.f;
  if (vel) {
    const float onorm = sqrtf(obs.x * obs.x + obs.y * obs.y + obs.z * obs.z);
    const float cm = tb.chi[tb.n_chi - 1] * (1.f - 1e-5f) - 0.01f - (telephoto ? onorm : 0.f);
    cm2 = cm > 0.f ? cm * cm * (1.f - 1e-6f) : -1.f;
  }
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    const float d0 = disp[3 * p + 0], d1 = disp[3 * p + 1], d2 = disp[3 * p + 2];
    int i = 0, j = 0, k = 0;
    if (!absolute) particle_ijk(g, p, i, j, k);
    const float c[3] = {((float)i + d0) / nx * box.x - obs.x, ((float)j + d1) / ny * box.y - obs.y,
                        ((float)k + d2) / nz * box.z - obs.z};
    float v[3] = {0.f, 0.f, 0.f}, vmag = 0.f;
    if (vel) {
      v[0] = vel[3 * p + 0];
      v[1] = vel[3 * p + 1];
      v[2] = vel[3 * p + 2];
      vmag = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
    const double wp = weights ? (double)weights[p] * (double)weight : (double)weight;
    const float dv = dbound * vmag;
    const float lo = (rmin - dv - 4e-3f) / (1.f + 4e-6f), hi = (rmax + dv + 4e-3f) / (1.f - 4e-6f);
    const float lo2 = lo > 0.f ? lo * lo * (1.f - 1e-6f) : -1.f, hi2 = hi * hi * (1.f + 1e-6f);
    double gc[3] = {0.0, 0.0, 0.0}, gvel[3] = {0.0, 0.0, 0.0}, gw = 0.0;
    for (int tile = 0; tile < ts.n; ++tile) {
      const signed char* M = ts.m[tile];
      float q[3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
        q[r] = (float)M[3 * r + 0] * c[0] + (float)M[3 * r + 1] * c[1] + (float)M[3 * r + 2] * c[2] + ts.shift[tile][r];
      const float qn2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
      if ((!vel || qn2 <= cm2) && (qn2 <= lo2 || qn2 > hi2)) continue;
      const double cd[3] = {((double)i + (double)d0) / nx * box.x - obs.x, ((double)j + (double)d1) / ny * box.y - obs.y,
                            ((double)k + (double)d2) / nz * box.z - obs.z};
      double qd[3], u[3] = {0.0, 0.0, 0.0}, dr[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int r = 0; r < 3; ++r)
        qd[r] = (double)M[3 * r + 0] * cd[0] + (double)M[3 * r + 1] * cd[1] + (double)M[3 * r + 2] * cd[2] +
                (double)ts.shift[tile][r];
      double D = 0.0, dD = 0.0;
      if (vel) {
        double e[3] = {qd[0], qd[1], qd[2]};
        if (telephoto) {
          e[0] -= obs.x;
          e[1] -= obs.y;
          e[2] -= obs.z;
        }
        const double dist = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        float s_a, s_g, s_d;
        const float at = interp_table_d((float)dist, tb.chi, tb.a_chi, tb.n_chi, s_a);
        const float ac = sqrtf(t * at);
        const float graw = interp_table_d(at, tb.ga, tb.g, tb.n_g, s_g);
        const float gp_at = fminf(fmaxf(graw, 0.f), 1.f);
        const float dgv = interp_table_d(ac, tb.da, tb.dgfa, tb.n_d, s_d);
        const float drift = (gp_at - gp_t) / dgv;
        D = (double)drift;
        const double dgp = (graw > 0.f && graw < 1.f) ? (double)s_g : 0.0;
        const double dac = ac > 0.f ? (double)t / (2.0 * (double)ac) : 0.0;
        dD = (double)s_a * (dgp * dgv - ((double)gp_at - gp_t) * (double)s_d * dac) / ((double)dgv * dgv);
        if (dist > 0.0) {
#pragma unroll
          for (int r = 0; r < 3; ++r) dr[r] = e[r] / dist;
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          u[r] = (double)M[3 * r + 0] * v[0] + (double)M[3 * r + 1] * v[1] + (double)M[3 * r + 2] * v[2];
          qd[r] += (double)(drift * (float)u[r]);
        }
      }
      const double rr = sqrt(qd[0] * qd[0] + qd[1] * qd[1] + qd[2] * qd[2]);
      if (!(rr > (double)rmin && rr <= (double)rmax)) continue;
      // the painter's adjoint at the painted vector qd
      const double zc = qd[2] / rr, phi = atan2(qd[1], qd[0]);
      long long pix[4] = {-1, -1, -1, -1};
      double w[4] = {0.0, 0.0, 0.0, 0.0}, dth[4] = {0.0, 0.0, 0.0, 0.0}, dph[4] = {0.0, 0.0, 0.0, 0.0};
      if (scheme == 0) {
        pix[0] = ang2pix_ring(zc, phi, nside);
        w[0] = 1.0;
      } else {
        interp_weights_grad(acos(fmin(1.0, fmax(-1.0, zc))), phi, nside, theta_tab, pix, w, dth, dph);
      }
      double g_th = 0.0, g_ph = 0.0, g_s = 0.0;
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) {
        if (pix[qq] < 0 || pix[qq] >= npix) continue;
        const double m = (double)__ldg(map_bar + pix[qq]);
        g_th += m * dth[qq];
        g_ph += m * dph[qq];
        g_s += m * w[qq];
      }
      gw += (double)weight * g_s;
      if (scheme == 0) continue;
      const double s2 = qd[0] * qd[0] + qd[1] * qd[1];
      if (!(s2 > 0.0)) continue;
      const double sxy = sqrt(s2), r2 = rr * rr;
      double gq[3] = {wp * (g_th * qd[2] * qd[0] / (r2 * sxy) - g_ph * qd[1] / s2),
                      wp * (g_th * qd[2] * qd[1] / (r2 * sxy) + g_ph * qd[0] / s2), wp * (-g_th * sxy / r2)};
      if (vel) {
        const double ug = u[0] * gq[0] + u[1] * gq[1] + u[2] * gq[2];
        // dL/dv += D M^T g  (before g gains the drift's distance term)
#pragma unroll
        for (int r = 0; r < 3; ++r)
          gvel[r] += D * ((double)M[0 * 3 + r] * gq[0] + (double)M[1 * 3 + r] * gq[1] + (double)M[2 * 3 + r] * gq[2]);
#pragma unroll
        for (int r = 0; r < 3; ++r) gq[r] += dD * ug * dr[r];
      }
#pragma unroll
      for (int r = 0; r < 3; ++r)
        gc[r] += (double)M[0 * 3 + r] * gq[0] + (double)M[1 * 3 + r] * gq[1] + (double)M[2 * 3 + r] * gq[2];
    }
    if (weights_bar) weights_bar[p] += (float)gw;
    disp_bar[3 * p + 0] += (float)(gc[0] * box.x / nx);
    disp_bar[3 * p + 1] += (float)(gc[1] * box.y / ny);
    disp_bar[3 * p + 2] += (float)(gc[2] * box.z / nz);
    if (vel && vel_bar) {
      vel_bar[3 * p + 0] += (float)gvel[0];
      vel_bar[3 * p + 1] += (float)gvel[1];
      vel_bar[3 * p + 2] += (float)gvel[2];
    }
  }
}

// Positions (Mpc/h) of one rotated, shifted replica, drifted to the light cone when vel is
// given, with the same conventions as k_healpix_paint_tiled (TelephotoInterp's flat planes
// beyond the box paint these with the flat-sky painter, pm/interp.py:643-699).
__global__ void k_replica_positions(const float* __restrict__ disp, int absolute, const float* __restrict__ vel,
                                    PGrid g, float3 box, float3 obs, TileSet ts, int telephoto, float t, float gp_t,
                                    DriftTables tb, float* __restrict__ out) {
  const long long b = blockIdx.y;
  disp += b * g.np * 3;
  out += b * g.np * 3;
  if (vel) vel += b * g.np * 3;
  const float nx = (float)g.nx, ny = (float)g.ny, nz = (float)g.nz;
  const signed char* M = ts.m[0];
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < g.np; p += gridDim.x * blockDim.x) {
    float x, y, z;
    if (absolute) {
      x = disp[3 * p + 0] / nx * box.x;
      y = disp[3 * p + 1] / ny * box.y;
      z = disp[3 * p + 2] / nz * box.z;
    } else {
      int i, j, k;
      particle_ijk(g, p, i, j, k);
      x = ((float)i + disp[3 * p + 0]) / nx * box.x;
      y = ((float)j + disp[3 * p + 1]) / ny * box.y;
      z = ((float)k + disp[3 * p + 2]) / nz * box.z;
    }
    const float c[3] = {x - obs.x, y - obs.y, z - obs.z};
    float q[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
      q[r] = (float)M[3 * r + 0] * c[0] + (float)M[3 * r + 1] * c[1] + (float)M[3 * r + 2] * c[2] + ts.shift[0][r];
    float o[3] = {q[0] + obs.x, q[1] + obs.y, q[2] + obs.z};
    if (vel) {
      const float v[3] = {vel[3 * p + 0], vel[3 * p + 1], vel[3 * p + 2]};
      float vr[3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
        vr[r] = (float)M[3 * r + 0] * v[0] + (float)M[3 * r + 1] * v[1] + (float)M[3 * r + 2] * v[2];
      float dist;
      if (telephoto) {
        const float ex = q[0] - obs.x, ey = q[1] - obs.y, ez = q[2] - obs.z;
        dist = sqrtf(ex * ex + ey * ey + ez * ez);
      } else {
        const float ex = o[0] - obs.x, ey = o[1] - obs.y, ez = o[2] - obs.z;
        dist = sqrtf(ex * ex + ey * ey + ez * ez);
      }
      const float at = interp_table(dist, tb.chi, tb.a_chi, tb.n_chi);
      const float ac = sqrtf(t * at);
      const float gp_at = fminf(fmaxf(interp_table(at, tb.ga, tb.g, tb.n_g), 0.f), 1.f);
      const float drift = (gp_at - gp_t) / interp_table(ac, tb.da, tb.dgfa, tb.n_d);
      if (telephoto) {
        const float ob[3] = {obs.x, obs.y, obs.z};
#pragma unroll
        for (int r = 0; r < 3; ++r) o[r] = (q[r] + drift * vr[r]) + ob[r];
      } else {
#pragma unroll
        for (int r = 0; r < 3; ++r) o[r] = o[r] + drift * vr[r];
      }
    }
    out[3 * p + 0] = o[0];
    out[3 * p + 1] = o[1];
    out[3 * p + 2] = o[2];
  }
}

cudaError_t replica_positions(const float* disp, int absolute, const float* vel, const MeshDims& d, const float* box,
                              const float* observer, const signed char* rotation, const float* shift, int telephoto,
                              float t, float gp_t, const DriftTables& tb, float* out, cudaStream_t s) {
  TileSet ts;
  ts.n = 1;
  for (int e = 0; e < 9; ++e) ts.m[0][e] = rotation[e];
  for (int e = 0; e < 3; ++e) ts.shift[0][e] = shift[e];
  k_replica_positions<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(
      disp, absolute, vel, make_pgrid(d), make_float3(box[0], box[1], box[2]),
      make_float3(observer[0], observer[1], observer[2]), ts, telephoto, t, gp_t, tb, out);
  note_launch();
  return cudaGetLastError();
}

// FP64 colatitudes of rings 0 .. 4 nside (entries 0 and 4 nside unused), one table per
// (device, nside), built once on the host: polar-cap rings from z = 1 - north^2 4 / npix
// (colatitude via atan2 of sin and cos), equatorial rings from z = (2 nside - north) 2 / (3 nside).
static std::mutex g_ring_mutex;
static std::map<std::pair<int, int>, double*> g_ring_tables;

static const double* ring_theta_table(int nside) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_ring_mutex);
  const auto key = std::make_pair(dev, nside);
  const auto it = g_ring_tables.find(key);
  if (it != g_ring_tables.end()) return it->second;
  const int nr = 4 * nside + 1;
  const double npix = 12.0 * nside * nside;
  std::vector<double> h(nr, 0.0);
  for (int ring = 1; ring < 4 * nside; ++ring) {
    const int north = ring > 2 * nside ? 4 * nside - ring : ring;
    double th;
    if (north < nside) {
      const double tmp = (double)north * north * (4.0 / npix);
      th = std::atan2(std::sqrt(tmp * (2.0 - tmp)), 1.0 - tmp);
    } else {
      th = std::acos((double)(2 * nside - north) * (2.0 / (3.0 * nside)));
    }
    h[ring] = north != ring ? M_PI - th : th;
  }
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double) * nr) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, h.data(), sizeof(double) * nr, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  g_ring_tables[key] = d;
  return d;
}

cudaError_t healpix_paint(const float* disp, int absolute, const float* weights, float weight, const MeshDims& d,
                          const float* box, const float* observer, float rmin, float rmax, int nside, int scheme,
                          float* map, cudaStream_t s, float sigma) {
  const double3 cell = make_double3((double)box[0] / d.nx, (double)box[1] / d.ny, (double)box[2] / d.nz);
  const double3 obs = make_double3(observer[0], observer[1], observer[2]);
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  long long blocks = (d.cells() + 255) / 256;
  if (blocks > (long long)nsm * 16) blocks = (long long)nsm * 16;
  const double* tab = ring_theta_table(nside);
  if (!tab) return cudaErrorMemoryAllocation;
  k_healpix_paint<<<dim3((unsigned)blocks, d.batch), 256, 0, s>>>(disp, absolute, weights, weight, d, cell, obs, rmin,
                                                                  rmax, nside, scheme, tab, map, sigma);
  note_launch();
  return cudaGetLastError();
}

cudaError_t healpix_paint_shells(const float* disp, int absolute, const float* weights, float weight,
                                 const MeshDims& d, const float* box, const float* observer, int nshells,
                                 const double* rmin, const double* rmax, const float* scale, int nside, int scheme,
                                 float* maps, cudaStream_t s, float sigma) {
  const double3 cell = make_double3((double)box[0] / d.nx, (double)box[1] / d.ny, (double)box[2] / d.nz);
  const double3 obs = make_double3(observer[0], observer[1], observer[2]);
  long long blocks = (d.cells() + 255) / 256;
  if (blocks > (long long)sm_count() * 16) blocks = (long long)sm_count() * 16;
  const double* tab = ring_theta_table(nside);
  if (!tab) return cudaErrorMemoryAllocation;
  const long long npix = 12LL * nside * nside;
  for (int s0 = 0; s0 < nshells; s0 += kMaxShellsPerPass) {
    ShellSet set;
    set.n = nshells - s0 < kMaxShellsPerPass ? nshells - s0 : kMaxShellsPerPass;
    for (int i = 0; i < set.n; ++i) {
      set.rmin[i] = rmin[s0 + i];
      set.rmax[i] = rmax[s0 + i];
      set.scale[i] = scale[s0 + i];
    }
    k_healpix_paint_shells<<<(unsigned)blocks, 256, 0, s>>>(disp, absolute, weights, weight, d, cell, obs, set, nside,
                                                            scheme, tab, maps + s0 * npix, sigma);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t healpix_paint_shells_adjoint(const float* disp, int absolute, const float* weights, float weight,
                                         const MeshDims& d, const float* box, const float* observer, int nshells,
                                         const double* rmin, const double* rmax, const float* scale, int nside,
                                         int scheme, const float* maps_bar, float* disp_bar, float* weights_bar,
                                         cudaStream_t s) {
  const double3 cell = make_double3((double)box[0] / d.nx, (double)box[1] / d.ny, (double)box[2] / d.nz);
  const double3 obs = make_double3(observer[0], observer[1], observer[2]);
  long long blocks = (d.cells() + 255) / 256;
  if (blocks > (long long)sm_count() * 16) blocks = (long long)sm_count() * 16;
  const double* tab = ring_theta_table(nside);
  if (!tab) return cudaErrorMemoryAllocation;
  const long long npix = 12LL * nside * nside;
  for (int s0 = 0; s0 < nshells; s0 += kMaxShellsPerPass) {
    ShellSet set;
    set.n = nshells - s0 < kMaxShellsPerPass ? nshells - s0 : kMaxShellsPerPass;
    for (int i = 0; i < set.n; ++i) {
      set.rmin[i] = rmin[s0 + i];
      set.rmax[i] = rmax[s0 + i];
      set.scale[i] = scale[s0 + i];
    }
    k_healpix_paint_shells_adjoint<<<(unsigned)blocks, 256, 0, s>>>(disp, absolute, weights, weight, d, cell, obs, set,
                                                                    nside, scheme, tab, maps_bar + s0 * npix,
                                                                    disp_bar, weights_bar);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t healpix_paint_tiled_adjoint(const float* disp, int absolute, const float* vel, const float* weights,
                                        float weight, const MeshDims& d, const float* box, const float* observer,
                                        int ntiles, const signed char* rotations, const float* shifts, int telephoto,
                                        float rmin, float rmax, float t, float gp_t, float dbound,
                                        const DriftTables& tb, int nside, int scheme, const float* map_bar,
                                        float* disp_bar, float* vel_bar, float* weights_bar, cudaStream_t s) {
  TileSet ts;
  ts.n = ntiles;
  for (int i = 0; i < ntiles; ++i) {
    for (int e = 0; e < 9; ++e) ts.m[i][e] = rotations[9 * i + e];
    for (int e = 0; e < 3; ++e) ts.shift[i][e] = shifts[3 * i + e];
  }
  const double* tab = ring_theta_table(nside);
  if (!tab) return cudaErrorMemoryAllocation;
  k_healpix_paint_tiled_adjoint<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(
      disp, absolute, vel, weights, weight, make_pgrid(d), make_float3(box[0], box[1], box[2]),
      make_float3(observer[0], observer[1], observer[2]), ts, telephoto, rmin, rmax, t, gp_t, dbound, tb, nside, scheme,
      tab, map_bar, disp_bar, vel_bar, weights_bar);
  note_launch();
  return cudaGetLastError();
}

cudaError_t healpix_paint_tiled(const float* disp, int absolute, const float* vel, const float* weights, float weight,
                                const MeshDims& d, const float* box, const float* observer, int ntiles,
                                const signed char* rotations, const float* shifts, int telephoto, float rmin,
                                float rmax, float t, float gp_t, float dbound, const DriftTables& tb, int nside,
                                int scheme, float* map, cudaStream_t s) {
  TileSet ts;
  ts.n = ntiles;
  for (int i = 0; i < ntiles; ++i) {
    for (int e = 0; e < 9; ++e) ts.m[i][e] = rotations[9 * i + e];
    for (int e = 0; e < 3; ++e) ts.shift[i][e] = shifts[3 * i + e];
  }
  const double* tab = ring_theta_table(nside);
  if (!tab) return cudaErrorMemoryAllocation;
  k_healpix_paint_tiled<<<particle_grid_dims(d.cells(), d.batch, 256, 16), 256, 0, s>>>(
      disp, absolute, vel, weights, weight, make_pgrid(d), make_float3(box[0], box[1], box[2]),
      make_float3(observer[0], observer[1], observer[2]), ts, telephoto, rmin, rmax, t, gp_t, dbound, tb, nside, scheme,
      tab, map);
  note_launch();
  return cudaGetLastError();
}

}  // namespace jfli
