/* CPU oracle: Legendre stages of the spherical harmonic transform (FP64, OpenMP) -- TEST
 * INFRASTRUCTURE ONLY.
 *
 * Only tests/ and the fixture generators under tests/golden/ reach this code (through
 * oracle/sht.py), as the checker of the library's GPU SHT; the product never does.
 *
 * The same arithmetic as oracle/sht.py::_lambda_m and its map2alm / alm2map loops, which
 * restate healpy's anafast (the reference's C_ell, _src/power/_compute.py:175-191):
 *   lambda_mm = (-1)^m sqrt((2m+1)/(4 pi) prod_{k<=m} (2k-1)/(2k)) sin^m theta, formed in
 *   log space; below FP64 range the recursion runs on values scaled by e^s and removes
 *   the scale (1e100 at a time) as they grow;
 *   lambda_{m+1,m} = x sqrt(2m+3) lambda_mm;
 *   lambda_lm = a (x lambda_{l-1,m} - b lambda_{l-2,m}),
 *     a = sqrt((4l^2-1)/(l^2-m^2)), b = sqrt(((l-1)^2-m^2)/(4(l-1)^2-1)).
 * Per-ring coefficients F[r][m] / G[r][m] are complex (interleaved doubles), m = 0..lmax;
 * a_lm is packed by m: a[m][l - m] at offset m (lmax + 1) - m (m - 1) / 2.
 */
#include <math.h>
#include <omp.h>
#include <stdlib.h>

static const double kBig = 1e100;

static long long alm_off(int m, int lmax) { return (long long)m * (lmax + 1) - (long long)m * (m - 1) / 2; }

typedef struct {
  double prev, cur, scale, escale, x;
  int m, l;
} Leg;

static double emit_scale(double scale) { return scale < 745.0 ? exp(-fmin(scale, 745.0)) : 0.0; }

/* lambda_mm at ring z; returns the emitted (unscaled) value */
static double leg_start(Leg* g, int m, double z, double logc) {
  const double sint = sqrt(fmax(0.0, 1.0 - z * z));
  double logv = logc + (m == 0 ? 0.0 : m * log(sint));
  if (!isfinite(logv)) logv = -INFINITY;
  g->scale = (logv < -600.0) ? -300.0 - logv : 0.0;
  if (!isfinite(g->scale)) g->scale = INFINITY;
  const double sign = (m & 1) ? -1.0 : 1.0;
  g->cur = isfinite(g->scale) ? sign * exp(logv + g->scale) : 0.0;
  g->prev = 0.0;
  g->escale = (g->scale < 745.0) ? exp(-fmin(g->scale, 745.0)) : 0.0;
  g->x = z;
  g->m = m;
  g->l = m;
  return g->cur * g->escale;
}

/* advance to l + 1; returns the emitted value */
static double leg_next(Leg* g) {
  const int l = g->l + 1, m = g->m;
  double nxt;
  if (l == m + 1) {
    nxt = g->x * sqrt(2.0 * m + 3.0) * g->cur;
  } else {
    const double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
    const double b = sqrt((((double)l - 1.0) * ((double)l - 1.0) - (double)m * m) /
                          (4.0 * ((double)l - 1.0) * ((double)l - 1.0) - 1.0));
    nxt = a * (g->x * g->cur - b * g->prev);
    if (fabs(nxt) > kBig && g->scale > 0.0) {
      nxt /= kBig;
      g->cur /= kBig;
      g->scale -= log(kBig);
      g->escale = emit_scale(g->scale);
    }
  }
  g->prev = g->cur;
  g->cur = nxt;
  g->l = l;
  return nxt * g->escale;
}

static double log_c(int m) {
  double s = 0.0;
  for (int k = 1; k <= m; ++k) s += log((2.0 * k - 1.0) / (2.0 * k));
  return 0.5 * log((2.0 * m + 1.0) / (4.0 * M_PI)) + 0.5 * s;
}

/* alm = w * sum_r lambda_lm(z_r) F[r][m] */
int oracle_sht_analysis(const double* F, const double* z, int nrings, int lmax, double w, double* alm) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int m = 0; m <= lmax; ++m) {
    const double logc = log_c(m);
    double* a = alm + 2 * alm_off(m, lmax);
    for (int l = m; l <= lmax; ++l) a[2 * (l - m)] = a[2 * (l - m) + 1] = 0.0;
    for (int r = 0; r < nrings; ++r) {
      const double fr = F[2 * ((long long)r * (lmax + 1) + m)], fi = F[2 * ((long long)r * (lmax + 1) + m) + 1];
      Leg g;
      double lam = leg_start(&g, m, z[r], logc);
      a[0] += lam * fr;
      a[1] += lam * fi;
      for (int l = m + 1; l <= lmax; ++l) {
        lam = leg_next(&g);
        a[2 * (l - m)] += lam * fr;
        a[2 * (l - m) + 1] += lam * fi;
      }
    }
    for (int l = m; l <= lmax; ++l) {
      a[2 * (l - m)] *= w;
      a[2 * (l - m) + 1] *= w;
    }
  }
  return 0;
}

/* G[r][m] = sum_l alm[m][l - m] lambda_lm(z_r) */
int oracle_sht_synthesis(const double* alm, const double* z, int nrings, int lmax, double* G) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int m = 0; m <= lmax; ++m) {
    const double logc = log_c(m);
    const double* a = alm + 2 * alm_off(m, lmax);
    for (int r = 0; r < nrings; ++r) {
      Leg g;
      double lam = leg_start(&g, m, z[r], logc);
      double sr = lam * a[0], si = lam * a[1];
      for (int l = m + 1; l <= lmax; ++l) {
        lam = leg_next(&g);
        sr += lam * a[2 * (l - m)];
        si += lam * a[2 * (l - m) + 1];
      }
      G[2 * ((long long)r * (lmax + 1) + m)] = sr;
      G[2 * ((long long)r * (lmax + 1) + m) + 1] = si;
    }
  }
  return 0;
}
