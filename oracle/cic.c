/* CPU oracle: CIC paint and readout in C with OpenMP -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load this library, and
 * only as the checker or the timed CPU restatement; the product never does.
 *
 * Same arithmetic as the NumPy restatement in oracle/pm.py (_cic_corners, cic_paint,
 * cic_read), which follows JaxPM's cic_paint_dx / cic_read_dx at the reference call sites
 * _src/fields/_painting.py:67,76 and fields/particles.py:203,210:
 *   position = grid point (i, j, k) + displacement (relative) or the position itself
 *   (absolute), in cells; per axis f = floor(pos), frac = pos - f, cells f and f + 1
 *   wrapped periodically; corner weight = prod_a (frac_a or 1 - frac_a), formed in the
 *   order x, y, z in the working precision.
 * Paint accumulates in FP64 for both precisions (NumPy's bincount does) and rounds the
 * mesh to the working precision at the end; each thread paints into a private FP64 mesh
 * and the meshes are summed cell by cell. Readout sums the 8 corner products in the
 * working precision with NumPy's 8-way pairwise order for a row of 8.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline int64_t wrap(int64_t i, int64_t n) {
  int64_t r = i % n;
  return r < 0 ? r + n : r;
}

/* corner order of oracle/pm.py::_cic_corners */
static const int kOff[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};

#define DEFINE_CORNERS(NAME, T, FLOOR)                                                                     \
  static inline void NAME(const T* pos, int64_t p, int64_t nx, int64_t ny, int64_t nz, int absolute,       \
                          int64_t idx[8], T w[8]) {                                                        \
    const int64_t n[3] = {nx, ny, nz};                                                                     \
    int64_t g[3] = {0, 0, 0};                                                                              \
    if (!absolute) {                                                                                       \
      g[0] = p / (ny * nz);                                                                                \
      g[1] = (p / nz) % ny;                                                                                \
      g[2] = p % nz;                                                                                       \
    }                                                                                                      \
    int64_t base[3];                                                                                       \
    T frac[3];                                                                                             \
    for (int a = 0; a < 3; ++a) {                                                                          \
      const T x = pos[3 * p + a];                                                                          \
      const T f = FLOOR(x);                                                                                \
      frac[a] = (T)(x - f);                                                                                \
      base[a] = g[a] + (int64_t)f;                                                                         \
    }                                                                                                      \
    for (int c = 0; c < 8; ++c) {                                                                          \
      int64_t ci[3];                                                                                       \
      T wc = (T)1;                                                                                         \
      for (int a = 0; a < 3; ++a) {                                                                        \
        ci[a] = wrap(base[a] + kOff[c][a], n[a]);                                                          \
        wc = (T)(wc * (kOff[c][a] ? frac[a] : (T)((T)1 - frac[a])));                                       \
      }                                                                                                    \
      idx[c] = (ci[0] * ny + ci[1]) * nz + ci[2];                                                          \
      w[c] = wc;                                                                                           \
    }                                                                                                      \
  }

DEFINE_CORNERS(corners_f64, double, floor)
DEFINE_CORNERS(corners_f32, float, floorf)

#define DEFINE_PAINT(NAME, T, CORNERS)                                                                     \
  int NAME(const T* pos, int64_t np, int64_t nx, int64_t ny, int64_t nz, int absolute, const T* weights,   \
           T weight, T* mesh) {                                                                            \
    const int64_t m = nx * ny * nz;                                                                        \
    if (!absolute && np != m) return -1;                                                                   \
    const int nt = omp_get_max_threads();                                                                  \
    double* priv = (double*)calloc((size_t)nt * (size_t)m, sizeof(double));                                \
    if (!priv) return -2;                                                                                  \
    _Pragma("omp parallel num_threads(nt)") {                                                              \
      double* acc = priv + (size_t)omp_get_thread_num() * (size_t)m;                                       \
      _Pragma("omp for schedule(static)") for (int64_t p = 0; p < np; ++p) {                               \
        int64_t idx[8];                                                                                    \
        T w[8];                                                                                            \
        CORNERS(pos, p, nx, ny, nz, absolute, idx, w);                                                     \
        const T s = weights ? (T)(weights[p]) : weight;                                                    \
        for (int c = 0; c < 8; ++c) acc[idx[c]] += (double)(T)(w[c] * s);                                  \
      }                                                                                                    \
      _Pragma("omp barrier")                                                                               \
      _Pragma("omp for schedule(static)") for (int64_t c = 0; c < m; ++c) {                                \
        double s = 0.0;                                                                                    \
        for (int t = 0; t < nt; ++t) s += priv[(size_t)t * (size_t)m + (size_t)c];                         \
        mesh[c] = (T)s;                                                                                    \
      }                                                                                                    \
    }                                                                                                      \
    free(priv);                                                                                            \
    return 0;                                                                                              \
  }

DEFINE_PAINT(oracle_cic_paint_f64, double, corners_f64)
DEFINE_PAINT(oracle_cic_paint_f32, float, corners_f32)

/* out[p * ncomp + q] = sum_c w_c meshes[q][idx_c]: ncomp meshes of nx*ny*nz read at the
 * same particles. */
#define DEFINE_READ(NAME, T, CORNERS)                                                                      \
  int NAME(const T* meshes, int ncomp, const T* pos, int64_t np, int64_t nx, int64_t ny, int64_t nz,       \
           int absolute, T* out) {                                                                         \
    const int64_t m = nx * ny * nz;                                                                        \
    if (!absolute && np != m) return -1;                                                                   \
    _Pragma("omp parallel for schedule(static)") for (int64_t p = 0; p < np; ++p) {                        \
      int64_t idx[8];                                                                                      \
      T w[8];                                                                                              \
      CORNERS(pos, p, nx, ny, nz, absolute, idx, w);                                                       \
      for (int q = 0; q < ncomp; ++q) {                                                                    \
        const T* mesh = meshes + (size_t)q * (size_t)m;                                                    \
        T r[8];                                                                                            \
        for (int c = 0; c < 8; ++c) r[c] = (T)(mesh[idx[c]] * w[c]);                                       \
        out[p * ncomp + q] = (T)((T)((T)(r[0] + r[1]) + (T)(r[2] + r[3])) +                                \
                                 (T)((T)(r[4] + r[5]) + (T)(r[6] + r[7])));                                \
      }                                                                                                    \
    }                                                                                                      \
    return 0;                                                                                              \
  }

DEFINE_READ(oracle_cic_read_f64, double, corners_f64)
DEFINE_READ(oracle_cic_read_f32, float, corners_f32)

int oracle_threads(void) { return omp_get_max_threads(); }
