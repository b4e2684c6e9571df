/* Resampler scatter of the CPU oracle in C (TEST INFRASTRUCTURE ONLY).
 *
 * The same arithmetic as oracle/paint.py:paint_mesh, which restates
 * resamplers.py:57-97 of jax-power:
 *   - kernels resamplers.py:57-63 in float32, no contraction (build with
 *     -ffp-contract=off): TSC 0.75 - s*s (s <= 0.5) or 0.5 * ((1.5 - s) * (1.5 - s)),
 *     PCS 1/6 * ((4 - 6 s^2) + 3 s^3) (s <= 1) or 1/6 * ((2 - s)^2 (2 - s)), CIC 1 - s;
 *   - base index round-half-even (odd order, jnp.round) or floor (even order),
 *     stencil offsets arange(order) - (order - 1) // 2 in itertools.product order
 *     (resamplers.py:84-85), periodic wrap;
 *   - contribution w * ((k0 * k1) * k2).
 * Two accumulations:
 *   - oracle_paint_serial: float32 adds, offset by offset and particle by particle
 *     (np.add.at order: the reference's serial CPU scatter order), bit-identical to
 *     paint_mesh(dtype=float32);
 *   - oracle_paint_f64: the same float32 contributions added in float64, particle by
 *     particle (rounded to float32 by the caller): paint_mesh(accum='f64') up to float64
 *     rounding;
 *   - oracle_paint_double: the whole computation in float64 (paint_mesh(dtype=float64)),
 *     particle by particle.
 * It exists so that the oracle finishes the 512^3 configurations in seconds; it is
 * never part of the product. */
#include <math.h>
#include <stdint.h>
#include <string.h>

static float kernel(int order, float s) {
  switch (order) {
    case 1:
      return 1.f;
    case 2:
      return 1.f - s;
    case 3:
      if (s <= 0.5f) return 0.75f - s * s;
      {
        const float t = 1.5f - s;
        return 0.5f * (t * t);
      }
    default: {
      const float sixth = 1.f / 6.f;  /* (bool) / 6 in float32 */
      if (s <= 1.f) {
        const float s2 = s * s, s3 = s2 * s;
        return sixth * ((4.f - 6.f * s2) + 3.f * s3);
      }
      const float t = 2.f - s;
      return sixth * ((t * t) * t);
    }
  }
}

static int64_t wrap(int64_t i, int64_t n) {
  const int64_t r = i % n;
  return r < 0 ? r + n : r;
}

static int64_t base_index(int order, float u) {
  return (order & 1) ? (int64_t)rintf(u) : (int64_t)floorf(u);
}

/* u: (n, 3) positions in cell units, already shifted; w: (n,) weights or NULL (1).
 * One stencil offset (a, b, c) at a time, over all particles. */
#define PAINT_BODY(ACCUM)                                                              \
  const int lo = -((order - 1) / 2);                                                   \
  for (int a = 0; a < order; ++a)                                                      \
    for (int b = 0; b < order; ++b)                                                    \
      for (int c = 0; c < order; ++c) {                                                \
        const int off[3] = {lo + a, lo + b, lo + c};                                   \
        for (int64_t p = 0; p < n; ++p) {                                              \
          float k[3];                                                                  \
          int64_t idx[3];                                                              \
          for (int d = 0; d < 3; ++d) {                                                \
            const float ud = u[3 * p + d];                                             \
            const int64_t i = base_index(order, ud) + off[d];                          \
            k[d] = kernel(order, fabsf((float)i - ud));                                \
            idx[d] = wrap(i, shape[d]);                                                \
          }                                                                            \
          const float ker = (k[0] * k[1]) * k[2];                                      \
          const float val = (w ? w[p] : 1.f) * ker;                                    \
          ACCUM;                                                                       \
        }                                                                              \
      }

void oracle_paint_serial(const float *u, const float *w, int64_t n, int order, const int64_t shape[3],
                         float *mesh) {
  PAINT_BODY(mesh[(idx[0] * shape[1] + idx[1]) * shape[2] + idx[2]] += val)
}

/* Particle by particle (all offsets of one particle in turn): the float64 sums differ from
 * the offset-major order only by float64 rounding, and the mesh is walked with locality. */
void oracle_paint_f64(const float *u, const float *w, int64_t n, int order, const int64_t shape[3],
                      double *acc) {
  const int lo = -((order - 1) / 2);
  for (int64_t p = 0; p < n; ++p) {
    float k[3][4];
    int64_t idx[3][4];
    for (int d = 0; d < 3; ++d) {
      const float ud = u[3 * p + d];
      const int64_t i0 = base_index(order, ud);
      for (int o = 0; o < order; ++o) {
        const int64_t i = i0 + lo + o;
        k[d][o] = kernel(order, fabsf((float)i - ud));
        idx[d][o] = wrap(i, shape[d]);
      }
    }
    const float wp = w ? w[p] : 1.f;
    for (int a = 0; a < order; ++a)
      for (int b = 0; b < order; ++b) {
        const float kab = k[0][a] * k[1][b];
        double *row = acc + (idx[0][a] * shape[1] + idx[1][b]) * shape[2];
        for (int c = 0; c < order; ++c) row[idx[2][c]] += (double)(wp * (kab * k[2][c]));
      }
  }
}

static double kernel_d(int order, double s) {
  switch (order) {
    case 1:
      return 1.;
    case 2:
      return 1. - s;
    case 3:
      if (s <= 0.5) return 0.75 - s * s;
      return 0.5 * ((1.5 - s) * (1.5 - s));
    default:
      if (s <= 1.) return (1. / 6.) * ((4. - 6. * s * s) + 3. * (s * s) * s);
      return (1. / 6.) * (((2. - s) * (2. - s)) * (2. - s));
  }
}

void oracle_paint_double(const double *u, const double *w, int64_t n, int order, const int64_t shape[3],
                         double *acc) {
  const int lo = -((order - 1) / 2);
  for (int64_t p = 0; p < n; ++p) {
    double k[3][4];
    int64_t idx[3][4];
    for (int d = 0; d < 3; ++d) {
      const double ud = u[3 * p + d];
      const int64_t i0 = (order & 1) ? (int64_t)rint(ud) : (int64_t)floor(ud);
      for (int o = 0; o < order; ++o) {
        const int64_t i = i0 + lo + o;
        k[d][o] = kernel_d(order, fabs((double)i - ud));
        idx[d][o] = wrap(i, shape[d]);
      }
    }
    const double wp = w ? w[p] : 1.;
    for (int a = 0; a < order; ++a)
      for (int b = 0; b < order; ++b) {
        const double kab = k[0][a] * k[1][b];
        double *row = acc + (idx[0][a] * shape[1] + idx[1][b]) * shape[2];
        for (int c = 0; c < order; ++c) row[idx[2][c]] += wp * (kab * k[2][c]);
      }
  }
}
