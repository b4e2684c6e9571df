// Correlation-function multipoles in the spherical-Bessel basis (BinMesh2CorrelationPoles
// with basis='bessel', mesh2.py:169-181, estimators mesh2.py:414-500 with basis 'bessel').
//
// The reference keeps the estimator's mode values A_ell(k) in Fourier space and projects
// them on j_ell(|k| s_b) for every separation bin b:
//   xi_ell[b] ~ (-1)^(ell/2) sum_k Re(A_ell(k)) j_ell(|k| s_b) / N^3
// summed over the stored (Hermitian half) modes, each once, without a Hermitian weight.
// A_ell is |d1|^2 L_ell(mu) (or conj(d1) d2 L_ell(mu)) for a fixed line of sight, and
// conj(sum_m F_lm Y_lm(khat)) A0 for the first point; the k = 0 mode is dropped for
// ell > 0 (remove_zero).  This kernel forms A_ell per mode, stages a chunk of modes in
// shared memory and lets every thread accumulate its separation bins over the chunk:
// a dense (bins x modes) projection whose matrix is generated on the fly.  j_ell is
// evaluated in float64 from the float32 argument |k| s_b (the reference's float32
// product); the reference's closed forms for x > 0.1 (utils.py:419-440) are the upward
// recurrence written out, its low-x branch the Taylor series, both used here.  Sums are
// float64, per CTA, then added in a fixed order (deterministic).
#include <math.h>

#include "common.cuh"
#include "ylm_table.cuh"

namespace pk {

constexpr int BES_THREADS = 512;        // = modes per staged chunk
constexpr int BES_BINS_PER_THREAD = 2;  // separation bins <= 1024
constexpr int BES_MAX_ELLS = 5;
constexpr int BES_MAX_TERMS = 32;
constexpr int BES_MAX_ORDER = 8;

// Legendre polynomials in the reference's float32 expression order (utils.py:341-360).
__device__ __forceinline__ float bessel_legendre(int ell, float x) {
  const float x2 = x * x;
  switch (ell) {
    case 0: return 1.f;
    case 1: return x;
    case 2: return 3.f * x2 / 2.f - 0.5f;
    case 3: return 5.f * (x2 * x) / 2.f - 3.f * x / 2.f;
    default: { const float x4 = x2 * x2; return 35.f * x4 / 8.f - 15.f * x2 / 4.f + 0.375f; }
  }
}

// j_0 .. j_LMAX at x (float64): x > 0.1 upward recurrence from sin and cos; x <= 0.1 the
// Taylor series x^l / (2l+1)!! sum_k (-x^2/2)^k / (k! (2l+3)(2l+5)...(2l+2k+1)), 6 terms
// (the reference truncates at x^10).  LMAX is a compile-time bound, so j stays in registers.
template <int LMAX>
__device__ __forceinline__ void spherical_jn(double x, double (&j)[LMAX + 1]) {
  if (x > 0.1) {
    double s, c;
    sincos(x, &s, &c);
    const double inv = 1.0 / x;
    j[0] = s * inv;
    if constexpr (LMAX >= 1) j[1] = (s * inv - c) * inv;
#pragma unroll
    for (int l = 1; l < LMAX; ++l) j[l + 1] = (2 * l + 1) * inv * j[l] - j[l - 1];
    return;
  }
  const double h = -0.5 * x * x;
  double lead = 1.0;  // x^l / (2l+1)!!
#pragma unroll
  for (int l = 0; l <= LMAX; ++l) {
    double term = lead, sum = lead;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      term *= h / ((k + 1) * (double)(2 * l + 2 * k + 3));
      sum += term;
    }
    j[l] = sum;
    lead *= x / (double)(2 * l + 3);
  }
}

struct BesselOp {
  int local;          // 0: fixed line of sight, 1: first point
  const float2 *d1;   // fixed los: delta1; first point: A0
  const float2 *d2;   // fixed los: delta2 (cross) or NULL; first point: B0 (cross, ell = 0) or NULL
  const float2 *f;    // first point: nterms transformed Y_lm-weighted meshes
  int64_t fstride;
  int nterms;
  int term_ell[BES_MAX_TERMS];
  int term_m[BES_MAX_TERMS];
  float los[3];
  int nells;
  int ells[BES_MAX_ELLS];
  int include_ell0;

  // Re(A_ell) of stored mode idx (no Hermitian weight).
  __device__ void operator()(int64_t idx, bool zero, float kx, float ky, float kz, float k2,
                             float v[BES_MAX_ELLS]) const {
    const float2 a = d1[idx];
    if (!local) {
      const float re = d2 ? a.x * d2[idx].x + a.y * d2[idx].y : a.x * a.x + a.y * a.y;
      const float num = (kx * los[0] + ky * los[1]) + kz * los[2];
      const float mu = k2 > 0.f ? num * rsqrtf(k2) : 0.f;
#pragma unroll
      for (int l = 0; l < BES_MAX_ELLS; ++l)
        v[l] = l >= nells ? 0.f : (ells[l] == 0 ? re : (zero ? 0.f : re * bessel_legendre(ells[l], mu)));
      return;
    }
    const float rn = k2 > 0.f ? rsqrtf(k2) : 0.f;
    const float xh = kx * rn, yh = ky * rn, zh = kz * rn;
#pragma unroll
    for (int l = 0; l < BES_MAX_ELLS; ++l) {
      const int ell = l < nells ? ells[l] : -1;
      v[l] = 0.f;
      if (ell < 0) continue;
      if (ell == 0) {
        if (!include_ell0) continue;
        v[l] = d2 ? d2[idx].x * a.x + d2[idx].y * a.y : a.x * a.x + a.y * a.y;
        continue;
      }
      if (zero) continue;
      float sr = 0.f, si = 0.f;
      for (int t = 0; t < nterms; ++t) {
        if (term_ell[t] != ell) continue;
        const float2 F = f[(int64_t)t * fstride + idx];
        const float y = ylm_eval(ell, term_m[t], xh, yh, zh);
        sr += F.x * y;
        si += F.y * y;
      }
      v[l] = sr * a.x + si * a.y;  // Re(conj(S) A0)
    }
  }
};

struct BesselGeom {
  Dims d;
  float kfun[3];
  int half;  // 1: 'jax' rfftfreq along the last axis
  int nbins;
  int use_klimit;
  float klimit[2];
};

template <int LMAX>
__global__ void __launch_bounds__(BES_THREADS, 1) bessel_project_kernel(BesselGeom g, BesselOp op,
                                                                     const double *__restrict__ sep,
                                                                     double *__restrict__ partials) {
  __shared__ float skn[BES_THREADS];
  __shared__ float sv[BES_MAX_ELLS][BES_THREADS];
  const int tid = threadIdx.x;
  int ells[BES_MAX_ELLS];
#pragma unroll
  for (int l = 0; l < BES_MAX_ELLS; ++l) ells[l] = l < op.nells ? op.ells[l] : -1;  // -1: no multipole, adds 0
  float s[BES_BINS_PER_THREAD];
  double acc[BES_BINS_PER_THREAD][BES_MAX_ELLS];
#pragma unroll
  for (int q = 0; q < BES_BINS_PER_THREAD; ++q) {
    const int b = tid + q * BES_THREADS;
    s[q] = b < g.nbins ? (float)sep[b] : 0.f;
#pragma unroll
    for (int l = 0; l < BES_MAX_ELLS; ++l) acc[q][l] = 0.;
  }
  const int64_t total = g.d.ncomplex();
  for (int64_t base = (int64_t)blockIdx.x * BES_THREADS; base < total; base += (int64_t)gridDim.x * BES_THREADS) {
    const int64_t idx = base + tid;
    float kn = 0.f, v[BES_MAX_ELLS];
#pragma unroll
    for (int l = 0; l < BES_MAX_ELLS; ++l) v[l] = 0.f;
    if (idx < total) {
      const int z = (int)(idx % g.d.nz);
      const int64_t row = idx / g.d.nz;
      const int j = (int)(row % g.d.n1), i = (int)(row / g.d.n1);
      const float kx = kcoord(i, g.d.n0, g.kfun[0], false);
      const float ky = kcoord(j, g.d.n1, g.kfun[1], false);
      const float kz = kcoord(z, g.d.n2, g.kfun[2], g.half != 0);
      const float k2 = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
      kn = __fsqrt_rn(k2);
      op(idx, i == 0 && j == 0 && z == 0, kx, ky, kz, k2, v);
      if (g.use_klimit && !(kn >= g.klimit[0] && kn < g.klimit[1]))
#pragma unroll
        for (int l = 0; l < BES_MAX_ELLS; ++l) v[l] = 0.f;
    }
    skn[tid] = kn;
#pragma unroll
    for (int l = 0; l < BES_MAX_ELLS; ++l) sv[l][tid] = v[l];
    __syncthreads();
    const int count = (int)min((int64_t)BES_THREADS, total - base);
    for (int m = 0; m < count; ++m) {
      const float knm = skn[m];
      double vm[BES_MAX_ELLS];
      bool any = false;
#pragma unroll
      for (int l = 0; l < BES_MAX_ELLS; ++l) {
        vm[l] = sv[l][m];
        any |= vm[l] != 0.;
      }
      if (!any) continue;  // uniform across the CTA (every thread reads mode m)
#pragma unroll
      for (int q = 0; q < BES_BINS_PER_THREAD; ++q) {
        if (tid + q * BES_THREADS >= g.nbins) break;
        double jn[LMAX + 1];
        spherical_jn<LMAX>((double)__fmul_rn(knm, s[q]), jn);
#pragma unroll
        for (int l = 0; l < BES_MAX_ELLS; ++l) {
          double jv = 0.;
#pragma unroll
          for (int o = 0; o <= LMAX; ++o) jv = o == ells[l] ? jn[o] : jv;
          acc[q][l] += vm[l] * jv;
        }
      }
    }
    __syncthreads();
  }
  // partials[cta][l][b]
#pragma unroll
  for (int q = 0; q < BES_BINS_PER_THREAD; ++q) {
    const int b = tid + q * BES_THREADS;
    if (b >= g.nbins) continue;
#pragma unroll
    for (int l = 0; l < BES_MAX_ELLS; ++l)
      if (l < op.nells) partials[((size_t)blockIdx.x * op.nells + l) * g.nbins + b] = acc[q][l];
  }
}

// out[l][b] (+)= sum over CTAs in index order of partials[cta][l][b].
__global__ void bessel_finalize_kernel(const double *__restrict__ partials, int nctas, int n, int accumulate,
                                       double *__restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double sum = 0.;
  for (int c = 0; c < nctas; ++c) sum += partials[(size_t)c * n + t];
  out[t] = accumulate ? out[t] + sum : sum;
}

static int bessel_ctas(const Dims &d) {
  const int64_t want = (d.ncomplex() + BES_THREADS - 1) / BES_THREADS;
  const int64_t cap = 4LL * sm_count();
  return (int)(want < cap ? want : cap);
}

}  // namespace pk

using namespace pk;

extern "C" pk_status pk_bin_bessel_workspace_size(const int32_t meshsize[3], int nbins, int nells, size_t *bytes) {
  Dims d;
  PK_REQUIRE(bytes && make_dims(meshsize, &d), PK_ERR_INVALID, "invalid arguments");
  PK_REQUIRE(nbins >= 1 && nbins <= BES_THREADS * BES_BINS_PER_THREAD, PK_ERR_RANGE,
             "the Bessel basis takes 1..%d separation bins", BES_THREADS * BES_BINS_PER_THREAD);
  PK_REQUIRE(nells >= 1 && nells <= BES_MAX_ELLS, PK_ERR_RANGE, "nells must be in 1..%d", BES_MAX_ELLS);
  *bytes = align_up((size_t)bessel_ctas(d) * nells * nbins * sizeof(double));
  return PK_OK;
}

extern "C" pk_status pk_bin_bessel(void *stream, const void *d1, const void *d2, const void *f, int nterms,
                                   const int32_t *term_ell, const int32_t *term_m, const int32_t meshsize[3],
                                   const float kfun[3], int backend, const float *los, const double *d_sep,
                                   int nbins, const float *klimit, int nells, const int32_t *ells,
                                   int include_ell0, int accumulate, double *d_out, void *workspace,
                                   size_t workspace_bytes) {
  BesselGeom g;
  PK_REQUIRE(make_dims(meshsize, &g.d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(d1 && d_sep && d_out && kfun && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nbins >= 1 && nbins <= BES_THREADS * BES_BINS_PER_THREAD, PK_ERR_RANGE,
             "the Bessel basis takes 1..%d separation bins", BES_THREADS * BES_BINS_PER_THREAD);
  PK_REQUIRE(nells >= 1 && nells <= BES_MAX_ELLS, PK_ERR_RANGE, "nells must be in 1..%d", BES_MAX_ELLS);
  PK_REQUIRE(nterms >= 0 && nterms <= BES_MAX_TERMS, PK_ERR_RANGE, "nterms must be in 0..%d", BES_MAX_TERMS);
  PK_REQUIRE(nterms == 0 || (f && term_ell && term_m && !los), PK_ERR_INVALID,
             "terms are first-point inputs (los must be NULL)");
  for (int c = 0; c < 3; ++c) g.kfun[c] = kfun[c];
  g.half = backend == PK_BACKEND_JAX;
  g.nbins = nbins;
  g.use_klimit = klimit != nullptr;
  g.klimit[0] = klimit ? klimit[0] : 0.f;
  g.klimit[1] = klimit ? klimit[1] : 0.f;
  BesselOp op{};
  op.local = los == nullptr;
  op.d1 = (const float2 *)d1;
  op.d2 = (const float2 *)d2;
  op.f = (const float2 *)f;
  op.fstride = g.d.ncomplex();
  op.nterms = nterms;
  for (int t = 0; t < nterms; ++t) {
    PK_REQUIRE(term_ell[t] >= 1 && term_ell[t] <= YLM_LMAX &&
                   term_m[t] >= -term_ell[t] && term_m[t] <= term_ell[t],
               PK_ERR_INVALID, "invalid (ell, m) = (%d, %d)", term_ell[t], term_m[t]);
    op.term_ell[t] = term_ell[t];
    op.term_m[t] = term_m[t];
  }
  for (int c = 0; c < 3; ++c) op.los[c] = los ? los[c] : 0.f;
  op.nells = nells;
  for (int l = 0; l < nells; ++l) {
    PK_REQUIRE(ells[l] >= 0 && ells[l] <= (los ? 4 : YLM_LMAX) && ells[l] <= BES_MAX_ORDER, PK_ERR_RANGE,
               "ell must be in 0..%d", los ? 4 : YLM_LMAX);
    op.ells[l] = ells[l];
  }
  op.include_ell0 = include_ell0;
  const int nctas = bessel_ctas(g.d);
  PK_REQUIRE(workspace && workspace_bytes >= (size_t)nctas * nells * nbins * sizeof(double), PK_ERR_WORKSPACE,
             "Bessel workspace too small");
  cudaStream_t s = (cudaStream_t)stream;
  double *partials = static_cast<double *>(workspace);
  int lmax = 0;
  for (int l = 0; l < nells; ++l) lmax = ells[l] > lmax ? ells[l] : lmax;
  switch (lmax) {
#define PK_BES_CASE(L)                                                          \
  case L:                                                                       \
    bessel_project_kernel<L><<<nctas, BES_THREADS, 0, s>>>(g, op, d_sep, partials); \
    break;
    PK_BES_CASE(0) PK_BES_CASE(1) PK_BES_CASE(2) PK_BES_CASE(3) PK_BES_CASE(4) PK_BES_CASE(5) PK_BES_CASE(6)
    PK_BES_CASE(7) PK_BES_CASE(8)
#undef PK_BES_CASE
  }
  PK_LAUNCH_CHECK();
  const int n = nells * nbins;
  bessel_finalize_kernel<<<(n + 255) / 256, 256, 0, s>>>(partials, nctas, n, accumulate, d_out);
  PK_LAUNCH_CHECK();
  return PK_OK;
}
