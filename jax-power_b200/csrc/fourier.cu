// Fourier-space passes: cuFFT plans, fused interlacing + compensation, and the
// real-space Y_lm premultiply of the first-point estimator.
#include <cufft.h>
#include <math.h>

#include "common.cuh"
#include "ylm_table.cuh"

struct pk_fft_plan_s {
  cufftHandle handle;
  int direction;
  int batch;
  pk::Dims d;
};

namespace pk {

struct FourierParams {
  Dims d;
  float cspacing[3];  // float32(2 pi / N_d): circular spacing (mesh.py:1627-1629)
  int nshifts;
  float shifts[8];
  float interlacing;
  int comp_order;
  int backend;
  int for_c2r;
  float scale;
};

// jnp.sinc(k / 2pi) with the reference's float32 operations (resamplers.py:21).
__device__ __forceinline__ float sinc_of(float kc) {
  const float x = __fdiv_rn(kc, 6.2831855f);  // float32(2 pi)
  if (x == 0.f) return 1.f;
  const float px = __fmul_rn(3.1415927f, x);
  return __fdiv_rn(sinf(px), px);
}

// (prod_d sinc)^(-order): lax.integer_pow by binary exponentiation, then 1/acc.
__device__ __forceinline__ float compensation(const FourierParams &p, float k0, float k1,
                                              float k2) {
  float ker = __fmul_rn(__fmul_rn(sinc_of(k0), sinc_of(k1)), sinc_of(k2));
  int y = p.comp_order;
  float acc = 1.f, x = ker;
  bool first = true;
  while (y > 0) {
    if (y & 1) {
      acc = first ? x : __fmul_rn(acc, x);
      first = false;
    }
    y >>= 1;
    if (y > 0) x = __fmul_rn(x, x);
  }
  return __fdiv_rn(1.f, acc);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// Interlaced + compensated value of stored mode (i, j, z).
__device__ __forceinline__ float2 combine(const FourierParams &p, const float2 *__restrict__ in,
                                          int i, int j, int z) {
  const Dims &d = p.d;
  const bool full = p.backend == PK_BACKEND_JAXDECOMP;
  const float k0 = ccoord(i, d.n0, p.cspacing[0], false);
  const float k1 = ccoord(j, d.n1, p.cspacing[1], false);
  const float k2 = ccoord(z, d.n2, p.cspacing[2], !full);
  const int64_t idx = ((int64_t)i * d.n1 + j) * d.nz + z;
  float2 acc;
  if (p.nshifts == 1 && p.shifts[0] == 0.f) {
    acc = in[idx];
  } else {
    const float ksum = __fadd_rn(__fadd_rn(k0, k1), k2);
    float ksum_neg = 0.f;
    if (full) {  // circular coordinates of the mirrored mode -k on the full grid
      const int in0 = (d.n0 - i) % d.n0, in1 = (d.n1 - j) % d.n1, in2 = (d.n2 - z) % d.n2;
      ksum_neg = __fadd_rn(__fadd_rn(ccoord(in0, d.n0, p.cspacing[0], false),
                                     ccoord(in1, d.n1, p.cspacing[1], false)),
                           ccoord(in2, d.n2, p.cspacing[2], false));
    }
    acc = make_float2(0.f, 0.f);
    for (int s = 0; s < p.nshifts; ++s) {
      const float2 v = in[(int64_t)s * d.ncomplex() + idx];
      float sn, cs;
      sincosf(__fmul_rn(p.shifts[s], ksum), &sn, &cs);
      float2 ph = make_float2(cs, sn);
      if (full) {  // Hermitian part of the full-grid phase: (e^{i t(k)} + e^{-i t(-k)}) / 2
        float sn2, cs2;
        sincosf(__fmul_rn(p.shifts[s], ksum_neg), &sn2, &cs2);
        ph = make_float2(0.5f * (cs + cs2), 0.5f * (sn - sn2));
      }
      float2 t = cmul(v, ph);
      t.x = __fdiv_rn(t.x, p.interlacing);  // value * phase / interlacing
      t.y = __fdiv_rn(t.y, p.interlacing);
      acc.x = __fadd_rn(acc.x, t.x);
      acc.y = __fadd_rn(acc.y, t.y);
    }
  }
  if (p.comp_order > 0) {
    const float c = compensation(p, k0, k1, k2);
    acc.x = __fmul_rn(acc.x, c);
    acc.y = __fmul_rn(acc.y, c);
  }
  return acc;
}

__global__ void interlace_kernel(FourierParams p, const float2 *__restrict__ in,
                                 float2 *__restrict__ out) {
  const Dims d = p.d;
  const int64_t total = d.ncomplex();
  const bool even = (d.n2 % 2) == 0;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(idx % d.nz);
    const int64_t r = idx / d.nz;
    const int j = (int)(r % d.n1);
    const int i = (int)(r / d.n1);
    float2 v = combine(p, in, i, j, z);
    if (p.for_c2r && (z == 0 || (even && z == d.nz - 1))) {
      const float2 m = combine(p, in, (d.n0 - i) % d.n0, (d.n1 - j) % d.n1, z);
      v = make_float2(0.5f * (v.x + m.x), 0.5f * (v.y - m.y));
    }
    v.x *= p.scale;
    v.y *= p.scale;
    out[idx] = v;
  }
}

__global__ void scale_kernel(float *__restrict__ x, int64_t n, float s) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= s;
}

struct YlmTerms {
  int n;
  int ell[32];
  int m[32];
};

// out[j] = rho(x) * Y_j(xhat), x the cell-corner position (observer at origin).
__global__ void ylm_premultiply_kernel(Dims d, float c0, float c1, float c2, float o0, float o1,
                                       float o2, YlmTerms terms, const float *__restrict__ rho,
                                       float *__restrict__ out) {
  const int64_t total = d.nreal();
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(idx % d.n2);
    const int64_t r = idx / d.n2;
    const int j = (int)(r % d.n1);
    const int i = (int)(r / d.n1);
    // rcoords: arange(n) * cellsize + (boxcenter - boxsize / 2)
    const float x = __fadd_rn(__fmul_rn((float)i, c0), o0);
    const float y = __fadd_rn(__fmul_rn((float)j, c1), o1);
    const float z = __fadd_rn(__fmul_rn((float)k, c2), o2);
    const float xn = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
    float xh = 0.f, yh = 0.f, zh = 0.f;
    if (xn != 0.f) {
      xh = __fdiv_rn(x, xn);
      yh = __fdiv_rn(y, xn);
      zh = __fdiv_rn(z, xn);
    }
    const float v = rho[idx];
    for (int t = 0; t < terms.n; ++t)
      out[(int64_t)t * total + idx] = __fmul_rn(v, ylm_eval(terms.ell[t], terms.m[t], xh, yh, zh));
  }
}

static int grid_for(int64_t n, int threads) {
  int64_t want = (n + threads - 1) / threads;
  int64_t cap = 32LL * sm_count();
  if (want < 1) want = 1;
  return (int)(want < cap ? want : cap);
}

}  // namespace pk

using namespace pk;

static const char *cufft_error_name(cufftResult r) {
  switch (r) {
    case CUFFT_SUCCESS: return "CUFFT_SUCCESS";
    case CUFFT_INVALID_PLAN: return "CUFFT_INVALID_PLAN";
    case CUFFT_ALLOC_FAILED: return "CUFFT_ALLOC_FAILED";
    case CUFFT_INVALID_VALUE: return "CUFFT_INVALID_VALUE";
    case CUFFT_INTERNAL_ERROR: return "CUFFT_INTERNAL_ERROR";
    case CUFFT_EXEC_FAILED: return "CUFFT_EXEC_FAILED";
    case CUFFT_SETUP_FAILED: return "CUFFT_SETUP_FAILED";
    case CUFFT_INVALID_SIZE: return "CUFFT_INVALID_SIZE";
    default: return "cufft error";
  }
}

#define PK_CUFFT(call)                                                         \
  do {                                                                         \
    cufftResult r_ = (call);                                                   \
    if (r_ != CUFFT_SUCCESS) {                                                 \
      ::pk::set_error("%s failed: %s", #call, cufft_error_name(r_));           \
      return PK_ERR_CUDA;                                                      \
    }                                                                          \
  } while (0)

extern "C" pk_status pk_fft_plan_create(const int32_t meshsize[3], int batch, int direction,
                                        pk_fft_plan *plan) {
  PK_REQUIRE(plan, PK_ERR_INVALID, "plan is NULL");
  Dims d;
  PK_REQUIRE(make_dims(meshsize, &d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(batch >= 1, PK_ERR_INVALID, "batch must be >= 1");
  PK_REQUIRE(direction == 0 || direction == 1, PK_ERR_INVALID, "direction must be 0 or 1");
  auto *p = new pk_fft_plan_s();
  p->direction = direction;
  p->batch = batch;
  p->d = d;
  int n[3] = {d.n0, d.n1, d.n2};
  // NULL embeds: contiguous meshes, batch distance = one real / one Hermitian mesh
  cufftResult r = cufftPlanMany(&p->handle, 3, n, nullptr, 1, 0, nullptr, 1, 0,
                                direction == 0 ? CUFFT_R2C : CUFFT_C2R, batch);
  if (r != CUFFT_SUCCESS) {
    delete p;
    set_error("cufftPlanMany failed: %s", cufft_error_name(r));
    return PK_ERR_CUDA;
  }
  *plan = p;
  return PK_OK;
}

extern "C" pk_status pk_fft_exec(pk_fft_plan plan, void *stream, void *in, void *out) {
  PK_REQUIRE(plan && in && out, PK_ERR_INVALID, "null plan / buffer");
  PK_CUFFT(cufftSetStream(plan->handle, (cudaStream_t)stream));
  if (plan->direction == 0)
    PK_CUFFT(cufftExecR2C(plan->handle, (cufftReal *)in, (cufftComplex *)out));
  else
    PK_CUFFT(cufftExecC2R(plan->handle, (cufftComplex *)in, (cufftReal *)out));
  return PK_OK;
}

extern "C" pk_status pk_fft_plan_destroy(pk_fft_plan plan) {
  if (!plan) return PK_OK;
  cufftDestroy(plan->handle);
  delete plan;
  return PK_OK;
}

extern "C" pk_status pk_interlace_compensate(void *stream, const void *in, int nshifts,
                                             const int32_t meshsize[3], int comp_order,
                                             int backend, int for_c2r, float scale, void *out) {
  PK_REQUIRE(in && out, PK_ERR_INVALID, "null buffer");
  FourierParams p;
  PK_REQUIRE(make_dims(meshsize, &p.d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(nshifts >= 1 && nshifts <= 8, PK_ERR_INVALID, "nshifts must be in 1..8");
  PK_REQUIRE(comp_order >= 0 && comp_order <= 4, PK_ERR_INVALID, "comp_order must be in 0..4");
  PK_REQUIRE(backend == PK_BACKEND_JAX || backend == PK_BACKEND_JAXDECOMP, PK_ERR_INVALID,
             "unknown backend %d", backend);
  PK_REQUIRE(in != out || (nshifts == 1 && !for_c2r), PK_ERR_INVALID,
             "in-place only for a single mesh without plane symmetrisation");
  const int ns[3] = {p.d.n0, p.d.n1, p.d.n2};
  for (int a = 0; a < 3; ++a) p.cspacing[a] = (float)(2. * M_PI / ns[a]);
  p.nshifts = nshifts;
  for (int s = 0; s < 8; ++s) p.shifts[s] = s < nshifts ? (float)s / (float)nshifts : 0.f;
  p.interlacing = (float)nshifts;
  p.comp_order = comp_order;
  p.backend = backend;
  p.for_c2r = for_c2r;
  p.scale = scale;
  const int threads = 256;
  interlace_kernel<<<grid_for(p.d.ncomplex(), threads), threads, 0, (cudaStream_t)stream>>>(
      p, (const float2 *)in, (float2 *)out);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_scale_real(void *stream, float *mesh, int64_t size, float scale) {
  PK_REQUIRE(mesh || size == 0, PK_ERR_INVALID, "null mesh");
  if (size == 0) return PK_OK;
  scale_kernel<<<grid_for(size, 256), 256, 0, (cudaStream_t)stream>>>(mesh, size, scale);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_ylm_premultiply(void *stream, const float *rho, const int32_t meshsize[3],
                                        const float cellsize[3], const float offset[3], int nterms,
                                        const int32_t *term_ell, const int32_t *term_m,
                                        float *out) {
  PK_REQUIRE(rho && out && cellsize && offset, PK_ERR_INVALID, "null pointer");
  Dims d;
  PK_REQUIRE(make_dims(meshsize, &d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(nterms >= 1 && nterms <= 32, PK_ERR_INVALID, "nterms must be in 1..32");
  YlmTerms t;
  t.n = nterms;
  for (int j = 0; j < nterms; ++j) {
    PK_REQUIRE(term_ell[j] >= 0 && term_ell[j] <= YLM_LMAX && term_m[j] >= -term_ell[j] &&
                   term_m[j] <= term_ell[j],
               PK_ERR_INVALID, "invalid (ell, m) = (%d, %d)", term_ell[j], term_m[j]);
    t.ell[j] = term_ell[j];
    t.m[j] = term_m[j];
  }
  ylm_premultiply_kernel<<<grid_for(d.nreal(), 256), 256, 0, (cudaStream_t)stream>>>(
      d, cellsize[0], cellsize[1], cellsize[2], offset[0], offset[1], offset[2], t, rho, out);
  PK_LAUNCH_CHECK();
  return PK_OK;
}
