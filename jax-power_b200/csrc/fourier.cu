// Fourier-space passes: cuFFT plans, fused interlacing + compensation, and the
// real-space Y_lm premultiply of the first-point estimator.
#include <cufft.h>
#include <math.h>

#include "common.cuh"
#include "fourier_common.cuh"
#include "ylm_block.cuh"

struct pk_fft_plan_s {
  cufftHandle handle;
  int direction;
  int batch;
  pk::Dims d;
};

namespace pk {

constexpr int IL_THREADS = 256;

// One warp per (i, j) row of the Hermitian mesh; lanes stride kz (coalesced).
template <int NS, bool FULL>
__global__ void __launch_bounds__(IL_THREADS) interlace_kernel(FourierParams p,
                                                               const float2 *__restrict__ in,
                                                               float2 *__restrict__ out) {
  // (in / out are advanced to this block's mesh of the batch below)
  extern __shared__ float4 ilsmem[];
  const Dims d = p.d;
  constexpr bool full = FULL;
  in += (int64_t)blockIdx.y * p.nshifts * d.ncomplex();  // batch of meshes along y
  out += (int64_t)blockIdx.y * d.ncomplex();
  const bool xy = use_xy_tables(d);
  ZTable t = xy ? ztable_at<XY_SMEM>(ilsmem, p, full) : ztable_at<XY_NONE>(ilsmem, p, full);
  if (xy) fill_ztable<FULL, XY_SMEM>(p, t);
  else fill_ztable<FULL, XY_NONE>(p, t);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  const bool even = (d.n2 % 2) == 0;
  for (RowWalker rw((int64_t)blockIdx.x * nwarps + warp, (int64_t)gridDim.x * nwarps, d.n1); rw.i < d.n0;
       rw.next()) {
    const int i = rw.i, j = rw.j;
    const int64_t row = (int64_t)i * d.n1 + j;
    RowFactor<NS> rf, rm;
    row_factor_rt<NS, FULL>(p, t, i, j, rf);
    const bool planes = p.for_c2r != 0;
    const int im = (d.n0 - i) % d.n0, jm = (d.n1 - j) % d.n1;
    if (planes) row_factor_rt<NS, FULL>(p, t, im, jm, rm);
    const int64_t rbase = row * d.nz;
    const int64_t mbase = ((int64_t)im * d.n1 + jm) * d.nz;
    // four kz per lane per iteration: 4 * NS independent loads in flight
    for (int zb = lane; zb < d.nz; zb += 128) {
      float2 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int z = zb + 32 * u;
        v[u] = z < d.nz ? combine_mode<NS, FULL>(p, rf, t, in, rbase + z, z) : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int z = zb + 32 * u;
        if (z >= d.nz) break;
        if (planes && (z == 0 || (even && z == d.nz - 1))) {
          const float2 m = combine_mode<NS, FULL>(p, rm, t, in, mbase + z, z);
          v[u] = make_float2(0.5f * (v[u].x + m.x), 0.5f * (v[u].y - m.y));
        }
        out[rbase + z] = make_float2(v[u].x * p.scale, v[u].y * p.scale);
      }
    }
  }
}

__global__ void scale_kernel(float *__restrict__ x, int64_t n, float s) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= s;
}

// Transpose of the normalised C2R: out (+)= r w_z / N, w_z = 2 off the self-conjugate kz planes.
__global__ void c2r_adjoint_kernel(Dims d, const float2 *__restrict__ r, int accumulate, float inv_n,
                                   float2 *__restrict__ out) {
  const int64_t total = d.ncomplex();
  const bool even = (d.n2 % 2) == 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(i % d.nz);
    const float s = (z == 0 || (even && z == d.nz - 1)) ? inv_n : 2.f * inv_n;
    float2 v = r[i];
    v.x *= s;
    v.y *= s;
    if (accumulate) {
      const float2 o = out[i];
      v.x += o.x;
      v.y += o.y;
    }
    out[i] = v;
  }
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
  const int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  IndexWalker3 w(start, stride, d.n1, d.n2);
  for (int64_t idx = start; idx < total; idx += stride, w.next()) {
    const int i = w.i, j = w.j, k = w.k;
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

// ylm_premultiply_kernel for whole-ell term lists (mask MASK): four consecutive cells
// along the last axis per thread (one float4 load of rho, one float4 store per term), each
// Y_lm a compile-time polynomial.  Needs n2 % 4 == 0.
template <int MASK>
__global__ void __launch_bounds__(256) ylm_premultiply_block_kernel(Dims d, float c0, float c1, float c2,
                                                                   float o0, float o1, float o2,
                                                                   const float4 *__restrict__ rho,
                                                                   float4 *__restrict__ out) {
  constexpr int NT = ylm_mask_terms(MASK);
  const int64_t nquad = d.nreal() / 4;
  const int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  IndexWalker3 w(start, stride, d.n1, d.n2 / 4);
  for (int64_t q = start; q < nquad; q += stride, w.next()) {
    const float x = __fadd_rn(__fmul_rn((float)w.i, c0), o0);
    const float y = __fadd_rn(__fmul_rn((float)w.j, c1), o1);
    const float xy2 = __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y));
    const float4 r = __ldcs(rho + q);
    const float rv[4] = {r.x, r.y, r.z, r.w};
    float val[4][NT];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const float z = __fadd_rn(__fmul_rn((float)(4 * w.k + u), c2), o2);
      const float xn = __fsqrt_rn(__fadd_rn(xy2, __fmul_rn(z, z)));
      float xh = 0.f, yh = 0.f, zh = 0.f;
      if (xn != 0.f) {
        xh = __fdiv_rn(x, xn);
        yh = __fdiv_rn(y, xn);
        zh = __fdiv_rn(z, xn);
      }
      float yl[NT];
      ylm_block<MASK>(xh, yh, zh, yl);
#pragma unroll
      for (int t = 0; t < NT; ++t) val[u][t] = __fmul_rn(rv[u], yl[t]);
    }
#pragma unroll
    for (int t = 0; t < NT; ++t)
      __stcs(out + (int64_t)t * nquad + q, make_float4(val[0][t], val[1][t], val[2][t], val[3][t]));
  }
}

// ylm_accumulate_kernel for whole-ell term lists (mask MASK), four cells per thread.
template <int MASK>
__global__ void __launch_bounds__(256) ylm_accumulate_block_kernel(Dims d, float c0, float c1, float c2,
                                                                  float o0, float o1, float o2,
                                                                  const float4 *__restrict__ r,
                                                                  float4 *__restrict__ rho_bar) {
  constexpr int NT = ylm_mask_terms(MASK);
  const int64_t nquad = d.nreal() / 4;
  const int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  IndexWalker3 w(start, stride, d.n1, d.n2 / 4);
  for (int64_t q = start; q < nquad; q += stride, w.next()) {
    const float x = __fadd_rn(__fmul_rn((float)w.i, c0), o0);
    const float y = __fadd_rn(__fmul_rn((float)w.j, c1), o1);
    const float xy2 = __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y));
    float4 rv[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) rv[t] = __ldcs(r + (int64_t)t * nquad + q);
    const float4 b = rho_bar[q];
    float acc[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const float z = __fadd_rn(__fmul_rn((float)(4 * w.k + u), c2), o2);
      const float xn = __fsqrt_rn(__fadd_rn(xy2, __fmul_rn(z, z)));
      float xh = 0.f, yh = 0.f, zh = 0.f;
      if (xn != 0.f) {
        xh = __fdiv_rn(x, xn);
        yh = __fdiv_rn(y, xn);
        zh = __fdiv_rn(z, xn);
      }
      float yl[NT];
      ylm_block<MASK>(xh, yh, zh, yl);
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const float4 v = rv[t];
        acc[u] += (u == 0 ? v.x : u == 1 ? v.y : u == 2 ? v.z : v.w) * yl[t];
      }
    }
    rho_bar[q] = make_float4(acc[0], acc[1], acc[2], acc[3]);
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

extern "C" pk_status pk_interlace_compensate_batch(void *stream, const void *in, int nbatch,
                                                   int nshifts, const int32_t meshsize[3],
                                                   int comp_order, int backend, int for_c2r,
                                                   float scale, void *out);

extern "C" pk_status pk_interlace_compensate(void *stream, const void *in, int nshifts,
                                             const int32_t meshsize[3], int comp_order,
                                             int backend, int for_c2r, float scale, void *out) {
  return pk_interlace_compensate_batch(stream, in, 1, nshifts, meshsize, comp_order, backend,
                                       for_c2r, scale, out);
}

extern "C" pk_status pk_interlace_compensate_batch(void *stream, const void *in, int nbatch,
                                                   int nshifts, const int32_t meshsize[3],
                                                   int comp_order, int backend, int for_c2r,
                                                   float scale, void *out) {
  PK_REQUIRE(nbatch >= 1 && nbatch <= 65535, PK_ERR_INVALID, "nbatch must be in 1..65535");
  PK_REQUIRE(in && out, PK_ERR_INVALID, "null buffer");
  FourierParams p;
  PK_REQUIRE(make_dims(meshsize, &p.d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(nshifts >= 1 && nshifts <= IL_MAX_SHIFTS, PK_ERR_INVALID, "nshifts must be in 1..8");
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
  const bool full = backend == PK_BACKEND_JAXDECOMP;
  p.gxy = nullptr;
  const size_t smem = ztable_bytes(p.d, nshifts, full, use_xy_tables(p.d));
  PK_REQUIRE(smem <= 200 * 1024, PK_ERR_RANGE, "mesh too large for the per-axis tables");
  const int64_t nrows = (int64_t)p.d.n0 * p.d.n1;
  const int64_t want = (nrows + IL_THREADS / 32 - 1) / (IL_THREADS / 32);
  const int64_t cap = 8LL * sm_count();
  const dim3 blocks((unsigned)(want < cap ? want : cap), (unsigned)nbatch);
  cudaStream_t st = (cudaStream_t)stream;
  switch (nshifts * 2 + (full ? 1 : 0)) {
#define PK_IL_CASE(N)                                                                          \
  case 2 * N:                                                                                  \
    PK_CUDA(cudaFuncSetAttribute(interlace_kernel<N, false>,                                   \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));     \
    interlace_kernel<N, false><<<blocks, IL_THREADS, smem, st>>>(p, (const float2 *)in,        \
                                                                 (float2 *)out);               \
    break;                                                                                     \
  case 2 * N + 1:                                                                              \
    PK_CUDA(cudaFuncSetAttribute(interlace_kernel<N, true>,                                    \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));     \
    interlace_kernel<N, true><<<blocks, IL_THREADS, smem, st>>>(p, (const float2 *)in,         \
                                                                (float2 *)out);                \
    break;
    PK_IL_CASE(1) PK_IL_CASE(2) PK_IL_CASE(3) PK_IL_CASE(4) PK_IL_CASE(5) PK_IL_CASE(6)
    PK_IL_CASE(7) PK_IL_CASE(8)
#undef PK_IL_CASE
  }
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

extern "C" pk_status pk_c2r_adjoint(void *stream, const void *r, const int32_t meshsize[3], int accumulate,
                                    void *out) {
  PK_REQUIRE(r && out, PK_ERR_INVALID, "null pointer");
  Dims d;
  PK_REQUIRE(make_dims(meshsize, &d), PK_ERR_INVALID, "invalid meshsize");
  const int64_t total = d.ncomplex();
  c2r_adjoint_kernel<<<grid_for(total, 256), 256, 0, (cudaStream_t)stream>>>(
      d, (const float2 *)r, accumulate, (float)(1.0 / (double)d.nreal()), (float2 *)out);
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
  const int mask = ylm_terms_mask(nterms, term_ell, term_m);
  const bool aligned = ((uintptr_t)rho % 16) == 0 && ((uintptr_t)out % 16) == 0;
  if (mask && ylm_mask_compiled(mask) && d.n2 % 4 == 0 && aligned) {
    const int grid = grid_for(d.nreal() / 4, 256);
#define PK_YLM_PRE_CASE(M)                                                                        \
  if (mask == (M)) {                                                                              \
    ylm_premultiply_block_kernel<M><<<grid, 256, 0, (cudaStream_t)stream>>>(                      \
        d, cellsize[0], cellsize[1], cellsize[2], offset[0], offset[1], offset[2], (const float4 *)rho, \
        (float4 *)out);                                                                           \
    PK_LAUNCH_CHECK();                                                                            \
    return PK_OK;                                                                                 \
  }
    PK_YLM_MASKS(PK_YLM_PRE_CASE)
#undef PK_YLM_PRE_CASE
  }
  ylm_premultiply_kernel<<<grid_for(d.nreal(), 256), 256, 0, (cudaStream_t)stream>>>(
      d, cellsize[0], cellsize[1], cellsize[2], offset[0], offset[1], offset[2], t, rho, out);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

// ------------------------------------------------------------------ adjoints
// Backward of _paint's Fourier part (mesh.py:2737-2752) for the 'jax' semantics.  The
// forward is delta = C / I sum_s e^{i theta_s} F_s, F_s = rfftn(rho_s), optionally
// followed by irfftn.  Given the cotangent of the output (R = rfftn(rho_bar) when the
// output was the real mesh rho, or the conjugate cotangent gbar of delta itself), this
// writes for every shift h_s = sym(C e^{-i theta_s} X / I) with X = R / (N0 N1 N2) or
// gbar / w', so that rho_bar_s = C2R(h_s) (unnormalised) is the cotangent of painted
// mesh s.  sym() Hermitian-symmetrises the kz = 0 and N/2 planes.
// The phase and window are the forward's per-axis factors (row factor x kz table), so this
// is the transpose of interlace_kernel's arithmetic: e^{-i theta_s} = conj of the forward
// phase, C / I = the same row scale times the kz window.  One warp per (i, j) row, four kz
// per lane.
template <int NS, bool FULL>
__global__ void __launch_bounds__(IL_THREADS) interlace_adjoint_kernel(FourierParams p,
                                                                       const float2 *__restrict__ in,
                                                                       int from_real,
                                                                       float2 *__restrict__ out) {
  extern __shared__ float4 ilsmem[];
  const Dims d = p.d;
  const bool xy = use_xy_tables(d);
  ZTable t = xy ? ztable_at<XY_SMEM>(ilsmem, p, FULL) : ztable_at<XY_NONE>(ilsmem, p, FULL);
  if (xy) fill_ztable<FULL, XY_SMEM>(p, t);
  else fill_ztable<FULL, XY_NONE>(p, t);
  __syncthreads();
  const int64_t total = d.ncomplex();
  const bool even = (d.n2 % 2) == 0;
  const float inv_n = 1.f / (float)d.nreal();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  for (RowWalker rw((int64_t)blockIdx.x * nwarps + warp, (int64_t)gridDim.x * nwarps, d.n1); rw.i < d.n0;
       rw.next()) {
    const int i = rw.i, j = rw.j;
    const int im = (d.n0 - i) % d.n0, jm = (d.n1 - j) % d.n1;
    RowFactor<NS> rf, rm;
    row_factor_rt<NS, FULL>(p, t, i, j, rf);
    row_factor_rt<NS, FULL>(p, t, im, jm, rm);
    const int64_t rbase = ((int64_t)i * d.n1 + j) * d.nz;
    const int64_t mbase = ((int64_t)im * d.n1 + jm) * d.nz;
    for (int zb = lane; zb < d.nz; zb += 128) {
      float2 x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int z = zb + 32 * u;
        x[u] = z < d.nz ? in[rbase + z] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int z = zb + 32 * u;
        if (z >= d.nz) break;
        const bool plane = z == 0 || (even && z == d.nz - 1);
        const float scale = from_real ? inv_n : (plane ? 1.f : 0.5f);
        const float c = rf.scale * t.comp[z] * scale;
        float2 xm = make_float2(0.f, 0.f);
        float cm = 0.f;
        if (plane) {
          xm = in[mbase + z];
          cm = rm.scale * t.comp[z] * scale;
        }
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const float2 ph = mode_phase<NS, FULL>(p, rf, t, s, z);  // the forward's phase (combine_mode)
          float2 v = cmul(x[u], make_float2(ph.x, -ph.y));
          v = make_float2(v.x * c, v.y * c);
          if (plane) {
            const float2 phm = mode_phase<NS, FULL>(p, rm, t, s, z);
            float2 m = cmul(xm, make_float2(phm.x, -phm.y));
            m = make_float2(m.x * cm, m.y * cm);
            v = make_float2(0.5f * (v.x + m.x), 0.5f * (v.y - m.y));
          }
          out[(int64_t)s * total + rbase + z] = v;
        }
      }
    }
  }
}

// rho_bar(x) += sum_j r_j(x) Y_j(xhat) (adjoint of the Y_lm premultiply).
__global__ void ylm_accumulate_kernel(Dims d, float c0, float c1, float c2, float o0, float o1,
                                      float o2, YlmTerms terms, const float *__restrict__ r,
                                      float *__restrict__ rho_bar) {
  const int64_t total = d.nreal();
  const int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  IndexWalker3 w(start, stride, d.n1, d.n2);
  for (int64_t idx = start; idx < total; idx += stride, w.next()) {
    const int i = w.i, j = w.j, k = w.k;
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
    float acc = rho_bar[idx];
    for (int t = 0; t < terms.n; ++t)
      acc += r[(int64_t)t * total + idx] * ylm_eval(terms.ell[t], terms.m[t], xh, yh, zh);
    rho_bar[idx] = acc;
  }
}

// carry(s) += sum_t r_t(s) Y_t(shat) on the real-space separation grid
// s_d = fftfreq(n_d)[i] * cellsize_d * n_d (the first-point correlation function,
// mesh2.py:436-446); shat = 0 at s = 0.
__global__ void ylm_separation_accumulate_kernel(Dims d, float c0, float c1, float c2, YlmTerms terms,
                                                 const float *__restrict__ r, float *__restrict__ carry) {
  const int64_t total = d.nreal();
  const int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  IndexWalker3 w(start, stride, d.n1, d.n2);
  for (int64_t idx = start; idx < total; idx += stride, w.next()) {
    const float x = kcoord(w.i, d.n0, c0, false);
    const float y = kcoord(w.j, d.n1, c1, false);
    const float z = kcoord(w.k, d.n2, c2, false);
    const float xn = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
    float xh = 0.f, yh = 0.f, zh = 0.f;
    if (xn != 0.f) {
      xh = __fdiv_rn(x, xn);
      yh = __fdiv_rn(y, xn);
      zh = __fdiv_rn(z, xn);
    }
    float acc = carry[idx];
    for (int t = 0; t < terms.n; ++t)
      acc += r[(int64_t)t * total + idx] * ylm_eval(terms.ell[t], terms.m[t], xh, yh, zh);
    carry[idx] = acc;
  }
}

// mesh_b(r) *= |r|^power for nmeshes real meshes: r the cell-corner position o + i cellsize (the
// x of the Y_lm(xhat) premultiply) or, separation != 0, the separation fftfreq(n)[i] cellsize n
// (the s of the Y_lm(shat) accumulation), |r| = sqrt((x^2 + y^2) + z^2) in float32; a positive
// power by repeated products, a negative one as 1 / (|r|^-power) (as JAX's integer powers).
__global__ void radial_power_kernel(Dims d, float c0, float c1, float c2, float o0, float o1, float o2,
                                    int separation, int power, int nmeshes, float *__restrict__ mesh) {
  const int64_t total = d.nreal();
  const int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  IndexWalker3 w(start, stride, d.n1, d.n2);
  for (int64_t idx = start; idx < total; idx += stride, w.next()) {
    float x, y, z;
    if (separation) {
      x = kcoord(w.i, d.n0, c0, false);
      y = kcoord(w.j, d.n1, c1, false);
      z = kcoord(w.k, d.n2, c2, false);
    } else {
      x = __fadd_rn(__fmul_rn((float)w.i, c0), o0);
      y = __fadd_rn(__fmul_rn((float)w.j, c1), o1);
      z = __fadd_rn(__fmul_rn((float)w.k, c2), o2);
    }
    const float rn = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
    const int ap = power < 0 ? -power : power;
    float f = 1.f;
    for (int q = 0; q < ap; ++q) f = __fmul_rn(f, rn);
    if (power < 0) f = __fdiv_rn(1.f, f);
    for (int b = 0; b < nmeshes; ++b) mesh[(int64_t)b * total + idx] = __fmul_rn(mesh[(int64_t)b * total + idx], f);
  }
}

// out_t = conj(f_t) * a for nterms complex meshes f_t of n modes each.
__global__ void conj_multiply_kernel(const float2 *__restrict__ f, const float2 *__restrict__ a, int nterms,
                                     int64_t n, float2 *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 b = a[i];
    for (int t = 0; t < nterms; ++t) {
      const float2 v = f[(int64_t)t * n + i];
      out[(int64_t)t * n + i] = make_float2(v.x * b.x + v.y * b.y, v.x * b.y - v.y * b.x);
    }
  }
}

extern "C" pk_status pk_interlace_adjoint(void *stream, const void *in, int from_real,
                                          int nshifts, const int32_t meshsize[3], int comp_order,
                                          int backend, void *out) {
  PK_REQUIRE(in && out && in != out, PK_ERR_INVALID, "null or aliased buffers");
  FourierParams p;
  PK_REQUIRE(make_dims(meshsize, &p.d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(nshifts >= 1 && nshifts <= IL_MAX_SHIFTS, PK_ERR_INVALID, "nshifts must be in 1..8");
  PK_REQUIRE(comp_order >= 0 && comp_order <= 4, PK_ERR_INVALID, "comp_order must be in 0..4");
  PK_REQUIRE(backend == PK_BACKEND_JAX || backend == PK_BACKEND_JAXDECOMP, PK_ERR_INVALID, "unknown backend %d",
             backend);
  const bool full = backend == PK_BACKEND_JAXDECOMP;
  const int ns[3] = {p.d.n0, p.d.n1, p.d.n2};
  for (int a = 0; a < 3; ++a) p.cspacing[a] = (float)(2. * M_PI / ns[a]);
  p.nshifts = nshifts;
  for (int s = 0; s < IL_MAX_SHIFTS; ++s) p.shifts[s] = s < nshifts ? (float)s / (float)nshifts : 0.f;
  p.interlacing = (float)nshifts;
  p.comp_order = comp_order;
  p.backend = backend;
  p.for_c2r = 1;
  p.scale = 1.f;
  p.gxy = nullptr;
  const size_t smem = ztable_bytes(p.d, nshifts, full, use_xy_tables(p.d));
  PK_REQUIRE(smem <= 200 * 1024, PK_ERR_RANGE, "mesh too large for the per-axis tables");
  const int64_t nrows = (int64_t)p.d.n0 * p.d.n1;
  const int64_t want = (nrows + IL_THREADS / 32 - 1) / (IL_THREADS / 32);
  const int64_t cap = 8LL * sm_count();
  const int blocks = (int)(want < cap ? want : cap);
  cudaStream_t st = (cudaStream_t)stream;
  switch (nshifts) {
#define PK_ILA_LAUNCH(N, F)                                                                            \
  PK_CUDA(cudaFuncSetAttribute(interlace_adjoint_kernel<N, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                               (int)smem));                                                            \
  interlace_adjoint_kernel<N, F><<<blocks, IL_THREADS, smem, st>>>(p, (const float2 *)in, from_real,     \
                                                                   (float2 *)out);
#define PK_ILA_CASE(N)                                                                                 \
  case N:                                                                                              \
    if (full) {                                                                                        \
      PK_ILA_LAUNCH(N, true)                                                                           \
    } else {                                                                                           \
      PK_ILA_LAUNCH(N, false)                                                                          \
    }                                                                                                  \
    break;
    PK_ILA_CASE(1) PK_ILA_CASE(2) PK_ILA_CASE(3) PK_ILA_CASE(4) PK_ILA_CASE(5) PK_ILA_CASE(6)
    PK_ILA_CASE(7) PK_ILA_CASE(8)
#undef PK_ILA_CASE
#undef PK_ILA_LAUNCH
  }
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_ylm_accumulate(void *stream, const float *r, const int32_t meshsize[3],
                                       const float cellsize[3], const float offset[3], int nterms,
                                       const int32_t *term_ell, const int32_t *term_m,
                                       float *rho_bar) {
  PK_REQUIRE(r && rho_bar && cellsize && offset, PK_ERR_INVALID, "null pointer");
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
  const int mask = ylm_terms_mask(nterms, term_ell, term_m);
  const bool aligned = ((uintptr_t)r % 16) == 0 && ((uintptr_t)rho_bar % 16) == 0;
  if (mask && ylm_mask_compiled(mask) && d.n2 % 4 == 0 && aligned) {
    const int grid = grid_for(d.nreal() / 4, 256);
#define PK_YLM_ACC_CASE(M)                                                                        \
  if (mask == (M)) {                                                                              \
    ylm_accumulate_block_kernel<M><<<grid, 256, 0, (cudaStream_t)stream>>>(                       \
        d, cellsize[0], cellsize[1], cellsize[2], offset[0], offset[1], offset[2], (const float4 *)r, \
        (float4 *)rho_bar);                                                                       \
    PK_LAUNCH_CHECK();                                                                            \
    return PK_OK;                                                                                 \
  }
    PK_YLM_MASKS(PK_YLM_ACC_CASE)
#undef PK_YLM_ACC_CASE
  }
  ylm_accumulate_kernel<<<grid_for(d.nreal(), 256), 256, 0, (cudaStream_t)stream>>>(
      d, cellsize[0], cellsize[1], cellsize[2], offset[0], offset[1], offset[2], t, r, rho_bar);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_ylm_separation_accumulate(void *stream, const float *r, const int32_t meshsize[3],
                                                  const float cellsize[3], int nterms, const int32_t *term_ell,
                                                  const int32_t *term_m, float *carry) {
  PK_REQUIRE(r && carry && cellsize && term_ell && term_m, PK_ERR_INVALID, "null pointer");
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
  ylm_separation_accumulate_kernel<<<grid_for(d.nreal(), 256), 256, 0, (cudaStream_t)stream>>>(
      d, cellsize[0], cellsize[1], cellsize[2], t, r, carry);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_radial_power(void *stream, float *mesh, int nmeshes, const int32_t meshsize[3],
                                     const float cellsize[3], const float offset[3], int separation, int power) {
  PK_REQUIRE(mesh && cellsize && (separation || offset), PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nmeshes >= 1 && power >= -8 && power <= 8, PK_ERR_INVALID, "invalid nmeshes or power");
  Dims d;
  PK_REQUIRE(make_dims(meshsize, &d), PK_ERR_INVALID, "invalid meshsize");
  radial_power_kernel<<<grid_for(d.nreal(), 256), 256, 0, (cudaStream_t)stream>>>(
      d, cellsize[0], cellsize[1], cellsize[2], separation ? 0.f : offset[0], separation ? 0.f : offset[1],
      separation ? 0.f : offset[2], separation, power, nmeshes, mesh);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_conj_multiply(void *stream, const void *f, const void *a, int nterms, int64_t n,
                                      void *out) {
  PK_REQUIRE(f && a && out && nterms >= 1 && n >= 0, PK_ERR_INVALID, "invalid arguments");
  if (n == 0) return PK_OK;
  conj_multiply_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>((const float2 *)f, (const float2 *)a,
                                                                            nterms, n, (float2 *)out);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

// ------------------------------------------------------ first-point mean spectrum
// compute_mesh2_spectrum_mean, first-point line of sight (mesh2.py:1607-1669): products of a
// half-complex mesh with real Y_lm(khat) (khat = k / |k|, 0 at k = 0, as the first-point
// estimator), and sums of real-mesh products.
constexpr int KGRID_MAX_TERMS = 32;

struct KgridTerms {
  int ell[KGRID_MAX_TERMS], m[KGRID_MAX_TERMS];
};

struct ProductCoefs {
  float c[KGRID_MAX_TERMS];
};

__global__ void ylm_kgrid_kernel(Dims d, float kf0, float kf1, float kf2, int nterms, KgridTerms t, float scale,
                                 int accumulate, const float2 *__restrict__ value, float2 *__restrict__ out) {
  const int64_t nc = d.ncomplex();
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nc; q += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(q % d.nz);
    const int64_t row = q / d.nz;
    const int j = (int)(row % d.n1), i = (int)(row / d.n1);
    const float kx = kcoord(i, d.n0, kf0, false), ky = kcoord(j, d.n1, kf1, false);
    const float kz = kcoord(z, d.n2, kf2, true);
    const float k2 = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
    const float rn = k2 > 0.f ? rsqrtf(k2) : 0.f;
    const float2 v = value[q];
    for (int s = 0; s < nterms; ++s) {
      const float y = ylm_eval(t.ell[s], t.m[s], kx * rn, ky * rn, kz * rn) * scale;
      float2 *o = out + (int64_t)s * nc + q;
      float2 r = make_float2(v.x * y, v.y * y);
      if (accumulate) {
        const float2 p = *o;
        r.x += p.x;
        r.y += p.y;
      }
      *o = r;
    }
  }
}

// out[i] (+)= sum_t coef[t] a[t n + i] b[t n + i]
__global__ void sum_products_kernel(float *__restrict__ out, const float *__restrict__ a, const float *__restrict__ b,
                                    int nterms, ProductCoefs coef, int64_t n, int accumulate) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float acc = accumulate ? out[i] : 0.f;
    for (int t = 0; t < nterms; ++t)
      acc += coef.c[t] * (a[(int64_t)t * n + i] * b[(int64_t)t * n + i]);
    out[i] = acc;
  }
}

extern "C" pk_status pk_ylm_kgrid_multiply(void *stream, const void *value, const int32_t meshsize[3],
                                           const float kfun[3], int nterms, const int32_t *term_ell,
                                           const int32_t *term_m, float scale, int accumulate, void *out) {
  Dims d;
  PK_REQUIRE(make_dims(meshsize, &d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(value && kfun && term_ell && term_m && out, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nterms >= 1 && nterms <= KGRID_MAX_TERMS, PK_ERR_INVALID, "nterms must be in 1..%d", KGRID_MAX_TERMS);
  KgridTerms t;
  for (int s = 0; s < KGRID_MAX_TERMS; ++s) {
    t.ell[s] = s < nterms ? term_ell[s] : 0;
    t.m[s] = s < nterms ? term_m[s] : 0;
    if (s < nterms)
      PK_REQUIRE(t.ell[s] >= 0 && t.ell[s] <= YLM_LMAX && t.m[s] >= -t.ell[s] && t.m[s] <= t.ell[s], PK_ERR_INVALID,
                 "invalid (ell, m) = (%d, %d)", t.ell[s], t.m[s]);
  }
  const int64_t want = (d.ncomplex() + 255) / 256;
  const int blocks = (int)(want < (int64_t)sm_count() * 8 ? want : (int64_t)sm_count() * 8);
  ylm_kgrid_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(d, kfun[0], kfun[1], kfun[2], nterms, t, scale,
                                                              accumulate, (const float2 *)value, (float2 *)out);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_sum_products(void *stream, float *out, const float *a, const float *b, int nterms,
                                     const float *coef, int64_t n, int accumulate) {
  PK_REQUIRE(out && a && b && coef, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nterms >= 1 && nterms <= KGRID_MAX_TERMS, PK_ERR_INVALID, "nterms must be in 1..%d", KGRID_MAX_TERMS);
  PK_REQUIRE(n >= 1, PK_ERR_INVALID, "empty meshes");
  ProductCoefs c;
  for (int s = 0; s < KGRID_MAX_TERMS; ++s) c.c[s] = s < nterms ? coef[s] : 0.f;
  const int64_t want = (n + 255) / 256;
  const int blocks = (int)(want < (int64_t)sm_count() * 8 ? want : (int64_t)sm_count() * 8);
  sum_products_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, a, b, nterms, c, n, accumulate);
  PK_LAUNCH_CHECK();
  return PK_OK;
}
