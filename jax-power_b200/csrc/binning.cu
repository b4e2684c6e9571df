// k-binning of Fourier meshes: BinMesh2SpectrumPoles (mesh2.py:25-119) and the
// estimators of compute_mesh2_spectrum (mesh2.py:253-374), fused so that the
// per-mode |k|, bin index, mu / Y_lm(khat) and products are computed on the fly
// from one streaming read of the complex mesh(es).
//
// Reduction (deterministic, no float atomics):
//   - one warp walks one (i, j) row of the Hermitian mesh in chunks of 32 kz;
//     |k| is non-decreasing along kz, so lanes of equal bin are contiguous and a
//     5-step segmented shuffle scan gives one float32 partial per (chunk, bin);
//   - segment tails (distinct bins) add their partial into the warp's private
//     float64 histogram in shared memory;
//   - per CTA, warp histograms are summed in warp order into a float64 partial
//     row in global memory; a final kernel sums the CTA rows in CTA order.
// The grid size depends only on the problem shape, so results are bitwise
// reproducible run to run.
#include <math.h>

#include "common.cuh"
#include "ylm_table.cuh"

namespace pk {

constexpr int BIN_THREADS = 256;
constexpr int MAX_FP_TERMS = 32;
constexpr int MAX_ELLS = 9;

struct BinGeom {
  Dims d;
  float kfun[3];
  int nedges;
  float step;  // > 0: uniform edges
  int backend;
};

// jnp.digitize(k, edges, right=False): number of edges <= k.
__device__ __forceinline__ int digitize(const float *__restrict__ e, int nedges, float step,
                                        float k) {
  int g;
  if (step > 0.f) {
    float t = floorf((k - e[0]) / step) + 1.f;
    g = t < 0.f ? 0 : (t > (float)nedges ? nedges : (int)t);
    while (g > 0 && e[g - 1] > k) --g;
    while (g < nedges && e[g] <= k) ++g;
  } else {
    int lo = 0, hi = nedges;  // first index with e[idx] > k
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (e[mid] <= k) lo = mid + 1;
      else hi = mid;
    }
    g = lo;
  }
  return g;
}

// Hermitian weight of stored mode z: 'jax' 1 + (kz > 0); 'jaxdecomp' counts the
// mirrored half of a full complex grid (self-conjugate planes once).
__device__ __forceinline__ float mode_weight(const BinGeom &g, int z) {
  if (g.backend == PK_BACKEND_JAX) return z > 0 ? 2.f : 1.f;
  const bool selfconj = (z == 0) || ((g.d.n2 % 2) == 0 && z == g.d.nz - 1);
  return selfconj ? 1.f : 2.f;
}

__device__ __forceinline__ float kz_coord(const BinGeom &g, int z) {
  // jaxdecomp: full-grid fftfreq (the Nyquist index is -N/2); jax: rfftfreq
  return kcoord(z, g.d.n2, g.kfun[2], g.backend == PK_BACKEND_JAX);
}

// Legendre polynomials with the reference's float32 expression order (utils.py:341-360).
__device__ __forceinline__ float legendre(int ell, float x) {
  const float x2 = x * x;
  switch (ell) {
    case 0: return 1.f;
    case 1: return x;
    case 2: return 3.f * x2 / 2.f - 0.5f;
    case 3: return 5.f * (x2 * x) / 2.f - 3.f * x / 2.f;
    case 4: { const float x4 = x2 * x2; return 35.f * x4 / 8.f - 15.f * x2 / 4.f + 0.375f; }
    case 5: { const float x4 = x2 * x2; return 63.f * (x4 * x) / 8.f - 35.f * (x2 * x) / 4.f + 15.f * x / 8.f; }
    case 6: { const float x4 = x2 * x2; return 231.f * (x4 * x2) / 16.f - 315.f * x4 / 16.f + 105.f * x2 / 16.f - 0.3125f; }
    case 7: { const float x4 = x2 * x2; return 429.f * (x4 * x2 * x) / 16.f - 693.f * (x4 * x) / 16.f + 315.f * (x2 * x) / 16.f - 35.f * x / 16.f; }
    default: { const float x4 = x2 * x2; return 6435.f * (x4 * x4) / 128.f - 3003.f * (x4 * x2) / 32.f + 3465.f * x4 / 64.f - 315.f * x2 / 32.f + 0.2734375f; }
  }
}

// ------------------------------------------------------------- per-mode ops
struct ModesOp {  // nmodes and sum of w |k|
  static constexpr int NV = 2;
  __device__ void operator()(int64_t, int, int, int, float, float, float, float knorm, float w,
                             float v[NV]) const {
    v[0] = w;
    v[1] = __fmul_rn(knorm, w);
  }
};

struct MeshOp {  // plain per-bin sum of a complex mesh value (BinMesh2SpectrumPoles.__call__)
  const float2 *v;
  int remove_zero;
  static constexpr int NV = 2;
  __device__ void operator()(int64_t idx, int i, int j, int z, float, float, float, float,
                             float w, float out[NV]) const {
    const float2 a = v[idx];
    const bool zero = remove_zero && i == 0 && j == 0 && z == 0;
    out[0] = zero ? 0.f : __fmul_rn(a.x, w);
    out[1] = zero ? 0.f : __fmul_rn(a.y, w);
  }
};

struct GlobalOp {
  const float2 *d1;
  const float2 *d2;
  float los[3];
  int nells;
  int ells[MAX_ELLS];
  static constexpr int NV = MAX_ELLS;
  __device__ void operator()(int64_t idx, int i, int j, int z, float kx, float ky, float kz,
                             float knorm, float w, float v[NV]) const {
    const float2 a = d1[idx];
    float re, im;
    if (d2) {
      const float2 b = d2[idx];  // conj(a) * b
      re = __fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
      im = __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x));
    } else {
      re = __fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y));
      im = 0.f;
    }
    const bool zero = (i == 0 && j == 0 && z == 0);
    const float num = __fadd_rn(__fadd_rn(__fadd_rn(0.f, __fmul_rn(kx, los[0])), __fmul_rn(ky, los[1])),
                                __fmul_rn(kz, los[2]));
    const float mu = __fdiv_rn(num, zero ? 1.f : knorm);
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      if (l < nells) {
        const int ell = ells[l];
        const float part = (ell & 1) ? im : re;
        if (ell == 0) {
          v[l] = __fmul_rn(part, w);
        } else {
          v[l] = zero ? 0.f : __fmul_rn(__fmul_rn(part, legendre(ell, mu)), w);
        }
      } else {
        v[l] = 0.f;
      }
    }
  }
};

struct FirstPointOp {
  const float2 *a0;
  const float2 *b0;
  const float2 *f;
  int64_t fstride;
  int nterms;
  int term_ell[MAX_FP_TERMS];
  int term_m[MAX_FP_TERMS];
  int nells;
  int ells[MAX_ELLS];
  int include_ell0;
  static constexpr int NV = MAX_ELLS;
  __device__ void operator()(int64_t idx, int i, int j, int z, float kx, float ky, float kz,
                             float knorm, float w, float v[NV]) const {
    const float2 A = a0[idx];
    const bool zero = (i == 0 && j == 0 && z == 0);
    float xh = 0.f, yh = 0.f, zh = 0.f;
    if (knorm != 0.f) {
      xh = __fdiv_rn(kx, knorm);
      yh = __fdiv_rn(ky, knorm);
      zh = __fdiv_rn(kz, knorm);
    }
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      v[l] = 0.f;
      if (l >= nells) continue;
      const int ell = ells[l];
      if (ell == 0) {
        if (!include_ell0) continue;
        float re, im;
        if (b0) {
          const float2 B = b0[idx];
          re = __fadd_rn(__fmul_rn(B.x, A.x), __fmul_rn(B.y, A.y));
          im = __fsub_rn(__fmul_rn(B.x, A.y), __fmul_rn(B.y, A.x));
        } else {
          re = __fadd_rn(__fmul_rn(A.x, A.x), __fmul_rn(A.y, A.y));
          im = 0.f;
        }
        (void)im;
        v[l] = __fmul_rn(re, w);
        continue;
      }
      float sr = 0.f, si = 0.f;
      bool any = false;
      for (int t = 0; t < nterms; ++t) {
        if (term_ell[t] != ell) continue;
        const float2 F = f[(int64_t)t * fstride + idx];
        const float y = ylm_eval(ell, term_m[t], xh, yh, zh);
        sr = __fadd_rn(sr, __fmul_rn(F.x, y));
        si = __fadd_rn(si, __fmul_rn(F.y, y));
        any = true;
      }
      if (!any || zero) continue;
      // conj(S) * A0
      const float re = __fadd_rn(__fmul_rn(sr, A.x), __fmul_rn(si, A.y));
      const float im = __fsub_rn(__fmul_rn(sr, A.y), __fmul_rn(si, A.x));
      v[l] = __fmul_rn((ell & 1) ? im : re, w);
    }
  }
};

// ------------------------------------------------------------ the reduction
template <class Op>
__global__ void __launch_bounds__(BIN_THREADS) bin_kernel(BinGeom g, Op op,
                                                          const float *__restrict__ edges,
                                                          int nv, int nwarps_hist,
                                                          double *__restrict__ partials) {
  constexpr int NV = Op::NV;
  extern __shared__ double smem[];
  const int nbins = g.nedges - 1;
  const int hist_len = nbins * nv;
  double *hist = smem;                                            // [warps][nbins][nv]
  float *sedges = reinterpret_cast<float *>(smem + (size_t)nwarps_hist * hist_len);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  for (int i = threadIdx.x; i < nwarps * hist_len; i += blockDim.x) hist[i] = 0.;
  for (int i = threadIdx.x; i < g.nedges; i += blockDim.x) sedges[i] = edges[i];
  __syncthreads();

  double *my = hist + (size_t)warp * hist_len;
  const int64_t nrows = (int64_t)g.d.n0 * g.d.n1;
  for (int64_t row = (int64_t)blockIdx.x * nwarps + warp; row < nrows;
       row += (int64_t)gridDim.x * nwarps) {
    const int i = (int)(row / g.d.n1), j = (int)(row % g.d.n1);
    const float kx = kcoord(i, g.d.n0, g.kfun[0], false);
    const float ky = kcoord(j, g.d.n1, g.kfun[1], false);
    const float kxy = __fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky));  // (0 + kx^2) + ky^2
    for (int z0 = 0; z0 < g.d.nz; z0 += 32) {
      const int z = z0 + lane;
      const bool valid = z < g.d.nz;
      float v[NV];
      int key = 0x7fffffff;
      if (valid) {
        const float kz = kz_coord(g, z);
        const float knorm = __fsqrt_rn(__fadd_rn(kxy, __fmul_rn(kz, kz)));
        key = digitize(sedges, g.nedges, g.step, knorm);
        op(row * g.d.nz + z, i, j, z, kx, ky, kz, knorm, mode_weight(g, z), v);
      } else {
#pragma unroll
        for (int c = 0; c < NV; ++c) v[c] = 0.f;
      }
      // segmented inclusive scan over contiguous equal keys
      const int prev = __shfl_up_sync(0xffffffffu, key, 1);
      const bool distinct = __all_sync(0xffffffffu, lane == 0 || prev != key);
      if (!distinct) {
#pragma unroll
        for (int dlt = 1; dlt < 32; dlt <<= 1) {
          const int ok = __shfl_up_sync(0xffffffffu, key, dlt) == key && lane >= dlt;
#pragma unroll
          for (int c = 0; c < NV; ++c) {
            if (c < nv) {
              const float t = __shfl_up_sync(0xffffffffu, v[c], dlt);
              if (ok) v[c] += t;
            }
          }
        }
      }
      const int next = __shfl_down_sync(0xffffffffu, key, 1);
      const bool tail = (lane == 31) || next != key;
      if (valid && tail && key >= 1 && key <= nbins) {
        double *h = my + (size_t)(key - 1) * nv;
#pragma unroll
        for (int c = 0; c < NV; ++c)
          if (c < nv) h[c] += (double)v[c];
      }
      __syncwarp();
    }
  }
  __syncthreads();
  double *out = partials + (size_t)blockIdx.x * hist_len;
  for (int e = threadIdx.x; e < hist_len; e += blockDim.x) {
    double s = 0.;
    for (int w = 0; w < nwarps; ++w) s += hist[(size_t)w * hist_len + e];
    out[e] = s;
  }
}

// out[e] (+)= sum over CTAs, in CTA order.
__global__ void bin_finalize_kernel(const double *__restrict__ partials, int nblocks,
                                    int hist_len, int nv, int nbins, int nout_values,
                                    int accumulate, double *__restrict__ out0,
                                    double *__restrict__ out1) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < hist_len;
       e += gridDim.x * blockDim.x) {
    double s = 0.;
    for (int b = 0; b < nblocks; ++b) s += partials[(size_t)b * hist_len + e];
    const int bin = e / nv, c = e % nv;
    if (c >= nout_values) continue;
    // transpose to [value][bin]
    double *dst = (c == 1 && out1) ? out1 : out0;
    const int64_t o = (c == 1 && out1) ? bin : (int64_t)c * nbins + bin;
    dst[o] = accumulate ? dst[o] + s : s;
  }
}

struct BinLaunch {
  int blocks;
  int nwarps;
  size_t smem;
  size_t partial_bytes;
};

static bool plan_bins(const Dims &d, int nedges, int nv, BinLaunch *L) {
  const int nbins = nedges - 1;
  const size_t per_warp = (size_t)nbins * nv * sizeof(double);
  const size_t edge_bytes = align_up((size_t)nedges * sizeof(float), 16);
  const size_t budget = 200 * 1024;
  int nwarps = BIN_THREADS / 32;
  if (per_warp + edge_bytes > budget) return false;
  while (nwarps > 1 && (size_t)nwarps * per_warp + edge_bytes > budget) nwarps >>= 1;
  L->nwarps = nwarps;
  L->smem = (size_t)nwarps * per_warp + edge_bytes;
  const int64_t nrows = (int64_t)d.n0 * d.n1;
  const int per_sm = L->smem > 110 * 1024 ? 1 : (L->smem > 72 * 1024 ? 2 : 4);
  int64_t blocks = (int64_t)per_sm * sm_count();
  const int64_t need = (nrows + nwarps - 1) / nwarps;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  L->blocks = (int)blocks;
  L->partial_bytes = (size_t)blocks * nbins * nv * sizeof(double);
  return true;
}

template <class Op>
static pk_status launch_bins(cudaStream_t s, const BinGeom &g, const Op &op, const float *edges,
                             int nv, int nout_values, int accumulate, double *out0, double *out1,
                             void *workspace, size_t workspace_bytes) {
  BinLaunch L;
  PK_REQUIRE(plan_bins(g.d, g.nedges, nv, &L), PK_ERR_RANGE,
             "too many bins x values (%d x %d) for the shared-memory histograms", g.nedges - 1, nv);
  PK_REQUIRE(workspace && workspace_bytes >= L.partial_bytes, PK_ERR_WORKSPACE,
             "binning workspace too small: need %zu bytes, got %zu", L.partial_bytes,
             workspace_bytes);
  double *partials = static_cast<double *>(workspace);
  PK_CUDA(cudaFuncSetAttribute(bin_kernel<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)L.smem));
  bin_kernel<Op><<<L.blocks, L.nwarps * 32, L.smem, s>>>(g, op, edges, nv, L.nwarps, partials);
  PK_LAUNCH_CHECK();
  const int hist_len = (g.nedges - 1) * nv;
  const int fb = (hist_len + 255) / 256;
  bin_finalize_kernel<<<fb, 256, 0, s>>>(partials, L.blocks, hist_len, nv, g.nedges - 1,
                                         nout_values, accumulate, out0, out1);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

static pk_status make_geom(const int32_t meshsize[3], const float kfun[3], int nedges, float step,
                           int backend, BinGeom *g) {
  PK_REQUIRE(make_dims(meshsize, &g->d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(kfun, PK_ERR_INVALID, "kfun is NULL");
  PK_REQUIRE(nedges >= 2, PK_ERR_INVALID, "need at least 2 edges");
  PK_REQUIRE(backend == PK_BACKEND_JAX || backend == PK_BACKEND_JAXDECOMP, PK_ERR_INVALID,
             "unknown backend %d", backend);
  for (int a = 0; a < 3; ++a) g->kfun[a] = kfun[a];
  g->nedges = nedges;
  g->step = step;
  g->backend = backend;
  return PK_OK;
}

}  // namespace pk

using namespace pk;

extern "C" pk_status pk_bin_workspace_size(const int32_t meshsize[3], int nedges, int nvalues,
                                           size_t *bytes) {
  PK_REQUIRE(bytes, PK_ERR_INVALID, "bytes is NULL");
  Dims d;
  PK_REQUIRE(make_dims(meshsize, &d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(nedges >= 2 && nvalues >= 1 && nvalues <= MAX_ELLS, PK_ERR_INVALID,
             "invalid nedges / nvalues");
  size_t most = 0;
  for (int nv = 1; nv <= MAX_ELLS; ++nv) {  // launches pick their grid from nv
    BinLaunch L;
    if (!plan_bins(d, nedges, nv, &L)) {
      PK_REQUIRE(nv > nvalues, PK_ERR_RANGE, "too many bins x values for the histograms");
      break;
    }
    if (L.partial_bytes > most) most = L.partial_bytes;
  }
  *bytes = most;
  return PK_OK;
}

extern "C" pk_status pk_bin_modes(void *stream, const int32_t meshsize[3], const float kfun[3],
                                  const float *d_edges, int nedges, float step, int backend,
                                  double *d_nmodes, double *d_ksum, void *workspace,
                                  size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(d_edges && d_nmodes && d_ksum, PK_ERR_INVALID, "null pointer");
  return launch_bins((cudaStream_t)stream, g, ModesOp(), d_edges, 2, 2, 0, d_nmodes, d_ksum,
                     workspace, workspace_bytes);
}

extern "C" pk_status pk_bin_mesh(void *stream, const void *value, const int32_t meshsize[3],
                                 const float kfun[3], const float *d_edges, int nedges, float step,
                                 int backend, int remove_zero, double *d_out, void *workspace,
                                 size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(value && d_edges && d_out, PK_ERR_INVALID, "null pointer");
  MeshOp op;
  op.v = (const float2 *)value;
  op.remove_zero = remove_zero;
  return launch_bins((cudaStream_t)stream, g, op, d_edges, 2, 2, 0, d_out, nullptr, workspace,
                     workspace_bytes);
}

extern "C" pk_status pk_bin_global(void *stream, const void *delta1, const void *delta2,
                                   const int32_t meshsize[3], const float kfun[3],
                                   const float los[3], const float *d_edges, int nedges,
                                   float step, int backend, int nells, const int32_t *ells,
                                   double *d_out, void *workspace, size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(delta1 && d_edges && d_out && los && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nells >= 1 && nells <= MAX_ELLS, PK_ERR_INVALID, "nells must be in 1..%d", MAX_ELLS);
  GlobalOp op;
  op.d1 = (const float2 *)delta1;
  op.d2 = (const float2 *)delta2;
  for (int a = 0; a < 3; ++a) op.los[a] = los[a];
  op.nells = nells;
  for (int l = 0; l < MAX_ELLS; ++l) {
    op.ells[l] = l < nells ? ells[l] : 0;
    PK_REQUIRE(l >= nells || (ells[l] >= 0 && ells[l] <= 8), PK_ERR_INVALID,
               "ell must be in 0..8");
  }
  return launch_bins((cudaStream_t)stream, g, op, d_edges, nells, nells, 0, d_out, nullptr,
                     workspace, workspace_bytes);
}

extern "C" pk_status pk_bin_firstpoint(void *stream, const void *a0, const void *b0,
                                       const void *f, int nterms, const int32_t *term_ell,
                                       const int32_t *term_m, const int32_t meshsize[3],
                                       const float kfun[3], const float *d_edges, int nedges,
                                       float step, int backend, int nells, const int32_t *ells,
                                       int include_ell0, int accumulate, double *d_out,
                                       void *workspace, size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(a0 && d_edges && d_out && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nterms >= 0 && nterms <= MAX_FP_TERMS, PK_ERR_INVALID, "nterms must be in 0..%d",
             MAX_FP_TERMS);
  PK_REQUIRE(nterms == 0 || (f && term_ell && term_m), PK_ERR_INVALID, "null term arrays");
  PK_REQUIRE(nells >= 1 && nells <= MAX_ELLS, PK_ERR_INVALID, "nells must be in 1..%d", MAX_ELLS);
  FirstPointOp op;
  op.a0 = (const float2 *)a0;
  op.b0 = (const float2 *)b0;
  op.f = (const float2 *)f;
  op.fstride = g.d.ncomplex();
  op.nterms = nterms;
  for (int t = 0; t < MAX_FP_TERMS; ++t) {
    op.term_ell[t] = t < nterms ? term_ell[t] : -1;
    op.term_m[t] = t < nterms ? term_m[t] : 0;
    PK_REQUIRE(t >= nterms || (term_ell[t] >= 0 && term_ell[t] <= YLM_LMAX &&
                               term_m[t] >= -term_ell[t] && term_m[t] <= term_ell[t]),
               PK_ERR_INVALID, "invalid (ell, m)");
  }
  op.nells = nells;
  for (int l = 0; l < MAX_ELLS; ++l) op.ells[l] = l < nells ? ells[l] : 0;
  op.include_ell0 = include_ell0;
  return launch_bins((cudaStream_t)stream, g, op, d_edges, nells, nells, accumulate, d_out,
                     nullptr, workspace, workspace_bytes);
}
