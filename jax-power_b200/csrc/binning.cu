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

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "fourier_common.cuh"
#include "ylm_block.cuh"

namespace pk {

constexpr int BIN_THREADS = 256;
constexpr int MAX_FP_TERMS = 32;
constexpr int MAX_ELLS = 9;

struct BinGeom {
  Dims d;          // separation grid: d.nz = n2 (the full real mesh)
  float kfun[3];   // separation grid: the cell size
  int nedges;
  float step;  // > 0: uniform edges
  int backend;
  int sep;     // 1: real-space separation grid (fftfreq * cellsize * n, unit weights)
  // mode oversampling (mesh2.py:48-61): the bin of a mode is that of |k + kshift|, the
  // shift added to each coordinate in float32 as the reference adds it; its value (mu,
  // khat) still comes from k.  Only the chunk walk (bin_chunks_kernel) takes a shift.
  int shifted;
  float kshift[3];
};

// |k + kshift|^2 = ((0 + (kx + sx)^2) + (ky + sy)^2) + (kz + sz)^2 in float32 (mesh2.py:50).
__device__ __forceinline__ float shifted_k2(const BinGeom &g, float kx, float ky, float kz) {
  const float a = __fadd_rn(kx, g.kshift[0]), b = __fadd_rn(ky, g.kshift[1]), c = __fadd_rn(kz, g.kshift[2]);
  return __fadd_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)), __fmul_rn(c, c));
}

// Hermitian weight of stored mode z: 'jax' 1 + (kz > 0); 'jaxdecomp' counts the
// mirrored half of a full complex grid (self-conjugate planes once).
__device__ __forceinline__ float mode_weight(const BinGeom &g, int z) {
  if (g.sep) return 1.f;
  if (g.backend == PK_BACKEND_JAX) return z > 0 ? 2.f : 1.f;
  const bool selfconj = (z == 0) || ((g.d.n2 % 2) == 0 && z == g.d.nz - 1);
  return selfconj ? 1.f : 2.f;
}

__device__ __forceinline__ float kz_coord(const BinGeom &g, int z) {
  // jaxdecomp: full-grid fftfreq (the Nyquist index is -N/2); jax: rfftfreq
  return kcoord(z, g.d.n2, g.kfun[2], !g.sep && g.backend == PK_BACKEND_JAX);
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

// Exact digitize on |k|^2: t_b = smallest float x with sqrt_rn(x) >= edges[b], so that
// #{b : k2 >= t_b} == #{b : edges[b] <= sqrt_rn(k2)} (sqrt_rn is monotone); this is
// jnp.digitize(sqrt(k2), edges, right=False) bit for bit, without a per-mode sqrt.
__device__ float sqrt_threshold(float e) {
  if (!(e > 0.f)) return -1.f;  // every k2 >= 0 passes
  if (isinf(e)) return e;
  float x = __fmul_rn(e, e);
  while (__fsqrt_rn(x) < e) x = nextafterf(x, INFINITY);
  for (;;) {
    const float p = nextafterf(x, 0.f);
    if (p >= 0.f && p < x && __fsqrt_rn(p) >= e) x = p;
    else break;
  }
  return x;
}

// Bin index from k2 without prior state: guess from an approximate |k| then correct.
__device__ __forceinline__ int bin_from_k2(const float *__restrict__ thr, int nedges, float e0,
                                           float inv_step, float k2) {
  int g;
  if (inv_step > 0.f) {
    const float k = k2 > 0.f ? k2 * rsqrtf(k2) : 0.f;
    const float t = floorf((k - e0) * inv_step) + 1.f;
    g = t < 0.f ? 0 : (t > (float)nedges ? nedges : (int)t);
    while (g > 0 && k2 < thr[g - 1]) --g;
    while (g < nedges && k2 >= thr[g]) ++g;
  } else {
    int lo = 0, hi = nedges;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (k2 >= thr[mid]) lo = mid + 1;
      else hi = mid;
    }
    g = lo;
  }
  return g;
}

// ------------------------------------------------------------- per-mode ops
// op(idx, i, j, z, kx, ky, kz, k2, w, v): values of stored mode (i, j, z), weight w.
struct ModesOp {  // nmodes and sum of w |k| (|k| = sqrt_rn(k2), as the reference's float32 knorm)
  static constexpr int NV = 2;
  int shifted = 0;  // mode oversampling: |k + kshift| instead
  float kshift[3] = {0.f, 0.f, 0.f};
  __device__ void operator()(int64_t, int, int, int, float kx, float ky, float kz, float k2, float w,
                             float v[NV]) const {
    if (shifted) {
      const float a = __fadd_rn(kx, kshift[0]), b = __fadd_rn(ky, kshift[1]), c = __fadd_rn(kz, kshift[2]);
      k2 = __fadd_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)), __fmul_rn(c, c));
    }
    v[0] = w;
    v[1] = __fmul_rn(__fsqrt_rn(k2), w);
  }
};

struct MeshOp {  // plain per-bin sum of a complex mesh value (BinMesh2SpectrumPoles.__call__)
  const float2 *v;
  int remove_zero;
  static constexpr int NV = 2;
  __device__ void operator()(int64_t idx, int i, int j, int z, float, float, float, float, float w,
                             float out[NV]) const {
    const float2 a = v[idx];
    const bool zero = remove_zero && i == 0 && j == 0 && z == 0;
    out[0] = zero ? 0.f : __fmul_rn(a.x, w);
    out[1] = zero ? 0.f : __fmul_rn(a.y, w);
  }
};

// w * value * L_ell(mu) of a real mesh on the separation grid, mu = s.los / |s| (|s|(0) = 1);
// the s = 0 cell is dropped for ell > 0 (compute_mesh2_correlation, mesh2.py:479-489).
template <int N>
struct SepLegendreOp {
  const float *v;
  float los[3];
  int ells[MAX_ELLS];
  static constexpr int NV = N;
  __device__ void operator()(int64_t idx, int i, int j, int z, float sx, float sy, float sz, float s2,
                             float w, float out[NV]) const {
    const float a = v[idx] * w;
    const bool zero = (i == 0 && j == 0 && z == 0);
    const float num = (sx * los[0] + sy * los[1]) + sz * los[2];
    const float mu = s2 > 0.f ? __fdiv_rn(num, __fsqrt_rn(s2)) : 0.f;
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      const int ell = ells[l];
      out[l] = ell == 0 ? a : (zero ? 0.f : a * legendre(ell, mu));
    }
  }
};

template <int N>
struct GlobalOp {  // w * Re/Im(A) * L_ell(mu), A = |d1|^2 or conj(d1) d2 (mesh2.py:346-374)
  const float2 *d1;
  const float2 *d2;
  float los[3];
  int ells[MAX_ELLS];
  static constexpr int NV = N;
  __device__ void operator()(int64_t idx, int i, int j, int z, float kx, float ky, float kz,
                             float k2, float w, float v[NV]) const {
    const float2 a = d1[idx];
    float re, im;
    if (d2) {
      const float2 b = d2[idx];
      re = a.x * b.x + a.y * b.y;
      im = a.x * b.y - a.y * b.x;
    } else {
      re = a.x * a.x + a.y * a.y;
      im = 0.f;
    }
    const bool zero = (i == 0 && j == 0 && z == 0);
    const float num = (kx * los[0] + ky * los[1]) + kz * los[2];
    const float mu = k2 > 0.f ? num * rsqrtf(k2) : 0.f;  // |k|(0) = 1 in the reference: mu(0) = 0
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      const int ell = ells[l];
      const float part = (ell & 1) ? im : re;
      v[l] = ell == 0 ? part * w : (zero ? 0.f : part * legendre(ell, mu) * w);
    }
  }
};

template <int N>
struct FirstPointOp {  // w * Re/Im(conj(sum_m F_m Y_lm(khat)) A0) (mesh2.py:293-344)
  const float2 *a0;
  const float2 *b0;
  const float2 *f;
  int64_t fstride;
  int nterms;
  int term_ell[MAX_FP_TERMS];
  int term_m[MAX_FP_TERMS];
  int ells[MAX_ELLS];
  int include_ell0;
  static constexpr int NV = N;
  __device__ void operator()(int64_t idx, int i, int j, int z, float kx, float ky, float kz,
                             float k2, float w, float v[NV]) const {
    const float2 A = a0[idx];
    const bool zero = (i == 0 && j == 0 && z == 0);
    const float rn = k2 > 0.f ? rsqrtf(k2) : 0.f;  // khat = k / |k|, 0 at k = 0
    const float xh = kx * rn, yh = ky * rn, zh = kz * rn;
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      v[l] = 0.f;
      const int ell = ells[l];
      if (ell == 0) {
        if (!include_ell0) continue;
        if (b0) {
          const float2 B = b0[idx];
          v[l] = (B.x * A.x + B.y * A.y) * w;
        } else {
          v[l] = (A.x * A.x + A.y * A.y) * w;
        }
        continue;
      }
      float sr = 0.f, si = 0.f;
      for (int t = 0; t < nterms; ++t) {
        if (term_ell[t] != ell) continue;
        const float2 F = f[(int64_t)t * fstride + idx];
        const float y = ylm_eval(ell, term_m[t], xh, yh, zh);
        sr += F.x * y;
        si += F.y * y;
      }
      if (zero) continue;
      const float re = sr * A.x + si * A.y;  // conj(S) * A0
      const float im = sr * A.y - si * A.x;
      v[l] = ((ell & 1) ? im : re) * w;
    }
  }
};

// Shared-memory layout of one binning CTA.
struct BinSmem {
  double *hist;  // [nwarps][nbins][NV]
  float *thr;    // [nedges]
  float *kz;     // [nz] (when tabulated)
  float *kz2;    // [nz]
};

__device__ __forceinline__ BinSmem bin_smem_init(const BinGeom &g, const float *edges, int nv,
                                                 int nwarps, bool tab) {
  extern __shared__ double smem[];
  BinSmem s;
  const int nbins = g.nedges - 1;
  s.hist = smem;
  s.thr = reinterpret_cast<float *>(smem + (size_t)nwarps * nbins * nv);
  s.kz = s.thr + ((g.nedges + 3) & ~3);
  s.kz2 = s.kz + ((g.d.nz + 3) & ~3);
  for (int i = threadIdx.x; i < nwarps * nbins * nv; i += blockDim.x) s.hist[i] = 0.;
  for (int i = threadIdx.x; i < g.nedges; i += blockDim.x) s.thr[i] = sqrt_threshold(edges[i]);
  if (tab)
    for (int z = threadIdx.x; z < g.d.nz; z += blockDim.x) {
      const float kz = kz_coord(g, z);
      s.kz[z] = kz;
      s.kz2[z] = __fmul_rn(kz, kz);
    }
  __syncthreads();
  return s;
}

__device__ __forceinline__ void bin_smem_flush(const BinSmem &s, int hist_len, int nwarps,
                                               double *__restrict__ partials) {
  __syncthreads();
  double *out = partials + (size_t)blockIdx.x * hist_len;
  for (int e = threadIdx.x; e < hist_len; e += blockDim.x) {
    double acc = 0.;
    for (int w = 0; w < nwarps; ++w) acc += s.hist[(size_t)w * hist_len + e];
    out[e] = acc;
  }
}

// --------------------------------------------------------- row-run reduction
// One warp per (i, j) row; lane l walks the contiguous run z in [l R, (l+1) R).  |k| is
// non-decreasing along the run, so the bin only moves forward: interior segments of a run
// belong to that lane alone and go straight to the warp's float64 histogram; the first
// and last segments of every run are merged across lanes by one segmented scan per row.
// SEP (real-space separation grid): |s| grows along z over z in [0, P), P = (n2 + 1) / 2, and
// along decreasing z over [P, n2); each row is walked as these two monotone half-rows.
template <int NV, class Op, bool SEP = false>
__global__ void __launch_bounds__(BIN_THREADS) bin_rows_kernel(BinGeom g, Op op,
                                                               const float *__restrict__ edges,
                                                               int nwarps_hist, int tab,
                                                               double *__restrict__ partials) {
  const int nbins = g.nedges - 1;
  const int hist_len = nbins * NV;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  const BinSmem s = bin_smem_init(g, edges, NV, nwarps_hist, tab);
  double *my = s.hist + (size_t)warp * hist_len;
  const float e0 = edges[0];
  const float inv_step = g.step > 0.f ? 1.f / g.step : 0.f;
  constexpr int NONE = 0x7fffffff;
  const int npos = SEP ? (g.d.n2 + 1) / 2 : g.d.nz;  // length of the first half-row
  for (RowWalker rw((int64_t)blockIdx.x * nwarps + warp, (int64_t)gridDim.x * nwarps, g.d.n1 * (SEP ? 2 : 1));
       rw.i < g.d.n0; rw.next()) {
    const int i = rw.i, j = SEP ? (rw.j >> 1) : rw.j;
    const int half = SEP ? (rw.j & 1) : 0;
    const int len = half ? g.d.n2 - npos : npos;
    const int R = (len + 31) / 32;
    const int z0 = lane * R, z1 = min(len, z0 + R);
    const int64_t row = (int64_t)i * g.d.n1 + j;
    const float kx = kcoord(i, g.d.n0, g.kfun[0], false);
    const float ky = kcoord(j, g.d.n1, g.kfun[1], false);
    const float kxy = __fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky));  // (0 + kx^2) + ky^2
    int cur = -1, lead = NONE, trail = NONE, nseg = 0;
    float acc[NV], facc[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c) acc[c] = facc[c] = 0.f;
    for (int t = z0; t < z1; ++t) {
      const int z = half ? g.d.n2 - 1 - t : t;
      float kz, kz2;
      if (tab) {
        kz = s.kz[z];
        kz2 = s.kz2[z];
      } else {
        kz = kz_coord(g, z);
        kz2 = __fmul_rn(kz, kz);
      }
      const float k2 = __fadd_rn(kxy, kz2);
      int gb = cur;
      if (cur < 0) gb = bin_from_k2(s.thr, g.nedges, e0, inv_step, k2);
      else
        while (gb < g.nedges && k2 >= s.thr[gb]) ++gb;
      if (gb != cur) {
        if (cur >= 0) {  // close the current segment
          if (nseg == 0) {
            lead = cur;
#pragma unroll
            for (int c = 0; c < NV; ++c) facc[c] = acc[c];
          } else if (cur >= 1 && cur <= nbins) {  // interior: exclusive to this lane
#pragma unroll
            for (int c = 0; c < NV; ++c) my[(size_t)(cur - 1) * NV + c] += (double)acc[c];
          }
          ++nseg;
        }
        cur = gb;
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = 0.f;
      }
      float v[NV];
      op(row * g.d.nz + z, i, j, z, kx, ky, kz, k2, mode_weight(g, z), v);
#pragma unroll
      for (int c = 0; c < NV; ++c) acc[c] += v[c];
    }
    // leading (L, facc) and trailing (T, tacc) entries of this lane's run
    float tacc[NV];
    if (cur < 0) {  // empty run
      lead = trail = NONE;
    } else if (nseg == 0) {  // a single segment
      lead = trail = cur;
#pragma unroll
      for (int c = 0; c < NV; ++c) facc[c] = tacc[c] = acc[c];
    } else {
      trail = cur;
#pragma unroll
      for (int c = 0; c < NV; ++c) tacc[c] = acc[c];
    }
    if (cur >= 0 && nseg == 0) {
#pragma unroll
      for (int c = 0; c < NV; ++c) facc[c] = 0.f;  // counted once, in the trailing entry
    }
    // inclusive segmented scan of trailing entries over lanes (keys are monotone)
    float S[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c) S[c] = tacc[c];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int k = __shfl_up_sync(0xffffffffu, trail, d);
      const bool ok = lane >= d && k == trail;
#pragma unroll
      for (int c = 0; c < NV; ++c) {
        const float t = __shfl_up_sync(0xffffffffu, S[c], d);
        if (ok) S[c] += t;
      }
    }
    const int prev_trail = __shfl_up_sync(0xffffffffu, trail, 1);
    float carry[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c) {
      const float t = __shfl_up_sync(0xffffffffu, S[c], 1);
      carry[c] = (lane > 0 && prev_trail == lead) ? t : 0.f;
    }
    const int next_lead = __shfl_down_sync(0xffffffffu, lead, 1);
    const int next_trail = __shfl_down_sync(0xffffffffu, trail, 1);
    // a multi-segment lane writes its leading bin with the carry of the lanes before it
    if (cur >= 0 && nseg > 0 && lead >= 1 && lead <= nbins) {
#pragma unroll
      for (int c = 0; c < NV; ++c) my[(size_t)(lead - 1) * NV + c] += (double)(facc[c] + carry[c]);
    }
    // the trailing total is written by the last lane of its key, unless the next lane
    // starts a multi-segment run with that key (then that lane writes it)
    const bool next_takes = lane < 31 && next_lead == trail;
    const bool next_continues = lane < 31 && next_trail == trail;
    if (cur >= 0 && !next_takes && !next_continues && trail >= 1 && trail <= nbins) {
#pragma unroll
      for (int c = 0; c < NV; ++c) my[(size_t)(trail - 1) * NV + c] += (double)S[c];
    }
    __syncwarp();
  }
  bin_smem_flush(s, hist_len, nwarps, partials);
}

// ------------------------------------------------------- chunk reduction
// One warp per row, lanes on consecutive kz (coalesced loads of many meshes); one
// segmented scan per 32 modes.  Used by the first-point estimator (14+ meshes per mode).
template <int NV, class Op>
__global__ void __launch_bounds__(BIN_THREADS) bin_chunks_kernel(BinGeom g, Op op,
                                                                 const float *__restrict__ edges,
                                                                 int nwarps_hist, int tab,
                                                                 double *__restrict__ partials) {
  const int nbins = g.nedges - 1;
  const int hist_len = nbins * NV;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  const BinSmem s = bin_smem_init(g, edges, NV, nwarps_hist, tab);
  double *my = s.hist + (size_t)warp * hist_len;
  const float e0 = edges[0];
  const float inv_step = g.step > 0.f ? 1.f / g.step : 0.f;
  for (RowWalker rw((int64_t)blockIdx.x * nwarps + warp, (int64_t)gridDim.x * nwarps, g.d.n1); rw.i < g.d.n0;
       rw.next()) {
    const int i = rw.i, j = rw.j;
    const int64_t row = (int64_t)i * g.d.n1 + j;
    const float kx = kcoord(i, g.d.n0, g.kfun[0], false);
    const float ky = kcoord(j, g.d.n1, g.kfun[1], false);
    const float kxy = __fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky));
    for (int zc = 0; zc < g.d.nz; zc += 32) {
      const int z = zc + lane;
      const bool valid = z < g.d.nz;
      float v[NV];
      int key = 0x7fffffff;
      if (valid) {
        float kz, kz2;
        if (tab) {
          kz = s.kz[z];
          kz2 = s.kz2[z];
        } else {
          kz = kz_coord(g, z);
          kz2 = __fmul_rn(kz, kz);
        }
        const float k2 = __fadd_rn(kxy, kz2);
        key = bin_from_k2(s.thr, g.nedges, e0, inv_step, g.shifted ? shifted_k2(g, kx, ky, kz) : k2);
        op(row * g.d.nz + z, i, j, z, kx, ky, kz, k2, mode_weight(g, z), v);
      } else {
#pragma unroll
        for (int c = 0; c < NV; ++c) v[c] = 0.f;
      }
      const int prev = __shfl_up_sync(0xffffffffu, key, 1);
      const bool head = lane == 0 || prev != key;
      if (!__all_sync(0xffffffffu, head)) {
        // segmented inclusive scan over runs of equal keys: a lane adds only lanes of its own
        // run (for monotone keys this is the same as comparing keys; with a k shift equal keys
        // may recur after another run)
        const unsigned heads = __ballot_sync(0xffffffffu, head);
        const int first = 31 - __clz(heads & (lane == 31 ? 0xffffffffu : ((2u << lane) - 1u)));
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const bool ok = lane - d >= first;
#pragma unroll
          for (int c = 0; c < NV; ++c) {
            const float t = __shfl_up_sync(0xffffffffu, v[c], d);
            if (ok) v[c] += t;
          }
        }
      }
      const int next = __shfl_down_sync(0xffffffffu, key, 1);
      const bool tail = valid && (lane == 31 || next != key) && key >= 1 && key <= nbins;
      if (!g.shifted) {  // keys are non-decreasing along a row: the run tails have distinct bins
        if (tail) {
#pragma unroll
          for (int c = 0; c < NV; ++c) my[(size_t)(key - 1) * NV + c] += (double)v[c];
        }
      } else {  // |k + shift| is not monotone: two runs may share a bin, add them one at a time
        for (unsigned tails = __ballot_sync(0xffffffffu, tail); tails; tails &= tails - 1) {
          if (lane == __ffs(tails) - 1) {
#pragma unroll
            for (int c = 0; c < NV; ++c) my[(size_t)(key - 1) * NV + c] += (double)v[c];
          }
          __syncwarp();
        }
      }
      __syncwarp();
    }
  }
  bin_smem_flush(s, hist_len, nwarps, partials);
}

// ------------------------------------------- first point, whole-ell term blocks
// The first-point pass (mesh2.py:293-344) when the terms are whole ells (mask MASK, every
// m of each ell in order): the F_lm of a mode are loaded together, Y_lm(khat) are
// compile-time polynomials at fixed register indices, and the modes are walked as one
// flat sequence of 32-mode chunks (a warp owns a contiguous range of chunks; a chunk may
// span rows, so bin keys carry the row's low 5 bits and equal bins of different rows stay
// separate runs -- a chunk spans at most 32 rows -- and the run tails of different rows,
// which may share a bin, add into the histogram one row after the other).  Values: 0 = the
// ell = 0 product, then one per ell of MASK, ascending.  Per mode the arithmetic is
// FirstPointOp's, term for term.

// sr + i si = sum_m F_{ELL m} Y_{ELL m}, terms T .. T + 2 ELL, in m order.
template <int ELL, int M, int T, int NT>
__device__ __forceinline__ void fp_ylm_sum(const float2 (&F)[NT], float x, float y, float z, float &sr,
                                           float &si) {
  const float yv = ylm_eval(ELL, M, x, y, z);
  sr += F[T].x * yv;
  si += F[T].y * yv;
  if constexpr (M < ELL) fp_ylm_sum<ELL, M + 1, T + 1>(F, x, y, z, sr, si);
}

template <int MASK, int ELL, int T, int V, int NT, int NV>
__device__ __forceinline__ void fp_block_values(const float2 (&F)[NT], float x, float y, float z, float2 A,
                                                bool zero, float w, float (&v)[NV]) {
  if constexpr (ELL <= YLM_LMAX) {
    if constexpr ((MASK >> ELL) & 1) {
      float sr = 0.f, si = 0.f;
      fp_ylm_sum<ELL, -ELL, T>(F, x, y, z, sr, si);
      const float re = sr * A.x + si * A.y;  // conj(S) * A0
      const float im = sr * A.y - si * A.x;
      v[V] = zero ? 0.f : ((ELL & 1) ? im : re) * w;
      fp_block_values<MASK, ELL + 1, T + 2 * ELL + 1, V + 1>(F, x, y, z, A, zero, w, v);
    } else {
      fp_block_values<MASK, ELL + 1, T, V>(F, x, y, z, A, zero, w, v);
    }
  }
}

template <int MASK, bool CROSS>
__global__ void __launch_bounds__(BIN_THREADS) bin_firstpoint_kernel(
    BinGeom g, const float2 *__restrict__ a0, const float2 *__restrict__ b0, const float2 *__restrict__ f,
    int64_t fstride, const float *__restrict__ edges, int nwarps_hist, int tab, int64_t chunks_per_warp,
    double *__restrict__ partials) {
  constexpr int NT = ylm_mask_terms(MASK);
  constexpr int NV = ylm_mask_ells(MASK) + 1;
  const int nbins = g.nedges - 1;
  const int hist_len = nbins * NV;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  const BinSmem s = bin_smem_init(g, edges, NV, nwarps_hist, tab);
  double *my = s.hist + (size_t)warp * hist_len;
  const float e0 = edges[0];
  const float inv_step = g.step > 0.f ? 1.f / g.step : 0.f;
  const int nz = g.d.nz, n1 = g.d.n1;
  const int64_t total = g.d.ncomplex();
  const int64_t nchunks = (total + 31) / 32;
  const int64_t c0 = ((int64_t)blockIdx.x * nwarps + warp) * chunks_per_warp;
  const int64_t c1 = min(nchunks, c0 + chunks_per_warp);
  if (c0 < c1) {
    int64_t m = c0 * 32 + lane;
    int z = (int)(m % nz);
    int j = (int)((m / nz) % n1);
    int i = (int)(m / ((int64_t)nz * n1));
    int ic = -1, jc = -1;
    float kx = 0.f, ky = 0.f, kxy = 0.f;
    const float thr_last = s.thr[g.nedges - 1];
    auto advance = [&]() {
      z += 32;
      while (z >= nz) {
        z -= nz;
        if (++j == n1) {
          j = 0;
          ++i;
        }
      }
    };
    for (int64_t c = c0; c < c1; ++c, m += 32) {
      const bool valid = m < total;
      float v[NV];
      int key = 0x7fffffff, bin = 0;
      float kz = 0.f, k2 = INFINITY;
      if (valid) {
        if (i != ic || j != jc) {
          kx = kcoord(i, g.d.n0, g.kfun[0], false);
          ky = kcoord(j, n1, g.kfun[1], false);
          kxy = __fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky));
          ic = i;
          jc = j;
        }
        float kz2;
        if (tab) {
          kz = s.kz[z];
          kz2 = s.kz2[z];
        } else {
          kz = kz_coord(g, z);
          kz2 = __fmul_rn(kz, kz);
        }
        k2 = __fadd_rn(kxy, kz2);
      }
      // a chunk whose modes all lie beyond the last edge adds nothing (warp-uniform skip)
      if (!__any_sync(0xffffffffu, k2 < thr_last)) {
        advance();
        continue;
      }
      if (valid) {
        bin = bin_from_k2(s.thr, g.nedges, e0, inv_step, k2);
        key = bin | ((int)((i * n1 + j) & 31) << 16);
        // modes outside the bins (beyond the last edge: the corners of the k cube) are not read
        const bool inr = bin >= 1 && bin <= nbins;
        float2 F[NT], A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
#pragma unroll
        for (int t = 0; t < NT; ++t) F[t] = make_float2(0.f, 0.f);
        if (inr) {
#pragma unroll
          for (int t = 0; t < NT; ++t) F[t] = __ldcs(f + (int64_t)t * fstride + m);
          A = a0[m];
          if (CROSS) B = b0[m];
        }
        const float w = mode_weight(g, z);
        if (CROSS) {
          v[0] = (B.x * A.x + B.y * A.y) * w;
        } else {
          v[0] = (A.x * A.x + A.y * A.y) * w;
        }
        const bool zero = (i == 0 && j == 0 && z == 0);
        const float rn = k2 > 0.f ? rsqrtf(k2) : 0.f;  // khat = k / |k|, 0 at k = 0
        fp_block_values<MASK, 0, 0, 1>(F, kx * rn, ky * rn, kz * rn, A, zero, w, v);
      } else {
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] = 0.f;
      }
      const int prev = __shfl_up_sync(0xffffffffu, key, 1);
      if (!__all_sync(0xffffffffu, lane == 0 || prev != key)) {
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const bool ok = __shfl_up_sync(0xffffffffu, key, d) == key && lane >= d;
#pragma unroll
          for (int q = 0; q < NV; ++q) {
            const float t = __shfl_up_sync(0xffffffffu, v[q], d);
            if (ok) v[q] += t;
          }
        }
      }
      const int next = __shfl_down_sync(0xffffffffu, key, 1);
      const bool tail = valid && (lane == 31 || next != key) && bin >= 1 && bin <= nbins;
      // a bin has one run tail per row: the rows of the chunk write in turn
      const int row = i * n1 + j;
      const int roff = row - __shfl_sync(0xffffffffu, row, 0);
      const int nrow = __reduce_max_sync(0xffffffffu, valid ? roff : 0);
      for (int p = 0; p <= nrow; ++p) {
        if (tail && roff == p) {
#pragma unroll
          for (int q = 0; q < NV; ++q) my[(size_t)(bin - 1) * NV + q] += (double)v[q];
        }
        __syncwarp();
      }
      advance();
    }
  }
  bin_smem_flush(s, hist_len, nwarps, partials);
}

// Output row of each value (n = 0: value c goes to row c); a negative row drops the value.
struct RowMap {
  int n;
  int row[MAX_ELLS + 1];
};

// out[e] (+)= sum over CTAs, transposed to [value][bin].  Deterministic two-level sum:
// 32 threads per entry each add a fixed contiguous range of CTA rows (4 independent loads
// in flight), then the 32 partials are added in a fixed order.  8 entries per CTA: a few
// hundred entries (bins x multipoles) still make a grid of ~100 CTAs, so the partial rows
// (one per binning CTA) are read with many loads in flight.
constexpr int FIN_ENTRIES = 8, FIN_SPLIT = 32;
__global__ void __launch_bounds__(FIN_ENTRIES * FIN_SPLIT) bin_finalize_kernel(
    const double *__restrict__ partials, int nblocks, int hist_len, int nv, int nbins,
    int accumulate, double *__restrict__ out0, double *__restrict__ out1, RowMap map) {
  __shared__ double part[FIN_SPLIT][FIN_ENTRIES];
  partials += (size_t)blockIdx.y * nblocks * hist_len;  // batch of histograms along y
  out0 += (size_t)blockIdx.y * hist_len;
  const int le = threadIdx.x % FIN_ENTRIES, sp = threadIdx.x / FIN_ENTRIES;
  const int e = blockIdx.x * FIN_ENTRIES + le;
  const int per = (nblocks + FIN_SPLIT - 1) / FIN_SPLIT;
  const int b0 = sp * per, b1 = min(nblocks, b0 + per);
  double a0 = 0., a1 = 0., a2 = 0., a3 = 0.;
  if (e < hist_len) {
    int b = b0;
    for (; b + 3 < b1; b += 4) {
      a0 += partials[(size_t)b * hist_len + e];
      a1 += partials[(size_t)(b + 1) * hist_len + e];
      a2 += partials[(size_t)(b + 2) * hist_len + e];
      a3 += partials[(size_t)(b + 3) * hist_len + e];
    }
    for (; b < b1; ++b) a0 += partials[(size_t)b * hist_len + e];
  }
  part[sp][le] = (a0 + a1) + (a2 + a3);
  __syncthreads();
  if (sp == 0 && e < hist_len) {
    double acc = 0.;
    for (int k = 0; k < FIN_SPLIT; ++k) acc += part[k][le];
    const int bin = e / nv, c = e % nv;
    const int r = map.n ? map.row[c] : c;
    if (r < 0) return;
    double *dst = (c == 1 && out1) ? out1 : out0;
    const int64_t o = (c == 1 && out1) ? bin : (int64_t)r * nbins + bin;
    dst[o] = accumulate ? dst[o] + acc : acc;
  }
}

static void launch_finalize(cudaStream_t s, const double *partials, int nblocks, int hist_len,
                            int nv, int nbins, int accumulate, double *out0, double *out1,
                            int nbatch = 1, RowMap map = RowMap{}) {
  const dim3 grid((hist_len + FIN_ENTRIES - 1) / FIN_ENTRIES, nbatch);
  bin_finalize_kernel<<<grid, FIN_ENTRIES * FIN_SPLIT, 0, s>>>(partials, nblocks, hist_len, nv, nbins,
                                                               accumulate, out0, out1, map);
}

struct BinLaunch {
  int blocks;
  int nwarps;
  int tab;
  size_t smem;
  size_t partial_bytes;
};

static bool plan_bins(const Dims &d, int nedges, int nv, BinLaunch *L,
                      size_t hist_elem = sizeof(double)) {
  const int nbins = nedges - 1;
  const size_t per_warp = (size_t)nbins * nv * hist_elem;
  const size_t thr_bytes = (size_t)((nedges + 3) & ~3) * sizeof(float);
  const size_t tab_bytes = 2 * (size_t)((d.nz + 3) & ~3) * sizeof(float);
  const size_t budget = 200 * 1024;
  L->tab = tab_bytes <= 32 * 1024;
  const size_t fixed = thr_bytes + (L->tab ? tab_bytes : 0);
  int nwarps = BIN_THREADS / 32;
  if (per_warp + fixed > budget) return false;
  while (nwarps > 1 && (size_t)nwarps * per_warp + fixed > budget) nwarps >>= 1;
  L->nwarps = nwarps;
  L->smem = align_up((size_t)nwarps * per_warp, 16) + fixed;
  const int64_t nrows = (int64_t)d.n0 * d.n1;
  int per_sm = (int)((228 * 1024) / (L->smem + 1024));
  if (per_sm > 8) per_sm = 8;
  if (per_sm < 1) per_sm = 1;
  int64_t blocks = (int64_t)per_sm * sm_count();
  const int64_t need = (nrows + nwarps - 1) / nwarps;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  L->blocks = (int)blocks;
  L->partial_bytes = (size_t)blocks * nbins * nv * sizeof(double);
  return true;
}

template <int NV, class Op, bool SEP = false>
static pk_status launch_bins(cudaStream_t s, const BinGeom &g, const Op &op, const float *edges,
                             bool rows, int accumulate, double *out0, double *out1,
                             void *workspace, size_t workspace_bytes) {
  BinLaunch L;
  PK_REQUIRE(plan_bins(g.d, g.nedges, NV, &L), PK_ERR_RANGE,
             "too many bins x values (%d x %d) for the shared-memory histograms", g.nedges - 1, NV);
  PK_REQUIRE(workspace && workspace_bytes >= L.partial_bytes, PK_ERR_WORKSPACE,
             "binning workspace too small: need %zu bytes, got %zu", L.partial_bytes,
             workspace_bytes);
  double *partials = static_cast<double *>(workspace);
  if (rows) {
    PK_CUDA(cudaFuncSetAttribute(bin_rows_kernel<NV, Op, SEP>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
    bin_rows_kernel<NV, Op, SEP><<<L.blocks, L.nwarps * 32, L.smem, s>>>(g, op, edges, L.nwarps, L.tab,
                                                                          partials);
  } else {
    PK_CUDA(cudaFuncSetAttribute(bin_chunks_kernel<NV, Op>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
    bin_chunks_kernel<NV, Op><<<L.blocks, L.nwarps * 32, L.smem, s>>>(g, op, edges, L.nwarps,
                                                                       L.tab, partials);
  }
  PK_LAUNCH_CHECK();
  const int hist_len = (g.nedges - 1) * NV;
  launch_finalize(s, partials, L.blocks, hist_len, NV, g.nedges - 1, accumulate, out0, out1);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

// ------------------------------------------------- global line of sight, fused
// The hot binning pass of the global-los estimator (mesh2.py:346-374), written out for
// throughput: per mode one complex load, |k|^2 from per-axis tables, the bin advanced
// against exact |k|^2 thresholds, mu^2 = (k.los)^2 / k^2 by a reciprocal, and every
// L_ell as Horner polynomials in mu^2 (times mu for odd ell).  Row runs and the per-row
// segmented scan as in bin_rows_kernel.
struct LegendreCoefs {
  float c[MAX_ELLS][5];  // L_ell(mu) = mu^(ell % 2) * sum_p c[p] mu^(2p)
  int odd[MAX_ELLS];
  int any_odd;
};

__host__ inline void legendre_coefs(int ell, float c[5], int *odd) {
  static const double table[9][5] = {
      {1., 0., 0., 0., 0.},
      {1., 0., 0., 0., 0.},
      {-0.5, 1.5, 0., 0., 0.},
      {-1.5, 2.5, 0., 0., 0.},
      {0.375, -3.75, 4.375, 0., 0.},
      {1.875, -8.75, 7.875, 0., 0.},
      {-0.3125, 6.5625, -19.6875, 14.4375, 0.},
      {-2.1875, 19.6875, -43.3125, 26.8125, 0.},
      {0.2734375, -9.84375, 54.140625, -93.84375, 50.2734375}};
  for (int p = 0; p < 5; ++p) c[p] = (float)table[ell][p];
  *odd = ell & 1;
}

// End of a row walk (bin_global_kernel, bin_interlaced_staged_kernel): join the lanes' lead and
// trail runs with a segmented scan over the lanes and add each bin's sum to the warp histogram
// once.  cur: the lane's last bin (-1: no mode), nseg: its finished runs, lead / facc: the first
// run (when nseg > 0), acc: the open run.
template <int NV>
__device__ __forceinline__ void finish_row_runs(int cur, int nseg, int lead, const float facc_in[NV],
                                                const float acc[NV], float *my, int nbins, int lane) {
  constexpr int NONE = 0x7fffffff;
  int trail;
  float facc[NV], tacc[NV];
  if (cur < 0) {
    lead = trail = NONE;
#pragma unroll
    for (int c = 0; c < NV; ++c) tacc[c] = facc[c] = 0.f;
  } else if (nseg == 0) {
    lead = trail = cur;
#pragma unroll
    for (int c = 0; c < NV; ++c) {
      tacc[c] = acc[c];
      facc[c] = 0.f;
    }
  } else {
    trail = cur;
#pragma unroll
    for (int c = 0; c < NV; ++c) {
      tacc[c] = acc[c];
      facc[c] = facc_in[c];
    }
  }
  float S[NV];
#pragma unroll
  for (int c = 0; c < NV; ++c) S[c] = tacc[c];
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int k = __shfl_up_sync(0xffffffffu, trail, d);
    const bool ok = lane >= d && k == trail;
#pragma unroll
    for (int c = 0; c < NV; ++c) {
      const float t = __shfl_up_sync(0xffffffffu, S[c], d);
      if (ok) S[c] += t;
    }
  }
  const int prev_trail = __shfl_up_sync(0xffffffffu, trail, 1);
  float carry[NV];
#pragma unroll
  for (int c = 0; c < NV; ++c) {
    const float t = __shfl_up_sync(0xffffffffu, S[c], 1);
    carry[c] = (lane > 0 && prev_trail == lead) ? t : 0.f;
  }
  const int next_lead = __shfl_down_sync(0xffffffffu, lead, 1);
  const int next_trail = __shfl_down_sync(0xffffffffu, trail, 1);
  if (cur >= 0 && nseg > 0 && lead >= 1 && lead <= nbins) {
#pragma unroll
    for (int c = 0; c < NV; ++c) my[(size_t)(lead - 1) * NV + c] += facc[c] + carry[c];
  }
  const bool next_takes = lane < 31 && next_lead == trail;
  const bool next_continues = lane < 31 && next_trail == trail;
  if (cur >= 0 && !next_takes && !next_continues && trail >= 1 && trail <= nbins) {
#pragma unroll
    for (int c = 0; c < NV; ++c) my[(size_t)(trail - 1) * NV + c] += S[c];
  }
  __syncwarp();
}

template <int NV>
__device__ __forceinline__ void moments_to_poles(const LegendreCoefs &lc, float m0, float m1, float m2,
                                                 float out[NV]) {
#pragma unroll
  for (int l = 0; l < NV; ++l) out[l] = __fmaf_rn(lc.c[l][2], m2, __fmaf_rn(lc.c[l][1], m1, lc.c[l][0] * m0));
}

// Shared layout of the fused kernel: float32 warp histograms [nwarps][nbins][NV] (warp
// partials), thresholds, kz tables.
struct GlobalSmem {
  float *hist;
  float *thr;
  float *kz;
  float *kz2;
};

// EVEN: every multipole even with ell <= 4 (L_ell a polynomial of degree <= 2 in mu^2, no
// odd parts), the usual (0, 2, 4) case; otherwise the general form (degree 4, odd ell).
// NS < 0: the binned value is Re(d1) itself, linear in the mesh (window-matrix columns).
// NS > 0: the mesh is not stored; each mode is formed on the fly from NS interlaced,
// uncompensated meshes at d1 (mesh s at d1 + s N_c), exactly as pk_interlace_compensate
// forms it (fp: its parameters; FULL: 'jaxdecomp' semantics), which saves writing and
// reading back the combined mesh.  MINB: CTAs per SM the register budget is sized for.  The
// fused form of a single mesh takes 3 (512^3, 3 shifts: 0.83 ms against 0.89 with 4 and 0.93
// with 2), batches of meshes 4 (29 x 192^3, 2 shifts: 1.58 ms against 1.78 with 3; 32 x 256^3:
// 3.34 against 3.76).
#ifndef PK_FUSED_MIN_CTAS
#define PK_FUSED_MIN_CTAS 3
#endif
#ifndef PK_FUSED_BATCH_MIN_CTAS
#define PK_FUSED_BATCH_MIN_CTAS 4
#endif
template <int NV, bool CROSS, bool EVEN, int NS = 0, bool FULL = false, int MINB = (NS > 0 ? PK_FUSED_MIN_CTAS : 4),
          int XYM = XY_NONE>
__global__ void __launch_bounds__(BIN_THREADS, MINB) bin_global_kernel(
    BinGeom g, const float2 *__restrict__ d1, const float2 *__restrict__ d2, float lx, float ly,
    float lz, LegendreCoefs lc, int zero_l0, const float *__restrict__ edges, int nwarps_hist,
    int tab, double *__restrict__ partials, FourierParams fp) {
  constexpr int NSR = NS > 0 ? NS : 1;
  const int nbins = g.nedges - 1;
  const int hist_len = nbins * NV;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  extern __shared__ double smem[];
  GlobalSmem s;
  s.hist = reinterpret_cast<float *>(smem);
  s.thr = s.hist + (((size_t)nwarps_hist * hist_len + 3) & ~(size_t)3);
  s.kz = s.thr + ((g.nedges + 3) & ~3);
  s.kz2 = s.kz + ((g.d.nz + 3) & ~3);
  ZTable zt;
  if (NS > 0) {
    zt = ztable_at<XYM>(s.kz2 + ((g.d.nz + 3) & ~3), fp, FULL);
    fill_ztable<FULL, XYM>(fp, zt);
  }
  for (int q = threadIdx.x; q < nwarps_hist * hist_len; q += blockDim.x) s.hist[q] = 0.f;
  for (int q = threadIdx.x; q < g.nedges; q += blockDim.x) s.thr[q] = sqrt_threshold(edges[q]);
  if (tab)
    for (int z = threadIdx.x; z < g.d.nz; z += blockDim.x) {
      const float kzz = kz_coord(g, z);
      s.kz[z] = kzz;
      s.kz2[z] = __fmul_rn(kzz, kzz);
    }
  __syncthreads();
  float *my = s.hist + (size_t)warp * hist_len;
  const float e0 = edges[0];
  const float inv_step = g.step > 0.f ? 1.f / g.step : 0.f;
  const int R = (g.d.nz + 31) / 32;
  const int z0 = lane * R, z1r = min(g.d.nz, z0 + R);
  const bool jaxw = g.backend == PK_BACKEND_JAX;
  const float thr_last = s.thr[g.nedges - 1];
  // batch of meshes along y: mesh blockIdx.y, its own partial rows
  d1 += (int64_t)blockIdx.y * (NS > 0 ? NS : 1) * g.d.ncomplex();
  if (CROSS) d2 += (int64_t)blockIdx.y * g.d.ncomplex();
  partials += (size_t)blockIdx.y * gridDim.x * hist_len;
  const int zself = (g.d.n2 % 2) == 0 ? g.d.nz - 1 : -1;  // self-conjugate last plane
  constexpr int NONE = 0x7fffffff;
  for (RowWalker rw((int64_t)blockIdx.x * nwarps + warp, (int64_t)gridDim.x * nwarps, g.d.n1); rw.i < g.d.n0;
       rw.next()) {
    const int i = rw.i, j = rw.j;
    const int64_t row = (int64_t)i * g.d.n1 + j;
    const float kx = kcoord(i, g.d.n0, g.kfun[0], false);
    const float ky = kcoord(j, g.d.n1, g.kfun[1], false);
    const float kxy = __fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky));
    // |k|^2 grows along the stored kz: the modes at or beyond the last edge (no bin) are the
    // row's tail, cut at the first one; rows beyond it entirely are skipped (warp-uniform)
    if (!(kxy < thr_last)) continue;
    int zcut = 0;
    {
      int lim = g.d.nz;
      while (zcut < lim) {
        const int mid = (zcut + lim) >> 1;
        float kz2m;
        if (tab) kz2m = s.kz2[mid];
        else {
          const float kzm = kz_coord(g, mid);
          kz2m = __fmul_rn(kzm, kzm);
        }
        if (__fadd_rn(kxy, kz2m) >= thr_last) lim = mid;
        else zcut = mid + 1;
      }
    }
    const int z1 = min(z1r, zcut);
    const float kl = kx * lx + ky * ly;
    RowFactor<NSR> rf;
    if (NS > 0) row_factor<NSR, FULL, XYM != XY_NONE>(fp, zt, i, j, rf);
    int cur = -1, lead = NONE, nseg = 0;
    float acc[NV], facc[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c) acc[c] = facc[c] = 0.f;
    const float2 *p1 = d1 + row * g.d.nz;
    const float2 *p2 = CROSS ? d2 + row * g.d.nz : nullptr;
    // the run's values are loaded RB at a time before use: several loads in flight per lane
    // (with 3 shifted meshes, RB = 2 measured 0.81 ms at 512^3 against 0.83 for 4 and 0.91
    // for 8: the wider batches cost registers)
#ifndef PK_FUSED_RB
#define PK_FUSED_RB 2
#endif
    constexpr int RB = CROSS ? 4 : (NS > 1 ? PK_FUSED_RB : 8);
    for (int zb = z0; zb < z1; zb += RB) {
      float2 va[RB], vb[CROSS ? RB : 1];
#pragma unroll
      for (int t = 0; t < RB; ++t) {
        const int z = zb + t;
        if (NS > 0)
          va[t] = z < z1 ? combine_mode<NSR, FULL>(fp, rf, zt, d1, row * g.d.nz + z, z) : make_float2(0.f, 0.f);
        else
          va[t] = z < z1 ? p1[z] : make_float2(0.f, 0.f);
        if (CROSS) vb[t] = z < z1 ? p2[z] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int t = 0; t < RB; ++t) {
        const int z = zb + t;
        if (z >= z1) break;
        float kz, kz2;
        if (tab) {
          kz = s.kz[z];
          kz2 = s.kz2[z];
        } else {
          kz = kz_coord(g, z);
          kz2 = __fmul_rn(kz, kz);
        }
        const float k2 = __fadd_rn(kxy, kz2);
        int gb = cur;
        if (cur < 0) gb = bin_from_k2(s.thr, g.nedges, e0, inv_step, k2);
        else
          while (gb < g.nedges && k2 >= s.thr[gb]) ++gb;
        if (gb != cur) {
          if (cur >= 0) {
            if (nseg == 0) {
              lead = cur;
#pragma unroll
              for (int c = 0; c < NV; ++c) facc[c] = acc[c];
            } else if (cur >= 1 && cur <= nbins) {
#pragma unroll
              for (int c = 0; c < NV; ++c) my[(size_t)(cur - 1) * NV + c] += acc[c];
            }
            ++nseg;
          }
          cur = gb;
#pragma unroll
          for (int c = 0; c < NV; ++c) acc[c] = 0.f;
        }
        const float2 a = va[t];
        float re, im = 0.f;
        if (CROSS) {
          const float2 b = vb[CROSS ? t : 0];
          re = a.x * b.x + a.y * b.y;
          im = a.x * b.y - a.y * b.x;
        } else {
          re = NS < 0 ? a.x : a.x * a.x + a.y * a.y;
        }
        const float w = jaxw ? (z > 0 ? 2.f : 1.f) : ((z == 0 || z == zself) ? 1.f : 2.f);
        const float num = kl + kz * lz;
        const float rk2 = k2 > 0.f ? __fdividef(1.f, k2) : 0.f;  // mu^2 enters L_ell only
        const float mu2 = num * num * rk2;
        const bool zero = (row == 0 && z == 0);  // remove_zero for ell > 0
        const float rw = re * w;
        if (EVEN) {
#pragma unroll
          for (int l = 0; l < NV; ++l) {
            const float L = __fmaf_rn(__fmaf_rn(lc.c[l][2], mu2, lc.c[l][1]), mu2, lc.c[l][0]);
            const bool drop = zero && !(zero_l0 & (1 << l));
            acc[l] += drop ? 0.f : rw * L;
          }
        } else {
          const float mu = lc.any_odd ? num * sqrtf(rk2) : 0.f;
          const float iw = im * w;
#pragma unroll
          for (int l = 0; l < NV; ++l) {
            float L = lc.c[l][4];
            L = L * mu2 + lc.c[l][3];
            L = L * mu2 + lc.c[l][2];
            L = L * mu2 + lc.c[l][1];
            L = L * mu2 + lc.c[l][0];
            if (lc.odd[l]) L *= mu;
            const float part = lc.odd[l] ? iw : rw;
            const bool drop = zero && !(zero_l0 & (1 << l));
            acc[l] += drop ? 0.f : part * L;
          }
        }
      }
    }
    finish_row_runs<NV>(cur, nseg, lead, facc, acc, my, nbins, lane);
  }
  __syncthreads();  // warp partials (float32) finished in float64, in warp order
  double *outp = partials + (size_t)blockIdx.x * hist_len;
  for (int q = threadIdx.x; q < hist_len; q += blockDim.x) {
    double a = 0.;
    for (int w = 0; w < nwarps; ++w) a += (double)s.hist[(size_t)w * hist_len + q];
    outp[q] = a;
  }
}

// ------------------------------------------------- fused interlaced binning, staged rows
// The interlaced + compensated global-los pass for even multipoles (ell <= 4) of 'jax'
// half-complex meshes (a single mesh or a batch).  A prologue (staged_rows_kernel) tabulates
// per (i, j) row |k_xy|^2, k_xy . los, the window scale, the interlacing phases and the row's
// cut: |k|^2 increases along kz, so the modes at or beyond the last edge form the row's tail,
// cut at the first such kz (rows whose first mode is already beyond it are skipped, meshes
// unread: with edges up to k_Nyq that is 48 % of the stored modes, the corners of the k cube;
// they would fall in no bin, so the sums do not change).  Then per row and warp:
//  1. lanes on consecutive kz form each mode's weighted power w |combine_mode(...)|^2 from
//     coalesced loads of the NS shifted meshes (one 128-byte line per 16 lanes and mesh) and
//     its mu^2, into the warp's row buffers in shared memory;
//  2. each lane walks a contiguous run of the row, following the bin by comparing |k|^2 with
//     the next exact threshold (the bin is non-decreasing along kz), and accumulates per bin
//     run the moments M_p = sum P mu^(2p), p = 0, 1, 2, in registers; a finished run becomes
//     its multipoles sum_p c_{ell,p} M_p once, and runs continuing across lanes are joined by
//     the segmented scan of bin_global_kernel.
// The k = 0 mode (row 0, kz 0) enters the monopole only (when ell = 0 is asked), added by lane 0
// on its own.  Mode values, row factors and bins are bit-identical to bin_global_kernel's (the
// same combine_mode, row_factor and exact thresholds); the multipoles differ by float32
// rounding in the run sums.
#ifndef PK_FUSED_STAGED
#define PK_FUSED_STAGED 1
#endif
#ifndef PK_STAGED_MIN_CTAS
#define PK_STAGED_MIN_CTAS 3
#endif
#ifndef PK_STAGED_UNROLL
#define PK_STAGED_UNROLL 3
#endif
#ifndef PK_STAGED_MIN_NZ
#define PK_STAGED_MIN_NZ 90  // shorter stored rows take bin_global_flat_kernel
#endif
constexpr int STAGED_MAX_SHIFTS = 4;
// shared-memory bytes of one warp's row buffers (power and mu^2, float) for nz modes
__host__ __device__ inline size_t staged_row_bytes(int nz) { return (size_t)32 * ((nz + 31) / 32) * 8; }
// global bytes of the row table: (|k_xy|^2, k_xy . los, scale, cut) per row, then the phases of
// shifts 1..NS-1 per row
inline size_t staged_table_bytes(const Dims &d, int nshifts) {
  return (size_t)d.n0 * d.n1 * (sizeof(float4) + (size_t)(nshifts - 1) * sizeof(float2));
}

template <int NS>
__global__ void staged_rows_kernel(BinGeom g, FourierParams fp, float lx, float ly, const float *__restrict__ edges,
                                   float4 *__restrict__ rowa, float2 *__restrict__ rowph) {
  const float thr_last = sqrt_threshold(edges[g.nedges - 1]);
  const ZTable zt = ztable_at<XY_GLOBAL>(nullptr, fp, false);  // the per-axis tables of fp.gxy
  const int64_t nrows = (int64_t)g.d.n0 * g.d.n1;
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < nrows;
       row += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(row / g.d.n1), j = (int)(row % g.d.n1);
    const float kx = kcoord(i, g.d.n0, g.kfun[0], false);
    const float ky = kcoord(j, g.d.n1, g.kfun[1], false);
    const float kxy = __fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky));
    int zhi = 0;  // the first kz whose |k|^2 reaches the last threshold (0: none below it)
    if (kxy < thr_last) {
      int lim = g.d.nz;
      while (zhi < lim) {
        const int mid = (zhi + lim) >> 1;
        const float kz = kz_coord(g, mid);
        if (__fadd_rn(kxy, __fmul_rn(kz, kz)) >= thr_last) lim = mid;
        else zhi = mid + 1;
      }
    }
    RowFactor<NS> rf;
    row_factor<NS, false, true>(fp, zt, i, j, rf);
    rowa[row] = make_float4(kxy, kx * lx + ky * ly, rf.scale, __int_as_float(zhi));
#pragma unroll
    for (int s = 1; s < NS; ++s) rowph[row * (NS - 1) + s - 1] = rf.ph[s];
  }
}

template <int NV, int NS, int MINB>
__global__ void __launch_bounds__(BIN_THREADS, MINB) bin_interlaced_staged_kernel(
    BinGeom g, const float2 *__restrict__ d1, float lz, LegendreCoefs lc, int zero_l0,
    const float *__restrict__ edges, int nwarps_hist, double *__restrict__ partials, FourierParams fp,
    const float4 *__restrict__ rowa, const float2 *__restrict__ rowph) {
  const int nbins = g.nedges - 1;
  const int hist_len = nbins * NV;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  const int nz = g.d.nz;
  const int S = 32 * ((nz + 31) / 32);  // row buffer slots
  extern __shared__ double smem[];
  float *hist = reinterpret_cast<float *>(smem);
  float *thr = hist + (((size_t)nwarps_hist * hist_len + 3) & ~(size_t)3);
  float *skz = thr + ((g.nedges + 3) & ~3);
  float *skz2 = skz + ((nz + 3) & ~3);
  float *pbuf_all = skz2 + ((nz + 3) & ~3);         // [nwarps][S] powers
  float *mbuf_all = pbuf_all + (size_t)nwarps * S;  // [nwarps][S] mu^2
  ZTable zt = ztable_at<XY_NONE>(mbuf_all + (size_t)nwarps * S, fp, false);
  fill_ztable<false, XY_NONE>(fp, zt);
  for (int q = threadIdx.x; q < nwarps_hist * hist_len; q += blockDim.x) hist[q] = 0.f;
  for (int q = threadIdx.x; q < g.nedges; q += blockDim.x) thr[q] = sqrt_threshold(edges[q]);
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    const float kzz = kz_coord(g, z);
    skz[z] = kzz;
    skz2[z] = __fmul_rn(kzz, kzz);
  }
  __syncthreads();
  float *my = hist + (size_t)warp * hist_len;
  float *pbuf = pbuf_all + (size_t)warp * S, *mbuf = mbuf_all + (size_t)warp * S;
  const float e0 = edges[0];
  const float inv_step = g.step > 0.f ? 1.f / g.step : 0.f;
  d1 += (int64_t)blockIdx.y * NS * g.d.ncomplex();
  partials += (size_t)blockIdx.y * gridDim.x * hist_len;
  RowWalker rw((int64_t)blockIdx.x * nwarps + warp, (int64_t)gridDim.x * nwarps, g.d.n1);
  // the row table entries of the warp's next row are loaded one row ahead
  float4 ra = make_float4(0.f, 0.f, 0.f, 0.f);
  float2 rp[NS > 1 ? NS - 1 : 1];
  if (rw.i < g.d.n0) {
    const int64_t r0 = (int64_t)rw.i * g.d.n1 + rw.j;
    ra = rowa[r0];
#pragma unroll
    for (int s = 1; s < NS; ++s) rp[s - 1] = rowph[r0 * (NS - 1) + s - 1];
  }
  for (; rw.i < g.d.n0;) {
    const int64_t row = (int64_t)rw.i * g.d.n1 + rw.j;
    const float4 rcur = ra;
    RowFactor<NS> rf;
#pragma unroll
    for (int s = 1; s < NS; ++s) rf.ph[s] = rp[s - 1];
    rw.next();
    if (rw.i < g.d.n0) {
      const int64_t rn = (int64_t)rw.i * g.d.n1 + rw.j;
      ra = rowa[rn];
#pragma unroll
      for (int s = 1; s < NS; ++s) rp[s - 1] = rowph[rn * (NS - 1) + s - 1];
    }
    const int zhi = __float_as_int(rcur.w);
    if (zhi == 0) continue;  // every mode of the row is beyond the last edge (warp-uniform)
    const float kxy = rcur.x, kl = rcur.y;
    rf.scale = rcur.z;
    const int Rz = (zhi + 31) >> 5;  // modes per lane
    // phase 1: lanes on consecutive kz: weighted power and mu^2 of each mode, PK_STAGED_UNROLL
    // modes (3 PK_STAGED_UNROLL mesh loads) in flight per lane
    constexpr int U = PK_STAGED_UNROLL;
    for (int t0 = 0; t0 < Rz; t0 += U) {
      float p[U], m[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int z = lane + 32 * (t0 + u);
        p[u] = m[u] = 0.f;
        if (t0 + u < Rz && z < zhi) {
          const float2 v = combine_mode<NS, false>(fp, rf, zt, d1, row * nz + z, z);
          p[u] = (v.x * v.x + v.y * v.y) * (z > 0 ? 2.f : 1.f);
          const float k2 = __fadd_rn(kxy, skz2[z]);
          const float num = kl + skz[z] * lz;
          m[u] = k2 > 0.f ? num * num * __fdividef(1.f, k2) : 0.f;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (t0 + u < Rz) {
          pbuf[lane + 32 * (t0 + u)] = p[u];
          mbuf[lane + 32 * (t0 + u)] = m[u];
        }
    }
    __syncwarp();
    // phase 2: contiguous runs per lane, the bin followed by threshold compares
    const int z0 = lane * Rz, z1 = min(zhi, z0 + Rz);
    int zs = z0;
    if (row == 0) {
      if (lane == 0) {  // the k = 0 mode: the monopole only
        const int gb = bin_from_k2(thr, g.nedges, e0, inv_step, 0.f);
        if (gb >= 1 && gb <= nbins)
#pragma unroll
          for (int l = 0; l < NV; ++l)
            if (zero_l0 & (1 << l)) my[(size_t)(gb - 1) * NV + l] += pbuf[0] * lc.c[l][0];
        zs = 1;
      }
      __syncwarp();
    }
    int cur = -1, lead = 0, nseg = 0;
    float thr_next = INFINITY;
    if (zs < z1) {
      cur = bin_from_k2(thr, g.nedges, e0, inv_step, __fadd_rn(kxy, skz2[zs]));  // < nedges: zs < zhi
      thr_next = thr[cur];
    }
    float m0 = 0.f, m1 = 0.f, m2 = 0.f;
    float facc[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c) facc[c] = 0.f;
    for (int z = zs; z < z1; ++z) {
      const float pz = pbuf[z], mu2 = mbuf[z];
      const float k2 = __fadd_rn(kxy, skz2[z]);
      if (k2 >= thr_next) {  // the run of bin cur ends before z
        float Sv[NV];
        moments_to_poles<NV>(lc, m0, m1, m2, Sv);
        const bool first = nseg == 0;
        lead = first ? cur : lead;
#pragma unroll
        for (int c = 0; c < NV; ++c) facc[c] = first ? Sv[c] : facc[c];
        if (!first && cur >= 1 && cur <= nbins) {
          float *h = my + (cur - 1) * NV;
#pragma unroll
          for (int c = 0; c < NV; ++c) h[c] += Sv[c];
        }
        ++nseg;
        do ++cur;
        while (cur < g.nedges - 1 && k2 >= thr[cur]);  // k2 < thr[nedges - 1]: z < zhi
        thr_next = thr[cur];
        m0 = m1 = m2 = 0.f;
      }
      const float pm = pz * mu2;
      m0 += pz;
      m1 += pm;
      m2 = __fmaf_rn(pm, mu2, m2);
    }
    float acc[NV];
    moments_to_poles<NV>(lc, m0, m1, m2, acc);
    finish_row_runs<NV>(cur, nseg, lead, facc, acc, my, nbins, lane);
  }
  __syncthreads();  // warp partials (float32) finished in float64, in warp order
  double *outp = partials + (size_t)blockIdx.x * hist_len;
  for (int q = threadIdx.x; q < hist_len; q += blockDim.x) {
    double a = 0.;
    for (int w = 0; w < nwarps; ++w) a += (double)hist[(size_t)w * hist_len + q];
    outp[q] = a;
  }
}

// The same pass with the modes walked as one flat sequence of 32-mode chunks (lanes on
// consecutive kz, coalesced loads), as bin_firstpoint_kernel: a warp owns a contiguous range
// of chunks, bin keys carry the row's low 5 bits, one segmented scan per chunk, and the run
// tails of different rows add into the warp's float32 histogram one row after the other.
// A lane recomputes its row's factors (k_x, k_y, phases, window) when it enters a new row.
template <int NV, bool CROSS, bool EVEN, int NS = 0, bool FULL = false, int XYM = XY_NONE>
__global__ void __launch_bounds__(BIN_THREADS, NS > 0 ? PK_FUSED_MIN_CTAS : 4) bin_global_flat_kernel(
    BinGeom g, const float2 *__restrict__ d1, const float2 *__restrict__ d2, float lx, float ly,
    float lz, LegendreCoefs lc, int zero_l0, const float *__restrict__ edges, int nwarps_hist,
    int64_t chunks_per_warp, double *__restrict__ partials, FourierParams fp) {
  constexpr int NSR = NS > 0 ? NS : 1;
  const int nbins = g.nedges - 1;
  const int hist_len = nbins * NV;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  extern __shared__ double smem[];
  GlobalSmem s;
  s.hist = reinterpret_cast<float *>(smem);
  s.thr = s.hist + (((size_t)nwarps_hist * hist_len + 3) & ~(size_t)3);
  s.kz = s.thr + ((g.nedges + 3) & ~3);
  s.kz2 = s.kz + ((g.d.nz + 3) & ~3);
  ZTable zt;
  if (NS > 0) {
    zt = ztable_at<XYM>(s.kz2 + ((g.d.nz + 3) & ~3), fp, FULL);
    fill_ztable<FULL, XYM>(fp, zt);
  }
  for (int q = threadIdx.x; q < nwarps_hist * hist_len; q += blockDim.x) s.hist[q] = 0.f;
  for (int q = threadIdx.x; q < g.nedges; q += blockDim.x) s.thr[q] = sqrt_threshold(edges[q]);
  for (int z = threadIdx.x; z < g.d.nz; z += blockDim.x) {
    const float kzz = kz_coord(g, z);
    s.kz[z] = kzz;
    s.kz2[z] = __fmul_rn(kzz, kzz);
  }
  __syncthreads();
  float *my = s.hist + (size_t)warp * hist_len;
  const float e0 = edges[0];
  const float inv_step = g.step > 0.f ? 1.f / g.step : 0.f;
  const bool jaxw = g.backend == PK_BACKEND_JAX;
  const int zself = (g.d.n2 % 2) == 0 ? g.d.nz - 1 : -1;  // self-conjugate last plane
  // batch of meshes along y: mesh blockIdx.y, its own partial rows
  d1 += (int64_t)blockIdx.y * NSR * g.d.ncomplex();
  if (CROSS) d2 += (int64_t)blockIdx.y * g.d.ncomplex();
  partials += (size_t)blockIdx.y * gridDim.x * hist_len;
  const int nz = g.d.nz, n1 = g.d.n1;
  const int64_t total = g.d.ncomplex();
  const int64_t nchunks = (total + 31) / 32;
  const int64_t c0 = ((int64_t)blockIdx.x * nwarps + warp) * chunks_per_warp;
  const int64_t c1 = min(nchunks, c0 + chunks_per_warp);
  if (c0 < c1) {
    int64_t m = c0 * 32 + lane;
    int z = (int)(m % nz);
    int j = (int)((m / nz) % n1);
    int i = (int)(m / ((int64_t)nz * n1));
    int ic = -1, jc = -1;
    float kxy = 0.f, kl = 0.f;
    RowFactor<NSR> rf;
    const float thr_last = s.thr[g.nedges - 1];
    auto advance = [&]() {
      z += 32;
      while (z >= nz) {
        z -= nz;
        if (++j == n1) {
          j = 0;
          ++i;
        }
      }
    };
    for (int64_t c = c0; c < c1; ++c, m += 32) {
      const bool valid = m < total;
      float v[NV];
      int key = 0x7fffffff, bin = 0;
      float kz = 0.f, k2 = INFINITY;
      if (valid) {
        if (i != ic || j != jc) {
          const float kx = kcoord(i, g.d.n0, g.kfun[0], false);
          const float ky = kcoord(j, n1, g.kfun[1], false);
          kxy = __fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky));
          kl = kx * lx + ky * ly;
          if (NS > 0) row_factor<NSR, FULL, XYM != XY_NONE>(fp, zt, i, j, rf);
          ic = i;
          jc = j;
        }
        kz = s.kz[z];
        k2 = __fadd_rn(kxy, s.kz2[z]);
      }
      // a chunk whose modes all lie beyond the last edge adds nothing (warp-uniform skip)
      if (!__any_sync(0xffffffffu, k2 < thr_last)) {
        advance();
        continue;
      }
      if (valid) {
        bin = bin_from_k2(s.thr, g.nedges, e0, inv_step, k2);
        key = bin | ((int)((i * n1 + j) & 31) << 16);
        // modes outside the bins (beyond the last edge: the corners of the k cube) are not read
        const bool inr = bin >= 1 && bin <= nbins;
        float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
        if (inr) {
          a = NS > 0 ? combine_mode<NSR, FULL>(fp, rf, zt, d1, m, z) : d1[m];
          if (CROSS) b = d2[m];
        }
        float re, im = 0.f;
        if (CROSS) {
          re = a.x * b.x + a.y * b.y;
          im = a.x * b.y - a.y * b.x;
        } else {
          re = NS < 0 ? a.x : a.x * a.x + a.y * a.y;
        }
        const float w = jaxw ? (z > 0 ? 2.f : 1.f) : ((z == 0 || z == zself) ? 1.f : 2.f);
        const float num = kl + kz * lz;
        const float rk2 = k2 > 0.f ? __fdividef(1.f, k2) : 0.f;  // mu^2 enters L_ell only
        const float mu2 = num * num * rk2;
        const bool zero = (i == 0 && j == 0 && z == 0);  // remove_zero for ell > 0
        const float rw = re * w;
        if (EVEN) {
#pragma unroll
          for (int l = 0; l < NV; ++l) {
            const float L = __fmaf_rn(__fmaf_rn(lc.c[l][2], mu2, lc.c[l][1]), mu2, lc.c[l][0]);
            const bool drop = zero && !(zero_l0 & (1 << l));
            v[l] = drop ? 0.f : rw * L;
          }
        } else {
          const float mu = lc.any_odd ? num * sqrtf(rk2) : 0.f;
          const float iw = im * w;
#pragma unroll
          for (int l = 0; l < NV; ++l) {
            float L = lc.c[l][4];
            L = L * mu2 + lc.c[l][3];
            L = L * mu2 + lc.c[l][2];
            L = L * mu2 + lc.c[l][1];
            L = L * mu2 + lc.c[l][0];
            if (lc.odd[l]) L *= mu;
            const float part = lc.odd[l] ? iw : rw;
            const bool drop = zero && !(zero_l0 & (1 << l));
            v[l] = drop ? 0.f : part * L;
          }
        }
      } else {
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] = 0.f;
      }
      const int prev = __shfl_up_sync(0xffffffffu, key, 1);
      if (!__all_sync(0xffffffffu, lane == 0 || prev != key)) {
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const bool ok = __shfl_up_sync(0xffffffffu, key, d) == key && lane >= d;
#pragma unroll
          for (int q = 0; q < NV; ++q) {
            const float t = __shfl_up_sync(0xffffffffu, v[q], d);
            if (ok) v[q] += t;
          }
        }
      }
      const int next = __shfl_down_sync(0xffffffffu, key, 1);
      const bool tail = valid && (lane == 31 || next != key) && bin >= 1 && bin <= nbins;
      // a bin has one run tail per row: the rows of the chunk write in turn
      const int row = i * n1 + j;
      const int roff = row - __shfl_sync(0xffffffffu, row, 0);
      const int nrow = __reduce_max_sync(0xffffffffu, valid ? roff : 0);
      for (int p = 0; p <= nrow; ++p) {
        if (tail && roff == p) {
#pragma unroll
          for (int q = 0; q < NV; ++q) my[(size_t)(bin - 1) * NV + q] += v[q];
        }
        __syncwarp();
      }
      advance();
    }
  }
  __syncthreads();  // warp partials (float32) finished in float64, in warp order
  double *outp = partials + (size_t)blockIdx.x * hist_len;
  for (int q = threadIdx.x; q < hist_len; q += blockDim.x) {
    double a = 0.;
    for (int w = 0; w < nwarps; ++w) a += (double)s.hist[(size_t)w * hist_len + q];
    outp[q] = a;
  }
}

// The flat walk wins on short rows, the row walk on long ones (measured, 3 shifts, ells 0/2/4:
// 128^3 x 27 meshes 0.68 ms flat against 0.82 ms; 192^3 x 29 1.88 against 1.78; 512^3 0.96
// against 0.83): the flat kernel takes meshes whose stored rows are shorter than this.
#ifndef PK_GLOBAL_FLAT_NZ
#define PK_GLOBAL_FLAT_NZ 90
#endif

// Fill the global per-axis tables of p.gxy (the same values fill_ztable would put in shared
// memory).
__global__ void fill_xy_tables_kernel(FourierParams p) {
  const Dims &d = p.d;
  float2 *phx = p.gxy, *phy = phx + (size_t)p.nshifts * d.n0;
  float *sx = reinterpret_cast<float *>(phy + (size_t)p.nshifts * d.n1), *sy = sx + d.n0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.n0 + d.n1; i += gridDim.x * blockDim.x) {
    const bool x = i < d.n0;
    const int a = x ? i : i - d.n0;
    const float k = x ? ccoord(a, d.n0, p.cspacing[0], false) : ccoord(a, d.n1, p.cspacing[1], false);
    for (int s = 0; s < p.nshifts; ++s) (x ? phx[s * d.n0 + a] : phy[s * d.n1 + a]) = expi(p.shifts[s] * k);
    (x ? sx[a] : sy[a]) = sinc_of(k);
  }
}

template <int NV, bool CROSS, bool EVEN, int NS = 0, bool FULL = false>
static pk_status launch_global(cudaStream_t st, const BinGeom &g, const float2 *d1,
                               const float2 *d2, const float los[3], const LegendreCoefs &lc,
                               int zero_l0, const float *edges, double *out, void *workspace,
                               size_t workspace_bytes, int nbatch,
                               const FourierParams *fp = nullptr) {
  BinLaunch L;
  PK_REQUIRE(plan_bins(g.d, g.nedges, NV, &L, sizeof(float)), PK_ERR_RANGE,
             "too many bins x values (%d x %d) for the shared-memory histograms", g.nedges - 1, NV);
  FourierParams fpv{};
  // fused form: the per-axis phase / window tables of the row factors sit in shared memory
  // for meshes with n0 + n1 <= 512, else in global memory after the partial histograms (read
  // through the L1 cache with one address per warp, without taking shared memory from it):
  // measured with 3 shifts, 512^3 0.80 ms with global tables against 0.83 with per-row sines
  // and 1.04 with shared-memory tables; batches of 128^3..256^3 are fastest with shared ones
  const bool xy_smem = use_xy_tables(g.d);
  const size_t table_off = align_up(L.partial_bytes * nbatch);
  const size_t need = (NS > 0 && !xy_smem) ? table_off + xy_table_bytes(g.d, NS) : L.partial_bytes * nbatch;
  if (NS > 0) {
    fpv = *fp;
    // the kz tables (binning and interlacing) always live in shared memory on this path
    if (!L.tab) L.smem += 2 * (size_t)((g.d.nz + 3) & ~3) * sizeof(float);
    L.tab = 1;
    L.smem += ztable_bytes(g.d, NS, FULL, xy_smem);
    PK_REQUIRE(L.smem <= 227 * 1024, PK_ERR_RANGE, "mesh too large along the last axis for the fused pass");
  }
  PK_REQUIRE(workspace && workspace_bytes >= need, PK_ERR_WORKSPACE,
             "binning workspace too small: need %zu bytes, got %zu", need, workspace_bytes);
  double *partials = static_cast<double *>(workspace);
  if (NS > 0 && !xy_smem) {
    fpv.gxy = reinterpret_cast<float2 *>(static_cast<char *>(workspace) + table_off);
    fill_xy_tables_kernel<<<(g.d.n0 + g.d.n1 + 127) / 128, 128, 0, st>>>(fpv);
    PK_LAUNCH_CHECK();
  }
  const int hist_len = (g.nedges - 1) * NV;
  int blocks = L.blocks;
#if PK_FUSED_STAGED
  if constexpr (NS > 0 && NS <= STAGED_MAX_SHIFTS && !CROSS && EVEN && !FULL && NV <= 3) {
    if (g.d.nz >= PK_STAGED_MIN_NZ) {
      // workspace: partial rows, the per-axis tables, the row table
      const size_t xy_off = align_up(L.partial_bytes * nbatch);
      const size_t rows_off = align_up(xy_off + xy_table_bytes(g.d, NS));
      PK_REQUIRE(workspace_bytes >= rows_off + staged_table_bytes(g.d, NS), PK_ERR_WORKSPACE,
                 "binning workspace too small: need %zu bytes, got %zu", rows_off + staged_table_bytes(g.d, NS),
                 workspace_bytes);
      fpv.gxy = reinterpret_cast<float2 *>(static_cast<char *>(workspace) + xy_off);
      if (xy_smem) {  // the row-run kernels keep these tables in shared memory; the prologue reads them here
        fill_xy_tables_kernel<<<(g.d.n0 + g.d.n1 + 127) / 128, 128, 0, st>>>(fpv);
        PK_LAUNCH_CHECK();
      }
      float4 *rowa = reinterpret_cast<float4 *>(static_cast<char *>(workspace) + rows_off);
      float2 *rowph = reinterpret_cast<float2 *>(rowa + (size_t)g.d.n0 * g.d.n1);
      const int64_t nrows = (int64_t)g.d.n0 * g.d.n1;
      staged_rows_kernel<NS><<<(int)std::min<int64_t>((nrows + 255) / 256, 4 * sm_count()), 256, 0, st>>>(
          g, fpv, los[0], los[1], edges, rowa, rowph);
      PK_LAUNCH_CHECK();
      // shared memory: histograms, thresholds, kz tables, row buffers, the kz phase / window tables
      const size_t smem = align_up((size_t)L.nwarps * (g.nedges - 1) * NV * sizeof(float), 16) +
                          (size_t)((g.nedges + 3) & ~3) * sizeof(float) +
                          2 * (size_t)((g.d.nz + 3) & ~3) * sizeof(float) +
                          (size_t)L.nwarps * staged_row_bytes(g.d.nz) + ztable_bytes(g.d, NS, false, false);
      PK_REQUIRE(smem <= 227 * 1024, PK_ERR_RANGE, "mesh too large along the last axis for the fused pass");
      auto kernel = bin_interlaced_staged_kernel<NV, NS, PK_STAGED_MIN_CTAS>;
      PK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      int per_sm = 0;
      PK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, L.nwarps * 32, smem));
      if (per_sm < 1) per_sm = 1;
      // one wave of resident CTAs (at most the planned partial rows)
      blocks = (int)std::min<int64_t>(L.blocks, std::max<int64_t>(1, (int64_t)per_sm * sm_count() / nbatch));
      kernel<<<dim3(blocks, nbatch), L.nwarps * 32, smem, st>>>(g, d1, los[2], lc, zero_l0, edges, L.nwarps, partials,
                                                                fpv, rowa, rowph);
      PK_LAUNCH_CHECK();
      launch_finalize(st, partials, blocks, hist_len, NV, g.nedges - 1, 0, out, nullptr, nbatch);
      PK_LAUNCH_CHECK();
      return PK_OK;
    }
  }
#endif
  if (g.d.nz < PK_GLOBAL_FLAT_NZ) {
    if (NS <= 0 && !L.tab) {  // the flat kernel always tabulates kz
      L.smem += 2 * (size_t)((g.d.nz + 3) & ~3) * sizeof(float);
      PK_REQUIRE(L.smem <= 227 * 1024, PK_ERR_RANGE, "mesh too large along the last axis for the kz table");
    }
    constexpr int XA = NS > 0 ? XY_SMEM : XY_NONE, XB = NS > 0 ? XY_GLOBAL : XY_NONE;
    auto kernel = xy_smem ? bin_global_flat_kernel<NV, CROSS, EVEN, NS, FULL, XA>
                          : bin_global_flat_kernel<NV, CROSS, EVEN, NS, FULL, XB>;
    PK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
    int per_sm = 0;
    PK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, L.nwarps * 32, L.smem));
    if (per_sm < 1) per_sm = 1;
    // one wave of resident CTAs per mesh of the batch, the chunks split evenly over their warps
    const int64_t nchunks = (g.d.ncomplex() + 31) / 32;
    int64_t nb = std::min<int64_t>(L.blocks, std::max<int64_t>(1, (int64_t)per_sm * sm_count() / nbatch));
    const int64_t cpw = (nchunks + nb * L.nwarps - 1) / (nb * L.nwarps);
    nb = ((nchunks + cpw - 1) / cpw + L.nwarps - 1) / L.nwarps;
    blocks = (int)nb;
    kernel<<<dim3(blocks, nbatch), L.nwarps * 32, L.smem, st>>>(g, d1, d2, los[0], los[1], los[2], lc, zero_l0,
                                                               edges, L.nwarps, cpw, partials, fpv);
  } else {
    constexpr int MINB1 = NS > 0 ? PK_FUSED_MIN_CTAS : 4;
    constexpr int MINB2 = NS > 0 ? PK_FUSED_BATCH_MIN_CTAS : 4;
    constexpr int XA = NS > 0 ? XY_SMEM : XY_NONE, XB = NS > 0 ? XY_GLOBAL : XY_NONE;
    auto kernel = nbatch > 1 ? (xy_smem ? bin_global_kernel<NV, CROSS, EVEN, NS, FULL, MINB2, XA>
                                        : bin_global_kernel<NV, CROSS, EVEN, NS, FULL, MINB2, XB>)
                             : (xy_smem ? bin_global_kernel<NV, CROSS, EVEN, NS, FULL, MINB1, XA>
                                        : bin_global_kernel<NV, CROSS, EVEN, NS, FULL, MINB1, XB>);
    PK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
    kernel<<<dim3(L.blocks, nbatch), L.nwarps * 32, L.smem, st>>>(g, d1, d2, los[0], los[1], los[2], lc, zero_l0,
                                                                  edges, L.nwarps, L.tab, partials, fpv);
  }
  PK_LAUNCH_CHECK();
  launch_finalize(st, partials, blocks, hist_len, NV, g.nedges - 1, 0, out, nullptr, nbatch);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

// Dispatch a runtime value count (1..MAX_ELLS) to the compile-time kernels.
template <template <int> class OpT, class Fill>
static pk_status dispatch_nv(int nv, Fill fill, cudaStream_t s, const BinGeom &g,
                             const float *edges, bool rows, int accumulate, double *out,
                             void *workspace, size_t workspace_bytes) {
  switch (nv) {
#define PK_NV_CASE(N)                                                                   \
  case N: {                                                                             \
    OpT<N> op;                                                                          \
    fill(op);                                                                           \
    return launch_bins<N>(s, g, op, edges, rows, accumulate, out, nullptr, workspace,   \
                          workspace_bytes);                                             \
  }
    PK_NV_CASE(1) PK_NV_CASE(2) PK_NV_CASE(3) PK_NV_CASE(4) PK_NV_CASE(5) PK_NV_CASE(6)
    PK_NV_CASE(7) PK_NV_CASE(8) PK_NV_CASE(9)
#undef PK_NV_CASE
    default:
      set_error("unsupported number of multipoles %d", nv);
      return PK_ERR_INVALID;
  }
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
  g->sep = 0;
  g->shifted = 0;
  g->kshift[0] = g->kshift[1] = g->kshift[2] = 0.f;
  return PK_OK;
}

static pk_status make_shifted_geom(const int32_t meshsize[3], const float kfun[3], const float kshift[3], int nedges,
                                   float step, int backend, BinGeom *g) {
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, g);
  if (st) return st;
  PK_REQUIRE(kshift, PK_ERR_INVALID, "kshift is NULL");
  for (int a = 0; a < 3; ++a) {
    PK_REQUIRE(isfinite(kshift[a]), PK_ERR_INVALID, "kshift must be finite");
    g->kshift[a] = kshift[a];
  }
  g->shifted = 1;
  return PK_OK;
}

}  // namespace pk

using namespace pk;

extern "C" pk_status pk_bin_workspace_size(const int32_t meshsize[3], int nedges, int nvalues,
                                           size_t *bytes);

extern "C" pk_status pk_bin_batch_workspace_size(const int32_t meshsize[3], int nedges,
                                                 int nvalues, int nbatch, size_t *bytes) {
  PK_REQUIRE(nbatch >= 1, PK_ERR_INVALID, "nbatch must be >= 1");
  pk_status st = pk_bin_workspace_size(meshsize, nedges, nvalues, bytes);
  if (st) return st;
  *bytes *= (size_t)nbatch;
  return PK_OK;
}

extern "C" pk_status pk_bin_workspace_size(const int32_t meshsize[3], int nedges, int nvalues,
                                           size_t *bytes) {
  PK_REQUIRE(bytes, PK_ERR_INVALID, "bytes is NULL");
  Dims d;
  PK_REQUIRE(make_dims(meshsize, &d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(nedges >= 2 && nvalues >= 1 && nvalues <= MAX_ELLS, PK_ERR_INVALID,
             "invalid nedges / nvalues");
  size_t most = 0;
  for (int nv = 1; nv <= MAX_ELLS; ++nv) {  // launches pick their grid from nv
    for (size_t elem : {sizeof(double), sizeof(float)}) {  // float64 / float32 warp histograms
      BinLaunch L;
      if (!plan_bins(d, nedges, nv, &L, elem)) {
        PK_REQUIRE(nv > nvalues, PK_ERR_RANGE, "too many bins x values for the histograms");
        continue;
      }
      if (L.partial_bytes > most) most = L.partial_bytes;
    }
  }
  // plus the per-axis tables and the row table of the fused interlacing pass (up to 4 shifts)
  most = align_up(align_up(most) + xy_table_bytes(d, 4)) + staged_table_bytes(d, STAGED_MAX_SHIFTS);
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
  return launch_bins<2>((cudaStream_t)stream, g, ModesOp(), d_edges, true, 0, d_nmodes, d_ksum,
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
  return launch_bins<2>((cudaStream_t)stream, g, op, d_edges, true, 0, d_out, nullptr, workspace,
                        workspace_bytes);
}

extern "C" pk_status pk_bin_global_batch(void *stream, const void *delta1, const void *delta2,
                                         int nbatch, const int32_t meshsize[3], const float kfun[3],
                                         const float los[3], const float *d_edges, int nedges,
                                         float step, int backend, int nells, const int32_t *ells,
                                         double *d_out, void *workspace, size_t workspace_bytes);

// ------------------------------------------------------------ mode oversampling
// BinMesh2SpectrumPoles(mode_oversampling=s) (mesh2.py:48-61): every integer shift in
// [-s, s]^3 bins the modes by |k + shift| (Hermitian weights and the binned values of k
// itself unchanged); the operator averages the per-shift sums (mesh.py:2894-2895).  One call
// per shift, each accumulating into d_out when `accumulate`; bins are found per mode (the
// chunk walk), since |k + shift| is not monotone along a row.

extern "C" pk_status pk_bin_modes_shifted(void *stream, const int32_t meshsize[3], const float kfun[3],
                                          const float kshift[3], const float *d_edges, int nedges, float step,
                                          int backend, int accumulate, double *d_nmodes, double *d_ksum,
                                          void *workspace, size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_shifted_geom(meshsize, kfun, kshift, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(d_edges && d_nmodes && d_ksum, PK_ERR_INVALID, "null pointer");
  ModesOp op;
  op.shifted = 1;
  for (int a = 0; a < 3; ++a) op.kshift[a] = kshift[a];
  return launch_bins<2>((cudaStream_t)stream, g, op, d_edges, false, accumulate, d_nmodes, d_ksum, workspace,
                        workspace_bytes);
}

extern "C" pk_status pk_bin_mesh_shifted(void *stream, const void *value, const int32_t meshsize[3],
                                         const float kfun[3], const float kshift[3], const float *d_edges,
                                         int nedges, float step, int backend, int remove_zero, int accumulate,
                                         double *d_out, void *workspace, size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_shifted_geom(meshsize, kfun, kshift, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(value && d_edges && d_out, PK_ERR_INVALID, "null pointer");
  MeshOp op;
  op.v = (const float2 *)value;
  op.remove_zero = remove_zero;
  return launch_bins<2>((cudaStream_t)stream, g, op, d_edges, false, accumulate, d_out, nullptr, workspace,
                        workspace_bytes);
}

extern "C" pk_status pk_bin_global_shifted(void *stream, const void *delta1, const void *delta2,
                                           const int32_t meshsize[3], const float kfun[3], const float kshift[3],
                                           const float los[3], const float *d_edges, int nedges, float step,
                                           int backend, int nells, const int32_t *ells, int accumulate,
                                           double *d_out, void *workspace, size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_shifted_geom(meshsize, kfun, kshift, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(delta1 && d_edges && d_out && los && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nells >= 1 && nells <= MAX_ELLS, PK_ERR_INVALID, "nells must be in 1..%d", MAX_ELLS);
  for (int l = 0; l < nells; ++l)
    PK_REQUIRE(ells[l] >= 0 && ells[l] <= 8, PK_ERR_INVALID, "ell must be in 0..8");
  auto fill = [&](auto &op) {
    op.d1 = (const float2 *)delta1;
    op.d2 = (const float2 *)delta2;
    for (int a = 0; a < 3; ++a) op.los[a] = los[a];
    for (int l = 0; l < MAX_ELLS; ++l) op.ells[l] = l < nells ? ells[l] : 0;
  };
  return dispatch_nv<GlobalOp>(nells, fill, (cudaStream_t)stream, g, d_edges, false, accumulate, d_out,
                               workspace, workspace_bytes);
}

extern "C" pk_status pk_bin_global(void *stream, const void *delta1, const void *delta2,
                                   const int32_t meshsize[3], const float kfun[3],
                                   const float los[3], const float *d_edges, int nedges,
                                   float step, int backend, int nells, const int32_t *ells,
                                   double *d_out, void *workspace, size_t workspace_bytes) {
  return pk_bin_global_batch(stream, delta1, delta2, 1, meshsize, kfun, los, d_edges, nedges, step,
                             backend, nells, ells, d_out, workspace, workspace_bytes);
}

extern "C" pk_status pk_bin_global_batch(void *stream, const void *delta1, const void *delta2,
                                         int nbatch, const int32_t meshsize[3], const float kfun[3],
                                         const float los[3], const float *d_edges, int nedges,
                                         float step, int backend, int nells, const int32_t *ells,
                                         double *d_out, void *workspace, size_t workspace_bytes) {
  PK_REQUIRE(nbatch >= 1 && nbatch <= 65535, PK_ERR_INVALID, "nbatch must be in 1..65535");
  BinGeom g;
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(delta1 && d_edges && d_out && los && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nells >= 1 && nells <= MAX_ELLS, PK_ERR_INVALID, "nells must be in 1..%d", MAX_ELLS);
  for (int l = 0; l < nells; ++l)
    PK_REQUIRE(ells[l] >= 0 && ells[l] <= 8, PK_ERR_INVALID, "ell must be in 0..8");
  LegendreCoefs lc;
  lc.any_odd = 0;
  int zero_l0 = 0, max_ell = 0;
  for (int l = 0; l < MAX_ELLS; ++l) {
    const int ell = l < nells ? ells[l] : 0;
    legendre_coefs(ell, lc.c[l], &lc.odd[l]);
    lc.any_odd |= (l < nells) && lc.odd[l];
    if (l < nells && ell == 0) zero_l0 |= 1 << l;  // ell = 0 keeps the k = 0 mode
    if (l < nells && ell > max_ell) max_ell = ell;
  }
  const bool even = !lc.any_odd && max_ell <= 4;
  cudaStream_t cs = (cudaStream_t)stream;
  const float2 *a = (const float2 *)delta1, *b = (const float2 *)delta2;
  switch (nells * 4 + (b ? 2 : 0) + (even ? 1 : 0)) {
#define PK_GL_CASE(N)                                                                           \
  case 4 * N:                                                                                   \
    return launch_global<N, false, false>(cs, g, a, b, los, lc, zero_l0, d_edges, d_out,        \
                                          workspace, workspace_bytes, nbatch);                  \
  case 4 * N + 1:                                                                               \
    return launch_global<N, false, true>(cs, g, a, b, los, lc, zero_l0, d_edges, d_out,         \
                                         workspace, workspace_bytes, nbatch);                   \
  case 4 * N + 2:                                                                               \
    return launch_global<N, true, false>(cs, g, a, b, los, lc, zero_l0, d_edges, d_out,         \
                                         workspace, workspace_bytes, nbatch);                   \
  case 4 * N + 3:                                                                               \
    return launch_global<N, true, true>(cs, g, a, b, los, lc, zero_l0, d_edges, d_out,          \
                                        workspace, workspace_bytes, nbatch);
    PK_GL_CASE(1) PK_GL_CASE(2) PK_GL_CASE(3) PK_GL_CASE(4) PK_GL_CASE(5) PK_GL_CASE(6)
    PK_GL_CASE(7) PK_GL_CASE(8) PK_GL_CASE(9)
#undef PK_GL_CASE
  }
  set_error("unsupported number of multipoles %d", nells);
  return PK_ERR_INVALID;
}

extern "C" pk_status pk_bin_global_interlaced(void *stream, const void *shifted, int nbatch, int nshifts,
                                              int comp_order, const int32_t meshsize[3], const float kfun[3],
                                              const float los[3], const float *d_edges, int nedges, float step,
                                              int backend, int nells, const int32_t *ells, double *d_out,
                                              void *workspace, size_t workspace_bytes) {
  PK_REQUIRE(nbatch >= 1 && nbatch <= 65535, PK_ERR_INVALID, "nbatch must be in 1..65535");
  BinGeom g;
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(shifted && d_edges && d_out && los && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nells >= 1 && nells <= MAX_ELLS, PK_ERR_INVALID, "nells must be in 1..%d", MAX_ELLS);
  FourierParams fp;
  PK_REQUIRE(make_fourier_params(meshsize, nshifts, comp_order, backend, 0, 1.f, &fp), PK_ERR_INVALID,
             "invalid meshsize / nshifts (1..8) / comp_order (0..4)");
  LegendreCoefs lc;
  lc.any_odd = 0;
  int zero_l0 = 0, max_ell = 0;
  for (int l = 0; l < MAX_ELLS; ++l) {
    const int ell = l < nells ? ells[l] : 0;
    PK_REQUIRE(l >= nells || (ell >= 0 && ell <= 8), PK_ERR_INVALID, "ell must be in 0..8");
    legendre_coefs(ell, lc.c[l], &lc.odd[l]);
    lc.any_odd |= (l < nells) && lc.odd[l];
    if (l < nells && ell == 0) zero_l0 |= 1 << l;  // ell = 0 keeps the k = 0 mode
    if (l < nells && ell > max_ell) max_ell = ell;
  }
  PK_REQUIRE(!lc.any_odd && max_ell <= 4 && nells <= 3 && nshifts <= 4, PK_ERR_RANGE,
             "the fused pass takes up to 3 even multipoles (ell <= 4) and up to 4 shifts; "
             "combine with pk_interlace_compensate and bin with pk_bin_global instead");
  cudaStream_t cs = (cudaStream_t)stream;
  const float2 *a = (const float2 *)shifted;
  const bool full = backend == PK_BACKEND_JAXDECOMP;
  switch ((nells * 8 + nshifts) * 2 + (full ? 1 : 0)) {
#define PK_GI_CASE(N, S)                                                                          \
  case (N * 8 + S) * 2:                                                                           \
    return launch_global<N, false, true, S, false>(cs, g, a, nullptr, los, lc, zero_l0, d_edges,  \
                                                   d_out, workspace, workspace_bytes, nbatch, &fp); \
  case (N * 8 + S) * 2 + 1:                                                                       \
    return launch_global<N, false, true, S, true>(cs, g, a, nullptr, los, lc, zero_l0, d_edges,   \
                                                  d_out, workspace, workspace_bytes, nbatch, &fp);
#define PK_GI_N(N) PK_GI_CASE(N, 1) PK_GI_CASE(N, 2) PK_GI_CASE(N, 3) PK_GI_CASE(N, 4)
    PK_GI_N(1) PK_GI_N(2) PK_GI_N(3)
#undef PK_GI_N
#undef PK_GI_CASE
  }
  set_error("unsupported fused binning configuration");
  return PK_ERR_INVALID;
}

static pk_status make_sep_geom(const int32_t meshsize[3], const float cellsize[3], int nedges, float step,
                               BinGeom *g) {
  pk_status st = make_geom(meshsize, cellsize, nedges, step, PK_BACKEND_JAX, g);
  if (st) return st;
  g->sep = 1;
  g->d.nz = g->d.n2;  // the full real mesh
  return PK_OK;
}

extern "C" pk_status pk_bin_separation_workspace_size(const int32_t meshsize[3], int nedges, int nvalues,
                                                      size_t *bytes) {
  PK_REQUIRE(bytes && meshsize, PK_ERR_INVALID, "null pointer");
  Dims d;
  PK_REQUIRE(make_dims(meshsize, &d), PK_ERR_INVALID, "invalid meshsize");
  d.nz = d.n2;
  BinLaunch L;
  PK_REQUIRE(plan_bins(d, nedges, nvalues, &L), PK_ERR_RANGE, "too many bins x values (%d x %d)", nedges - 1,
             nvalues);
  *bytes = L.partial_bytes;
  return PK_OK;
}

extern "C" pk_status pk_bin_separation_modes(void *stream, const int32_t meshsize[3], const float cellsize[3],
                                             const float *d_edges, int nedges, float step, double *d_nmodes,
                                             double *d_ssum, void *workspace, size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_sep_geom(meshsize, cellsize, nedges, step, &g);
  if (st) return st;
  PK_REQUIRE(d_edges && d_nmodes && d_ssum, PK_ERR_INVALID, "null pointer");
  return launch_bins<2, ModesOp, true>((cudaStream_t)stream, g, ModesOp(), d_edges, true, 0, d_nmodes, d_ssum,
                                       workspace, workspace_bytes);
}

// Mode oversampling of BinMesh2CorrelationPoles (_make_edges2('real'), mesh2.py:48-61): the
// separations binned by |s + shift| (the chunk walk, which takes a shift), their values (and
// mu) from s; one call per shift, added (accumulate) and averaged by the caller.
static pk_status make_sep_shifted_geom(const int32_t meshsize[3], const float cellsize[3], const float sshift[3],
                                       int nedges, float step, BinGeom *g) {
  pk_status st = make_sep_geom(meshsize, cellsize, nedges, step, g);
  if (st) return st;
  PK_REQUIRE(sshift, PK_ERR_INVALID, "sshift is NULL");
  for (int a = 0; a < 3; ++a) {
    PK_REQUIRE(isfinite(sshift[a]), PK_ERR_INVALID, "sshift must be finite");
    g->kshift[a] = sshift[a];
  }
  g->shifted = 1;
  return PK_OK;
}

extern "C" pk_status pk_bin_separation_modes_shifted(void *stream, const int32_t meshsize[3],
                                                     const float cellsize[3], const float sshift[3],
                                                     const float *d_edges, int nedges, float step, int accumulate,
                                                     double *d_nmodes, double *d_ssum, void *workspace,
                                                     size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_sep_shifted_geom(meshsize, cellsize, sshift, nedges, step, &g);
  if (st) return st;
  PK_REQUIRE(d_edges && d_nmodes && d_ssum, PK_ERR_INVALID, "null pointer");
  ModesOp op;
  op.shifted = 1;
  for (int a = 0; a < 3; ++a) op.kshift[a] = sshift[a];
  return launch_bins<2>((cudaStream_t)stream, g, op, d_edges, false, accumulate, d_nmodes, d_ssum, workspace,
                        workspace_bytes);
}

extern "C" pk_status pk_bin_separation_global_shifted(void *stream, const float *value, const int32_t meshsize[3],
                                                      const float cellsize[3], const float sshift[3],
                                                      const float los[3], const float *d_edges, int nedges,
                                                      float step, int nells, const int32_t *ells, int accumulate,
                                                      double *d_out, void *workspace, size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_sep_shifted_geom(meshsize, cellsize, sshift, nedges, step, &g);
  if (st) return st;
  PK_REQUIRE(value && d_edges && d_out && los && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nells >= 1 && nells <= 3, PK_ERR_INVALID, "nells must be in 1..3");
  for (int l = 0; l < nells; ++l) PK_REQUIRE(ells[l] >= 0 && ells[l] <= 8, PK_ERR_INVALID, "ell must be in 0..8");
  cudaStream_t cs = (cudaStream_t)stream;
#define PK_SEPS_CASE(N)                                                                            \
  if (nells == N) {                                                                                \
    SepLegendreOp<N> op;                                                                           \
    op.v = value;                                                                                  \
    for (int a = 0; a < 3; ++a) op.los[a] = los[a];                                                \
    for (int l = 0; l < MAX_ELLS; ++l) op.ells[l] = l < nells ? ells[l] : 0;                       \
    return launch_bins<N>(cs, g, op, d_edges, false, accumulate, d_out, nullptr, workspace, workspace_bytes); \
  }
  PK_SEPS_CASE(1) PK_SEPS_CASE(2) PK_SEPS_CASE(3)
#undef PK_SEPS_CASE
  return PK_ERR_INVALID;
}

extern "C" pk_status pk_bin_separation_global(void *stream, const float *value, const int32_t meshsize[3],
                                              const float cellsize[3], const float los[3], const float *d_edges,
                                              int nedges, float step, int nells, const int32_t *ells,
                                              double *d_out, void *workspace, size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_sep_geom(meshsize, cellsize, nedges, step, &g);
  if (st) return st;
  PK_REQUIRE(value && d_edges && d_out && los && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nells >= 1 && nells <= 3, PK_ERR_INVALID, "nells must be in 1..3");
  for (int l = 0; l < nells; ++l) PK_REQUIRE(ells[l] >= 0 && ells[l] <= 8, PK_ERR_INVALID, "ell must be in 0..8");
  cudaStream_t cs = (cudaStream_t)stream;
#define PK_SEP_CASE(N)                                                                             \
  if (nells == N) {                                                                                \
    SepLegendreOp<N> op;                                                                           \
    op.v = value;                                                                                  \
    for (int a = 0; a < 3; ++a) op.los[a] = los[a];                                                \
    for (int l = 0; l < MAX_ELLS; ++l) op.ells[l] = l < nells ? ells[l] : 0;                       \
    return launch_bins<N, SepLegendreOp<N>, true>(cs, g, op, d_edges, true, 0, d_out, nullptr, workspace, \
                                                  workspace_bytes);                                \
  }
  PK_SEP_CASE(1) PK_SEP_CASE(2) PK_SEP_CASE(3)
#undef PK_SEP_CASE
  return PK_ERR_INVALID;
}

// ------------------------------------------------------------ window matrix
// compute_mesh2_spectrum_window, global line of sight, mesh input power (mesh2.py:1013-1133).
// Column (ell_in, [k_lo, k_hi)) of the window is the binned Re(A) L_ell(mu) of
//   A = N 1{k_lo <= |k| < k_hi} L_ell_in(mu)             (periodic box), or
//   A = r2c(Q c2r(N 1{k_lo <= |k| < k_hi} L_ell_in(mu)))  (selection Q = c2r(W1 W2*) / N),
// with |k| = sqrt((kx^2 + ky^2) + kz^2) and mu = k.los / |k| (|k| = 1 at k = 0) in float32.
// The reference bins Aell * (L_ell(mu) + L_ell(-mu)) for odd ell, which is zero term by term.

constexpr int WINDOW_MAX_COLUMNS = 16;

struct WindowColumns {
  float klo[WINDOW_MAX_COLUMNS], khi[WINDOW_MAX_COLUMNS];
};

__device__ __forceinline__ float window_mu(float kx, float ky, float kz, float k2, const float los[3],
                                           float *knorm) {
  const float num = __fadd_rn(__fadd_rn(__fmul_rn(kx, los[0]), __fmul_rn(ky, los[1])), __fmul_rn(kz, los[2]));
  *knorm = __fsqrt_rn(k2);
  return __fdiv_rn(num, k2 > 0.f ? *knorm : 1.f);
}

// ncol half-complex meshes (column c at out + c N_c): N 1{k_lo[c] <= |k| < k_hi[c]} L_ell_in(mu) + 0i.
__global__ void window_fill_kernel(Dims d, float kf0, float kf1, float kf2, float l0, float l1, float l2,
                                   int ellin, float scale, int ncol, WindowColumns cols, float2 *__restrict__ out) {
  const int64_t nc = d.ncomplex();
  const float los[3] = {l0, l1, l2};
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nc; q += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(q % d.nz);
    const int64_t row = q / d.nz;
    const int j = (int)(row % d.n1), i = (int)(row / d.n1);
    const float kx = kcoord(i, d.n0, kf0, false), ky = kcoord(j, d.n1, kf1, false);
    const float kz = kcoord(z, d.n2, kf2, true);
    const float k2 = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
    float knorm;
    const float mu = window_mu(kx, ky, kz, k2, los, &knorm);
    const float v = __fmul_rn(legendre(ellin, mu), scale);
    for (int c = 0; c < ncol; ++c) {
      const bool in = knorm >= cols.klo[c] && knorm < cols.khi[c];
      out[(int64_t)c * nc + q] = make_float2(in ? v : 0.f, 0.f);
    }
  }
}

// meshes[c N + q] *= q[q] for c < ncol (float4 when N is a multiple of 4).
__global__ void window_multiply_kernel(float *__restrict__ meshes, const float *__restrict__ qmesh, int64_t n,
                                       int ncol) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  if ((n & 3) == 0) {
    const int64_t n4 = n >> 2;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n4; t += stride) {
      const float4 w = reinterpret_cast<const float4 *>(qmesh)[t];
      for (int c = 0; c < ncol; ++c) {
        float4 *p = reinterpret_cast<float4 *>(meshes + (int64_t)c * n) + t;
        float4 v = *p;
        v.x *= w.x; v.y *= w.y; v.z *= w.z; v.w *= w.w;
        *p = v;
      }
    }
  } else {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
      const float w = qmesh[t];
      for (int c = 0; c < ncol; ++c) meshes[(int64_t)c * n + t] *= w;
    }
  }
}

// w Re(A) L_ell(mu) per mode, k = 0 dropped for every ell (_bin of the reference passes
// remove_zero=True); A formed from the column (periodic box), or read from v if set.
template <int N>
struct WindowOp {
  const float2 *v;
  float los[3];
  int ells[MAX_ELLS];
  int ellin;
  float klo, khi, scale;
  static constexpr int NV = N;
  __device__ void operator()(int64_t idx, int i, int j, int z, float kx, float ky, float kz, float k2, float w,
                             float out[NV]) const {
    float knorm;
    const float mu = window_mu(kx, ky, kz, k2, los, &knorm);
    float a;
    if (v) a = v[idx].x;
    else a = (knorm >= klo && knorm < khi) ? __fmul_rn(legendre(ellin, mu), scale) : 0.f;
    const bool zero = (i == 0 && j == 0 && z == 0);
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      const int ell = ells[l];
      out[l] = (zero || (ell & 1)) ? 0.f : __fmul_rn(__fmul_rn(a, legendre(ell, mu)), w);
    }
  }
};

// The same row for a mesh A (the selection-function columns): no |k| comparison is made, so
// mu^2 = (k.los)^2 / k^2 by a fast reciprocal and L_ell as Horner polynomials in mu^2 (odd
// ell: zero coefficients).
template <int N>
struct WindowMeshOp {
  const float2 *v;
  float los[3];
  float c[MAX_ELLS][5];
  static constexpr int NV = N;
  __device__ void operator()(int64_t idx, int i, int j, int z, float kx, float ky, float kz, float k2, float w,
                             float out[NV]) const {
    const float num = (kx * los[0] + ky * los[1]) + kz * los[2];
    const float rk2 = k2 > 0.f ? __fdividef(1.f, k2) : 0.f;
    const float mu2 = num * num * rk2;
    const float a = (i == 0 && j == 0 && z == 0) ? 0.f : v[idx].x * w;
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      float L = c[l][4];
      L = L * mu2 + c[l][3];
      L = L * mu2 + c[l][2];
      L = L * mu2 + c[l][1];
      L = L * mu2 + c[l][0];
      out[l] = a * L;
    }
  }
};

// Periodic window, every column of an ell_in at once: binned on the union of the output and
// input edges, each merged interval lies in one (output bin, input bin) pair, so value l is
// w N L_ell_in[l](mu) L_ell[l](mu) (the per-column product, same rounding) for pairs
// (ell[l], ell_in[l]).
template <int N>
struct WindowPairsOp {
  float los[3];
  int ell[MAX_ELLS], ellin[MAX_ELLS];
  float scale;
  static constexpr int NV = N;
  __device__ void operator()(int64_t, int i, int j, int z, float kx, float ky, float kz, float k2, float w,
                             float out[NV]) const {
    float knorm;
    const float mu = window_mu(kx, ky, kz, k2, los, &knorm);
    const bool zero = (i == 0 && j == 0 && z == 0);
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      const float a = __fmul_rn(legendre(ellin[l], mu), scale);
      out[l] = (zero || (ell[l] & 1)) ? 0.f : __fmul_rn(__fmul_rn(a, legendre(ell[l], mu)), w);
    }
  }
};

template <int MASK, bool CROSS>
static pk_status launch_firstpoint_block(cudaStream_t s, const BinGeom &g, const float2 *a0, const float2 *b0,
                                         const float2 *f, const float *edges, const RowMap &map, double *out,
                                         void *workspace, size_t workspace_bytes) {
  constexpr int NV = ylm_mask_ells(MASK) + 1;
  BinLaunch L;
  PK_REQUIRE(plan_bins(g.d, g.nedges, NV, &L), PK_ERR_RANGE,
             "too many bins x values (%d x %d) for the shared-memory histograms", g.nedges - 1, NV);
  auto kernel = bin_firstpoint_kernel<MASK, CROSS>;
  PK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
  int per_sm = 0;
  PK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, L.nwarps * 32, L.smem));
  if (per_sm < 1) per_sm = 1;
  // one wave of resident CTAs, the chunks split evenly over their warps
  const int64_t nchunks = (g.d.ncomplex() + 31) / 32;
  int64_t blocks = std::min<int64_t>(L.blocks, (int64_t)per_sm * sm_count());
  const int64_t cpw = (nchunks + blocks * L.nwarps - 1) / (blocks * L.nwarps);
  blocks = ((nchunks + cpw - 1) / cpw + L.nwarps - 1) / L.nwarps;
  const int hist_len = (g.nedges - 1) * NV;
  const size_t need = (size_t)blocks * hist_len * sizeof(double);
  PK_REQUIRE(workspace && workspace_bytes >= need, PK_ERR_WORKSPACE,
             "binning workspace too small: need %zu bytes, got %zu", need, workspace_bytes);
  double *partials = static_cast<double *>(workspace);
  kernel<<<(int)blocks, L.nwarps * 32, L.smem, s>>>(g, a0, b0, f, g.d.ncomplex(), edges, L.nwarps, L.tab, cpw,
                                                    partials);
  PK_LAUNCH_CHECK();
  launch_finalize(s, partials, (int)blocks, hist_len, NV, g.nedges - 1, 1, out, nullptr, 1, map);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

static pk_status dispatch_firstpoint_block(int mask, cudaStream_t s, const BinGeom &g, const float2 *a0,
                                           const float2 *b0, const float2 *f, const float *edges,
                                           const RowMap &map, double *out, void *workspace,
                                           size_t workspace_bytes) {
#define PK_FP_BLOCK_CASE(M)                                                                            \
  if (mask == (M))                                                                                     \
    return b0 ? launch_firstpoint_block<M, true>(s, g, a0, b0, f, edges, map, out, workspace, workspace_bytes) \
              : launch_firstpoint_block<M, false>(s, g, a0, b0, f, edges, map, out, workspace, workspace_bytes);
  PK_YLM_MASKS(PK_FP_BLOCK_CASE)
#undef PK_FP_BLOCK_CASE
  set_error("no first-point kernel for term mask 0x%x", mask);
  return PK_ERR_INVALID;
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
  for (int t = 0; t < nterms; ++t)
    PK_REQUIRE(term_ell[t] >= 0 && term_ell[t] <= YLM_LMAX && term_m[t] >= -term_ell[t] &&
                   term_m[t] <= term_ell[t],
               PK_ERR_INVALID, "invalid (ell, m)");
  // whole ells (every m, in order) and distinct output ells: the compiled per-mask kernel
  const int mask = ylm_terms_mask(nterms, term_ell, term_m);
  bool distinct = true;
  for (int l = 0; l < nells; ++l)
    for (int q = 0; q < l; ++q) distinct &= ells[l] != ells[q];
  if (nterms > 0 && mask && ylm_mask_compiled(mask) && distinct) {
    RowMap map{};
    map.n = 1;
    auto row_of = [&](int ell) {
      for (int l = 0; l < nells; ++l)
        if (ells[l] == ell) return l;
      return -1;
    };
    map.row[0] = include_ell0 ? row_of(0) : -1;
    int q = 1;
    for (int ell = 1; ell <= YLM_LMAX; ++ell)
      if ((mask >> ell) & 1) map.row[q++] = row_of(ell);
    cudaStream_t cs = (cudaStream_t)stream;
    if (!accumulate) PK_CUDA(cudaMemsetAsync(d_out, 0, (size_t)nells * (nedges - 1) * sizeof(double), cs));
    return dispatch_firstpoint_block(mask, cs, g, (const float2 *)a0, (const float2 *)b0, (const float2 *)f,
                                     d_edges, map, d_out, workspace, workspace_bytes);
  }
  const int64_t stride = g.d.ncomplex();
  auto fill = [&](auto &op) {
    op.a0 = (const float2 *)a0;
    op.b0 = (const float2 *)b0;
    op.f = (const float2 *)f;
    op.fstride = stride;
    op.nterms = nterms;
    for (int t = 0; t < MAX_FP_TERMS; ++t) {
      op.term_ell[t] = t < nterms ? term_ell[t] : -1;
      op.term_m[t] = t < nterms ? term_m[t] : 0;
    }
    for (int l = 0; l < MAX_ELLS; ++l) op.ells[l] = l < nells ? ells[l] : 0;
    op.include_ell0 = include_ell0;
  };
  return dispatch_nv<FirstPointOp>(nells, fill, (cudaStream_t)stream, g, d_edges, false,
                                   accumulate, d_out, workspace, workspace_bytes);
}

extern "C" pk_status pk_bin_firstpoint_shifted(void *stream, const void *a0, const void *b0, const void *f,
                                               int nterms, const int32_t *term_ell, const int32_t *term_m,
                                               const int32_t meshsize[3], const float kfun[3],
                                               const float kshift[3], const float *d_edges, int nedges, float step,
                                               int backend, int nells, const int32_t *ells, int include_ell0,
                                               int accumulate, double *d_out, void *workspace,
                                               size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_shifted_geom(meshsize, kfun, kshift, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(a0 && d_edges && d_out && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nterms >= 0 && nterms <= MAX_FP_TERMS, PK_ERR_INVALID, "nterms must be in 0..%d",
             MAX_FP_TERMS);
  PK_REQUIRE(nterms == 0 || (f && term_ell && term_m), PK_ERR_INVALID, "null term arrays");
  PK_REQUIRE(nells >= 1 && nells <= MAX_ELLS, PK_ERR_INVALID, "nells must be in 1..%d", MAX_ELLS);
  for (int t = 0; t < nterms; ++t)
    PK_REQUIRE(term_ell[t] >= 0 && term_ell[t] <= YLM_LMAX && term_m[t] >= -term_ell[t] &&
                   term_m[t] <= term_ell[t],
               PK_ERR_INVALID, "invalid (ell, m)");
  const int64_t stride = g.d.ncomplex();
  auto fill = [&](auto &op) {
    op.a0 = (const float2 *)a0;
    op.b0 = (const float2 *)b0;
    op.f = (const float2 *)f;
    op.fstride = stride;
    op.nterms = nterms;
    for (int t = 0; t < MAX_FP_TERMS; ++t) {
      op.term_ell[t] = t < nterms ? term_ell[t] : -1;
      op.term_m[t] = t < nterms ? term_m[t] : 0;
    }
    for (int l = 0; l < MAX_ELLS; ++l) op.ells[l] = l < nells ? ells[l] : 0;
    op.include_ell0 = include_ell0;
  };
  return dispatch_nv<FirstPointOp>(nells, fill, (cudaStream_t)stream, g, d_edges, false, accumulate, d_out,
                                   workspace, workspace_bytes);
}

// ------------------------------------------------------------ allocation-free variant
// Some callers cannot allocate device memory at the point of the call: code running
// inside a host callback or a foreign runtime that owns the allocator (an XLA custom
// call without a scratch operand, a plugin loaded by a host that forbids cudaMalloc after
// start-up).  pk_bin_global_noalloc takes its scratch (the per-CTA partial histograms of
// the global-los binning) from this fixed array instead of a caller workspace.
//
// - The array is NOALLOC_SCRATCH_BYTES = 16 MiB; every GPU that loads the library holds
//   it until the process exits.
// - Host code cannot use the symbol as a device address; the address is looked up per
//   device, with that device current, by cudaGetSymbolAddress.  The first call on a device
//   does this set-up, so make that first call before any stream capture.  Later calls on a
//   stream that is not capturing look the address up again (it is cheap), so a context
//   that was destroyed and recreated (cudaDeviceReset) never leaves a stale address behind;
//   a call on a capturing stream reuses the address of the last call on that device.
// - Every call shares the array.  Each call overwrites all the partial rows it reads, so
//   nothing needs clearing between calls, but calls that overlap on the GPU (different
//   streams, or several host threads) race on it.
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

static pk_status noalloc_scratch(cudaStream_t stream, void **out) {
  static std::mutex lock;
  static void *address[256] = {};
  int dev = 0;
  PK_CUDA(cudaGetDevice(&dev));
  PK_REQUIRE(dev >= 0 && dev < 256, PK_ERR_RANGE, "device index %d out of range", dev);
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &capture) != cudaSuccess) {
    (void)cudaGetLastError();  // e.g. the legacy stream while another stream captures
    capture = cudaStreamCaptureStatusActive;
  }
  std::lock_guard<std::mutex> guard(lock);
  if (!address[dev] || capture == cudaStreamCaptureStatusNone) {
    void *p = nullptr;
    PK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    address[dev] = p;
  }
  *out = address[dev];
  return PK_OK;
}

extern "C" pk_status pk_bin_global_noalloc(void *stream, const void *delta1, const void *delta2,
                                           const int32_t meshsize[3], const float kfun[3],
                                           const float los[3], const float *d_edges, int nedges,
                                           float step, int backend, int nells, const int32_t *ells,
                                           double *d_out) {
  Dims d;
  PK_REQUIRE(make_dims(meshsize, &d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(nedges >= 2, PK_ERR_INVALID, "need at least 2 edges");
  PK_REQUIRE(nells >= 1 && nells <= MAX_ELLS, PK_ERR_INVALID, "nells must be in 1..%d", MAX_ELLS);
  BinLaunch L;
  PK_REQUIRE(plan_bins(d, nedges, nells, &L, sizeof(float)), PK_ERR_RANGE,
             "too many bins x multipoles (%d x %d)", nedges - 1, nells);
  PK_REQUIRE(L.partial_bytes <= NOALLOC_SCRATCH_BYTES, PK_ERR_RANGE,
             "pk_bin_global_noalloc: %d bins x %d multipoles need %zu bytes of scratch, more than "
             "the fixed %zu; use pk_bin_global with a workspace",
             nedges - 1, nells, L.partial_bytes, NOALLOC_SCRATCH_BYTES);
  void *scratch = nullptr;
  pk_status st = noalloc_scratch((cudaStream_t)stream, &scratch);
  if (st) return st;
  return pk_bin_global(stream, delta1, delta2, meshsize, kfun, los, d_edges, nedges, step, backend,
                       nells, ells, d_out, scratch, NOALLOC_SCRATCH_BYTES);
}

// ------------------------------------------------------------------ adjoints
// Backward of the binned estimators.  Given per-bin cotangent coefficients
// coef[l][b] (dLoss/dnum_l[b] times the estimator's per-bin factor, e.g. (2l+1)/nmodes),
// each stored mode gets G_l(k) = w_k coef[l][b(k)] (ell > 0: 0 at k = 0) and the
// conjugate cotangent (dL/dRe + i dL/dIm) of the mesh(es) it was computed from.  With
// for_c2r the cotangent is divided by the C2R weight w' (2 off the self-conjugate
// planes) and Hermitian-symmetrised on the kz = 0 / N/2 planes, so that an unnormalised
// C2R of it is the cotangent of the real mesh the modes were transformed from.

constexpr int ADJ_MAX_KSHIFTS = 125;  // mode_oversampling <= 2: (2 s + 1)^3 shifts

struct AdjGeom {
  BinGeom g;
  int nbins;
  int nells;
  int ells[MAX_ELLS];
  LegendreCoefs lc;
  float los[3];
  float e0, inv_step;
  int for_c2r;
  int nkshift;  // mode oversampling: the k shifts of the forward's bins (0: none)
  float kshift[ADJ_MAX_KSHIFTS][3];
};

// Bin index of a stored mode (thresholds in a global table).
__device__ __forceinline__ int adj_bin(const AdjGeom &a, const float *thr, float k2) {
  return bin_from_k2(thr, a.g.nedges, a.e0, a.inv_step, k2);
}

// Mode oversampling (mesh2.py:48-61): the forward averages the sums of the shifted binnings
// (the bin of |k + shift|, shifted_k2's float32 expression), so a mode's cotangent coefficient
// for multipole row l is the mean over the shifts of coef[l][b_s - 1]; false when no shift puts
// the mode in a bin.
__device__ __forceinline__ bool adj_shifted_coefs(const AdjGeom &a, const float *thr, const float *coef, float kx,
                                                  float ky, float kz, float (&csum)[MAX_ELLS]) {
#pragma unroll
  for (int l = 0; l < MAX_ELLS; ++l) csum[l] = 0.f;
  bool any = false;
  for (int q = 0; q < a.nkshift; ++q) {
    const float x = __fadd_rn(kx, a.kshift[q][0]), y = __fadd_rn(ky, a.kshift[q][1]), z = __fadd_rn(kz, a.kshift[q][2]);
    const float k2s = __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
    const int b = adj_bin(a, thr, k2s);
    if (b < 1 || b > a.nbins) continue;
    any = true;
#pragma unroll
    for (int l = 0; l < MAX_ELLS; ++l)
      if (l < a.nells) csum[l] += coef[(size_t)l * a.nbins + (b - 1)];
  }
  const float inv = 1.f / (float)a.nkshift;
#pragma unroll
  for (int l = 0; l < MAX_ELLS; ++l) csum[l] *= inv;
  return any;
}

__device__ __forceinline__ float c2r_weight(const BinGeom &g, int z) {
  return (z == 0 || ((g.d.n2 % 2) == 0 && z == g.d.nz - 1)) ? 1.f : 2.f;
}

__global__ void thresholds_kernel(const float *__restrict__ edges, int nedges,
                                  float *__restrict__ thr) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nedges; i += gridDim.x * blockDim.x)
    thr[i] = sqrt_threshold(edges[i]);
}

// global line of sight: gbar_k = 2 G_k delta_k, G_k = w_k sum_l coef_l[b] L_l(mu)
template <bool SHIFTED>
__device__ __forceinline__ float2 global_adj_mode(const AdjGeom &a, const float *thr,
                                                  const float *coef, const float2 *delta, int i,
                                                  int j, int z) {
  const BinGeom &g = a.g;
  const float kx = kcoord(i, g.d.n0, g.kfun[0], false);
  const float ky = kcoord(j, g.d.n1, g.kfun[1], false);
  const float kz = kz_coord(g, z);
  const float k2 = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
  int b = 1;
  float csum[MAX_ELLS];
  if (SHIFTED) {
    if (!adj_shifted_coefs(a, thr, coef, kx, ky, kz, csum)) return make_float2(0.f, 0.f);
  } else {
    b = adj_bin(a, thr, k2);
    if (b < 1 || b > a.nbins) return make_float2(0.f, 0.f);
  }
  const float num = (kx * a.los[0] + ky * a.los[1]) + kz * a.los[2];
  const float rk2 = k2 > 0.f ? 1.f / k2 : 0.f;
  const float mu2 = num * num * rk2;
  const float mu = num * sqrtf(rk2);
  const bool zero = (i == 0 && j == 0 && z == 0);
  float G = 0.f;
  for (int l = 0; l < a.nells; ++l) {
    if ((a.ells[l] > 0 && zero) || a.lc.odd[l]) continue;  // odd ell of an auto spectrum is 0
    float L = a.lc.c[l][4];
    L = L * mu2 + a.lc.c[l][3];
    L = L * mu2 + a.lc.c[l][2];
    L = L * mu2 + a.lc.c[l][1];
    L = L * mu2 + a.lc.c[l][0];
    if (a.lc.odd[l]) L *= mu;  // odd multipoles bin Im(A): handled by the caller's coef sign
    G += (SHIFTED ? csum[l] : coef[(size_t)l * a.nbins + (b - 1)]) * L;
  }
  G *= mode_weight(g, z);
  const float2 d = delta[((int64_t)i * g.d.n1 + j) * g.d.nz + z];
  return make_float2(2.f * G * d.x, 2.f * G * d.y);
}

template <bool SHIFTED>
__global__ void global_adjoint_kernel(AdjGeom a, const float *__restrict__ thr,
                                      const float *__restrict__ coef,
                                      const float2 *__restrict__ delta,
                                      float2 *__restrict__ out) {
  const BinGeom &g = a.g;
  const int64_t total = g.d.ncomplex();
  const bool even = (g.d.n2 % 2) == 0;
  const int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  IndexWalker3 w(start, stride, g.d.n1, g.d.nz);
  for (int64_t idx = start; idx < total; idx += stride, w.next()) {
    const int i = w.i, j = w.j, z = w.k;
    float2 v = global_adj_mode<SHIFTED>(a, thr, coef, delta, i, j, z);
    if (a.for_c2r) {
      if (z == 0 || (even && z == g.d.nz - 1)) {
        const float2 m = global_adj_mode<SHIFTED>(a, thr, coef, delta, (g.d.n0 - i) % g.d.n0,
                                                  (g.d.n1 - j) % g.d.n1, z);
        v = make_float2(0.5f * (v.x + m.x), 0.5f * (v.y - m.y));
      } else {
        v = make_float2(0.5f * v.x, 0.5f * v.y);
      }
    }
    out[idx] = v;
  }
}

// first point: per mode the cotangents of A0 and of each F_j in the batch.
struct FPAdj {
  int nterms;
  int term_ell[MAX_FP_TERMS];
  int term_m[MAX_FP_TERMS];
  int term_l[MAX_FP_TERMS];  // index of the term's ell in ells
};

template <bool SHIFTED>
__device__ __forceinline__ void fp_adj_mode(const AdjGeom &a, const FPAdj &t, const float *thr,
                                            const float *coef, const float2 *a0, const float2 *f,
                                            int i, int j, int z, float2 *ga0, float2 *gf) {
  const BinGeom &g = a.g;
  const float kx = kcoord(i, g.d.n0, g.kfun[0], false);
  const float ky = kcoord(j, g.d.n1, g.kfun[1], false);
  const float kz = kz_coord(g, z);
  const float k2 = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
  const int64_t idx = ((int64_t)i * g.d.n1 + j) * g.d.nz + z;
  const int64_t stride = g.d.ncomplex();
  *ga0 = make_float2(0.f, 0.f);
  for (int q = 0; q < t.nterms; ++q) gf[q] = make_float2(0.f, 0.f);
  int b = 1;
  float csum[MAX_ELLS];
  if (SHIFTED) {
    if (!adj_shifted_coefs(a, thr, coef, kx, ky, kz, csum)) return;
  } else {
    b = adj_bin(a, thr, k2);
    if (b < 1 || b > a.nbins) return;
  }
  const bool zero = (i == 0 && j == 0 && z == 0);
  const float w = mode_weight(g, z);
  const float rn = k2 > 0.f ? rsqrtf(k2) : 0.f;
  const float xh = kx * rn, yh = ky * rn, zh = kz * rn;
  const float2 A = a0[idx];
  float2 acc = make_float2(0.f, 0.f);
  for (int l = 0; l < a.nells; ++l)
    if (a.ells[l] == 0) {  // ell = 0: |A0|^2 -> 2 G0 A0
      const float G0 = w * (SHIFTED ? csum[l] : coef[(size_t)l * a.nbins + (b - 1)]);
      acc.x += 2.f * G0 * A.x;
      acc.y += 2.f * G0 * A.y;
    }
  if (!zero)
    for (int q = 0; q < t.nterms; ++q) {
      const int l = t.term_l[q];
      const float G = w * (SHIFTED ? csum[l] : coef[(size_t)l * a.nbins + (b - 1)]);
      const float y = ylm_eval(t.term_ell[q], t.term_m[q], xh, yh, zh);
      const float2 F = f[(int64_t)q * stride + idx];
      const float gy = G * y;
      if (t.term_ell[q] & 1) {  // odd ell bins Im(conj(S) A0) = Re(conj(i S) A0) = Re(S conj(-i A0))
        acc.x -= gy * F.y;      // d/dA0 = G i S
        acc.y += gy * F.x;
        gf[q] = make_float2(gy * A.y, -gy * A.x);  // d/dF = G Y (-i A0)
      } else {
        acc.x += gy * F.x;  // d/dA0 of G Re(conj(S) A0) = G S
        acc.y += gy * F.y;
        gf[q] = make_float2(gy * A.x, gy * A.y);  // d/dF of G Re(S conj(A0)) = G Y A0
      }
    }
  *ga0 = acc;
}

template <bool SHIFTED>
__global__ void firstpoint_adjoint_kernel(AdjGeom a, FPAdj t, const float *__restrict__ thr,
                                          const float *__restrict__ coef,
                                          const float2 *__restrict__ a0,
                                          const float2 *__restrict__ f,
                                          float2 *__restrict__ out_a0, int accumulate_a0,
                                          float2 *__restrict__ out_f) {
  const BinGeom &g = a.g;
  const int64_t total = g.d.ncomplex();
  const bool even = (g.d.n2 % 2) == 0;
  float2 gf[MAX_FP_TERMS], gfm[MAX_FP_TERMS];
  const int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  IndexWalker3 w(start, stride, g.d.n1, g.d.nz);
  for (int64_t idx = start; idx < total; idx += stride, w.next()) {
    const int i = w.i, j = w.j, z = w.k;
    float2 ga0;
    fp_adj_mode<SHIFTED>(a, t, thr, coef, a0, f, i, j, z, &ga0, gf);
    const bool plane = z == 0 || (even && z == g.d.nz - 1);
    if (a.for_c2r) {
      if (plane) {
        float2 ga0m;
        fp_adj_mode<SHIFTED>(a, t, thr, coef, a0, f, (g.d.n0 - i) % g.d.n0, (g.d.n1 - j) % g.d.n1, z,
                             &ga0m, gfm);
        if (a.for_c2r == 1) ga0 = make_float2(0.5f * (ga0.x + ga0m.x), 0.5f * (ga0.y - ga0m.y));
        for (int q = 0; q < t.nterms; ++q)
          gf[q] = make_float2(0.5f * (gf[q].x + gfm[q].x), 0.5f * (gf[q].y - gfm[q].y));
      } else {
        if (a.for_c2r == 1) ga0 = make_float2(0.5f * ga0.x, 0.5f * ga0.y);
        for (int q = 0; q < t.nterms; ++q) gf[q] = make_float2(0.5f * gf[q].x, 0.5f * gf[q].y);
      }
    }
    if (out_a0) {
      if (accumulate_a0) {
        const float2 o = out_a0[idx];
        out_a0[idx] = make_float2(o.x + ga0.x, o.y + ga0.y);
      } else {
        out_a0[idx] = ga0;
      }
    }
    for (int q = 0; q < t.nterms; ++q) out_f[(int64_t)q * total + idx] = gf[q];
  }
}

// firstpoint_adjoint_kernel for whole-ell term blocks (mask MASK): the same per-mode
// arithmetic with every term at a fixed register index and Y_lm as compile-time polynomials.
struct FPAdjRows {
  int row[YLM_LMAX + 1];  // row of each ell of the mask in ells (coef rows)
};

template <int ELL, int M, int T, int NT>
__device__ __forceinline__ void fp_adj_terms(float G, float x, float y, float z, float2 A,
                                             const float2 *__restrict__ f, int64_t stride, int64_t idx,
                                             float2 &acc, float2 (&gf)[NT]) {
  const float gy = G * ylm_eval(ELL, M, x, y, z);
  const float2 F = f[(int64_t)T * stride + idx];
  if constexpr (ELL & 1) {  // odd ell: Im(conj(S) A0); d/dA0 = G i S, d/dF = G Y (-i A0)
    acc.x -= gy * F.y;
    acc.y += gy * F.x;
    gf[T] = make_float2(gy * A.y, -gy * A.x);
  } else {
    acc.x += gy * F.x;  // d/dA0 of G Re(conj(S) A0) = G S
    acc.y += gy * F.y;
    gf[T] = make_float2(gy * A.x, gy * A.y);  // d/dF of G Re(S conj(A0)) = G Y A0
  }
  if constexpr (M < ELL) fp_adj_terms<ELL, M + 1, T + 1>(G, x, y, z, A, f, stride, idx, acc, gf);
}

template <int MASK, int ELL, int T, int NT>
__device__ __forceinline__ void fp_adj_ells(const FPAdjRows &r, const float *__restrict__ coef, int nbins, int b,
                                            float w, float x, float y, float z, float2 A,
                                            const float2 *__restrict__ f, int64_t stride, int64_t idx, float2 &acc,
                                            float2 (&gf)[NT]) {
  if constexpr (ELL <= YLM_LMAX) {
    if constexpr ((MASK >> ELL) & 1) {
      const float G = w * coef[(size_t)r.row[ELL] * nbins + (b - 1)];
      fp_adj_terms<ELL, -ELL, T>(G, x, y, z, A, f, stride, idx, acc, gf);
      fp_adj_ells<MASK, ELL + 1, T + 2 * ELL + 1>(r, coef, nbins, b, w, x, y, z, A, f, stride, idx, acc, gf);
    } else {
      fp_adj_ells<MASK, ELL + 1, T>(r, coef, nbins, b, w, x, y, z, A, f, stride, idx, acc, gf);
    }
  }
}

template <int MASK, int NT>
__device__ __forceinline__ void fp_adj_block_mode(const AdjGeom &a, const FPAdjRows &r, const float *thr,
                                                  const float *coef, const float2 *__restrict__ a0,
                                                  const float2 *__restrict__ f, int i, int j, int z, float2 &ga0,
                                                  float2 (&gf)[NT]) {
  const BinGeom &g = a.g;
  const float kx = kcoord(i, g.d.n0, g.kfun[0], false);
  const float ky = kcoord(j, g.d.n1, g.kfun[1], false);
  const float kz = kz_coord(g, z);
  const float k2 = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
  const int b = adj_bin(a, thr, k2);
  const int64_t idx = ((int64_t)i * g.d.n1 + j) * g.d.nz + z;
  ga0 = make_float2(0.f, 0.f);
#pragma unroll
  for (int q = 0; q < NT; ++q) gf[q] = make_float2(0.f, 0.f);
  if (b < 1 || b > a.nbins) return;
  const bool zero = (i == 0 && j == 0 && z == 0);
  const float w = mode_weight(g, z);
  const float rn = k2 > 0.f ? rsqrtf(k2) : 0.f;
  const float2 A = a0[idx];
  float2 acc = make_float2(0.f, 0.f);
  for (int l = 0; l < a.nells; ++l)
    if (a.ells[l] == 0) {  // ell = 0: |A0|^2 -> 2 G0 A0
      const float G0 = w * coef[(size_t)l * a.nbins + (b - 1)];
      acc.x += 2.f * G0 * A.x;
      acc.y += 2.f * G0 * A.y;
    }
  if (!zero)
    fp_adj_ells<MASK, 0, 0>(r, coef, a.nbins, b, w, kx * rn, ky * rn, kz * rn, A, f, g.d.ncomplex(), idx, acc, gf);
  ga0 = acc;
}

template <int MASK>
__global__ void __launch_bounds__(256) firstpoint_adjoint_block_kernel(
    AdjGeom a, FPAdjRows r, const float *__restrict__ thr, const float *__restrict__ coef,
    const float2 *__restrict__ a0, const float2 *__restrict__ f, float2 *__restrict__ out_a0, int accumulate_a0,
    float2 *__restrict__ out_f) {
  constexpr int NT = ylm_mask_terms(MASK);
  const BinGeom &g = a.g;
  const int64_t total = g.d.ncomplex();
  const bool even = (g.d.n2 % 2) == 0;
  const int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  IndexWalker3 w(start, stride, g.d.n1, g.d.nz);
  for (int64_t idx = start; idx < total; idx += stride, w.next()) {
    const int i = w.i, j = w.j, z = w.k;
    float2 ga0, gf[NT];
    fp_adj_block_mode<MASK>(a, r, thr, coef, a0, f, i, j, z, ga0, gf);
    if (a.for_c2r) {
      if (z == 0 || (even && z == g.d.nz - 1)) {
        float2 ga0m, gfm[NT];
        fp_adj_block_mode<MASK>(a, r, thr, coef, a0, f, (g.d.n0 - i) % g.d.n0, (g.d.n1 - j) % g.d.n1, z, ga0m,
                                gfm);
        if (a.for_c2r == 1) ga0 = make_float2(0.5f * (ga0.x + ga0m.x), 0.5f * (ga0.y - ga0m.y));
#pragma unroll
        for (int q = 0; q < NT; ++q) gf[q] = make_float2(0.5f * (gf[q].x + gfm[q].x), 0.5f * (gf[q].y - gfm[q].y));
      } else {
        if (a.for_c2r == 1) ga0 = make_float2(0.5f * ga0.x, 0.5f * ga0.y);
#pragma unroll
        for (int q = 0; q < NT; ++q) gf[q] = make_float2(0.5f * gf[q].x, 0.5f * gf[q].y);
      }
    }
    if (out_a0) {
      if (accumulate_a0) {
        const float2 o = out_a0[idx];
        out_a0[idx] = make_float2(o.x + ga0.x, o.y + ga0.y);
      } else {
        out_a0[idx] = ga0;
      }
    }
#pragma unroll
    for (int q = 0; q < NT; ++q) __stcs(out_f + (int64_t)q * total + idx, gf[q]);
  }
}

static pk_status make_adj(const int32_t meshsize[3], const float kfun[3], int nedges, float step,
                          int backend, int nells, const int32_t *ells, const float *d_edges,
                          int for_c2r, AdjGeom *a) {
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, &a->g);
  if (st) return st;
  PK_REQUIRE(d_edges && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nells >= 1 && nells <= MAX_ELLS, PK_ERR_INVALID, "nells must be in 1..%d", MAX_ELLS);
  a->nbins = nedges - 1;
  a->nells = nells;
  a->lc.any_odd = 0;
  for (int l = 0; l < MAX_ELLS; ++l) {
    a->ells[l] = l < nells ? ells[l] : 0;
    PK_REQUIRE(l >= nells || (ells[l] >= 0 && ells[l] <= 8), PK_ERR_INVALID, "ell must be in 0..8");
    legendre_coefs(a->ells[l], a->lc.c[l], &a->lc.odd[l]);
  }
  a->e0 = 0.f;  // refined on the device from edges[0]
  a->inv_step = step > 0.f ? 1.f / step : 0.f;
  a->for_c2r = for_c2r;
  a->nkshift = 0;
  return PK_OK;
}

static pk_status set_adj_kshifts(AdjGeom *a, int nkshift, const float *kshifts) {
  PK_REQUIRE(nkshift >= 0 && nkshift <= ADJ_MAX_KSHIFTS, PK_ERR_RANGE, "nkshift must be in 0..%d", ADJ_MAX_KSHIFTS);
  PK_REQUIRE(nkshift == 0 || kshifts, PK_ERR_INVALID, "null kshifts");
  a->nkshift = nkshift;
  for (int q = 0; q < nkshift; ++q)
    for (int c = 0; c < 3; ++c) a->kshift[q][c] = kshifts[3 * q + c];
  return PK_OK;
}

extern "C" pk_status pk_adjoint_workspace_size(int nedges, size_t *bytes) {
  PK_REQUIRE(bytes && nedges >= 2, PK_ERR_INVALID, "invalid arguments");
  *bytes = align_up((size_t)nedges * sizeof(float));
  return PK_OK;
}

static pk_status bin_global_adjoint(void *stream, const void *delta, const int32_t meshsize[3], const float kfun[3],
                                    const float los[3], const float *d_edges, int nedges, float step, float edge0,
                                    int backend, int nells, const int32_t *ells, const float *d_coef, int for_c2r,
                                    int nkshift, const float *kshifts, void *out, void *workspace,
                                    size_t workspace_bytes) {
  AdjGeom a;
  pk_status st = make_adj(meshsize, kfun, nedges, step, backend, nells, ells, d_edges, for_c2r, &a);
  if (st) return st;
  st = set_adj_kshifts(&a, nkshift, kshifts);
  if (st) return st;
  PK_REQUIRE(delta && d_coef && out && los, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(delta != out, PK_ERR_INVALID, "out must not alias delta");
  PK_REQUIRE(workspace && workspace_bytes >= (size_t)nedges * sizeof(float), PK_ERR_WORKSPACE,
             "adjoint workspace too small");
  a.e0 = edge0;
  for (int c = 0; c < 3; ++c) a.los[c] = los[c];
  cudaStream_t s = (cudaStream_t)stream;
  float *thr = static_cast<float *>(workspace);
  thresholds_kernel<<<(nedges + 255) / 256, 256, 0, s>>>(d_edges, nedges, thr);
  PK_LAUNCH_CHECK();
  const int64_t total = a.g.d.ncomplex();
  const int64_t want = (total + 255) / 256, cap = 32LL * sm_count();
  if (a.nkshift)
    global_adjoint_kernel<true><<<(int)(want < cap ? want : cap), 256, 0, s>>>(
        a, thr, d_coef, (const float2 *)delta, (float2 *)out);
  else
    global_adjoint_kernel<false><<<(int)(want < cap ? want : cap), 256, 0, s>>>(
        a, thr, d_coef, (const float2 *)delta, (float2 *)out);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_bin_global_adjoint(void *stream, const void *delta,
                                           const int32_t meshsize[3], const float kfun[3],
                                           const float los[3], const float *d_edges, int nedges,
                                           float step, float edge0, int backend, int nells,
                                           const int32_t *ells, const float *d_coef, int for_c2r,
                                           void *out, void *workspace, size_t workspace_bytes) {
  return bin_global_adjoint(stream, delta, meshsize, kfun, los, d_edges, nedges, step, edge0, backend, nells, ells,
                            d_coef, for_c2r, 0, nullptr, out, workspace, workspace_bytes);
}

extern "C" pk_status pk_bin_global_adjoint_shifted(void *stream, const void *delta, const int32_t meshsize[3],
                                                   const float kfun[3], const float los[3], const float *d_edges,
                                                   int nedges, float step, float edge0, int backend, int nells,
                                                   const int32_t *ells, const float *d_coef, int for_c2r,
                                                   int nkshift, const float *kshifts, void *out, void *workspace,
                                                   size_t workspace_bytes) {
  return bin_global_adjoint(stream, delta, meshsize, kfun, los, d_edges, nedges, step, edge0, backend, nells, ells,
                            d_coef, for_c2r, nkshift, kshifts, out, workspace, workspace_bytes);
}

static pk_status bin_firstpoint_adjoint(void *stream, const void *a0, const void *f, int nterms,
                                        const int32_t *term_ell, const int32_t *term_m, const int32_t meshsize[3],
                                        const float kfun[3], const float *d_edges, int nedges, float step,
                                        float edge0, int backend, int nells, const int32_t *ells,
                                        const float *d_coef, int for_c2r, int nkshift, const float *kshifts,
                                        void *out_a0, int accumulate_a0, void *out_f, void *workspace,
                                        size_t workspace_bytes) {
  AdjGeom a;
  pk_status st = make_adj(meshsize, kfun, nedges, step, backend, nells, ells, d_edges, for_c2r, &a);
  if (st) return st;
  st = set_adj_kshifts(&a, nkshift, kshifts);
  if (st) return st;
  PK_REQUIRE(a0 && d_coef, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nterms >= 0 && nterms <= MAX_FP_TERMS, PK_ERR_INVALID, "nterms must be in 0..%d",
             MAX_FP_TERMS);
  PK_REQUIRE(nterms == 0 || (f && out_f && term_ell && term_m), PK_ERR_INVALID, "null term arrays");
  PK_REQUIRE(workspace && workspace_bytes >= (size_t)nedges * sizeof(float), PK_ERR_WORKSPACE,
             "adjoint workspace too small");
  a.e0 = edge0;
  FPAdj t;
  t.nterms = nterms;
  for (int q = 0; q < MAX_FP_TERMS; ++q) {
    t.term_ell[q] = q < nterms ? term_ell[q] : 0;
    t.term_m[q] = q < nterms ? term_m[q] : 0;
    t.term_l[q] = -1;
    for (int l = 0; l < nells && q < nterms; ++l)
      if (ells[l] == term_ell[q]) t.term_l[q] = l;
    PK_REQUIRE(q >= nterms || (t.term_l[q] >= 0 && term_ell[q] >= 1 && term_ell[q] <= YLM_LMAX &&
                               term_m[q] >= -term_ell[q] && term_m[q] <= term_ell[q]),
               PK_ERR_INVALID, "term (%d, %d) is not one of the requested multipoles",
               q < nterms ? term_ell[q] : 0, q < nterms ? term_m[q] : 0);
  }
  cudaStream_t s = (cudaStream_t)stream;
  float *thr = static_cast<float *>(workspace);
  thresholds_kernel<<<(nedges + 255) / 256, 256, 0, s>>>(d_edges, nedges, thr);
  PK_LAUNCH_CHECK();
  const int64_t total = a.g.d.ncomplex();
  const int64_t want = (total + 255) / 256, cap = 32LL * sm_count();
  const int mask = ylm_terms_mask(nterms, term_ell, term_m);
  if (a.nkshift) {  // mode oversampling: the general kernel with shift-averaged coefficients
    firstpoint_adjoint_kernel<true><<<(int)(want < cap ? want : cap), 256, 0, s>>>(
        a, t, thr, d_coef, (const float2 *)a0, (const float2 *)f, (float2 *)out_a0, accumulate_a0,
        (float2 *)out_f);
    PK_LAUNCH_CHECK();
    return PK_OK;
  }
  if (nterms > 0 && mask && ylm_mask_compiled(mask)) {
    FPAdjRows r{};
    for (int q = 0; q < nterms; ++q) r.row[term_ell[q]] = t.term_l[q];
#define PK_FP_ADJ_CASE(M)                                                                                \
  if (mask == (M)) {                                                                                     \
    firstpoint_adjoint_block_kernel<M><<<(int)(want < cap ? want : cap), 256, 0, s>>>(                   \
        a, r, thr, d_coef, (const float2 *)a0, (const float2 *)f, (float2 *)out_a0, accumulate_a0,       \
        (float2 *)out_f);                                                                                \
    PK_LAUNCH_CHECK();                                                                                   \
    return PK_OK;                                                                                        \
  }
    PK_YLM_MASKS(PK_FP_ADJ_CASE)
#undef PK_FP_ADJ_CASE
  }
  firstpoint_adjoint_kernel<false><<<(int)(want < cap ? want : cap), 256, 0, s>>>(
      a, t, thr, d_coef, (const float2 *)a0, (const float2 *)f, (float2 *)out_a0, accumulate_a0,
      (float2 *)out_f);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_bin_firstpoint_adjoint(void *stream, const void *a0, const void *f,
                                               int nterms, const int32_t *term_ell,
                                               const int32_t *term_m, const int32_t meshsize[3],
                                               const float kfun[3], const float *d_edges,
                                               int nedges, float step, float edge0, int backend,
                                               int nells, const int32_t *ells,
                                               const float *d_coef, int for_c2r, void *out_a0,
                                               int accumulate_a0, void *out_f, void *workspace,
                                               size_t workspace_bytes) {
  return bin_firstpoint_adjoint(stream, a0, f, nterms, term_ell, term_m, meshsize, kfun, d_edges, nedges, step,
                                edge0, backend, nells, ells, d_coef, for_c2r, 0, nullptr, out_a0, accumulate_a0,
                                out_f, workspace, workspace_bytes);
}

extern "C" pk_status pk_bin_firstpoint_adjoint_shifted(void *stream, const void *a0, const void *f, int nterms,
                                                       const int32_t *term_ell, const int32_t *term_m,
                                                       const int32_t meshsize[3], const float kfun[3],
                                                       const float *d_edges, int nedges, float step, float edge0,
                                                       int backend, int nells, const int32_t *ells,
                                                       const float *d_coef, int for_c2r, int nkshift,
                                                       const float *kshifts, void *out_a0, int accumulate_a0,
                                                       void *out_f, void *workspace, size_t workspace_bytes) {
  return bin_firstpoint_adjoint(stream, a0, f, nterms, term_ell, term_m, meshsize, kfun, d_edges, nedges, step,
                                edge0, backend, nells, ells, d_coef, for_c2r, nkshift, kshifts, out_a0,
                                accumulate_a0, out_f, workspace, workspace_bytes);
}

extern "C" pk_status pk_window_fill(void *stream, const int32_t meshsize[3], const float kfun[3], int backend,
                                    const float los[3], int ellin, float scale, int ncolumns, const float *klo,
                                    const float *khi, void *out) {
  Dims d;
  PK_REQUIRE(make_dims(meshsize, &d), PK_ERR_INVALID, "invalid meshsize");
  PK_REQUIRE(backend == PK_BACKEND_JAX, PK_ERR_INVALID, "the window fill takes the 'jax' (rfftn) layout");
  PK_REQUIRE(kfun && los && klo && khi && out, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(ellin >= 0 && ellin <= 8, PK_ERR_INVALID, "ellin must be in 0..8");
  PK_REQUIRE(ncolumns >= 1 && ncolumns <= WINDOW_MAX_COLUMNS, PK_ERR_INVALID, "ncolumns must be in 1..%d",
             WINDOW_MAX_COLUMNS);
  WindowColumns cols;
  for (int c = 0; c < WINDOW_MAX_COLUMNS; ++c) {
    cols.klo[c] = c < ncolumns ? klo[c] : 0.f;
    cols.khi[c] = c < ncolumns ? khi[c] : 0.f;
  }
  const int64_t nc = d.ncomplex();
  const int64_t want = (nc + 255) / 256;
  const int blocks = (int)(want < (int64_t)sm_count() * 8 ? want : (int64_t)sm_count() * 8);
  window_fill_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(d, kfun[0], kfun[1], kfun[2], los[0], los[1],
                                                                  los[2], ellin, scale, ncolumns, cols,
                                                                  (float2 *)out);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_window_multiply(void *stream, float *meshes, int ncolumns, const float *q, int64_t n) {
  PK_REQUIRE(meshes && q, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(n >= 1 && ncolumns >= 1, PK_ERR_INVALID, "empty meshes");
  PK_REQUIRE(((uintptr_t)meshes & 15) == 0 && ((uintptr_t)q & 15) == 0, PK_ERR_INVALID,
             "meshes must be 16-byte aligned");
  const int64_t want = ((n & 3) == 0 ? n / 4 : n + 255) / 256 + 1;
  const int blocks = (int)(want < (int64_t)sm_count() * 8 ? want : (int64_t)sm_count() * 8);
  window_multiply_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(meshes, q, n, ncolumns);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_bin_window(void *stream, const void *value, const int32_t meshsize[3], const float kfun[3],
                                   const float los[3], const float *d_edges, int nedges, float step, int backend,
                                   int nells, const int32_t *ells, int ellin, float klo, float khi, float scale,
                                   double *d_out, void *workspace, size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(backend == PK_BACKEND_JAX, PK_ERR_INVALID, "the window binning takes the 'jax' (rfftn) layout");
  PK_REQUIRE(d_edges && d_out && los && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nells >= 1 && nells <= MAX_ELLS, PK_ERR_INVALID, "nells must be in 1..%d", MAX_ELLS);
  PK_REQUIRE(ellin >= 0 && ellin <= 8, PK_ERR_INVALID, "ellin must be in 0..8");
  for (int l = 0; l < nells; ++l) PK_REQUIRE(ells[l] >= 0 && ells[l] <= 8, PK_ERR_INVALID, "ell must be in 0..8");
  if (value) {
    auto fill = [&](auto &op) {
      op.v = (const float2 *)value;
      for (int a = 0; a < 3; ++a) op.los[a] = los[a];
      for (int l = 0; l < MAX_ELLS; ++l) {
        int odd = 0;
        legendre_coefs(l < nells ? ells[l] : 0, op.c[l], &odd);
        if (odd)
          for (int q = 0; q < 5; ++q) op.c[l][q] = 0.f;
      }
    };
    return dispatch_nv<WindowMeshOp>(nells, fill, (cudaStream_t)stream, g, d_edges, true, 0, d_out, workspace,
                                     workspace_bytes);
  }
  auto fill = [&](auto &op) {
    op.v = nullptr;
    for (int a = 0; a < 3; ++a) op.los[a] = los[a];
    for (int l = 0; l < MAX_ELLS; ++l) op.ells[l] = l < nells ? ells[l] : 0;
    op.ellin = ellin;
    op.klo = klo;
    op.khi = khi;
    op.scale = scale;
  };
  return dispatch_nv<WindowOp>(nells, fill, (cudaStream_t)stream, g, d_edges, true, 0, d_out, workspace,
                               workspace_bytes);
}

extern "C" pk_status pk_bin_window_pairs(void *stream, const int32_t meshsize[3], const float kfun[3],
                                         const float los[3], const float *d_edges, int nedges, float step,
                                         int backend, int npairs, const int32_t *pair_ell,
                                         const int32_t *pair_ellin, float scale, double *d_out, void *workspace,
                                         size_t workspace_bytes) {
  BinGeom g;
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(backend == PK_BACKEND_JAX, PK_ERR_INVALID, "the window binning takes the 'jax' (rfftn) layout");
  PK_REQUIRE(d_edges && d_out && los && pair_ell && pair_ellin, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(npairs >= 1 && npairs <= MAX_ELLS, PK_ERR_INVALID, "npairs must be in 1..%d", MAX_ELLS);
  for (int l = 0; l < npairs; ++l)
    PK_REQUIRE(pair_ell[l] >= 0 && pair_ell[l] <= 8 && pair_ellin[l] >= 0 && pair_ellin[l] <= 8, PK_ERR_INVALID,
               "ell must be in 0..8");
  auto fill = [&](auto &op) {
    for (int a = 0; a < 3; ++a) op.los[a] = los[a];
    for (int l = 0; l < MAX_ELLS; ++l) {
      op.ell[l] = l < npairs ? pair_ell[l] : 0;
      op.ellin[l] = l < npairs ? pair_ellin[l] : 0;
    }
    op.scale = scale;
  };
  return dispatch_nv<WindowPairsOp>(npairs, fill, (cudaStream_t)stream, g, d_edges, true, 0, d_out, workspace,
                                    workspace_bytes);
}

extern "C" pk_status pk_bin_window_batch(void *stream, const void *value, int nbatch, const int32_t meshsize[3],
                                         const float kfun[3], const float los[3], const float *d_edges, int nedges,
                                         float step, int backend, int nells, const int32_t *ells, int remove_zero,
                                         double *d_out, void *workspace, size_t workspace_bytes) {
  PK_REQUIRE(nbatch >= 1 && nbatch <= 65535, PK_ERR_INVALID, "nbatch must be in 1..65535");
  BinGeom g;
  pk_status st = make_geom(meshsize, kfun, nedges, step, backend, &g);
  if (st) return st;
  PK_REQUIRE(backend == PK_BACKEND_JAX, PK_ERR_INVALID, "the window binning takes the 'jax' (rfftn) layout");
  PK_REQUIRE(value && d_edges && d_out && los && ells, PK_ERR_INVALID, "null pointer");
  PK_REQUIRE(nells >= 1 && nells <= 5, PK_ERR_INVALID, "nells must be in 1..5");
  LegendreCoefs lc;
  lc.any_odd = 0;
  int max_ell = 0;
  for (int l = 0; l < MAX_ELLS; ++l) {
    const int ell = l < nells ? ells[l] : 0;
    if (l < nells) PK_REQUIRE(ell >= 0 && ell <= 8 && ell % 2 == 0, PK_ERR_INVALID, "ell must be even, 0..8");
    legendre_coefs(ell, lc.c[l], &lc.odd[l]);
    if (l < nells && ell > max_ell) max_ell = ell;
  }
  const bool even = max_ell <= 4;
  cudaStream_t cs = (cudaStream_t)stream;
  const float2 *a = (const float2 *)value;
  // remove_zero: k = 0 dropped for every ell (no ell keeps it), else kept for all
  const int keep = remove_zero ? 0 : (1 << nells) - 1;
  switch (nells * 2 + (even ? 1 : 0)) {
#define PK_WB_CASE(N)                                                                                       \
  case 2 * N:                                                                                               \
    return launch_global<N, false, false, -1>(cs, g, a, nullptr, los, lc, keep, d_edges, d_out, workspace,  \
                                              workspace_bytes, nbatch);                                     \
  case 2 * N + 1:                                                                                           \
    return launch_global<N, false, true, -1>(cs, g, a, nullptr, los, lc, keep, d_edges, d_out, workspace,   \
                                             workspace_bytes, nbatch);
    PK_WB_CASE(1) PK_WB_CASE(2) PK_WB_CASE(3) PK_WB_CASE(4) PK_WB_CASE(5)
#undef PK_WB_CASE
  }
  set_error("unsupported number of multipoles %d", nells);
  return PK_ERR_INVALID;
}
