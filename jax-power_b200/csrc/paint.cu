// Particle painting and reading (resampler scatter / gather) for sm_100a.
//
// Paint = resamplers.paint (resamplers.py:66-97) driven by _paint
// (mesh.py:2673-2729) for all interlacing shifts at once, for one catalog or a batch of
// catalogs (mocks) sharing a mesh geometry.
//
// Design (HBM-bound, deterministic, no global float atomics):
//   1. bucket_kernel<count>: per particle, normalise the position exactly as the
//      reference (float32 IEEE ops, mesh.py:2684), find every mesh tile its stencil can
//      reach for any shift (tiles of all mocks share one index space), and count it there
//      (warp-aggregated int atomics); also track max|w| (fixed-point scale).
//   2. exclusive scan of the tile counts (CUB).
//   3. bucket_kernel<fill>: write (u, w) as a float4 into each reached tile's bucket.
//   4. paint_tiles_kernel: one CTA per tile; every shifted mesh of the tile is accumulated
//      in shared memory as 64-bit fixed point held in two 32-bit words (native shared
//      atomics, exact carries), so the sum does not depend on the order of the additions;
//      then it is converted once to float32 and written with coalesced float4 stores.
//      Each output cell is written exactly once; the mesh is never memset.
// Tile shapes / CTA sizes are compile-time configurations chosen by the caller's
// autotuner (pk_paint uses configuration 0).
#include <algorithm>

#include <cub/device/device_scan.cuh>
#include <math.h>

#include "common.cuh"

namespace pk {

constexpr int MAX_SHIFTS = 4;
constexpr int MAX_ORDER = 4;
constexpr float MAX_CELL_COORD = 4194304.f;  // 2^22 cells
constexpr int NUM_TILE_CONFIGS = 11;

// Tile configurations: (cells along axes 0, 1, 2; threads per CTA; SWZ: shared-memory rows
// swizzled, see paint_swizzle; ROWS36: the per-shift kernel paint_shift_tile_kernel, see
// there).  Configurations 4..7 are 0..3 with the swizzle; 8 to 10 take the per-shift
// kernel where the mesh allows it (last axis a multiple of 32, at least 64; the others a
// multiple of 8), else the all-shifts kernel with the same tile.
template <int C>
struct TileConfig;
#define PK_TILE_CONFIG(C, A, B, TH, S, R)                                                         \
  template <>                                                                                     \
  struct TileConfig<C> {                                                                          \
    static constexpr int T0 = A, T1 = B, T2 = 32, THREADS = TH;                                   \
    static constexpr bool SWZ = S, ROWS36 = R;                                                    \
  };
PK_TILE_CONFIG(0, 8, 16, 512, false, false)
PK_TILE_CONFIG(1, 8, 16, 256, false, false)
PK_TILE_CONFIG(2, 8, 8, 256, false, false)
PK_TILE_CONFIG(3, 4, 16, 256, false, false)
PK_TILE_CONFIG(4, 8, 16, 512, true, false)
PK_TILE_CONFIG(5, 8, 16, 256, true, false)
PK_TILE_CONFIG(6, 8, 8, 256, true, false)
PK_TILE_CONFIG(7, 4, 16, 256, true, false)
PK_TILE_CONFIG(8, 8, 16, 256, false, true)
PK_TILE_CONFIG(9, 16, 16, 256, false, true)
PK_TILE_CONFIG(10, 16, 16, 512, false, true)
#undef PK_TILE_CONFIG

static void tile_dims(int config, int t[3], int *threads) {
  switch (config) {
#define PK_TC(C)                       \
  case C:                              \
    t[0] = TileConfig<C>::T0;          \
    t[1] = TileConfig<C>::T1;          \
    t[2] = TileConfig<C>::T2;          \
    *threads = TileConfig<C>::THREADS; \
    return;
    PK_TC(0) PK_TC(1) PK_TC(2) PK_TC(3) PK_TC(4) PK_TC(5) PK_TC(6) PK_TC(7) PK_TC(8) PK_TC(9) PK_TC(10)
#undef PK_TC
  }
}

struct PaintGeom {
  Dims d;
  float half[3], center[3], cell[3];
  int order;
  int nshifts;
  float shifts[MAX_SHIFTS];
  int reach_lo, reach_hi;  // stencil reach below / above floor(u), all shifts
  int tile[3];             // tile shape (powers of two)
  int tshift[3];           // log2 of the tile shape
  int nt[3];               // tiles per axis (one mock)
  int64_t tiles_per_mock;
  int nmocks;
  const int64_t *offsets;  // device, nmocks + 1 particle offsets (NULL: one mock)
  int64_t n;               // particles (one mock)
};

__device__ __forceinline__ float normalise(float p, float half, float center, float cell) {
  // ((pos + boxsize / 2.) - boxcenter) / cellsize, mesh.py:2684, no contraction
  return __fdiv_rn(__fsub_rn(__fadd_rn(p, half), center), cell);
}

__device__ __forceinline__ int wrapi(int i, int n) {
  if (i >= 0 && i < n) return i;
  if (i < 0 && i >= -n) return i + n;
  if (i >= n && i < 2 * n) return i - n;
  const int r = i % n;
  return r < 0 ? r + n : r;
}

// The reference's kernels (resamplers.py:57-63) in float32 without contraction.
__device__ __forceinline__ float bspline(int order, float s) {
  switch (order) {
    case 1:
      return 1.f;
    case 2:
      return __fsub_rn(1.f, s);
    case 3:
      if (s <= 0.5f) return __fsub_rn(0.75f, __fmul_rn(s, s));
      {
        float t = __fsub_rn(1.5f, s);
        return __fmul_rn(0.5f, __fmul_rn(t, t));
      }
    default: {
      const float sixth = 0.16666667f;  // (bool) / 6 in float32
      if (s <= 1.f) {
        float s2 = __fmul_rn(s, s);
        float s3 = __fmul_rn(s, s2);
        float p = __fadd_rn(__fsub_rn(4.f, __fmul_rn(6.f, s2)), __fmul_rn(3.f, s3));
        return __fmul_rn(sixth, p);
      }
      float t = __fsub_rn(2.f, s);
      return __fmul_rn(sixth, __fmul_rn(t, __fmul_rn(t, t)));
    }
  }
}

// dW/ds of the kernels above.
__device__ __forceinline__ float bspline_deriv(int order, float s) {
  switch (order) {
    case 1:
      return 0.f;
    case 2:
      return -1.f;
    case 3:
      return s <= 0.5f ? -2.f * s : -(1.5f - s);
    default:
      return s <= 1.f ? (-12.f * s + 9.f * s * s) / 6.f : -0.5f * (2.f - s) * (2.f - s);
  }
}

// Base index: floor for even orders, round-half-to-even for odd (jnp.round).
__device__ __forceinline__ int base_index(int order, float u) {
  return (order & 1) ? (int)rintf(u) : (int)floorf(u);
}

__device__ __forceinline__ int offset_lo(int order) { return -((order - 1) / 2); }

// Distinct tiles of the wrapped cell span [c - lo, c + hi] along one axis.  When every
// tile on the axis is at least as long as the span (the usual case), the span touches the
// tiles of its two ends only.
__device__ __forceinline__ int span_tiles(int c, int lo, int hi, int n, int tshift, int nt,
                                          int out[3]) {
  const int last = n - ((nt - 1) << tshift);
  if (last >= lo + hi || nt == 1) {
    const int a = wrapi(c - lo, n) >> tshift, b = wrapi(c + hi, n) >> tshift;
    out[0] = a;
    out[1] = b;
    return a == b ? 1 : 2;
  }
  // short last tile: up to 3 distinct tiles, kept in registers (no dynamic indexing)
  int count = 0, t0 = -1, t1 = -1, t2 = -1;
  for (int x = c - lo; x <= c + hi; ++x) {
    const int t = wrapi(x, n) >> tshift;
    if (t == t0 || t == t1 || t == t2) continue;
    if (count == 0) t0 = t;
    else if (count == 1) t1 = t;
    else if (count == 2) t2 = t;
    count += count < 3;
  }
  out[0] = t0;
  out[1] = t1;
  out[2] = t2;
  return count;
}

__device__ __forceinline__ bool load_particle(const PaintGeom &g, const float *pos,
                                              const float *w, int64_t p, float u[3],
                                              float *wp) {
  const float *q = pos + 3 * p;
  bool ok = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    u[d] = normalise(q[d], g.half[d], g.center[d], g.cell[d]);
    ok &= isfinite(u[d]) && fabsf(u[d]) < MAX_CELL_COORD;
  }
  *wp = w ? w[p] : 1.f;
  return ok;
}

// Mock of particle p (offsets sorted, offsets[0] = 0, offsets[nmocks] = n).
__device__ __forceinline__ int mock_of(const PaintGeom &g, int64_t p) {
  if (g.nmocks <= 1 || !g.offsets) return 0;
  int lo = 0, hi = g.nmocks - 1;  // largest m with offsets[m] <= p
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(g.offsets + mid) <= p) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Mock of particle base + lane for a warp's 32 consecutive particles: one search by lane 0
// when the whole warp lies in one mock (the usual case), else one per lane.
__device__ __forceinline__ int warp_mock_of(const PaintGeom &g, int64_t base, int64_t n) {
  if (g.nmocks <= 1 || !g.offsets) return 0;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int m0 = 0;
  bool same = false;
  if (lane == 0) {
    m0 = mock_of(g, base);
    const int64_t last = min(base + 31, n - 1);
    same = __ldg(g.offsets + m0 + 1) > last;
  }
  m0 = __shfl_sync(FULL, m0, 0);
  same = __shfl_sync(FULL, (int)same, 0) != 0;
  if (same) return m0;
  return base + lane < n ? mock_of(g, base + lane) : m0;
}

// The tiles reached by a warp's particles base .. base + 31 (those below `end`), every
// interlacing shift at once: per axis the base cell c (floor for even orders, round-half-even
// for odd ones, as the shift-0 stencil) and the reach [c - reach_lo, c + reach_hi] over all
// shifts.  Each reached tile goes to `sink` as a run of consecutive lanes with the same tile
// (catalogs are often sorted by cell, so neighbouring particles usually share tiles); the
// run leader makes one atomic for the whole run and its lanes take consecutive slots.
//   sink.particle(ok, wp)                  once per lane (validity, weight)
//   sink.run(act, lead, leads, runlen, tile, u, wp)   once per candidate copy (warp-uniform)
// A lane's raw position and weight (0 beyond `end`): loaded one warp iteration ahead by the
// shared-histogram passes, so that the next loads are in flight while a warp works on its runs.
struct RawParticle {
  float x, y, z, w;
};

__device__ __forceinline__ RawParticle load_raw(const float *__restrict__ pos, const float *__restrict__ w,
                                                int64_t p, int64_t end) {
  RawParticle r{0.f, 0.f, 0.f, 0.f};
  if (p < end) {
    const float *q = pos + 3 * p;
    r.x = q[0];
    r.y = q[1];
    r.z = q[2];
    r.w = w ? w[p] : 1.f;
  }
  return r;
}

template <class Sink>
__device__ __forceinline__ void warp_tile_runs_raw(const PaintGeom &g, int64_t n, int64_t end, int64_t base,
                                                   const RawParticle &raw, Sink &sink);

template <class Sink>
__device__ __forceinline__ void warp_tile_runs(const PaintGeom &g, const float *__restrict__ pos,
                                               const float *__restrict__ w, int64_t n, int64_t end,
                                               int64_t base, Sink &sink) {
  warp_tile_runs_raw(g, n, end, base, load_raw(pos, w, base + (threadIdx.x & 31), end), sink);
}

template <class Sink>
__device__ __forceinline__ void warp_tile_runs_raw(const PaintGeom &g, int64_t n, int64_t end, int64_t base,
                                                   const RawParticle &raw, Sink &sink) {
  const int ns[3] = {g.d.n0, g.d.n1, g.d.n2};
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t p = base + lane;
  float u[3] = {0.f, 0.f, 0.f}, wp = 0.f;
  bool ok = false;
  const int mock = warp_mock_of(g, base, n);
  if (p < end) {
    const float q[3] = {raw.x, raw.y, raw.z};
    ok = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      u[d] = normalise(q[d], g.half[d], g.center[d], g.cell[d]);
      ok &= isfinite(u[d]) && fabsf(u[d]) < MAX_CELL_COORD;
    }
    wp = raw.w;
    ok = ok && isfinite(wp);
  }
  sink.particle(p < end, ok, wp);
  int t[3][3], nt[3] = {0, 0, 0};
  if (ok) {
#pragma unroll
    for (int d = 0; d < 3; ++d)
      nt[d] = span_tiles(base_index(g.order, u[d]), g.reach_lo, g.reach_hi, ns[d], g.tshift[d], g.nt[d], t[d]);
  }
  const int m0 = __reduce_max_sync(FULL, nt[0]), m1 = __reduce_max_sync(FULL, nt[1]),
            m2 = __reduce_max_sync(FULL, nt[2]);
  const int64_t mbase = (int64_t)mock * g.tiles_per_mock;
  // the copies in (axis 0, 1, 2) order; loop bounds are warp-uniform
#pragma unroll
  for (int c0 = 0; c0 < 3; ++c0) {
    if (c0 >= m0) break;
#pragma unroll
    for (int c1 = 0; c1 < 3; ++c1) {
      if (c1 >= m1) break;
#pragma unroll
      for (int c2 = 0; c2 < 3; ++c2) {
        if (c2 >= m2) break;
        const bool act = c0 < nt[0] && c1 < nt[1] && c2 < nt[2];
        int tile = -1;
        if (act) tile = (int)(mbase + ((int64_t)t[0][c0] * g.nt[1] + t[1][c1]) * g.nt[2] + t[2][c2]);
        // a run ends at the next leader or inactive lane
        const int prev = __shfl_up_sync(FULL, tile, 1);
        const bool lead = act && (lane == 0 || prev != tile);
        const unsigned leads = __ballot_sync(FULL, lead);
        const unsigned ends = leads | ~__ballot_sync(FULL, act);
        const unsigned above = lane == 31 ? 0u : (ends & (0xffffffffu << (lane + 1)));
        const unsigned runlen = (unsigned)((above ? __ffs(above) - 1 : 32) - lane);
        sink.run(act, lead, leads, runlen, tile, u, wp);
      }
    }
  }
}

// Slot of each lane of a run: the leader's atomic result, shuffled to its run, plus the
// lane's place in the run.
__device__ __forceinline__ unsigned run_slot(unsigned leader_base, unsigned leads) {
  const int lane = threadIdx.x & 31;
  const unsigned upto = leads & (lane == 31 ? 0xffffffffu : ((2u << lane) - 1u));
  const int my_lead = upto ? 31 - __clz(upto) : lane;
  return __shfl_sync(0xffffffffu, leader_base, my_lead) + (unsigned)(lane - my_lead);
}

// Global-memory counters (any number of tiles): bucket_kernel<false> counts the copies per
// tile, bucket_kernel<true> fills the bucket from the scanned offsets.
template <bool FILL>
struct GlobalSink {
  unsigned *counts;
  const int *offsets;
  unsigned *cursors;
  float4 *bucket;
  unsigned *wmax_bits;
  int *status;
  __device__ __forceinline__ void particle(bool in, bool ok, float wp) {
    if (FILL) return;
    if (in && !ok && status) atomicExch(status, 1);
    const unsigned wb = __reduce_max_sync(0xffffffffu, ok ? __float_as_uint(fabsf(wp)) : 0u);
    if ((threadIdx.x & 31) == 0 && wb) atomicMax(wmax_bits, wb);
  }
  __device__ __forceinline__ void run(bool act, bool lead, unsigned leads, unsigned runlen, int tile,
                                      const float u[3], float wp) {
    if (!FILL) {
      if (lead) atomicAdd(counts + tile, runlen);
      return;
    }
    unsigned b0 = 0;
    if (lead) b0 = atomicAdd(cursors + tile, runlen);
    const unsigned slot = run_slot(b0, leads);
    if (act) bucket[(int64_t)offsets[tile] + slot] = make_float4(u[0], u[1], u[2], wp);
  }
};

template <bool FILL>
__global__ void bucket_kernel(PaintGeom g, const float *__restrict__ pos,
                              const float *__restrict__ w, int64_t n,
                              unsigned *__restrict__ counts, const int *__restrict__ offsets,
                              unsigned *__restrict__ cursors, float4 *__restrict__ bucket,
                              unsigned *__restrict__ wmax_bits, int *__restrict__ status) {
  GlobalSink<FILL> sink{counts, offsets, cursors, bucket, wmax_bits, status};
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = warp * 32; base < n; base += nwarps * 32) warp_tile_runs(g, pos, w, n, n, base, sink);
}

// Shared-memory counters (tile index spaces up to HIST_MAX_TILES): each CTA takes a
// contiguous range of particles and counts its copies per tile in shared memory; the
// counts form a (CTA, tile) matrix whose column scan gives each CTA its own slots in every
// tile.  The fill pass then assigns slots with shared-memory atomics only.  Versus global
// counters this removes the global atomics (and their latency) from both passes.
constexpr int HIST_THREADS = 1024;
constexpr int HIST_MAX_TILES = 48 * 1024;  // 192 KB of counters per CTA

template <bool PLACE>
struct SharedSink {
  unsigned *hist;  // shared counters (count) or cursors (place)
  float4 *bucket;
  unsigned wmax;   // per-lane max |w| bits (count)
  int bad;
  __device__ __forceinline__ void particle(bool in, bool ok, float wp) {
    if (PLACE) return;
    bad |= in && !ok;
    if (ok) wmax = max(wmax, __float_as_uint(fabsf(wp)));
  }
  __device__ __forceinline__ void run(bool act, bool lead, unsigned leads, unsigned runlen, int tile,
                                      const float u[3], float wp) {
    if (!PLACE) {
      if (lead) atomicAdd(hist + tile, runlen);
      return;
    }
    unsigned b0 = 0;
    if (lead) b0 = atomicAdd(hist + tile, runlen);
    const unsigned slot = run_slot(b0, leads);
    if (act) bucket[slot] = make_float4(u[0], u[1], u[2], wp);
  }
};

// colmat[c * ntiles + t]: the copies CTA c makes in tile t (count); after
// bucket_colscan_kernel the first of them within tile t, to which PLACE adds tile_start[t].
template <bool PLACE>
__global__ void __launch_bounds__(HIST_THREADS) bucket_hist_kernel(
    PaintGeom g, const float *__restrict__ pos, const float *__restrict__ w, int64_t n, int64_t chunk,
    int ntiles, unsigned *__restrict__ colmat, const int *__restrict__ tile_start, float4 *__restrict__ bucket,
    unsigned *__restrict__ wmax_bits, int *__restrict__ status) {
  extern __shared__ unsigned hist[];
  unsigned *row = colmat + (size_t)blockIdx.x * ntiles;
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) hist[t] = PLACE ? (unsigned)tile_start[t] + row[t] : 0u;
  __syncthreads();
  SharedSink<PLACE> sink{hist, bucket, 0u, 0};
  const int64_t begin = (int64_t)blockIdx.x * chunk;
  const int64_t end = min(n, begin + chunk);
  const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t wstride = (int64_t)nwarps * 32;
  int64_t base = begin + (int64_t)warp * 32;
  RawParticle cur = load_raw(pos, w, base + lane, end);
  for (; base < end; base += wstride) {
    const RawParticle next = load_raw(pos, w, base + wstride + lane, end);  // one iteration ahead
    warp_tile_runs_raw(g, n, end, base, cur, sink);
    cur = next;
  }
  if (!PLACE) {
    const unsigned wb = __reduce_max_sync(0xffffffffu, sink.wmax);
    if ((threadIdx.x & 31) == 0 && wb) atomicMax(wmax_bits, wb);
    if (__any_sync(0xffffffffu, sink.bad) && (threadIdx.x & 31) == 0 && status) atomicExch(status, 1);
  }
  __syncthreads();
  if (!PLACE)
    for (int t = threadIdx.x; t < ntiles; t += blockDim.x) row[t] = hist[t];
}

// Exclusive scan of every tile's column of the (CTA, tile) count matrix, in place, and the
// tile totals (totals[ntiles] = 0, so that the scan of totals ends on the bucket size).
__global__ void bucket_colscan_kernel(unsigned *__restrict__ colmat, int nctas, int ntiles,
                                      unsigned *__restrict__ totals) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > ntiles) return;
  if (t == ntiles) {
    totals[t] = 0u;
    return;
  }
  // 16 rows in flight per thread: the loads of a batch are independent (the column is ~150 rows)
  constexpr int B = 16;
  unsigned acc = 0u;
  for (int c0 = 0; c0 < nctas; c0 += B) {
    unsigned v[B];
#pragma unroll
    for (int k = 0; k < B; ++k) v[k] = c0 + k < nctas ? colmat[(size_t)(c0 + k) * ntiles + t] : 0u;
#pragma unroll
    for (int k = 0; k < B; ++k) {
      if (c0 + k < nctas) colmat[(size_t)(c0 + k) * ntiles + t] = acc;
      acc += v[k];
    }
  }
  totals[t] = acc;
}

// Fixed-point exponent e such that count * max|w| * 2^e < 2^62, count = the particles of the
// catalog: every partial sum of a cell fits in a signed 64-bit integer (each particle adds
// at most |w| to a cell).  It depends on the catalog only, not on the tiling, so every tile
// configuration rounds each contribution identically and paints the same bits.  For tiny
// weights e exceeds float32's largest power of two (127; max|w| subnormal gives up to 187),
// so the scale is applied as two exact factors (fixed_scales).
__device__ __forceinline__ int fixed_exponent(unsigned wmax_bits, long long count) {
  const float wmax = __uint_as_float(wmax_bits);
  if (!(wmax > 0.f) || !isfinite(wmax)) return 40;
  const int ew = (int)((wmax_bits >> 23) & 0xff) - 126;  // wmax < 2^ew (subnormals: 2^-126)
  const int en = 64 - __clzll(count > 0 ? count : 1);     // count < 2^en
  return 62 - ew - en;                                    // in [-129, 187]
}

// 2^e as two float32 factors, each a power of two within float32's normal range or (e < -126)
// an exact subnormal: (w * s0) * s1 is w 2^e exactly whenever that is a normal float.
__device__ __forceinline__ void fixed_scales(int e, float *s0, float *s1) {
  const int e0 = e > 120 ? 120 : e;
  *s0 = ldexpf(1.f, e0);
  *s1 = ldexpf(1.f, e - e0);
}

// A cell's 64-bit fixed-point sum (units 2^-e) to float32: one correctly rounded int64 ->
// float32 conversion, then the exact power-of-two scaling 2^-e in two factors (inv from
// fixed_inverse); only a result below float32's normal range rounds again.
__device__ __forceinline__ void fixed_inverse(int e, float *inv0, float *inv1) {
  const int e0 = e > 120 ? 120 : (e < -120 ? -120 : e);
  *inv0 = ldexpf(1.f, -e0);
  *inv1 = ldexpf(1.f, e0 - e);
}

__device__ __forceinline__ float fixed_to_float(unsigned lo, unsigned hi, float inv0, float inv1) {
  const long long fx = (long long)(((unsigned long long)hi << 32) | lo);
  return __fmul_rn(__fmul_rn(__ll2float_rn(fx), inv0), inv1);
}

// Shared-memory atomics on 32-bit shared-window addresses.
__device__ __forceinline__ unsigned atom_add_shared(unsigned addr, unsigned v) {
  unsigned old;
  asm volatile("atom.shared.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(addr), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ void red_add_shared(unsigned addr, unsigned v) {
  asm volatile("red.shared.add.u32 [%0], %1;" : : "r"(addr), "r"(v) : "memory");
}

// hi + the carry out of old + lo (the low word's addition), with the add's carry flag.
__device__ __forceinline__ unsigned add_carry_hi(unsigned old, unsigned lo, unsigned hi) {
  unsigned r;
  asm("{\n\t.reg .u32 t;\n\tadd.cc.u32 t, %1, %2;\n\taddc.u32 %0, %3, 0;\n\t}" : "=r"(r) : "r"(old), "r"(lo), "r"(hi));
  return r;
}

// bspline() at stencil point O (0 .. ORDER - 1) of a compile-time order.  Which polynomial
// piece applies is known from O: with i0 = rint(u) (odd order) or floor(u) (even order) the
// distance s = |i0 + OLO + O - u| lies in [0, 0.5] for TSC's middle point and in [0.5, 1.5]
// for its outer ones, in [0, 1] for PCS's two middle points and in [1, 2] for its outer ones
// (float32 rounding cannot cross these representable bounds).  At a shared bound both pieces
// give the same float32 value (TSC 0.5 at s = 0.5, PCS 1/6 at s = 1), so this equals
// bspline() bit for bit without evaluating the other piece.
template <int ORDER, int O>
__device__ __forceinline__ float bspline_at(float s) {
  if (ORDER == 1) return 1.f;
  if (ORDER == 2) return __fsub_rn(1.f, s);
  if (ORDER == 3) {
    if (O == 1) return __fsub_rn(0.75f, __fmul_rn(s, s));
    const float t = __fsub_rn(1.5f, s);
    return __fmul_rn(0.5f, __fmul_rn(t, t));
  }
  const float sixth = 0.16666667f;
  if (O == 1 || O == 2) {
    const float s2 = __fmul_rn(s, s);
    const float s3 = __fmul_rn(s, s2);
    return __fmul_rn(sixth, __fadd_rn(__fsub_rn(4.f, __fmul_rn(6.f, s2)), __fmul_rn(3.f, s3)));
  }
  const float t = __fsub_rn(2.f, s);
  return __fmul_rn(sixth, __fmul_rn(t, __fmul_rn(t, t)));
}

// Shared-memory position of tile cell (x, y, z) in the swizzled configurations: row (x, y)
// holds its z in an order XORed by a multiple of 4 that varies with the row, so that the same
// z in neighbouring rows and planes falls in different banks (groups of 4 consecutive z stay
// contiguous for the float4 write-out).  It pays on catalogs stored in spatial order (a warp's
// lanes then paint nearby cells): at 512^3 the benchmark's lognormal catalog paints in 1.74
// ms instead of 2.07, a dense 128^3 mock in 1.33 instead of 1.81; on randomly ordered
// particles it costs its few instructions (the cut-sky catalog: 6.14 against 5.90 ms).
template <bool SWZ>
__device__ __forceinline__ int paint_swizzle(int x, int y) {
  return SWZ ? (((y + 3 * x) & 7) << 2) : 0;
}

template <int ORDER, int CFG>
__global__ void __launch_bounds__(TileConfig<CFG>::THREADS) paint_tiles_kernel(
    PaintGeom g, const float4 *__restrict__ bucket, const int *__restrict__ offsets,
    const unsigned *__restrict__ wmax_bits, float *__restrict__ out) {
  using TC = TileConfig<CFG>;
  constexpr int T0 = TC::T0, T1 = TC::T1, T2 = TC::T2, CELLS = T0 * T1 * T2;
  // Per-cell 64-bit fixed point as two 32-bit words (native shared atomics): the low word's
  // returned old value gives the exact carry into the high word, so the integer sum stays
  // exact and independent of the order of the additions.
  extern __shared__ __align__(16) unsigned acc32[];  // lo[nshifts][CELLS], scratch[32], hi[nshifts][CELLS], scratch[32]
  const int64_t gtile = blockIdx.x;
  const int mock = (int)(gtile / g.tiles_per_mock);
  const int tile = (int)(gtile % g.tiles_per_mock);
  const int t2i = tile % g.nt[2];
  const int t1i = (tile / g.nt[2]) % g.nt[1];
  const int t0i = tile / (g.nt[2] * g.nt[1]);
  const int los[3] = {t0i * T0, t1i * T1, t2i * T2};
  const int begin = offsets[gtile], end = offsets[gtile + 1];
  const unsigned count = (unsigned)(end - begin);
  const bool vec = (g.d.n2 % 4) == 0;
  float *mock_out = out + (int64_t)mock * g.nshifts * g.d.nreal();

  if (count > 0) {
    {
      uint4 *z4 = reinterpret_cast<uint4 *>(acc32);  // 2 nshifts CELLS words, CELLS % 4 == 0
      for (int i = threadIdx.x; i < (2 * g.nshifts * CELLS + 64) / 4; i += blockDim.x) z4[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();
    const long long ncat = g.offsets ? (long long)(g.offsets[mock + 1] - g.offsets[mock]) : (long long)g.n;
    const int fexp = fixed_exponent(*wmax_bits, ncat);
    float fscale0, fscale1;  // exact power-of-two scaling of each contribution, 2^fexp
    fixed_scales(fexp, &fscale0, &fscale1);
    const int ns[3] = {g.d.n0, g.d.n1, g.d.n2};
    const int tl[3] = {T0, T1, T2};
    constexpr int OLO = -((ORDER - 1) / 2);
    // a stencil wraps past the mesh end at most once when every axis has >= ORDER cells
    const bool one_wrap = g.d.n0 >= ORDER && g.d.n1 >= ORDER && g.d.n2 >= ORDER;
    const unsigned acc_base = (unsigned)__cvta_generic_to_shared(acc32);
    // The bucket is cut into 32 runs of S entries; lane l of a warp takes entry l S + jj of
    // slot jj, so the lanes of a warp sit S entries apart (on different cells: bucket order
    // follows the particles' input order, often spatial) and every entry is visited once.
    // A slot paints all shifts of its entries; a sparse tile (fewer slots than warps) splits
    // its slots per shift instead, so that its few entries still spread over all warps.
    const int nwarps = blockDim.x >> 5, lane = threadIdx.x & 31;
    const unsigned S = (count + 31) >> 5;
    const bool split = S < (unsigned)nwarps;
    const unsigned nslots = split ? S * (unsigned)g.nshifts : S;
    for (unsigned j = threadIdx.x >> 5; j < nslots; j += (unsigned)nwarps) {
      const unsigned jj = split ? j % S : j;
      const int s_begin = split ? (int)(j / S) : 0, s_end = split ? s_begin + 1 : g.nshifts;
      const unsigned e = lane * S + jj;
      const bool has = e < count;
      const float4 q = bucket[begin + (has ? e : 0u)];
      const float uq[3] = {q.x, q.y, q.z};
      // w 2^fexp is exact, so (w 2^fexp) * ker rounds like the reference's w * ker, scaled;
      // lanes past the end of the bucket add zeros (to their scratch words)
      const float wq = has ? __fmul_rn(__fmul_rn(q.w, fscale0), fscale1) : 0.f;
      for (int s = s_begin; s < s_end; ++s) {
        float k[3][ORDER];
        int l[3][ORDER];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float u = __fadd_rn(uq[d], g.shifts[s]);
          const float fi0 = (ORDER & 1) ? rintf(u) : floorf(u);
          const int i0 = (int)fi0;
          // tile-relative cell of the first stencil point; stencil stays within one period
          const int w0 = wrapi(i0 + OLO, ns[d]) - los[d];
          const int lim = ns[d] - los[d];
          k[d][0] = bspline_at<ORDER, 0>(fabsf(__fsub_rn(__fadd_rn(fi0, (float)OLO), u)));
          if (ORDER > 1) k[d][ORDER > 1 ? 1 : 0] = bspline_at<ORDER, 1>(fabsf(__fsub_rn(__fadd_rn(fi0, (float)(OLO + 1)), u)));
          if (ORDER > 2) k[d][ORDER > 2 ? 2 : 0] = bspline_at<ORDER, 2>(fabsf(__fsub_rn(__fadd_rn(fi0, (float)(OLO + 2)), u)));
          if (ORDER > 3) k[d][ORDER > 3 ? 3 : 0] = bspline_at<ORDER, 3>(fabsf(__fsub_rn(__fadd_rn(fi0, (float)(OLO + 3)), u)));
#pragma unroll
          for (int o = 0; o < ORDER; ++o) {
            // (float)(i0 + OLO + o) exactly above, without an int -> float conversion
            int loc = w0 + o;
            if (one_wrap) {
              loc -= loc >= lim ? ns[d] : 0;
            } else {
#pragma unroll
              for (int r = 0; r < ORDER - 1; ++r) loc -= loc >= lim ? ns[d] : 0;  // tiny meshes
            }
            l[d][o] = (loc >= 0 && loc < tl[d]) ? loc : -1;
          }
        }
        // layout: lo[nshifts][CELLS], 32 scratch words, hi[nshifts][CELLS], 32 scratch words, so
        // that every high word (scratch included) sits a fixed distance after its low word
        const unsigned dummy = acc_base + 4u * (unsigned)(g.nshifts * CELLS + (threadIdx.x & 31));
        const unsigned hi_delta = 4u * (unsigned)(g.nshifts * CELLS + 32);
        const unsigned lo_base = acc_base + 4u * (unsigned)(s * CELLS);
        unsigned zoff[ORDER];  // byte offset of each stencil z in a row
        bool zin[ORDER];
#pragma unroll
        for (int c = 0; c < ORDER; ++c) {
          zoff[c] = 4u * (unsigned)l[2][c];
          zin[c] = l[2][c] >= 0;
        }
#pragma unroll
        for (int a = 0; a < ORDER; ++a) {
#pragma unroll
          for (int b = 0; b < ORDER; ++b) {
            const float kab = __fmul_rn(k[0][a], k[1][b]);
            const bool vab = has && (l[0][a] | l[1][b]) >= 0;
            const unsigned rowbase = lo_base + 4u * (unsigned)((l[0][a] * T1 + l[1][b]) * T2);
            const unsigned sw4 = 4u * (unsigned)paint_swizzle<TC::SWZ>(l[0][a], l[1][b]);
#pragma unroll
            for (int c = 0; c < ORDER; ++c) {
              const float v = __fmul_rn(wq, __fmul_rn(kab, k[2][c]));  // (w * ker) 2^fexp
              const long long fx = __float2ll_rn(v);
              const unsigned lo = (unsigned)fx;
              // invalid cells go to this lane's scratch words (never read): no branch, and
              // the scratch words of a warp sit in distinct banks
              const unsigned addr = (vab && zin[c]) ? rowbase + (zoff[c] ^ sw4) : dummy;
              const unsigned old = atom_add_shared(addr, lo);
              red_add_shared(addr + hi_delta, add_carry_hi(old, lo, (unsigned)(fx >> 32)));
            }
          }
        }
      }
    }
    __syncthreads();
    float inv0, inv1;
    fixed_inverse(fexp, &inv0, &inv1);
    for (int s = 0; s < g.nshifts; ++s) {
      float *mesh = mock_out + (int64_t)s * g.d.nreal();
      const unsigned *alo = acc32 + s * CELLS;
      const unsigned *ahi = acc32 + g.nshifts * CELLS + 32 + s * CELLS;
      for (int i = threadIdx.x * 4; i < CELLS; i += blockDim.x * 4) {
        const int c2 = i % T2, c1 = (i / T2) % T1, c0 = i / (T2 * T1);
        const int x0 = los[0] + c0, x1 = los[1] + c1, x2 = los[2] + c2;
        if (x0 >= g.d.n0 || x1 >= g.d.n1) continue;
        const int64_t base = ((int64_t)x0 * g.d.n1 + x1) * g.d.n2 + x2;
        const int is = i - c2 + (c2 ^ paint_swizzle<TC::SWZ>(c0, c1));  // 4 contiguous cells
        const uint4 lo4 = *reinterpret_cast<const uint4 *>(alo + is);
        const uint4 hi4 = *reinterpret_cast<const uint4 *>(ahi + is);
        const unsigned los4[4] = {lo4.x, lo4.y, lo4.z, lo4.w}, his4[4] = {hi4.x, hi4.y, hi4.z, hi4.w};
        float v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = fixed_to_float(los4[j], his4[j], inv0, inv1);
        if (vec) {
          if (x2 < g.d.n2) *reinterpret_cast<float4 *>(mesh + base) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (x2 + j < g.d.n2) mesh[base + j] = v[j];
        }
      }
    }
  } else {
    for (int s = 0; s < g.nshifts; ++s) {
      float *mesh = mock_out + (int64_t)s * g.d.nreal();
      for (int i = threadIdx.x * 4; i < CELLS; i += blockDim.x * 4) {
        const int c2 = i % T2, c1 = (i / T2) % T1, c0 = i / (T2 * T1);
        const int x0 = los[0] + c0, x1 = los[1] + c1, x2 = los[2] + c2;
        if (x0 >= g.d.n0 || x1 >= g.d.n1) continue;
        const int64_t base = ((int64_t)x0 * g.d.n1 + x1) * g.d.n2 + x2;
        if (vec) {
          if (x2 < g.d.n2) *reinterpret_cast<float4 *>(mesh + base) = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (x2 + j < g.d.n2) mesh[base + j] = 0.f;
        }
      }
    }
  }
}

// ------------------------------------------------------------ per-shift tile kernel
// One CTA per (tile, interlacing shift), tiles T0 x T1 x 32, on meshes whose last axis is a
// multiple of 4 and at least 64 cells (paint_run falls back to paint_tiles_kernel otherwise).
//
// Shared memory holds the low and the high words of the tile's 64-bit fixed-point cells in
// rows of ROW_WORDS = 37 words: tile row (x, y) starts at word (x T1 + y) 37 and cell z sits
// at + z + 4, so cells z in [-4, 33) are in the row and z in [33, 36) fall on the next row's
// first words, which hold cells z < 0 of that row: cells outside the tile, never written out.
// The odd row length spreads the cells of neighbouring rows over the banks.
// A particle's ORDER stencil cells along z are therefore immediate offsets from one address,
// with no per-cell test.
//
// Lane l of a warp takes entry l S + j of slot j (S = ceil(count / 32)): the lanes of one
// atomic instruction sit S entries apart in the bucket, which keeps the catalog's order (often
// spatial), so they rarely paint the same cell.  The three shifts of a tile are consecutive
// CTAs (blockIdx.x = tile * nshifts + shift), so they read the tile's bucket from L2.  The
// contributions, their fixed-point rounding and the write-out are those of
// paint_tiles_kernel, so every configuration paints the same bits.
constexpr int ROW_WORDS = 37;  // odd: the bank of a cell mixes its row (x, y) and z
constexpr int ROW_ZOFF = 4;

template <int T0, int T1>
struct ShiftTileLayout {
  static constexpr int ROWS = T0 * T1;
  // 32 words after the rows (and the 3 words the last row's z >= 33 cells spill into): one per
  // lane that adds nothing to the tile
  static constexpr int IDLE = ROWS * ROW_WORDS + 4;
  // low words rounded to 32 words so that a high word shares its low word's bank
  static constexpr int LO_WORDS = (IDLE + 32 + 31) / 32 * 32;
  static constexpr int ACC_WORDS = 2 * LO_WORDS;
  static constexpr size_t BYTES = (size_t)ACC_WORDS * 4;
};

// First stencil cell of shift value `shift` along one axis (global index) and its kernel weights.
template <int ORDER>
__device__ __forceinline__ int stencil_axis(float u, float shift, float k[ORDER]) {
  constexpr int OLO = -((ORDER - 1) / 2);
  const float us = __fadd_rn(u, shift);
  const float fi0 = (ORDER & 1) ? rintf(us) : floorf(us);
  k[0] = bspline_at<ORDER, 0>(fabsf(__fsub_rn(__fadd_rn(fi0, (float)OLO), us)));
  if (ORDER > 1) k[ORDER > 1 ? 1 : 0] = bspline_at<ORDER, 1>(fabsf(__fsub_rn(__fadd_rn(fi0, (float)(OLO + 1)), us)));
  if (ORDER > 2) k[ORDER > 2 ? 2 : 0] = bspline_at<ORDER, 2>(fabsf(__fsub_rn(__fadd_rn(fi0, (float)(OLO + 2)), us)));
  if (ORDER > 3) k[ORDER > 3 ? 3 : 0] = bspline_at<ORDER, 3>(fabsf(__fsub_rn(__fadd_rn(fi0, (float)(OLO + 3)), us)));
  return (int)fi0 + OLO;
}

// First stencil cell along the last axis relative to the tile origin z0, as the representative
// of (first - z0) mod n in [-8, n - 8) (n >= 64): for every bucket copy of the tile it lies in
// [-4, 32], the periodic wrap included.
__device__ __forceinline__ int tile_z(int first, int z0, int n) {
  int r = wrapi(first - z0, n);
  return r >= n - 8 ? r - n : r;
}

template <int ORDER, int T0, int T1, int SHIFT_TILE_THREADS>
__global__ void __launch_bounds__(SHIFT_TILE_THREADS) paint_shift_tile_kernel(
    PaintGeom g, const float4 *__restrict__ bucket, const int *__restrict__ offsets,
    const unsigned *__restrict__ wmax_bits, float *__restrict__ out) {
  using L = ShiftTileLayout<T0, T1>;
  constexpr int T2 = 32;
  constexpr int NWARPS = SHIFT_TILE_THREADS / 32;
  constexpr int GROUPS = T0 * T1 * (T2 / 4);  // float4 groups of the write-out
  extern __shared__ __align__(16) unsigned acc[];  // lo [LO_WORDS], hi [LO_WORDS]
  const int64_t gtile = blockIdx.x / g.nshifts;
  const int s = (int)(blockIdx.x % g.nshifts);
  const int mock = (int)(gtile / g.tiles_per_mock);
  const int tile = (int)(gtile % g.tiles_per_mock);
  const int t2i = tile % g.nt[2];
  const int t1i = (tile / g.nt[2]) % g.nt[1];
  const int t0i = tile / (g.nt[2] * g.nt[1]);
  const int x0 = t0i * T0, y0 = t1i * T1, z0 = t2i * T2;
  const int begin = offsets[gtile];
  const int count = offsets[gtile + 1] - begin;
  float *mesh = out + ((int64_t)mock * g.nshifts + s) * g.d.nreal();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  if (count == 0) {
    for (int i = tid; i < GROUPS; i += SHIFT_TILE_THREADS) {
      const int row = i / (T2 / 4), z = (i % (T2 / 4)) * 4;
      const int x = x0 + row / T1, y = y0 + row % T1;
      if (x < g.d.n0 && y < g.d.n1 && z0 + z < g.d.n2)
        *reinterpret_cast<float4 *>(mesh + ((int64_t)x * g.d.n1 + y) * g.d.n2 + z0 + z) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    return;
  }
  {
    uint4 *z4 = reinterpret_cast<uint4 *>(acc);
    for (int i = tid; i < L::ACC_WORDS / 4; i += SHIFT_TILE_THREADS) z4[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  __syncthreads();
  const long long ncat = g.offsets ? (long long)(g.offsets[mock + 1] - g.offsets[mock]) : (long long)g.n;
  const int fexp = fixed_exponent(*wmax_bits, ncat);
  float fscale0, fscale1;
  fixed_scales(fexp, &fscale0, &fscale1);
  const float shift = g.shifts[s];
  const unsigned acc_base = (unsigned)__cvta_generic_to_shared(acc);
  constexpr unsigned HI = 4u * L::LO_WORDS;  // byte distance from a low word to its high word
  const unsigned idle_addr = acc_base + 4u * (unsigned)(L::IDLE + lane);
  const float4 *entries = bucket + begin;

  const int S = (count + 31) >> 5;
  // each lane's entry of the warp's next slot is loaded one slot ahead (L2 latency behind the atomics)
  float4 qn = warp < S && lane * S + warp < count ? entries[lane * S + warp] : make_float4(0.f, 0.f, 0.f, 0.f);
  for (int j = warp; j < S; j += NWARPS) {
    const int e = lane * S + j;
    const bool has = e < count;
    const float4 q = qn;
    const int en = e + NWARPS;
    if (j + NWARPS < S && en < count) qn = entries[en];
    const float wq = has ? __fmul_rn(__fmul_rn(q.w, fscale0), fscale1) : 0.f;
    float kx[ORDER], ky[ORDER], kz[ORDER];
    const int fx = stencil_axis<ORDER>(q.x, shift, kx);
    const int fy = stencil_axis<ORDER>(q.y, shift, ky);
    const int fz = stencil_axis<ORDER>(q.z, shift, kz);
    const unsigned zbyte = 4u * (unsigned)(tile_z(fz, z0, g.d.n2) + ROW_ZOFF);
    int xr[ORDER], yr[ORDER];
#pragma unroll
    for (int o = 0; o < ORDER; ++o) {
      xr[o] = wrapi(fx + o, g.d.n0) - x0;
      yr[o] = wrapi(fy + o, g.d.n1) - y0;
    }
#pragma unroll
    for (int a = 0; a < ORDER; ++a) {
#pragma unroll
      for (int b = 0; b < ORDER; ++b) {
        const float kab = __fmul_rn(kx[a], ky[b]);
        // a lane without an entry, or whose stencil row is outside the tile, adds to its own
        // idle word (lanes of one instruction then never share a word there)
        const bool in = has && (unsigned)xr[a] < (unsigned)T0 && (unsigned)yr[b] < (unsigned)T1;
        const unsigned addr = in ? acc_base + 4u * (unsigned)((xr[a] * T1 + yr[b]) * ROW_WORDS) + zbyte : idle_addr;
        const unsigned step = in ? 4u : 0u;
#pragma unroll
        for (int c = 0; c < ORDER; ++c) {
          const long long v = __float2ll_rn(__fmul_rn(wq, __fmul_rn(kab, kz[c])));  // (w * ker) 2^fexp
          const unsigned lo = (unsigned)v;
          const unsigned old = atom_add_shared(addr + step * c, lo);
          red_add_shared(addr + step * c + HI, add_carry_hi(old, lo, (unsigned)(v >> 32)));
        }
      }
    }
  }
  __syncthreads();
  float inv0, inv1;
  fixed_inverse(fexp, &inv0, &inv1);
  for (int i = tid; i < GROUPS; i += SHIFT_TILE_THREADS) {
    const int row = i / (T2 / 4), z = (i % (T2 / 4)) * 4;
    const int x = x0 + row / T1, y = y0 + row % T1;
    if (x >= g.d.n0 || y >= g.d.n1 || z0 + z >= g.d.n2) continue;
    const unsigned *lo = acc + row * ROW_WORDS + ROW_ZOFF + z, *hi = lo + L::LO_WORDS;  // rows are not 16 B aligned
    *reinterpret_cast<float4 *>(mesh + ((int64_t)x * g.d.n1 + y) * g.d.n2 + z0 + z) =
        make_float4(fixed_to_float(lo[0], hi[0], inv0, inv1), fixed_to_float(lo[1], hi[1], inv0, inv1),
                    fixed_to_float(lo[2], hi[2], inv0, inv1), fixed_to_float(lo[3], hi[3], inv0, inv1));
  }
}

// Gather (resamplers.read) plus the position gradient of paint's adjoint, read at u + shift.
template <int ORDER>
__global__ void __launch_bounds__(256) read_kernel(PaintGeom g, const float *__restrict__ mesh, float shift,
                                                   const float *__restrict__ pos, const float *__restrict__ w,
                                                   int64_t n, float scale, float *__restrict__ out,
                                                   float *__restrict__ grad, int accumulate) {
  const int ns[3] = {g.d.n0, g.d.n1, g.d.n2};
  constexpr int OLO = -((ORDER - 1) / 2);
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    float u[3], wp;
    load_particle(g, pos, w, p, u, &wp);
    float k[3][ORDER], dk[3][ORDER];
    int idx[3][ORDER];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float ud = __fadd_rn(u[d], shift);
      const int i0 = base_index(ORDER, ud);
#pragma unroll
      for (int q = 0; q < ORDER; ++q) {
        const int ii = i0 + OLO + q;
        const float diff = __fsub_rn((float)ii, ud);
        const float sd = fabsf(diff);
        k[d][q] = bspline(ORDER, sd);
        // ds/du = -sign(idx - u); sign(0) = 0 as in JAX's abs derivative
        const float sgn = diff > 0.f ? -1.f : (diff < 0.f ? 1.f : 0.f);
        dk[d][q] = bspline_deriv(ORDER, sd) * sgn;
        idx[d][q] = wrapi(ii, ns[d]);
      }
    }
    float acc = 0.f, g0 = 0.f, g1 = 0.f, g2 = 0.f;
#pragma unroll
    for (int a = 0; a < ORDER; ++a)
#pragma unroll
      for (int b = 0; b < ORDER; ++b) {
        const int64_t row = ((int64_t)idx[0][a] * g.d.n1 + idx[1][b]) * g.d.n2;
        const float kab = __fmul_rn(k[0][a], k[1][b]);
#pragma unroll
        for (int c = 0; c < ORDER; ++c) {
          const float m = mesh[row + idx[2][c]];
          acc = __fadd_rn(acc, __fmul_rn(m, __fmul_rn(kab, k[2][c])));
          if (grad) {
            g0 += m * dk[0][a] * k[1][b] * k[2][c];
            g1 += m * k[0][a] * dk[1][b] * k[2][c];
            g2 += m * kab * dk[2][c];
          }
        }
      }
    if (out) out[p] = accumulate ? out[p] + scale * acc : scale * acc;
    if (grad) {
      const float f = scale * wp;
      const float v0 = f * g0 / g.cell[0], v1 = f * g1 / g.cell[1], v2 = f * g2 / g.cell[2];
      float *gp = grad + 3 * p;
      if (accumulate) {
        gp[0] += v0;
        gp[1] += v1;
        gp[2] += v2;
      } else {
        gp[0] = v0;
        gp[1] = v1;
        gp[2] = v2;
      }
    }
  }
}

static pk_status launch_read(cudaStream_t stream, const PaintGeom &g, const float *mesh, float shift,
                             const float *positions, const float *weights, int64_t n, float scale, float *out,
                             float *grad, int accumulate) {
  if (n == 0) return PK_OK;
  const int threads = 256;
  const int64_t want = (n + threads - 1) / threads;
  const int blocks = (int)(want < 64LL * sm_count() ? want : 64LL * sm_count());
  switch (g.order) {
#define PK_READ_CASE(O)                                                                                   \
  case O:                                                                                                 \
    read_kernel<O><<<blocks, threads, 0, stream>>>(g, mesh, shift, positions, weights, n, scale, out, grad, \
                                                   accumulate);                                           \
    break;
    PK_READ_CASE(1) PK_READ_CASE(2) PK_READ_CASE(3) PK_READ_CASE(4)
#undef PK_READ_CASE
  }
  PK_LAUNCH_CHECK();
  return PK_OK;
}

static bool fill_geom(const int32_t meshsize[3], const float boxsize[3], const float boxcenter[3],
                      const float cellsize[3], int order, int nshifts, const float *shifts,
                      int config, int nmocks, PaintGeom *g) {
  if (!make_dims(meshsize, &g->d)) return false;
  if (order < 1 || order > MAX_ORDER) return false;
  if (nshifts < 1 || nshifts > MAX_SHIFTS) return false;
  if (config < 0 || config >= NUM_TILE_CONFIGS) return false;
  if (nmocks < 1) return false;
  for (int d = 0; d < 3; ++d) {
    g->half[d] = boxsize[d] / 2.f;
    g->center[d] = boxcenter[d];
    g->cell[d] = cellsize[d];
    if (!(cellsize[d] > 0.f)) return false;
  }
  g->order = order;
  g->nshifts = nshifts;
  bool shifted = false;
  for (int s = 0; s < MAX_SHIFTS; ++s) {
    g->shifts[s] = s < nshifts ? shifts[s] : 0.f;
    shifted |= (s < nshifts && shifts[s] != 0.f);
  }
  // stencil of shift s: base_index(u + s) + [-lo, hi], and base_index(u + s) is base_index(u)
  // or base_index(u) + 1 for 0 <= s < 1: the bucket key is base_index(u), reach [-lo, hi + 1]
  const int hi = order - 1 - (order - 1) / 2;
  g->reach_lo = (order - 1) / 2;
  g->reach_hi = hi + (shifted ? 1 : 0);
  int threads;
  tile_dims(config, g->tile, &threads);
  for (int d = 0; d < 3; ++d) {
    g->nt[d] = (meshsize[d] + g->tile[d] - 1) / g->tile[d];
    g->tshift[d] = 0;
    while ((1 << g->tshift[d]) < g->tile[d]) ++g->tshift[d];
    if ((1 << g->tshift[d]) != g->tile[d]) return false;
  }
  g->tiles_per_mock = (int64_t)g->nt[0] * g->nt[1] * g->nt[2];
  g->nmocks = nmocks;
  g->offsets = nullptr;
  g->n = 0;
  return true;
}

static int max_copies_axis(int n, int tile, int nt, int span) {
  if (nt <= 1) return 1;
  int last = n - (nt - 1) * tile;
  int c = (last >= span - 1 || last == tile) ? 2 : 3;
  return c < nt ? c : nt;
}

struct PaintLayout {
  int64_t ntiles;
  int64_t max_entries;
  size_t scan_bytes;
  size_t total;
};

constexpr int HIST_MAX_CTAS = 256;

// The shared-histogram bucket passes serve tile index spaces that fit in shared memory.
static bool hist_bucket(const PaintLayout &L) { return L.ntiles <= HIST_MAX_TILES; }

static pk_status paint_layout(int64_t n, const PaintGeom &g, PaintLayout *L) {
  L->ntiles = g.tiles_per_mock * g.nmocks;
  PK_REQUIRE(L->ntiles < (int64_t)INT32_MAX / 2, PK_ERR_RANGE, "too many tiles (%lld)",
             (long long)L->ntiles);
  const int span = g.reach_lo + g.reach_hi + 1;
  const int ns[3] = {g.d.n0, g.d.n1, g.d.n2};
  int64_t copies = 1;
  for (int d = 0; d < 3; ++d) copies *= max_copies_axis(ns[d], g.tile[d], g.nt[d], span);
  L->max_entries = n * copies;
  PK_REQUIRE(L->max_entries < (int64_t)INT32_MAX, PK_ERR_RANGE,
             "too many particles for one paint call (%lld x %lld tile copies)", (long long)n,
             (long long)copies);
  L->scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, L->scan_bytes, (unsigned *)nullptr, (int *)nullptr,
                                (int)(L->ntiles + 1));
  Carver c(nullptr);
  c.take<unsigned>(L->ntiles + 1);  // counts
  c.take<int>(L->ntiles + 1);       // offsets
  c.take<unsigned>(L->ntiles);      // cursors
  c.take<unsigned>(4);              // wmax bits
  c.take<char>(L->scan_bytes);
  c.take<float4>(L->max_entries);
  if (hist_bucket(*L)) c.take<unsigned>((size_t)HIST_MAX_CTAS * L->ntiles);  // (CTA, tile) counts
  L->total = align_up(c.used);
  return PK_OK;
}

// Configurations 8 to 10 take the per-shift tile kernel when the last axis is a multiple of 4
// (float4 rows) and has at least 64 cells (unambiguous tile-relative z, see tile_z); on other
// meshes they stand for configuration 4 (effective_config).
static bool shift_tile_mesh(const int32_t meshsize[3]) { return meshsize[2] % 4 == 0 && meshsize[2] >= 64; }

static bool shift_tile_config(int config) { return config >= 8 && config < NUM_TILE_CONFIGS; }

static int effective_config(int config, const int32_t meshsize[3]) {
  return (shift_tile_config(config) && meshsize && !shift_tile_mesh(meshsize)) ? 4 : config;
}

static bool shift_tile_eligible(int config, const PaintGeom &g) {
  const int32_t ms[3] = {g.d.n0, g.d.n1, g.d.n2};
  return shift_tile_config(config) && shift_tile_mesh(ms);
}

template <int ORDER, int C>
static pk_status launch_shift_tile(cudaStream_t s, const PaintGeom &g, const float4 *bucket, const int *offsets,
                                   const unsigned *wmax, float *out, int64_t ntiles) {
  using TC = TileConfig<C>;
  const size_t smem = ShiftTileLayout<TC::T0, TC::T1>::BYTES;
  PK_REQUIRE(ntiles * g.nshifts < (int64_t)INT32_MAX, PK_ERR_RANGE, "too many tiles x shifts (%lld)",
             (long long)(ntiles * g.nshifts));
  auto kernel = paint_shift_tile_kernel<ORDER, TC::T0, TC::T1, TC::THREADS>;
  PK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kernel<<<(unsigned)(ntiles * g.nshifts), TC::THREADS, smem, s>>>(g, bucket, offsets, wmax, out);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

static pk_status launch_shift_tiles(cudaStream_t s, const PaintGeom &g, int config, const float4 *bucket,
                                    const int *offsets, const unsigned *wmax, float *out, int64_t ntiles) {
  switch (config * 8 + g.order) {
#define PK_ST_CASE(C, O) \
  case C * 8 + O:        \
    return launch_shift_tile<O, C>(s, g, bucket, offsets, wmax, out, ntiles);
#define PK_ST_CFG(C) PK_ST_CASE(C, 1) PK_ST_CASE(C, 2) PK_ST_CASE(C, 3) PK_ST_CASE(C, 4)
    PK_ST_CFG(8) PK_ST_CFG(9) PK_ST_CFG(10)
#undef PK_ST_CFG
#undef PK_ST_CASE
  }
  set_error("no per-shift tile kernel for order %d", g.order);
  return PK_ERR_INVALID;
}

static pk_status paint_run(cudaStream_t s, const float *positions, const float *weights,
                           int64_t n, PaintGeom g, int config, float *out, void *workspace,
                           size_t workspace_bytes, int *d_status) {
  PaintLayout L;
  g.n = n;
  pk_status st = paint_layout(n, g, &L);
  if (st) return st;
  PK_REQUIRE(workspace && workspace_bytes >= L.total, PK_ERR_WORKSPACE,
             "paint workspace too small: need %zu bytes, got %zu", L.total, workspace_bytes);
  Carver c(workspace);
  unsigned *counts = c.take<unsigned>(L.ntiles + 1);
  int *offsets = c.take<int>(L.ntiles + 1);
  unsigned *cursors = c.take<unsigned>(L.ntiles);
  unsigned *wmax = c.take<unsigned>(4);
  void *scan_tmp = c.take<char>(L.scan_bytes);
  float4 *bucket = c.take<float4>(L.max_entries);

  PK_CUDA(cudaMemsetAsync(wmax, 0, 4 * sizeof(unsigned), s));
  size_t scan_bytes = L.scan_bytes;
  if (hist_bucket(L)) {
    // per-CTA shared counters over contiguous particle ranges, a column scan of the
    // (CTA, tile) counts, the tile offsets, then the placement (shared-memory atomics only)
    unsigned *colmat = c.take<unsigned>((size_t)HIST_MAX_CTAS * L.ntiles);
    const int ntiles = (int)L.ntiles;
    const int64_t want = (n + HIST_THREADS - 1) / HIST_THREADS;
    const int nctas = (int)std::max<int64_t>(1, std::min<int64_t>(want, std::min(sm_count(), HIST_MAX_CTAS)));
    const int64_t chunk = (n + nctas - 1) / nctas;
    const size_t hsmem = (size_t)ntiles * sizeof(unsigned);
    PK_CUDA(cudaFuncSetAttribute(bucket_hist_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem));
    PK_CUDA(cudaFuncSetAttribute(bucket_hist_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem));
    bucket_hist_kernel<false><<<nctas, HIST_THREADS, hsmem, s>>>(g, positions, weights, n, chunk, ntiles, colmat,
                                                                 nullptr, nullptr, wmax, d_status);
    PK_LAUNCH_CHECK();
    bucket_colscan_kernel<<<(ntiles + 1 + 255) / 256, 256, 0, s>>>(colmat, nctas, ntiles, counts);
    PK_LAUNCH_CHECK();
    PK_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, counts, offsets, ntiles + 1, s));
    bucket_hist_kernel<true><<<nctas, HIST_THREADS, hsmem, s>>>(g, positions, weights, n, chunk, ntiles, colmat,
                                                                offsets, bucket, nullptr, nullptr);
    PK_LAUNCH_CHECK();
  } else {
    PK_CUDA(cudaMemsetAsync(counts, 0, (L.ntiles + 1) * sizeof(unsigned), s));
    PK_CUDA(cudaMemsetAsync(cursors, 0, L.ntiles * sizeof(unsigned), s));
    const int threads = 256;
    const int64_t want = (n + threads - 1) / threads;
    const int blocks = (int)(want < 64LL * sm_count() ? (want > 0 ? want : 1) : 64LL * sm_count());
    if (n > 0) {
      bucket_kernel<false><<<blocks, threads, 0, s>>>(g, positions, weights, n, counts, nullptr,
                                                      nullptr, nullptr, wmax, d_status);
      PK_LAUNCH_CHECK();
    }
    PK_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, counts, offsets,
                                          (int)(L.ntiles + 1), s));
    if (n > 0) {
      bucket_kernel<true><<<blocks, threads, 0, s>>>(g, positions, weights, n, nullptr, offsets,
                                                     cursors, bucket, nullptr, nullptr);
      PK_LAUNCH_CHECK();
    }
  }
  int tdims[3], tthreads;
  tile_dims(config, tdims, &tthreads);
  if (shift_tile_eligible(config, g)) return launch_shift_tiles(s, g, config, bucket, offsets, wmax, out, L.ntiles);
  // accumulators (lo, hi words per shift and cell) + 64 scratch words for masked-off lanes
  const size_t smem = ((size_t)g.nshifts * tdims[0] * tdims[1] * tdims[2] * 2 + 64) * sizeof(unsigned);
  switch (config * 8 + g.order) {  // all-shifts tile kernel
#define PK_PAINT_CASE(C, O)                                                                    \
  case C * 8 + O:                                                                              \
    PK_CUDA(cudaFuncSetAttribute(paint_tiles_kernel<O, C>,                                     \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));     \
    paint_tiles_kernel<O, C><<<(unsigned)L.ntiles, TileConfig<C>::THREADS, smem, s>>>(        \
        g, bucket, offsets, wmax, out);                                                        \
    break;
#define PK_PAINT_CFG(C) PK_PAINT_CASE(C, 1) PK_PAINT_CASE(C, 2) PK_PAINT_CASE(C, 3) PK_PAINT_CASE(C, 4)
    PK_PAINT_CFG(0) PK_PAINT_CFG(1) PK_PAINT_CFG(2) PK_PAINT_CFG(3) PK_PAINT_CFG(4) PK_PAINT_CFG(5)
    PK_PAINT_CFG(6) PK_PAINT_CFG(7)
    default:  // 8 to 10 took the per-shift kernel above or were mapped to 4 (effective_config)
      set_error("no tile kernel for configuration %d", config);
      return PK_ERR_INVALID;
#undef PK_PAINT_CFG
#undef PK_PAINT_CASE
  }
  PK_LAUNCH_CHECK();
  return PK_OK;
}

static pk_status make_shifts(int interlacing, int shift_begin, int nshifts, float shifts[MAX_SHIFTS]) {
  PK_REQUIRE(interlacing >= 1 && shift_begin >= 0 && nshifts >= 1 && nshifts <= MAX_SHIFTS &&
                 shift_begin + nshifts <= interlacing,
             PK_ERR_INVALID, "invalid interlacing %d / shift range [%d, %d)", interlacing,
             shift_begin, shift_begin + nshifts);
  for (int s = 0; s < MAX_SHIFTS; ++s)  // arange(I) * 1. / I in float32 (mesh.py:2679)
    shifts[s] = s < nshifts ? (float)(shift_begin + s) / (float)interlacing : 0.f;
  return PK_OK;
}

}  // namespace pk

using namespace pk;

extern "C" pk_status pk_paint_batch_workspace_size(int64_t n, int nmocks, const int32_t meshsize[3],
                                                   int order, int nshifts, int tile_config,
                                                   size_t *bytes) {
  PK_REQUIRE(bytes, PK_ERR_INVALID, "bytes is NULL");
  PK_REQUIRE(n >= 0, PK_ERR_INVALID, "negative particle count");
  float box[3] = {1.f, 1.f, 1.f}, cen[3] = {0.f, 0.f, 0.f}, cell[3] = {1.f, 1.f, 1.f};
  // worst-case reach: any nonzero shift
  float shifts[MAX_SHIFTS] = {0.f, 0.5f, 0.5f, 0.5f};
  if (nshifts > MAX_SHIFTS) nshifts = MAX_SHIFTS;
  if (meshsize) tile_config = effective_config(tile_config, meshsize);
  PaintGeom g;
  PK_REQUIRE(fill_geom(meshsize, box, cen, cell, order, nshifts, shifts, tile_config, nmocks, &g),
             PK_ERR_INVALID,
             "invalid meshsize / order (1..4) / nshifts (1..%d) / tile config / nmocks", MAX_SHIFTS);
  PaintLayout L;
  pk_status st = paint_layout(n, g, &L);
  if (st) return st;
  *bytes = L.total;
  return PK_OK;
}

extern "C" pk_status pk_paint_workspace_size(int64_t n, const int32_t meshsize[3], int order,
                                             int nshifts, size_t *bytes) {
  // the larger workspace of the two configurations pk_paint may pick
  PK_REQUIRE(bytes, PK_ERR_INVALID, "bytes is NULL");
  size_t a = 0, b = 0;
  pk_status st = pk_paint_batch_workspace_size(n, 1, meshsize, order, nshifts, 4, &a);
  if (st) return st;
  st = pk_paint_batch_workspace_size(n, 1, meshsize, order, nshifts, 9, &b);
  if (st) return st;
  *bytes = a > b ? a : b;
  return PK_OK;
}

extern "C" pk_status pk_paint_batch(void *stream, const float *positions, const float *weights,
                                    const int64_t *d_offsets, int64_t n, int nmocks,
                                    const int32_t meshsize[3], const float boxsize[3],
                                    const float boxcenter[3], const float cellsize[3], int order,
                                    int interlacing, int shift_begin, int nshifts, int tile_config,
                                    float *out, void *workspace, size_t workspace_bytes,
                                    int *d_status) {
  PK_REQUIRE(out, PK_ERR_INVALID, "out is NULL");
  PK_REQUIRE(n == 0 || positions, PK_ERR_INVALID, "positions is NULL");
  PK_REQUIRE(boxsize && boxcenter && cellsize, PK_ERR_INVALID, "geometry pointer is NULL");
  PK_REQUIRE(nmocks == 1 || d_offsets, PK_ERR_INVALID, "offsets are required for several mocks");
  float shifts[MAX_SHIFTS];
  pk_status st = make_shifts(interlacing, shift_begin, nshifts, shifts);
  if (st) return st;
  if (meshsize) tile_config = effective_config(tile_config, meshsize);
  PaintGeom g;
  PK_REQUIRE(fill_geom(meshsize, boxsize, boxcenter, cellsize, order, nshifts, shifts, tile_config,
                       nmocks, &g),
             PK_ERR_INVALID,
             "invalid meshsize / order (1..4) / nshifts (1..%d) / cellsize / tile config / nmocks",
             MAX_SHIFTS);
  g.offsets = nmocks > 1 ? d_offsets : nullptr;
  return paint_run((cudaStream_t)stream, positions, weights, n, g, tile_config, out, workspace,
                   workspace_bytes, d_status);
}

extern "C" pk_status pk_paint(void *stream, const float *positions, const float *weights,
                              int64_t n, const int32_t meshsize[3], const float boxsize[3],
                              const float boxcenter[3], const float cellsize[3], int order,
                              int interlacing, int shift_begin, int nshifts, float *out,
                              void *workspace, size_t workspace_bytes, int *d_status) {
  // the per-shift tile kernel (16 x 16 x 32 tiles) where the mesh allows it, else the swizzled
  // all-shifts kernel
  const int config = (meshsize && shift_tile_mesh(meshsize)) ? 9 : 4;
  return pk_paint_batch(stream, positions, weights, nullptr, n, 1, meshsize, boxsize, boxcenter,
                        cellsize, order, interlacing, shift_begin, nshifts, config, out, workspace,
                        workspace_bytes, d_status);
}

extern "C" pk_status pk_read(void *stream, const float *mesh, const float *positions,
                             const float *weights, int64_t n, const int32_t meshsize[3],
                             const float boxsize[3], const float boxcenter[3],
                             const float cellsize[3], int order, float shift, float scale,
                             float *out, float *grad, int accumulate) {
  PK_REQUIRE(mesh && (n == 0 || positions), PK_ERR_INVALID, "mesh / positions is NULL");
  PK_REQUIRE(out || grad, PK_ERR_INVALID, "nothing to write (out and grad NULL)");
  float shifts[MAX_SHIFTS] = {0.f, 0.f, 0.f, 0.f};
  PaintGeom g;
  PK_REQUIRE(fill_geom(meshsize, boxsize, boxcenter, cellsize, order, 1, shifts, 0, 1, &g),
             PK_ERR_INVALID, "invalid meshsize / order / cellsize");
  return launch_read((cudaStream_t)stream, g, mesh, shift, positions, weights, n, scale, out, grad, accumulate);
}

extern "C" pk_status pk_read_interlaced(void *stream, const float *meshes, int interlacing,
                                        const float *positions, const float *weights, int64_t n,
                                        const int32_t meshsize[3], const float boxsize[3],
                                        const float boxcenter[3], const float cellsize[3], int order,
                                        float scale, float *out, float *grad, int accumulate) {
  PK_REQUIRE(meshes && (n == 0 || positions), PK_ERR_INVALID, "meshes / positions is NULL");
  PK_REQUIRE(out || grad, PK_ERR_INVALID, "nothing to write (out and grad NULL)");
  PK_REQUIRE(interlacing >= 1 && interlacing <= 8, PK_ERR_INVALID, "interlacing must be in 1..8");
  float shifts[MAX_SHIFTS] = {0.f, 0.f, 0.f, 0.f};
  PaintGeom g;
  PK_REQUIRE(fill_geom(meshsize, boxsize, boxcenter, cellsize, order, 1, shifts, 0, 1, &g),
             PK_ERR_INVALID, "invalid meshsize / order / cellsize");
  // one pass per shifted mesh, each adding into the previous: a pass reads a single mesh,
  // whose random-access working set the L2 holds far better than all meshes at once
  for (int s = 0; s < interlacing; ++s) {
    pk_status st = launch_read((cudaStream_t)stream, g, meshes + (int64_t)s * g.d.nreal(),
                               (float)s / (float)interlacing, positions, weights, n, scale, out, grad,
                               s > 0 || accumulate);
    if (st) return st;
  }
  return PK_OK;
}
