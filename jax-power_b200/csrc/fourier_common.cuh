// Interlacing + compensation arithmetic shared by the Fourier-space kernels (fourier.cu)
// and the fused interlace + binning kernel (binning.cu).  The combination of the shifted
// meshes follows _paint (mesh.py:2737-2752): sum_s e^{i s (kx + ky + kz)} F_s / I, with the
// circular k grid (mesh.py:1627-1629), times the compensation prod_d sinc(k_d / 2pi)^-p
// (resamplers.py:16-26).  Phases and windows are factored per axis: a per-row factor (x, y)
// times a per-kz factor from a shared-memory table, which differs from the reference's
// single product by float32 rounding only.
#pragma once
#include <math.h>

#include "common.cuh"

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
  // Per-axis tables in global memory (phx [nshifts][n0], phy [nshifts][n1], then sx [n0] and
  // sy [n1] as floats), filled by fill_xy_tables_kernel; NULL: the kernel keeps them in shared
  // memory (when use_xy_tables) or computes its row factors.
  float2 *gxy;
};

// jnp.sinc(k / 2pi) with the reference's float32 operations (resamplers.py:21).
__device__ __forceinline__ float sinc_of(float kc) {
  const float x = __fdiv_rn(kc, 6.2831855f);  // float32(2 pi)
  if (x == 0.f) return 1.f;
  const float px = __fmul_rn(3.1415927f, x);
  return __fdiv_rn(sinf(px), px);
}

// (window)^(-order): lax.integer_pow by binary exponentiation, then the reciprocal.
__device__ __forceinline__ float inverse_power(float ker, int order) {
  int y = order;
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
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 expi(float t) {
  float sn, cs;
  sincosf(t, &sn, &cs);
  return make_float2(cs, sn);
}

constexpr int IL_MAX_SHIFTS = 8;

// Per-CTA tables (shared memory).  Along kz: for each shift s, e^{i s kz(z)} and, for the
// 'jaxdecomp' semantics, e^{-i s kz(-z)} on the full grid; plus sinc(kz / 2pi)^-p.  Along
// kx and ky (when use_xy_tables): e^{i s k(i)} per shift and sinc(k / 2pi), from which the
// per-row factors are formed with a complex product and a multiply instead of sines and
// divisions per row.
struct ZTable {
  float2 *ph;    // [nshifts][nz]
  float2 *phm;   // [nshifts][nz] (jaxdecomp)
  float2 *phx;   // [nshifts][n0]
  float2 *phy;   // [nshifts][n1]
  float *comp;   // [nz]: sinc(kz / 2pi)^-p (1 without compensation)
  float *sx;     // [n0]: sinc(kx / 2pi)
  float *sy;     // [n1]: sinc(ky / 2pi)
};

// The x / y tables are kept for meshes with n0 + n1 <= 512: they replace the per-row sines
// and divisions, which matters on short rows (batched 128^3..256^3 fused binning: 15-27 %
// faster), while on long rows the per-row cost is small and the tables' shared memory would
// be taken from the L1 cache that the row walk's strided loads rely on (512^3: 1.04 ms with
// the tables against 0.81 ms without).
__host__ __device__ inline bool use_xy_tables(const Dims &d) { return d.n0 + d.n1 <= 512; }

// Row factors: the phase over x, y per shift, and the row's real scale.
template <int NS>
struct RowFactor {
  float2 ph[NS];
  float2 phm[NS];
  float scale;  // (sinc(kx / 2pi) sinc(ky / 2pi))^-p / I (1 / I without compensation)
};

// XY (the tables exist, use_xy_tables): e^{i s kx} e^{i s ky} (and, jaxdecomp, the conjugate
// of the mirrored row's) and the window product sinc(kx / 2pi) sinc(ky / 2pi) from the
// per-axis tables; else computed for the row: e^{i s (kx + ky)} and the same window product.
template <int NS, bool FULL, bool XY>
__device__ __forceinline__ void row_factor(const FourierParams &p, const ZTable &t, int i, int j,
                                           RowFactor<NS> &r) {
  const Dims &d = p.d;
  constexpr bool full = FULL;
  const float inv = 1.f / p.interlacing;
  const int i2 = (d.n0 - i) % d.n0, j2 = (d.n1 - j) % d.n1;
  if constexpr (!XY) {
    const float k0 = ccoord(i, d.n0, p.cspacing[0], false);
    const float k1 = ccoord(j, d.n1, p.cspacing[1], false);
    const float kxy = k0 + k1;
    const float kxym = ccoord(i2, d.n0, p.cspacing[0], false) + ccoord(j2, d.n1, p.cspacing[1], false);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      r.ph[s] = expi(p.shifts[s] * kxy);
      if (full) r.phm[s] = expi(-p.shifts[s] * kxym);
    }
    r.scale = (p.comp_order > 0 ? inverse_power(__fmul_rn(sinc_of(k0), sinc_of(k1)), p.comp_order) : 1.f) * inv;
    return;
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    r.ph[s] = cmul(t.phx[s * d.n0 + i], t.phy[s * d.n1 + j]);
    if (full) {
      const float2 m = cmul(t.phx[s * d.n0 + i2], t.phy[s * d.n1 + j2]);
      r.phm[s] = make_float2(m.x, -m.y);
    }
  }
  r.scale = (p.comp_order > 0 ? inverse_power(__fmul_rn(t.sx[i], t.sy[j]), p.comp_order) : 1.f) * inv;
}

// row_factor with the table choice made at run time (kernels where it is not register-critical).
template <int NS, bool FULL>
__device__ __forceinline__ void row_factor_rt(const FourierParams &p, const ZTable &t, int i, int j,
                                              RowFactor<NS> &r) {
  if (use_xy_tables(p.d)) row_factor<NS, FULL, true>(p, t, i, j, r);
  else row_factor<NS, FULL, false>(p, t, i, j, r);
}

// Phase of shift s at stored mode (row factor r, z) in the interlaced sum: e^{i s/I (kx + ky + kz)}
// ('jax'), or FULL ('jaxdecomp', full-grid circular coordinates) the Hermitian part
// (e^{i t(k)} + e^{-i t(-k)}) / 2, which differs from e^{i t(k)} on the Nyquist planes only.
template <int NS, bool FULL>
__device__ __forceinline__ float2 mode_phase(const FourierParams &p, const RowFactor<NS> &r, const ZTable &t,
                                             int s, int z) {
  float2 ph = cmul(r.ph[s], t.ph[s * p.d.nz + z]);
  if (FULL) {
    const float2 m = cmul(r.phm[s], t.phm[s * p.d.nz + z]);
    ph = make_float2(0.5f * (ph.x + m.x), 0.5f * (ph.y + m.y));
  }
  return ph;
}

// Interlaced + compensated value of stored mode (row r, z): shift 0 has phase 1, so its
// value enters as is; the others are rotated by their phase; the sum is scaled once by the
// window and 1 / I.
template <int NS, bool FULL>
__device__ __forceinline__ float2 combine_mode(const FourierParams &p, const RowFactor<NS> &r,
                                               const ZTable &t, const float2 *__restrict__ in,
                                               int64_t idx, int z) {
  constexpr bool full = FULL;
  float2 acc = in[idx];
  const int64_t mesh = p.d.ncomplex();
#pragma unroll
  for (int s = 1; s < NS; ++s) {
    const float2 v = in[s * mesh + idx];
    float2 ph = cmul(r.ph[s], t.ph[s * p.d.nz + z]);
    if (full) {  // Hermitian part of the full-grid phase: (e^{i t(k)} + e^{-i t(-k)}) / 2
      const float2 m = cmul(r.phm[s], t.phm[s * p.d.nz + z]);
      ph = make_float2(0.5f * (ph.x + m.x), 0.5f * (ph.y + m.y));
    }
    const float2 c = cmul(v, ph);
    acc.x += c.x;
    acc.y += c.y;
  }
  const float c = r.scale * t.comp[z];
  return make_float2(acc.x * c, acc.y * c);
}

// Where a kernel's per-axis x / y tables are: none (row factors computed per row), in shared
// memory, or in global memory (FourierParams::gxy).
enum { XY_NONE = 0, XY_SMEM = 1, XY_GLOBAL = 2 };

// Fill the per-CTA kz table (and, XY_SMEM, the x / y tables; all threads of the block; call
// __syncthreads() after).
template <bool FULL, int XYM>
__device__ __forceinline__ void fill_ztable(const FourierParams &p, ZTable &t) {
  const Dims &d = p.d;
  for (int z = threadIdx.x; z < d.nz; z += blockDim.x) {
    const float k2 = ccoord(z, d.n2, p.cspacing[2], !FULL);
    const int zm = (d.n2 - z) % d.n2;
    const float k2m = ccoord(zm, d.n2, p.cspacing[2], false);
    for (int s = 0; s < p.nshifts; ++s) {
      t.ph[s * d.nz + z] = expi(p.shifts[s] * k2);
      if (FULL) t.phm[s * d.nz + z] = expi(-p.shifts[s] * k2m);
    }
    t.comp[z] = p.comp_order > 0 ? inverse_power(sinc_of(k2), p.comp_order) : 1.f;
  }
  for (int i = threadIdx.x; XYM == XY_SMEM && i < d.n0 + d.n1; i += blockDim.x) {
    const bool x = i < d.n0;
    const int a = x ? i : i - d.n0;
    const float k = x ? ccoord(a, d.n0, p.cspacing[0], false) : ccoord(a, d.n1, p.cspacing[1], false);
    for (int s = 0; s < p.nshifts; ++s) (x ? t.phx[s * d.n0 + a] : t.phy[s * d.n1 + a]) = expi(p.shifts[s] * k);
    (x ? t.sx[a] : t.sy[a]) = sinc_of(k);
  }
}

// Bytes of the shared-memory tables for nshifts shifts (xy: with the per-axis ones).
inline size_t ztable_bytes(const Dims &d, int nshifts, bool full, bool xy) {
  const size_t nxy = xy ? (size_t)d.n0 + d.n1 : 0;
  return ((size_t)nshifts * (d.nz * (full ? 2 : 1) + nxy)) * sizeof(float2) + (d.nz + nxy) * sizeof(float);
}

// Lay the tables out from `base` (shared memory, 8-byte aligned).
template <int XYM>
__device__ __forceinline__ ZTable ztable_at(void *base, const FourierParams &p, bool full) {
  ZTable t;
  t.ph = reinterpret_cast<float2 *>(base);
  t.phm = t.ph + (size_t)p.nshifts * p.d.nz;
  constexpr bool xy = XYM == XY_SMEM;
  t.phx = t.phm + (full ? (size_t)p.nshifts * p.d.nz : 0);
  t.phy = t.phx + (xy ? (size_t)p.nshifts * p.d.n0 : 0);
  t.comp = reinterpret_cast<float *>(t.phy + (xy ? (size_t)p.nshifts * p.d.n1 : 0));
  t.sx = t.comp + p.d.nz;
  t.sy = t.sx + (xy ? p.d.n0 : 0);
  if (XYM == XY_GLOBAL) {  // per-axis tables in global memory
    t.phx = p.gxy;
    t.phy = t.phx + (size_t)p.nshifts * p.d.n0;
    t.sx = reinterpret_cast<float *>(t.phy + (size_t)p.nshifts * p.d.n1);
    t.sy = t.sx + p.d.n0;
  }
  return t;
}

// Bytes of the global per-axis tables for nshifts shifts.
inline size_t xy_table_bytes(const Dims &d, int nshifts) {
  return (size_t)nshifts * (d.n0 + d.n1) * sizeof(float2) + (size_t)(d.n0 + d.n1) * sizeof(float);
}

// Interlacing shifts s / I and circular spacings: the host-side set-up of FourierParams.
inline bool make_fourier_params(const int32_t meshsize[3], int nshifts, int comp_order, int backend,
                                int for_c2r, float scale, FourierParams *p) {
  if (!make_dims(meshsize, &p->d)) return false;
  if (nshifts < 1 || nshifts > IL_MAX_SHIFTS || comp_order < 0 || comp_order > 4) return false;
  const int ns[3] = {p->d.n0, p->d.n1, p->d.n2};
  for (int a = 0; a < 3; ++a) p->cspacing[a] = (float)(2. * M_PI / ns[a]);
  p->nshifts = nshifts;
  for (int s = 0; s < 8; ++s) p->shifts[s] = s < nshifts ? (float)s / (float)nshifts : 0.f;
  p->interlacing = (float)nshifts;
  p->comp_order = comp_order;
  p->backend = backend;
  p->for_c2r = for_c2r;
  p->scale = scale;
  p->gxy = nullptr;
  return true;
}

}  // namespace pk
