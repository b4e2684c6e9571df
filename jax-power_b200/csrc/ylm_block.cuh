// Y_lm(xhat) for whole ells at compile time.
//
// A "mask" names a set of multipoles (bit ell set for each ell); its terms are every
// (ell, m) of those ells, ell ascending, m = -ell .. ell (the order of _firstpoint_terms in
// mesh2.py).  The helpers below expand ylm_eval with constant (ell, m), so each Y_lm is its
// own short polynomial instead of a run-time switch, and every term sits at a fixed
// register index.
#pragma once

#include "ylm_table.cuh"

namespace pk {

__host__ __device__ constexpr int ylm_mask_terms(int mask) {
  int n = 0;
  for (int ell = 0; ell <= YLM_LMAX; ++ell)
    if ((mask >> ell) & 1) n += 2 * ell + 1;
  return n;
}

__host__ __device__ constexpr int ylm_mask_ells(int mask) {
  int n = 0;
  for (int ell = 0; ell <= YLM_LMAX; ++ell) n += (mask >> ell) & 1;
  return n;
}

// Masks with a compiled kernel: every single ell 1..8, {1, 3}, {2, 4}, {1, 2, 3, 4}, {2, 4, 6}.
#define PK_YLM_MASKS(X) \
  X(0x002) X(0x004) X(0x008) X(0x010) X(0x020) X(0x040) X(0x080) X(0x100) X(0x00A) X(0x014) X(0x01E) X(0x054)

// The mask of a term list that is whole ells in canonical order, 0 otherwise.
inline int ylm_terms_mask(int nterms, const int32_t *term_ell, const int32_t *term_m) {
  int mask = 0, t = 0, prev = 0;
  while (t < nterms) {
    const int ell = term_ell[t];
    if (ell <= prev || ell > YLM_LMAX) return 0;
    for (int m = -ell; m <= ell; ++m, ++t)
      if (t >= nterms || term_ell[t] != ell || term_m[t] != m) return 0;
    mask |= 1 << ell;
    prev = ell;
  }
  return mask;
}

inline bool ylm_mask_compiled(int mask) {
#define PK_YLM_MASK_EQ(M) if (mask == (M)) return true;
  PK_YLM_MASKS(PK_YLM_MASK_EQ)
#undef PK_YLM_MASK_EQ
  return false;
}

// out[T + (m + ELL)] = Y_{ELL m}(x, y, z) for every term of MASK from ELL on.
template <int MASK, int ELL, int M, int T, int NT>
__device__ __forceinline__ void ylm_fill(float x, float y, float z, float (&out)[NT]) {
  if constexpr (ELL <= YLM_LMAX) {
    if constexpr ((MASK >> ELL) & 1) {
      out[T] = ylm_eval(ELL, M, x, y, z);
      if constexpr (M < ELL) ylm_fill<MASK, ELL, M + 1, T + 1>(x, y, z, out);
      else ylm_fill<MASK, ELL + 1, -(ELL + 1), T + 1>(x, y, z, out);
    } else {
      ylm_fill<MASK, ELL + 1, -(ELL + 1), T>(x, y, z, out);
    }
  }
}

template <int MASK, int NT>
__device__ __forceinline__ void ylm_block(float x, float y, float z, float (&out)[NT]) {
  static_assert(NT == ylm_mask_terms(MASK), "term count");
  ylm_fill<MASK, 0, 0, 0>(x, y, z, out);
}

}  // namespace pk
