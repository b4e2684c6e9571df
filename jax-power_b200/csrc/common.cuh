// Shared helpers for the jaxpower_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>

#include "../../include/jaxpower_b200.h"

namespace pk {

// ---------------------------------------------------------------- errors
void set_error(const char *fmt, ...);

#define PK_REQUIRE(cond, code, ...)      \
  do {                                   \
    if (!(cond)) {                       \
      ::pk::set_error(__VA_ARGS__);      \
      return (code);                     \
    }                                    \
  } while (0)

#define PK_CUDA(call)                                                             \
  do {                                                                            \
    cudaError_t err_ = (call);                                                    \
    if (err_ != cudaSuccess) {                                                    \
      ::pk::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_),  \
                      __FILE__, __LINE__);                                        \
      return PK_ERR_CUDA;                                                         \
    }                                                                             \
  } while (0)

#define PK_LAUNCH_CHECK() PK_CUDA(cudaGetLastError())

inline int sm_count() {
  static int count = 0;
  if (!count) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
    if (count <= 0) count = 148;
  }
  return count;
}

inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// Carve aligned sub-buffers out of a caller workspace.
struct Carver {
  char *base;
  size_t used = 0;
  explicit Carver(void *p) : base(static_cast<char *>(p)) {}
  template <class T>
  T *take(size_t count) {
    used = align_up(used);
    T *p = reinterpret_cast<T *>(base ? base + used : nullptr);
    used += count * sizeof(T);
    return p;
  }
};

struct Dims {
  int n0, n1, n2;   // real mesh shape
  int nz;           // n2 / 2 + 1
  __host__ __device__ int64_t nreal() const { return (int64_t)n0 * n1 * n2; }
  __host__ __device__ int64_t ncomplex() const { return (int64_t)n0 * n1 * nz; }
};

inline bool make_dims(const int32_t meshsize[3], Dims *d) {
  if (!meshsize) return false;
  for (int i = 0; i < 3; ++i)
    if (meshsize[i] <= 0 || meshsize[i] > (1 << 15)) return false;
  d->n0 = meshsize[0];
  d->n1 = meshsize[1];
  d->n2 = meshsize[2];
  d->nz = meshsize[2] / 2 + 1;
  return true;
}

// ------------------------------------------------------- exact arithmetic
// jnp.fft.fftfreq / rfftfreq index (signed) of position i on an axis of n.
__host__ __device__ inline int signed_freq(int i, int n, bool half) {
  return (half || i < (n + 1) / 2) ? i : i - n;
}

// kcoords (mesh.py:1605-1636): (fftfreq(n)[i] * spacing) * n in float32 with the
// reference's rounding: fftfreq = (float)signed / (float)n (IEEE division).
__device__ __forceinline__ float kcoord(int i, int n, float spacing, bool half) {
  float f = __fdiv_rn((float)signed_freq(i, n, half), (float)n);
  return __fmul_rn(__fmul_rn(f, spacing), (float)n);
}

// Circular coordinate in [-pi, pi): spacing = float32(2 pi / n).
__device__ __forceinline__ float ccoord(int i, int n, float cspacing, bool half) {
  return kcoord(i, n, cspacing, half);
}

struct Complex {
  float re, im;
};

// Row-major (i, j) rows of an n0 x n1 grid visited from `start` with a fixed `stride`,
// advanced without a division per step (one 64-bit division at construction).
struct RowWalker {
  int i, j, si, sj, n1;
  __device__ __forceinline__ RowWalker(int64_t start, int64_t stride, int n1_) : n1(n1_) {
    i = (int)(start / n1_);
    j = (int)(start % n1_);
    si = (int)(stride / n1_);
    sj = (int)(stride % n1_);
  }
  __device__ __forceinline__ void next() {
    j += sj;
    i += si;
    if (j >= n1) {
      j -= n1;
      ++i;
    }
  }
};

// (i, j, k) of a row-major n0 x n1 x n2 grid visited from `start` with a fixed `stride`
// (grid-stride loops), advanced with carries instead of a division per element.
struct IndexWalker3 {
  int i, j, k, si, sj, sk, n1, n2;
  __device__ __forceinline__ IndexWalker3(int64_t start, int64_t stride, int n1_, int n2_)
      : n1(n1_), n2(n2_) {
    k = (int)(start % n2_);
    const int64_t r = start / n2_;
    j = (int)(r % n1_);
    i = (int)(r / n1_);
    sk = (int)(stride % n2_);
    const int64_t sr = stride / n2_;
    sj = (int)(sr % n1_);
    si = (int)(sr / n1_);
  }
  __device__ __forceinline__ void next() {
    k += sk;
    j += sj;
    i += si;
    if (k >= n2) {
      k -= n2;
      ++j;
    }
    if (j >= n1) {
      j -= n1;
      ++i;
    }
  }
};

}  // namespace pk
