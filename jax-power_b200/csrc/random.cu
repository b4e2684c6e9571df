// Per-particle random variates keyed by particle ids, for the split (disjoint random
// subsample) FKP normalisation.
//
// The reference draws them with create_sharded_random(jax.random.uniform, (seed, ids))
// (mesh.py:237-271, 284-329): one scalar uniform per id from the key
// fold_in(fold_in(key(seed), lo32(id)), hi32(id)) (_fold_in, mesh.py:215-233, int64 ids as
// with jax_enable_x64).  jax.random's generator is Threefry-2x32 with 20 rounds (Salmon,
// Moraes, Dror and Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011):
//   - key schedule k0, k1, k2 = k0 ^ k1 ^ 0x1BD11BDA, injected every 4 rounds with the
//     injection count added to the second word;
//   - rotations 13 15 26 6 17 29 16 24;
//   - fold_in(key, d) = threefry(key, (0, d));
//   - a float64 uniform from key k: bits = threefry(k, (0, 0)) as (word0 << 32 | word1),
//     then the 52 high mantissa bits over 1.0, minus 1.
// One thread per id; the variates are a pure function of (seed, id), so any sharding or
// ordering of the particles draws the same value for the same id.
#include "common.cuh"

namespace pk {

__device__ __forceinline__ unsigned rotl32(unsigned x, int r) { return (x << r) | (x >> (32 - r)); }

__device__ __forceinline__ void threefry2x32_20(unsigned k0, unsigned k1, unsigned c0, unsigned c1,
                                                unsigned *y0, unsigned *y1) {
  const unsigned ks[3] = {k0, k1, k0 ^ k1 ^ 0x1BD11BDAu};
  const int rot[8] = {13, 15, 26, 6, 17, 29, 16, 24};
  unsigned x0 = c0 + ks[0], x1 = c1 + ks[1];
#pragma unroll
  for (int block = 0; block < 5; ++block) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      x0 += x1;
      x1 = rotl32(x1, rot[(block & 1) * 4 + r]);
      x1 ^= x0;
    }
    x0 += ks[(block + 1) % 3];
    x1 += ks[(block + 2) % 3] + (unsigned)(block + 1);
  }
  *y0 = x0;
  *y1 = x1;
}

// ids NULL: jax.random.uniform(key, (n,)) of the whole array instead, element i drawn from
// counter (hi32(i), lo32(i)) (JAX's partitionable Threefry layout).
__global__ void uniform_ids_kernel(unsigned k0, unsigned k1, const int64_t *__restrict__ ids, int64_t n,
                                   double *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    unsigned y0, y1;
    if (ids) {
      const unsigned long long id = (unsigned long long)ids[i];
      unsigned a0, a1, b0, b1;
      threefry2x32_20(k0, k1, 0u, (unsigned)(id & 0xffffffffull), &a0, &a1);  // fold in the low word
      threefry2x32_20(a0, a1, 0u, (unsigned)(id >> 32), &b0, &b1);          // then the high word
      threefry2x32_20(b0, b1, 0u, 0u, &y0, &y1);                              // 64 random bits
    } else {
      threefry2x32_20(k0, k1, (unsigned)((unsigned long long)i >> 32), (unsigned)i, &y0, &y1);
    }
    const unsigned long long bits = ((unsigned long long)y0 << 32) | y1;
    out[i] = __longlong_as_double((long long)((bits >> 12) | 0x3FF0000000000000ull)) - 1.0;
  }
}

}  // namespace pk

using namespace pk;

extern "C" pk_status pk_uniform_ids(void *stream, uint64_t seed, const int64_t *d_ids, int64_t n, double *d_out) {
  PK_REQUIRE(n >= 0, PK_ERR_INVALID, "negative count");
  if (n == 0) return PK_OK;
  PK_REQUIRE(d_out, PK_ERR_INVALID, "out is NULL");
  const int threads = 256;
  const int64_t want = (n + threads - 1) / threads;
  const int blocks = (int)(want < 32LL * sm_count() ? want : 32LL * sm_count());
  // jax.random.key(seed): the two 32-bit halves of the 64-bit seed
  uniform_ids_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>((unsigned)(seed >> 32), (unsigned)seed, d_ids,
                                                                    n, d_out);
  PK_LAUNCH_CHECK();
  return PK_OK;
}
