// Small BF16 MLP for the learned aliasing correction of low-resolution spectra:
// 4 dense layers (16 -> 128 -> 128 -> 128 -> 1), SiLU activations, BF16 weights and
// activations as tensor-core operands with FP32 accumulation (mma.sync m16n8k16 bf16),
// FP32 master weights, biases and Adam state.
//   - mlp_forward_kernel: one warp per 16 samples, layer by layer through shared memory;
//     optionally keeps pre-activations Z and activations H for the backward pass;
//   - mlp_mse_kernel: weighted mean-squared-error loss and its gradient dL/dy (one CTA,
//     fixed-order reduction);
//   - mlp_forward_tc_kernel: the forward pass on the tcgen05 tensor cores;
//   - mlp_backward_kernel: per CTA (64 samples) the weight and bias gradients of its
//     samples, written as one partial row; mlp_reduce_kernel adds the rows in CTA order,
//     so the gradient is deterministic;
//   - mlp_backward_tc_kernel: the backward pass on the tcgen05 tensor cores (weight gradients
//     accumulated in tensor memory over a persistent CTA's tiles, one partial row per CTA);
//   - mlp_adam_kernel: AdamW update of the FP32 master weights and their BF16 copies.
// Samples can be gathered through an index array (minibatches of a resident training set).
// There is no counterpart in the reference: the learned correction is a new method.
#include <cuda_bf16.h>
#include <math.h>

#include "common.cuh"

namespace pk {

constexpr int MLP_IN = 16;      // padded input features
constexpr int MLP_H = 128;      // hidden width
constexpr int MLP_OUT = 8;      // padded output rows of the last layer (row 0 used)
constexpr int MLP_WARPS = 4;    // warps per CTA
constexpr int MLP_ROWS = 16;    // samples per warp
constexpr int MLP_CTA_ROWS = MLP_WARPS * MLP_ROWS;
constexpr int MLP_LD = MLP_H + 8;  // padded shared-memory row (bank-conflict-free fragments)

// Parameter layout (float32 master weights and their bf16 copies share it):
//   W0 [H][IN], b0 [H], W1 [H][H], b1 [H], W2 [H][H], b2 [H], W3 [OUT][H], b3 [OUT]
constexpr int OFF_W0 = 0;
constexpr int OFF_B0 = OFF_W0 + MLP_H * MLP_IN;
constexpr int OFF_W1 = OFF_B0 + MLP_H;
constexpr int OFF_B1 = OFF_W1 + MLP_H * MLP_H;
constexpr int OFF_W2 = OFF_B1 + MLP_H;
constexpr int OFF_B2 = OFF_W2 + MLP_H * MLP_H;
constexpr int OFF_W3 = OFF_B2 + MLP_H;
constexpr int OFF_B3 = OFF_W3 + MLP_OUT * MLP_H;
constexpr int MLP_NPARAMS = OFF_B3 + MLP_OUT;

__device__ __forceinline__ float sigmoid(float z) { return 1.f / (1.f + expf(-z)); }

__device__ __forceinline__ unsigned pack_raw(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
}

// D(16x8) += A(16x16, row-major) * B(16x8, column-major); bf16 operands, f32 accumulators.
__device__ __forceinline__ void mma16816(float d[4], const unsigned a[4], const unsigned b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Operand fragments through accessors: A(r, k), r < 16, k < 16; B(k, n), k < 16, n < 8.
// Lane (g = lane / 4, t = lane % 4) holds A rows g, g + 8, columns 2t, 2t + 1, 2t + 8, 2t + 9
// and B rows 2t, 2t + 1, 2t + 8, 2t + 9 of column g (the PTX m16n8k16 fragment layout).
template <class FA>
__device__ __forceinline__ void load_a(unsigned a[4], FA A) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  a[0] = pack_raw(A(g, 2 * t), A(g, 2 * t + 1));
  a[1] = pack_raw(A(g + 8, 2 * t), A(g + 8, 2 * t + 1));
  a[2] = pack_raw(A(g, 2 * t + 8), A(g, 2 * t + 9));
  a[3] = pack_raw(A(g + 8, 2 * t + 8), A(g + 8, 2 * t + 9));
}

template <class FB>
__device__ __forceinline__ void load_b(unsigned b[2], FB B) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  b[0] = pack_raw(B(2 * t, g), B(2 * t + 1, g));
  b[1] = pack_raw(B(2 * t + 8, g), B(2 * t + 9, g));
}

// Accumulator q of this lane sits at row acc_row(q), column acc_col(q) of the 16x8 tile.
__device__ __forceinline__ int acc_row(int q) { return ((threadIdx.x & 31) >> 2) + (q >= 2 ? 8 : 0); }
__device__ __forceinline__ int acc_col(int q) { return 2 * (threadIdx.x & 3) + (q & 1); }

// One warp: acc (16 x NT*8) = act (16 x K) W^T, W [NT*8][K] bf16 row-major (out x in).
template <int K, int NT>
__device__ __forceinline__ void dense_warp(const __nv_bfloat16 (*act)[MLP_LD],
                                           const __nv_bfloat16 *__restrict__ W, float acc[NT][4]) {
#pragma unroll
  for (int nt = 0; nt < NT; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
#pragma unroll 2
  for (int kk = 0; kk < K; kk += 16) {
    unsigned a[4];
    load_a(a, [&](int r, int k) { return act[r][kk + k]; });
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      unsigned b[2];
      load_b(b, [&](int k, int n) { return W[(nt * 8 + n) * K + kk + k]; });
      mma16816(acc[nt], a, b);
    }
  }
}

__device__ __forceinline__ int sample_of(const int *__restrict__ idx, int row) {
  return idx ? idx[row] : row;
}

// Forward pass.  X [*][MLP_IN] float32 (zero-padded features), rows gathered through idx
// (or the first `batch` rows); y [batch].  With Z and H, stores the pre-activations
// Z[l][batch][H] and activations H[l][batch][H] of the hidden layers l < 3.
__global__ void __launch_bounds__(MLP_WARPS * 32) mlp_forward_kernel(
    const float *__restrict__ X, const int *__restrict__ idx, int batch,
    const __nv_bfloat16 *__restrict__ Wb, const float *__restrict__ Wf, float *__restrict__ y,
    float *__restrict__ Z, float *__restrict__ H) {
  __shared__ __nv_bfloat16 act_all[MLP_WARPS][MLP_ROWS][MLP_LD];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = (blockIdx.x * MLP_WARPS + warp) * MLP_ROWS;
  __nv_bfloat16(*act)[MLP_LD] = act_all[warp];
  for (int i = lane; i < MLP_ROWS * MLP_IN; i += 32) {
    const int r = i / MLP_IN, c = i % MLP_IN;
    const float v = (row0 + r < batch) ? X[(int64_t)sample_of(idx, row0 + r) * MLP_IN + c] : 0.f;
    act[r][c] = __float2bfloat16_rn(v);
  }
  __syncwarp();
  for (int l = 0; l < 3; ++l) {
    float acc[MLP_H / 8][4];
    if (l == 0) dense_warp<MLP_IN, MLP_H / 8>(act, Wb + OFF_W0, acc);
    else dense_warp<MLP_H, MLP_H / 8>(act, Wb + (l == 1 ? OFF_W1 : OFF_W2), acc);
    const float *bias = Wf + (l == 0 ? OFF_B0 : (l == 1 ? OFF_B1 : OFF_B2));
    __syncwarp();
#pragma unroll
    for (int nt = 0; nt < MLP_H / 8; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = acc_row(q), c = nt * 8 + acc_col(q);
        const float z = acc[nt][q] + bias[c];
        const float h = z * sigmoid(z);
        act[r][c] = __float2bfloat16_rn(h);
        if (Z && row0 + r < batch) {
          Z[((int64_t)l * batch + row0 + r) * MLP_H + c] = z;
          H[((int64_t)l * batch + row0 + r) * MLP_H + c] = h;
        }
      }
    __syncwarp();
  }
  float acc[1][4];
  dense_warp<MLP_H, 1>(act, Wb + OFF_W3, acc);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int r = acc_row(q);
    if (acc_col(q) == 0 && row0 + r < batch) y[row0 + r] = acc[0][q] + Wf[OFF_B3];
  }
}

// ------------------------------------------------------------- tcgen05 forward pass
// The same network on the 5th-generation tensor cores.  One CTA (TC_GROUPS warpgroups)
// takes 128 samples; each layer is D[128 x N] = A[128 x K] B[N x K]^T with A (bf16
// activations) and B (bf16 weights, out x in) in shared memory in the no-swizzle K-major
// canonical layout and D (float32) in tensor memory: one elected thread issues the K / 16
// tcgen05.mma.kind::f16 instructions and commits them to an mbarrier; after the (bounded)
// wait, warp w reads rows 32 (w % 4) .. +31 of D (its warpgroup's lane quarter) and its
// warpgroup's share of the columns with tcgen05.ld, adds the bias (shared memory), applies
// SiLU and writes the next layer's bf16 operand back to shared memory.  The epilogue is the
// longest part of a layer, so the warpgroups split its columns (measured on 1M rows: 68
// TFLOP/s with one warpgroup, 124 with two, 156 with four).  CTAs are persistent (two per
// SM): the weights and biases are loaded into shared memory once per CTA.
#ifndef PK_TC_GROUPS
#define PK_TC_GROUPS 4
#endif
constexpr int TC_ROWS = 128;
constexpr int TC_GROUPS = PK_TC_GROUPS;         // warpgroups per CTA, each a share of the columns
constexpr int TC_THREADS = 128 * TC_GROUPS;
constexpr int TC_COLS = 128 / TC_GROUPS;         // accumulator columns per warpgroup
constexpr int TC_FEAT = MLP_IN / TC_GROUPS;      // input features per thread
constexpr int TC_N3 = 16;  // last layer's N (rows 8..15 of its weight tile are zero)
constexpr int TC_TMEM_COLS = 128;
constexpr unsigned TC_WAIT_LIMIT = 1u << 22;  // mbarrier polls before giving up
constexpr size_t TC_SMEM = 4096 + 32768 + 32768 + 4096 + 4096 + 32768 + 3 * 128 * 4 + 64;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of element (r, k) of an R x K bf16 matrix in the canonical no-swizzle
// K-major layout: 8 x 8 core matrices of 128 contiguous bytes (row r & 7 at 16 (r & 7),
// column k & 7 at 2 (k & 7)), laid out by row group, then by group of 8 columns.
__device__ __forceinline__ uint32_t canon_off(int r, int k, int K) {
  return (uint32_t)((((r >> 3) * (K >> 3)) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (sm_100): start address, leading byte offset (between the
// two 8-column groups of one K = 16 step), stride byte offset (between row groups), all >> 4;
// descriptor version 1 at bit 46; no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: f32 accumulator (bits 4-5 = 1), bf16 A and B (bits 7-9,
// 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24 (M = 128).
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_ROWS >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (unsigned it = 0; it < TC_WAIT_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive float32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t v[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// rows [0, rows) of a row-major bf16 matrix (rows x K) into the canonical layout of a
// (rows_total x K) tile; rows [rows, rows_total) are zero.  16-byte chunks.
__device__ __forceinline__ void load_canon(unsigned char *dst, const __nv_bfloat16 *__restrict__ src, int rows,
                                           int rows_total, int K) {
  const int chunks = rows_total * (K >> 3);
  for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
    const int r = c / (K >> 3), kc = c % (K >> 3);
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (r < rows) v = *reinterpret_cast<const uint4 *>(src + (size_t)r * K + kc * 8);
    *reinterpret_cast<uint4 *>(dst + canon_off(r, kc * 8, K)) = v;
  }
}

__global__ void __launch_bounds__(TC_THREADS, TC_GROUPS >= 4 ? 2 : 1) mlp_forward_tc_kernel(
    const float *__restrict__ X, const int *__restrict__ idx, int batch, const __nv_bfloat16 *__restrict__ Wb,
    const float *__restrict__ Wf, float *__restrict__ y, float *__restrict__ Z, float *__restrict__ H,
    int *__restrict__ status) {
  extern __shared__ __align__(1024) unsigned char tcsm[];
  unsigned char *sW0 = tcsm, *sW1 = sW0 + 4096, *sW2 = sW1 + 32768, *sW3 = sW2 + 32768, *sA0 = sW3 + 4096,
                *sA = sA0 + 4096;
  float *sBias = reinterpret_cast<float *>(sA + 32768);  // b0, b1, b2
  uint64_t *bar = reinterpret_cast<uint64_t *>(sBias + 3 * MLP_H);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int r = tid & (TC_ROWS - 1);  // this thread's row of the tile (and D lane)
  const int half = tid >> 7;          // warpgroup: its share of the columns
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");  // visible to the commit
  }
  load_canon(sW0, Wb + OFF_W0, MLP_H, MLP_H, MLP_IN);
  load_canon(sW1, Wb + OFF_W1, MLP_H, MLP_H, MLP_H);
  load_canon(sW2, Wb + OFF_W2, MLP_H, MLP_H, MLP_H);
  load_canon(sW3, Wb + OFF_W3, MLP_OUT, TC_N3, MLP_H);
  for (int q = tid; q < 3 * MLP_H; q += TC_THREADS)
    sBias[q] = Wf[(q < MLP_H ? OFF_B0 : (q < 2 * MLP_H ? OFF_B1 : OFF_B2)) + q % MLP_H];
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const int ntiles = (batch + TC_ROWS - 1) / TC_ROWS;
  bool ok = true;
  uint32_t phase = 0;
  // persistent: the weights stay in shared memory while the CTA walks its 128-row tiles
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int row = tile * TC_ROWS + r;  // this thread's sample
    {  // input features of this thread's sample, its warpgroup's share (bf16, zero past the batch)
      const bool in = row < batch;
      const float *xr = X + (int64_t)(in ? sample_of(idx, row) : 0) * MLP_IN;
      const int kc = TC_FEAT * half;
      unsigned pk[TC_FEAT / 2];
#pragma unroll
      for (int q = 0; q < TC_FEAT / 2; ++q) {
        const float a = in ? xr[kc + 2 * q] : 0.f, b = in ? xr[kc + 2 * q + 1] : 0.f;
        pk[q] = pack_raw(__float2bfloat16_rn(a), __float2bfloat16_rn(b));
      }
      if constexpr (TC_FEAT == 8)
        *reinterpret_cast<uint4 *>(sA0 + canon_off(r, kc, MLP_IN)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
      else
        *reinterpret_cast<uint2 *>(sA0 + canon_off(r, kc, MLP_IN)) = make_uint2(pk[0], pk[1]);
    }
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    for (int l = 0; l < 4 && ok; ++l) {
      const int K = l == 0 ? MLP_IN : MLP_H;
      const int N = l == 3 ? TC_N3 : MLP_H;
      const unsigned char *A = l == 0 ? sA0 : sA;
      const unsigned char *B = l == 0 ? sW0 : (l == 1 ? sW1 : (l == 2 ? sW2 : sW3));
      if (tid == 0) {
        const uint32_t idesc = umma_idesc_bf16(N);
        const uint32_t sbo = (uint32_t)(K >> 3) * 128u;
        for (int j = 0; j < K / 16; ++j)
          tc_mma(tmem, umma_desc(smem_u32(A) + 256u * j, 128u, sbo), umma_desc(smem_u32(B) + 256u * j, 128u, sbo),
                 idesc, j > 0 ? 1u : 0u);
        tc_commit(smem_u32(bar));
      }
      ok = __syncthreads_and(mbar_wait(smem_u32(bar), phase & 1u) ? 1 : 0) != 0;
      ++phase;
      tc_fence_after();
      if (!ok) break;
      if (l < 3) {
        const float *bias = sBias + l * MLP_H;
        for (int c0 = TC_COLS * half; c0 < TC_COLS * half + TC_COLS; c0 += 32) {
          uint32_t v[32];
          tmem_ld32(lane_addr + (uint32_t)c0, v);
#pragma unroll
          for (int c = 0; c < 32; c += 8) {
            unsigned pk[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const float z0 = __uint_as_float(v[c + 2 * q]) + bias[c0 + c + 2 * q];
              const float z1 = __uint_as_float(v[c + 2 * q + 1]) + bias[c0 + c + 2 * q + 1];
              const float h0 = z0 * sigmoid(z0), h1 = z1 * sigmoid(z1);
              pk[q] = pack_raw(__float2bfloat16_rn(h0), __float2bfloat16_rn(h1));
              if (Z && row < batch) {
                const int64_t o = ((int64_t)l * batch + row) * MLP_H + c0 + c + 2 * q;
                Z[o] = z0;
                Z[o + 1] = z1;
                H[o] = h0;
                H[o + 1] = h1;
              }
            }
            *reinterpret_cast<uint4 *>(sA + canon_off(r, c0 + c, MLP_H)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          }
        }
      } else if (half == 0) {
        uint32_t v[32];
        tmem_ld32(lane_addr, v);
        if (row < batch) y[row] = __uint_as_float(v[0]) + Wf[OFF_B3];
      }
      // the next MMA (this tile's next layer or the next tile's first) reads shared memory
      // written above and overwrites the accumulators read above
      async_proxy_fence();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
    }
  }
  if (!ok && tid == 0 && status) atomicExch(status, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                 : "memory");
}

// loss = sum_i w_i (y_i - t_i)^2 / batch, dy_i = 2 w_i (y_i - t_i) / batch; one CTA,
// fixed-order reduction.  Targets and sample weights are gathered through idx.
constexpr int MSE_THREADS = 1024;
__global__ void __launch_bounds__(MSE_THREADS) mlp_mse_kernel(
    const float *__restrict__ y, const float *__restrict__ target, const float *__restrict__ weight,
    const int *__restrict__ idx, int batch, float *__restrict__ dy, float *__restrict__ loss) {
  __shared__ double part[MSE_THREADS / 32];
  double s = 0.;
  const float inv = 1.f / (float)batch;
  for (int i = threadIdx.x; i < batch; i += MSE_THREADS) {
    const int j = sample_of(idx, i);
    const float w = weight ? weight[j] : 1.f;
    const float d = y[i] - target[j];
    dy[i] = 2.f * w * d * inv;
    s += (double)(w * d * d);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int w = 0; w < MSE_THREADS / 32; ++w) t += part[w];
    if (loss) *loss = (float)(t / batch);
  }
}

struct BackwardShared {
  __nv_bfloat16 dz[MLP_CTA_ROWS][MLP_LD];   // dL/dZ of the current layer (bf16 operand)
  __nv_bfloat16 hin[MLP_CTA_ROWS][MLP_LD];  // the layer's input activations (bf16)
  float dzf[MLP_CTA_ROWS][MLP_H];           // dL/dZ in float (bias gradients)
  float dh[MLP_CTA_ROWS][MLP_H];            // dL/dH of the current layer
};

// Backward pass of the loss gradient dy [batch].  Each CTA writes the gradients of its
// 64 samples into partial[blockIdx.x][MLP_NPARAMS].  The operands are rounded as in the
// forward pass: dW = bf16(dZ)^T bf16(A), dH_prev = bf16(dZ) bf16(W), both in f32.
__global__ void __launch_bounds__(MLP_WARPS * 32) mlp_backward_kernel(
    const float *__restrict__ X, const int *__restrict__ idx, int batch,
    const __nv_bfloat16 *__restrict__ Wb, const float *__restrict__ Z, const float *__restrict__ H,
    const float *__restrict__ dy, float *__restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BackwardShared &sh = *reinterpret_cast<BackwardShared *>(smem_raw);
  const int warp = threadIdx.x >> 5;
  const int cta_row0 = blockIdx.x * MLP_CTA_ROWS;
  float *out = partial + (size_t)blockIdx.x * MLP_NPARAMS;
  // output layer y = bf16(H2) . W3[0] + b3:  dH2 = dy W3[0], dW3[0] = sum dy bf16(H2), db3 = sum dy
  for (int i = threadIdx.x; i < MLP_CTA_ROWS * MLP_H; i += blockDim.x) {
    const int r = i / MLP_H, c = i % MLP_H, row = cta_row0 + r;
    const float g = row < batch ? dy[row] : 0.f;
    sh.dh[r][c] = g * __bfloat162float(Wb[OFF_W3 + c]);
  }
  for (int c = threadIdx.x; c < MLP_H; c += blockDim.x) {
    float s = 0.f;
    for (int r = 0; r < MLP_CTA_ROWS; ++r) {
      const int row = cta_row0 + r;
      if (row < batch)
        s += dy[row] * __bfloat162float(__float2bfloat16_rn(H[((int64_t)2 * batch + row) * MLP_H + c]));
    }
    out[OFF_W3 + c] = s;
  }
  for (int c = MLP_H + threadIdx.x; c < MLP_OUT * MLP_H + MLP_OUT; c += blockDim.x) {
    float s = 0.f;
    if (c == MLP_OUT * MLP_H)
      for (int r = 0; r < MLP_CTA_ROWS; ++r)
        if (cta_row0 + r < batch) s += dy[cta_row0 + r];
    out[OFF_W3 + c] = s;  // unused output rows and bias entries get zero gradient
  }
  __syncthreads();
  for (int l = 2; l >= 0; --l) {
    for (int i = threadIdx.x; i < MLP_CTA_ROWS * MLP_H; i += blockDim.x) {
      const int r = i / MLP_H, c = i % MLP_H, row = cta_row0 + r;
      float g = 0.f, hv = 0.f;
      if (row < batch) {
        const float z = Z[((int64_t)l * batch + row) * MLP_H + c];
        const float s = sigmoid(z);
        g = sh.dh[r][c] * (s * (1.f + z * (1.f - s)));
        if (l > 0) hv = H[((int64_t)(l - 1) * batch + row) * MLP_H + c];
        else if (c < MLP_IN) hv = X[(int64_t)sample_of(idx, row) * MLP_IN + c];
      }
      sh.dzf[r][c] = g;
      sh.dz[r][c] = __float2bfloat16_rn(g);
      sh.hin[r][c] = __float2bfloat16_rn(hv);
    }
    __syncthreads();
    const int boff = l == 0 ? OFF_B0 : (l == 1 ? OFF_B1 : OFF_B2);
    for (int c = threadIdx.x; c < MLP_H; c += blockDim.x) {
      float s = 0.f;
      for (int r = 0; r < MLP_CTA_ROWS; ++r) s += sh.dzf[r][c];
      out[boff + c] = s;
    }
    // dW[n][k] = sum_r dZ[r][n] A[r][k]: M = 128 outputs (2 m-tiles per warp), N = inputs,
    // reduction over the CTA's 64 samples
    const int K = l == 0 ? MLP_IN : MLP_H;
    const int woff = l == 0 ? OFF_W0 : (l == 1 ? OFF_W1 : OFF_W2);
    for (int mt = warp * 2; mt < warp * 2 + 2; ++mt) {
      unsigned a[MLP_CTA_ROWS / 16][4];
#pragma unroll
      for (int ks = 0; ks < MLP_CTA_ROWS / 16; ++ks)
        load_a(a[ks], [&](int m, int k) { return sh.dz[ks * 16 + k][mt * 16 + m]; });
      for (int nt = 0; nt < K / 8; ++nt) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ks = 0; ks < MLP_CTA_ROWS / 16; ++ks) {
          unsigned b[2];
          load_b(b, [&](int k, int n) { return sh.hin[ks * 16 + k][nt * 8 + n]; });
          mma16816(acc, a[ks], b);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
          out[woff + (mt * 16 + acc_row(q)) * K + nt * 8 + acc_col(q)] = acc[q];
      }
    }
    if (l > 0) {
      // dH_prev = dZ W: rows = the warp's 16 samples, N = 128 inputs, reduction over outputs
      __syncthreads();
      const __nv_bfloat16 *W = Wb + (l == 1 ? OFF_W1 : OFF_W2);
      for (int nt = 0; nt < MLP_H / 8; ++nt) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
        for (int kk = 0; kk < MLP_H; kk += 16) {
          unsigned a[4], b[2];
          load_a(a, [&](int r, int k) { return sh.dz[warp * 16 + r][kk + k]; });
          load_b(b, [&](int k, int n) { return W[(kk + k) * MLP_H + nt * 8 + n]; });
          mma16816(acc, a, b);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) sh.dh[warp * 16 + acc_row(q)][nt * 8 + acc_col(q)] = acc[q];
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------- tcgen05 backward pass
// The gradient on the 5th-generation tensor cores.  Per 128-sample tile, for l = 2, 1, 0:
//   dZ_l = dH_l silu'(Z_l)            float, per thread: its sample and 32 columns
//   dW_l += bf16(dZ_l)^T bf16(A_l)    M = 128 outputs, N = K_l inputs, reduction over samples
//   dH_{l-1} = bf16(dZ_l) bf16(W_l)   M = 128 samples, N = 128 inputs, reduction over outputs
// with dH_2 = dy W3[0].  The operands stay in the layouts of the forward pass: the sample-major
// tiles (dZ, A_l: element (r, c) at canon_off(r, c, K)) and the weights (W_l[n][k] at
// canon_off(n, k, 128)).  Where the contiguous index is the reduction index they are K-major
// operands; where it is the output index they are MN-major operands (instruction descriptor
// bits 15 / 16).  A no-swizzle MN-major core matrix is 8 contiguous MN elements x 8 K rows of
// 16 bytes, with SBO the byte step between MN groups and LBO the step between K groups, so
// the same bytes serve both ways and no transposed copy is made.  The dW_l accumulate in
// tensor memory over all of the CTA's tiles (columns 128, 256, 384); dH_{l-1} goes to
// columns 0-127.  The bias and W3 gradients are float column sums over the samples (the
// oracle's float dZ), read from a float copy in shared memory in a fixed order while the MMAs
// run.  One CTA per SM (all 512 tensor-memory columns, ~200 KB of shared memory), persistent;
// each CTA writes one partial row, added in CTA order by mlp_reduce_kernel.  With every index
// bound, a descriptor read with LBO and SBO exchanged would still stay inside the CTA's shared
// memory (largest reach: 59.6 KB past the start of a 32 KB operand tile).
constexpr int BT_THREADS = 512;  // 4 warpgroups; warpgroup q takes columns [32 q, 32 q + 32)
constexpr int BT_TMEM_COLS = 512;
constexpr uint32_t BT_DH = 0, BT_DW2 = 128, BT_DW1 = 256, BT_DW0 = 384;  // tensor-memory columns
constexpr int BT_LDF = MLP_H + 1;  // float staging row: conflict-free column writes and reads
constexpr int BT_DZ = 0;                              // bf16 dZ tile (128 x 128)
constexpr int BT_A = BT_DZ + 32768;                   // bf16 A_l tile, l = 1, 2 (128 x 128)
constexpr int BT_A0 = BT_A + 32768;                   // bf16 input features (128 x 16)
constexpr int BT_W1 = BT_A0 + 4096;                   // bf16 W1 (128 x 128)
constexpr int BT_W2 = BT_W1 + 32768;                  // bf16 W2
constexpr int BT_F = BT_W2 + 32768;                   // float [128][129] staging
constexpr int BT_PART = BT_F + TC_ROWS * BT_LDF * 4;  // float [4][128] partial column sums
constexpr int BT_ACC = BT_PART + 4 * MLP_H * 4;       // float [4][128]: db0, db1, db2, dW3 row 0
constexpr int BT_W3 = BT_ACC + 4 * MLP_H * 4;         // float [128]: bf16 W3 row 0
constexpr int BT_DY = BT_W3 + MLP_H * 4;              // float [128]: the tile's dy
constexpr int BT_BAR = BT_DY + TC_ROWS * 4;           // mbarrier, tensor-memory slot
constexpr size_t BT_SMEM = BT_BAR + 16;
static_assert(BT_SMEM <= 227 * 1024, "backward tile exceeds the shared memory of one CTA");
static_assert(BT_BAR % 8 == 0, "mbarrier alignment");

// sums[c] += the column sum of sF over the tile's 128 rows, in a fixed order (four sums of 32
// rows, then theirs).  Every thread calls it; threads < 128 write sums after a barrier.
__device__ __forceinline__ void bt_column_sums(const float (*sF)[BT_LDF], float (*sPart)[MLP_H], float *sums) {
  const int c = threadIdx.x & (MLP_H - 1), rq = threadIdx.x >> 7;
  float s = 0.f;
#pragma unroll 8
  for (int i = 0; i < 32; ++i) s += sF[rq * 32 + i][c];
  sPart[rq][c] = s;
  __syncthreads();
  if (threadIdx.x < MLP_H) sums[c] += (sPart[0][c] + sPart[1][c]) + (sPart[2][c] + sPart[3][c]);
}

__global__ void __launch_bounds__(BT_THREADS, 1) mlp_backward_tc_kernel(
    const float *__restrict__ X, const int *__restrict__ idx, int batch, const __nv_bfloat16 *__restrict__ Wb,
    const float *__restrict__ Z, const float *__restrict__ H, const float *__restrict__ dy,
    float *__restrict__ partial, int *__restrict__ status) {
  extern __shared__ __align__(1024) unsigned char btsm[];
  unsigned char *sDZ = btsm + BT_DZ, *sA = btsm + BT_A, *sA0 = btsm + BT_A0, *sW1 = btsm + BT_W1,
                *sW2 = btsm + BT_W2;
  float(*sF)[BT_LDF] = reinterpret_cast<float(*)[BT_LDF]>(btsm + BT_F);
  float(*sPart)[MLP_H] = reinterpret_cast<float(*)[MLP_H]>(btsm + BT_PART);
  float(*sAcc)[MLP_H] = reinterpret_cast<float(*)[MLP_H]>(btsm + BT_ACC);
  float *sW3 = reinterpret_cast<float *>(btsm + BT_W3);
  float *sDY = reinterpret_cast<float *>(btsm + BT_DY);
  uint64_t *bar = reinterpret_cast<uint64_t *>(btsm + BT_BAR);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(btsm + BT_BAR + 8);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int r = tid & (TC_ROWS - 1), q = tid >> 7, c0 = 32 * q;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(BT_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  load_canon(sW1, Wb + OFF_W1, MLP_H, MLP_H, MLP_H);
  load_canon(sW2, Wb + OFF_W2, MLP_H, MLP_H, MLP_H);
  for (int i = tid; i < MLP_H; i += BT_THREADS) sW3[i] = __bfloat162float(Wb[OFF_W3 + i]);
  for (int i = tid; i < 4 * MLP_H; i += BT_THREADS) (&sAcc[0][0])[i] = 0.f;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const int ntiles = (batch + TC_ROWS - 1) / TC_ROWS;
  float db3 = 0.f;  // thread 0
  bool ok = true, first = true;
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int row = tile * TC_ROWS + r;
    const bool in = row < batch;
    const int64_t rowc = in ? row : 0;
    const float g = in ? dy[row] : 0.f;
    if (q == 0) sDY[r] = g;
    float dh[32];
    {  // output layer: dH_2 = dy W3[0]; dW3[0] from the column sums of dy bf16(H_2)
      const float *hr = H + ((int64_t)2 * batch + rowc) * MLP_H + c0;
#pragma unroll
      for (int c = 0; c < 32; c += 4) {
        const float4 hv = in ? *reinterpret_cast<const float4 *>(hr + c) : make_float4(0.f, 0.f, 0.f, 0.f);
        sF[r][c0 + c] = g * __bfloat162float(__float2bfloat16_rn(hv.x));
        sF[r][c0 + c + 1] = g * __bfloat162float(__float2bfloat16_rn(hv.y));
        sF[r][c0 + c + 2] = g * __bfloat162float(__float2bfloat16_rn(hv.z));
        sF[r][c0 + c + 3] = g * __bfloat162float(__float2bfloat16_rn(hv.w));
      }
#pragma unroll
      for (int c = 0; c < 32; ++c) dh[c] = g * sW3[c0 + c];
    }
    __syncthreads();
    bt_column_sums(sF, sPart, sAcc[3]);
    if (tid == 0)
      for (int i = 0; i < TC_ROWS; ++i) db3 += sDY[i];
    __syncthreads();
    for (int l = 2; l >= 0 && ok; --l) {
      if (l < 2) {
        uint32_t v[32];
        tmem_ld32(lane_addr + BT_DH + (uint32_t)c0, v);
#pragma unroll
        for (int c = 0; c < 32; ++c) dh[c] = __uint_as_float(v[c]);
      }
      {  // dZ_l: float copy for the bias sums, bf16 tile for the MMAs
        const float *zr = Z + ((int64_t)l * batch + rowc) * MLP_H + c0;
#pragma unroll
        for (int c = 0; c < 32; c += 8) {
          unsigned pk[4];
#pragma unroll
          for (int u = 0; u < 8; u += 4) {
            const float4 zv = in ? *reinterpret_cast<const float4 *>(zr + c + u) : make_float4(0.f, 0.f, 0.f, 0.f);
            const float zz[4] = {zv.x, zv.y, zv.z, zv.w};
            float d[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const float s = sigmoid(zz[e]);
              d[e] = in ? dh[c + u + e] * (s * (1.f + zz[e] * (1.f - s))) : 0.f;
              sF[r][c0 + c + u + e] = d[e];
            }
            pk[u / 2] = pack_raw(__float2bfloat16_rn(d[0]), __float2bfloat16_rn(d[1]));
            pk[u / 2 + 1] = pack_raw(__float2bfloat16_rn(d[2]), __float2bfloat16_rn(d[3]));
          }
          *reinterpret_cast<uint4 *>(sDZ + canon_off(r, c0 + c, MLP_H)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
      }
      if (l > 0) {  // A_l = bf16(H_{l-1})
        const float *ar = H + ((int64_t)(l - 1) * batch + rowc) * MLP_H + c0;
#pragma unroll
        for (int c = 0; c < 32; c += 8) {
          const float4 a = in ? *reinterpret_cast<const float4 *>(ar + c) : make_float4(0.f, 0.f, 0.f, 0.f);
          const float4 b = in ? *reinterpret_cast<const float4 *>(ar + c + 4) : make_float4(0.f, 0.f, 0.f, 0.f);
          *reinterpret_cast<uint4 *>(sA + canon_off(r, c0 + c, MLP_H)) =
              make_uint4(pack_raw(__float2bfloat16_rn(a.x), __float2bfloat16_rn(a.y)),
                         pack_raw(__float2bfloat16_rn(a.z), __float2bfloat16_rn(a.w)),
                         pack_raw(__float2bfloat16_rn(b.x), __float2bfloat16_rn(b.y)),
                         pack_raw(__float2bfloat16_rn(b.z), __float2bfloat16_rn(b.w)));
        }
      } else {  // A_0 = bf16(X): 4 of the 16 features per warpgroup
        const float *xr = X + (int64_t)(in ? sample_of(idx, row) : 0) * MLP_IN + 4 * q;
        const float x0 = in ? xr[0] : 0.f, x1 = in ? xr[1] : 0.f, x2 = in ? xr[2] : 0.f, x3 = in ? xr[3] : 0.f;
        *reinterpret_cast<uint2 *>(sA0 + canon_off(r, 4 * q, MLP_IN)) =
            make_uint2(pack_raw(__float2bfloat16_rn(x0), __float2bfloat16_rn(x1)),
                       pack_raw(__float2bfloat16_rn(x2), __float2bfloat16_rn(x3)));
      }
      async_proxy_fence();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      if (tid == 0) {
        const int K = l == 0 ? MLP_IN : MLP_H;
        const unsigned char *A = l == 0 ? sA0 : sA;
        const uint32_t dw = tmem + (l == 2 ? BT_DW2 : (l == 1 ? BT_DW1 : BT_DW0));
        // dW_l += dZ^T A_l: A = dZ tile MN-major (MN groups of 8 outputs 128 B apart, K groups
        // of 8 samples 2048 B apart), B = A_l tile MN-major (input groups 128 B apart, sample
        // groups 16 K B apart); 16 samples per instruction
        const uint32_t idw = umma_idesc_bf16(K) | (1u << 15) | (1u << 16);
        for (int j = 0; j < TC_ROWS / 16; ++j)
          tc_mma(dw, umma_desc(smem_u32(sDZ) + 4096u * j, 2048u, 128u),
                 umma_desc(smem_u32(A) + (uint32_t)(32 * K) * j, (uint32_t)(16 * K), 128u), idw,
                 (first && j == 0) ? 0u : 1u);
        if (l > 0) {
          // dH_{l-1} = dZ W_l: A = dZ tile K-major (as in the forward pass), B = W_l MN-major
          // (input groups 128 B apart, output groups 2048 B apart); 16 outputs per instruction
          const unsigned char *W = l == 2 ? sW2 : sW1;
          const uint32_t idh = umma_idesc_bf16(MLP_H) | (1u << 16);
          for (int j = 0; j < MLP_H / 16; ++j)
            tc_mma(tmem + BT_DH, umma_desc(smem_u32(sDZ) + 256u * j, 128u, 2048u),
                   umma_desc(smem_u32(W) + 4096u * j, 2048u, 128u), idh, j > 0 ? 1u : 0u);
        }
        tc_commit(smem_u32(bar));
      }
      bt_column_sums(sF, sPart, sAcc[l]);  // while the MMAs run
      ok = __syncthreads_and(mbar_wait(smem_u32(bar), phase & 1u) ? 1 : 0) != 0;
      ++phase;
      tc_fence_after();
    }
    first = false;
  }
  if (ok) {
    float *out = partial + (size_t)blockIdx.x * MLP_NPARAMS;
    uint32_t v[32];
    tmem_ld32(lane_addr + BT_DW2 + (uint32_t)c0, v);  // lane = output r, columns = inputs
#pragma unroll
    for (int c = 0; c < 32; ++c) out[OFF_W2 + r * MLP_H + c0 + c] = __uint_as_float(v[c]);
    tmem_ld32(lane_addr + BT_DW1 + (uint32_t)c0, v);
#pragma unroll
    for (int c = 0; c < 32; ++c) out[OFF_W1 + r * MLP_H + c0 + c] = __uint_as_float(v[c]);
    if (q == 0) {  // warp-uniform; columns 400-415 are read but not used
      tmem_ld32(lane_addr + BT_DW0, v);
#pragma unroll
      for (int c = 0; c < MLP_IN; ++c) out[OFF_W0 + r * MLP_IN + c] = __uint_as_float(v[c]);
    }
    for (int i = tid; i < MLP_H; i += BT_THREADS) {
      out[OFF_B0 + i] = sAcc[0][i];
      out[OFF_B1 + i] = sAcc[1][i];
      out[OFF_B2 + i] = sAcc[2][i];
      out[OFF_W3 + i] = sAcc[3][i];
    }
    for (int i = MLP_H + tid; i < MLP_OUT * MLP_H + MLP_OUT; i += BT_THREADS)
      if (i != MLP_OUT * MLP_H) out[OFF_W3 + i] = 0.f;  // unused output rows and biases
    if (tid == 0) out[OFF_B3] = db3;
  } else if (tid == 0 && status) {
    atomicExch(status, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BT_TMEM_COLS)
                 : "memory");
}

// grad[p] = sum over the CTA partial rows, in CTA order.
__global__ void mlp_reduce_kernel(const float *__restrict__ partial, int nblocks, float *__restrict__ grad) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < MLP_NPARAMS; p += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nblocks; ++b) s += partial[(size_t)b * MLP_NPARAMS + p];
    grad[p] = s;
  }
}

// AdamW step t + 1 with t = *step (then *step = t + 1): m, v moments, bias corrections
// 1 - beta^(t+1), decoupled weight decay, learning rate lr_table[min(t, ntable - 1)].  One
// CTA, so the step counter advances after every thread has read it; the whole training
// step can then be replayed from a CUDA graph.
constexpr int ADAM_THREADS = 1024;
__global__ void __launch_bounds__(ADAM_THREADS) mlp_adam_kernel(
    float *__restrict__ w, __nv_bfloat16 *__restrict__ wb, float *__restrict__ m, float *__restrict__ v,
    const float *__restrict__ g, const float *__restrict__ lr_table, int ntable, int *__restrict__ step,
    float beta1, float beta2, float eps, float wd) {
  const int t = *step;
  const float rate = lr_table[min(t, ntable - 1)];
  const float c1 = 1.f - powf(beta1, (float)(t + 1)), c2 = 1.f - powf(beta2, (float)(t + 1));
  for (int p = threadIdx.x; p < MLP_NPARAMS; p += ADAM_THREADS) {
    const float gp = g[p];
    const float mp = beta1 * m[p] + (1.f - beta1) * gp;
    const float vp = beta2 * v[p] + (1.f - beta2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    const float wp = w[p] - rate * ((mp / c1) / (sqrtf(vp / c2) + eps) + wd * w[p]);
    w[p] = wp;
    wb[p] = __float2bfloat16_rn(wp);
  }
  __syncthreads();
  if (threadIdx.x == 0) *step = t + 1;
}

__global__ void mlp_cast_kernel(const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < MLP_NPARAMS; p += gridDim.x * blockDim.x)
    wb[p] = __float2bfloat16_rn(w[p]);
}

}  // namespace pk

using namespace pk;

extern "C" int pk_mlp_num_params(void) { return MLP_NPARAMS; }

extern "C" pk_status pk_mlp_cast(void *stream, const float *w, void *wb) {
  PK_REQUIRE(w && wb, PK_ERR_INVALID, "mlp_cast: null pointer");
  mlp_cast_kernel<<<(MLP_NPARAMS + 255) / 256, 256, 0, (cudaStream_t)stream>>>(w, (__nv_bfloat16 *)wb);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_mlp_forward(void *stream, const float *x, const int *idx, int batch, const void *wb,
                                    const float *w, float *y, float *z, float *h) {
  PK_REQUIRE(x && wb && w && y && batch >= 0, PK_ERR_INVALID, "mlp_forward: invalid arguments");
  PK_REQUIRE((z == nullptr) == (h == nullptr), PK_ERR_INVALID, "mlp_forward: z and h go together");
  if (batch == 0) return PK_OK;
  const int blocks = (batch + MLP_CTA_ROWS - 1) / MLP_CTA_ROWS;
  mlp_forward_kernel<<<blocks, MLP_WARPS * 32, 0, (cudaStream_t)stream>>>(
      x, idx, batch, (const __nv_bfloat16 *)wb, w, y, z, h);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_mlp_forward_tc(void *stream, const float *x, const int *idx, int batch, const void *wb,
                                       const float *w, float *y, float *z, float *h, int *d_status) {
  PK_REQUIRE(x && wb && w && y && batch >= 0, PK_ERR_INVALID, "mlp_forward_tc: invalid arguments");
  PK_REQUIRE((z == nullptr) == (h == nullptr), PK_ERR_INVALID, "mlp_forward_tc: z and h go together");
  PK_REQUIRE(((uintptr_t)wb & 15u) == 0, PK_ERR_INVALID, "mlp_forward_tc: bf16 weights must be 16-byte aligned");
  if (batch == 0) return PK_OK;
  PK_CUDA(cudaFuncSetAttribute(mlp_forward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  const int ntiles = (batch + TC_ROWS - 1) / TC_ROWS;
  const int blocks = ntiles < 2 * sm_count() ? ntiles : 2 * sm_count();  // persistent, 2 CTAs per SM
  mlp_forward_tc_kernel<<<blocks, TC_THREADS, TC_SMEM, (cudaStream_t)stream>>>(
      x, idx, batch, (const __nv_bfloat16 *)wb, w, y, z, h, d_status);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_mlp_mse(void *stream, const float *y, const float *target, const float *weight,
                                const int *idx, int batch, float *dy, float *loss) {
  PK_REQUIRE(y && target && dy && batch > 0, PK_ERR_INVALID, "mlp_mse: invalid arguments");
  mlp_mse_kernel<<<1, MSE_THREADS, 0, (cudaStream_t)stream>>>(y, target, weight, idx, batch, dy, loss);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_mlp_backward_workspace_size(int batch, size_t *bytes) {
  PK_REQUIRE(bytes && batch >= 0, PK_ERR_INVALID, "mlp_backward_workspace_size: invalid arguments");
  const int blocks = (batch + MLP_CTA_ROWS - 1) / MLP_CTA_ROWS;
  *bytes = (size_t)(blocks > 0 ? blocks : 1) * MLP_NPARAMS * sizeof(float);
  return PK_OK;
}

extern "C" pk_status pk_mlp_backward(void *stream, const float *x, const int *idx, int batch, const void *wb,
                                     const float *z, const float *h, const float *dy, float *grad,
                                     void *workspace, size_t workspace_bytes) {
  PK_REQUIRE(x && wb && z && h && dy && grad && batch > 0, PK_ERR_INVALID, "mlp_backward: invalid arguments");
  const int blocks = (batch + MLP_CTA_ROWS - 1) / MLP_CTA_ROWS;
  PK_REQUIRE(workspace && workspace_bytes >= (size_t)blocks * MLP_NPARAMS * sizeof(float), PK_ERR_WORKSPACE,
             "mlp_backward: workspace too small");
  cudaStream_t s = (cudaStream_t)stream;
  const int smem = (int)sizeof(BackwardShared);
  PK_CUDA(cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  float *partial = static_cast<float *>(workspace);
  mlp_backward_kernel<<<blocks, MLP_WARPS * 32, smem, s>>>(x, idx, batch, (const __nv_bfloat16 *)wb, z, h, dy,
                                                           partial);
  PK_LAUNCH_CHECK();
  mlp_reduce_kernel<<<(MLP_NPARAMS + 255) / 256, 256, 0, s>>>(partial, blocks, grad);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_mlp_backward_tc(void *stream, const float *x, const int *idx, int batch, const void *wb,
                                        const float *z, const float *h, const float *dy, float *grad,
                                        void *workspace, size_t workspace_bytes, int *d_status) {
  PK_REQUIRE(x && wb && z && h && dy && grad && batch > 0, PK_ERR_INVALID, "mlp_backward_tc: invalid arguments");
  PK_REQUIRE((((uintptr_t)wb | (uintptr_t)z | (uintptr_t)h) & 15u) == 0, PK_ERR_INVALID,
             "mlp_backward_tc: wb, z and h must be 16-byte aligned");
  const int ntiles = (batch + TC_ROWS - 1) / TC_ROWS;
  const int blocks = ntiles < sm_count() ? ntiles : sm_count();  // persistent, one CTA per SM
  PK_REQUIRE(workspace && workspace_bytes >= (size_t)blocks * MLP_NPARAMS * sizeof(float), PK_ERR_WORKSPACE,
             "mlp_backward_tc: workspace too small");
  cudaStream_t s = (cudaStream_t)stream;
  PK_CUDA(cudaFuncSetAttribute(mlp_backward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BT_SMEM));
  float *partial = static_cast<float *>(workspace);
  mlp_backward_tc_kernel<<<blocks, BT_THREADS, BT_SMEM, s>>>(x, idx, batch, (const __nv_bfloat16 *)wb, z, h, dy,
                                                             partial, d_status);
  PK_LAUNCH_CHECK();
  mlp_reduce_kernel<<<(MLP_NPARAMS + 255) / 256, 256, 0, s>>>(partial, blocks, grad);
  PK_LAUNCH_CHECK();
  return PK_OK;
}

extern "C" pk_status pk_mlp_adam(void *stream, float *w, void *wb, float *m, float *v, const float *grad,
                                 const float *lr_table, int ntable, int *step, float beta1, float beta2,
                                 float eps, float weight_decay) {
  PK_REQUIRE(w && wb && m && v && grad && lr_table && step && ntable >= 1, PK_ERR_INVALID,
             "mlp_adam: invalid arguments");
  mlp_adam_kernel<<<1, ADAM_THREADS, 0, (cudaStream_t)stream>>>(w, (__nv_bfloat16 *)wb, m, v, grad, lr_table,
                                                                ntable, step, beta1, beta2, eps, weight_decay);
  PK_LAUNCH_CHECK();
  return PK_OK;
}
