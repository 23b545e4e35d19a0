// Mean-field surrogate: a small MLP (BF16 weights and activations, FP32
// accumulation) trained and evaluated with hand-written 5th-generation
// tensor-core kernels.  It has no counterpart in the reference; it maps sweep
// parameters (per-group drive, excitatory and inhibitory gains) to
// per-region firing rates and a hyperactivity logit, and screens parameter
// grids whose candidates the simulator then verifies.
//
// GEMM: C[M x N] = A[M x K] . B[N x K]^T, A and B BF16 row-major (K
// contiguous).  One CTA per 128-row tile holds the whole K (<= 256) and N
// (<= 256) in shared memory in the no-swizzle K-major core-matrix layout
// (8 rows x 16 bytes per core matrix); one thread issues K/16 tcgen05.mma
// (kind::f16, BF16 x BF16 -> FP32) into a TMEM accumulator; tcgen05.commit
// arrives on an mbarrier; the four warps read their 32 TMEM lanes back
// (tcgen05.ld 32x32b) for a fused epilogue: bias, ReLU, the ReLU mask of the
// backward pass, FP32 / BF16 / transposed-BF16 outputs.
//
// Training: one Adam step over a batch of 256 rows is 4 forward GEMMs, the
// loss kernel, 4 weight-gradient and 3 input-gradient GEMMs, bias sums and
// the Adam updates; the step is captured once into a CUDA graph (batch
// index and Adam step count live in device counters) and replayed.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include "flysim_b200.h"

namespace fsm {

typedef __nv_bfloat16 bf16;
constexpr int kThreads = 128;  // four warps: one quarter of the 128 TMEM lanes each
constexpr int kTileM = 128;
constexpr uint32_t kSpin = 1u << 26;  // bounded mbarrier wait

struct GemmArgs {
  const bf16 *A;
  int lda;
  const bf16 *B;
  int ldb;
  int M, N, K;
  const float *bias;  // [N] or null
  int relu;
  const bf16 *mask;   // [M x N]: output zeroed where mask <= 0 (ReLU backward), or null
  int ldm;
  float *Cf;          // FP32 [M x N] or null
  int ldcf;
  bf16 *Cb;           // BF16 [M x N] or null
  int ldcb;
  bf16 *Ct;           // BF16 [N x M] (transposed) or null
  int ldct;
  int *err;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (no swizzle, K-major): `lbo` = bytes
// between the two 8-element K halves of a 16-wide K step, `sbo` = bytes
// between consecutive 8-row groups; descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;
  return d;  // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

constexpr int kKC = 64;   // K columns per load chunk (4 MMAs, one mbarrier)
constexpr int kCW = 64;   // output columns per epilogue chunk
constexpr int kSP = kCW + 4;  // staging row pitch (floats)
constexpr int kMaxChunks = 256 / kKC;

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          dst),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t it = 0; it < kSpin; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Grid: x over 128-row tiles, y over column tiles of g.N / gridDim.y columns.
// Operands arrive by TMA (cp.async.bulk.tensor, no swizzle): each 8-wide K
// column of a tile is one box of rows x 16 bytes, which is exactly a stack
// of K-major core matrices (8 rows x 16 bytes, 128 bytes apart), so one
// thread issues every box of the tile up front, K chunk by K chunk on its
// own mbarrier, and starts each chunk's MMAs as soon as it lands.  Rows past
// M are the TMA's zero fill.  The epilogue goes through shared memory
// (reusing the operand space once the accumulator is complete) so that
// every global store is coalesced.
__global__ void __launch_bounds__(kThreads) k_gemm_tn(const __grid_constant__ GemmArgs g,
                                                      const __grid_constant__ CUtensorMap ta,
                                                      const __grid_constant__ CUtensorMap tb) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int K = g.K, N = g.N / (int)gridDim.y, nkb = K >> 3;  // 8-wide K columns
  const int n0 = blockIdx.y * N;  // first column of this CTA
  uint8_t *sA = smem;                              // nkb boxes of 128 rows x 16 B
  uint8_t *sB = smem + (size_t)nkb * kTileM * 16;  // nkb boxes of N rows x 16 B
  const size_t opnd = (size_t)nkb * (kTileM + N) * 16, stage = (size_t)kTileM * kSP * 4;
  uint64_t *mbar = (uint64_t *)(smem + (opnd > stage ? opnd : stage));  // [0] MMA, [1..] K chunks
  uint32_t *tslot = (uint32_t *)(mbar + 1 + kMaxChunks);
  float *stg = (float *)smem;                      // epilogue staging [128][kSP]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTileM;
  const int nch = (K + kKC - 1) / kKC;
  uint32_t ncols = 32;
  while (ncols < (uint32_t)N) ncols <<= 1;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int c = 0; c <= nch; c++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(mbar + c)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  bool loads_ok = true;
  if (tid == 0) {
    // every box of the tile, chunk by chunk
    for (int c = 0; c < nch; c++) {
      const int kb0 = c * (kKC / 8), kb1 = min(nkb, kb0 + kKC / 8);
      const uint32_t bytes = (uint32_t)(kb1 - kb0) * (uint32_t)(kTileM + N) * 16u;
      const uint32_t bar = smem_u32(mbar + 1 + c);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
      for (int kb = kb0; kb < kb1; kb++) {
        tma_load_2d(smem_u32(sA + (size_t)kb * kTileM * 16), &ta, kb * 8, m0, bar);
        tma_load_2d(smem_u32(sB + (size_t)kb * N * 16), &tb, kb * 8, n0, bar);
      }
    }
    // MMAs as the chunks land: slab s (16 wide) = boxes 2s (LBO away: 2s+1)
    const uint32_t id = idesc_bf16(kTileM, (uint32_t)N);
    for (int c = 0; c < nch && loads_ok; c++) {
      loads_ok = mbar_wait(smem_u32(mbar + 1 + c), 0);
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int s0 = c * (kKC / 16), s1 = min(K >> 4, s0 + kKC / 16);
      for (int sl = s0; sl < s1 && loads_ok; sl++) {
        const uint64_t ad = sdesc(smem_u32(sA + (size_t)(2 * sl) * kTileM * 16), kTileM * 16, 128);
        const uint64_t bd = sdesc(smem_u32(sB + (size_t)(2 * sl) * N * 16), (uint32_t)N * 16, 128);
        mma_bf16(tmem, ad, bd, id, sl > 0 ? 1u : 0u);
      }
    }
    if (!loads_ok && g.err) atomicExch(g.err, 4);
  }
  if (tid == 0)
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(mbar))
                 : "memory");
  // wait for the accumulator (bounded); the commit covers every MMA issued
  const bool ok = mbar_wait(smem_u32(mbar), 0);
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (!ok) {
    if (g.err && tid == 0) atomicExch(g.err, 3);
  } else {
    const int rl = warp * 32 + lane;  // this thread's accumulator row
    for (int cc = 0; cc < N; cc += kCW) {
      const int cw = min(kCW, N - cc);
      // TMEM -> registers -> (bias, ReLU) -> staging
      for (int c0 = 0; c0 < cw; c0 += 16) {
        uint32_t v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cc + c0), v);
#pragma unroll
        for (int j = 0; j < 16; j++) {
          float x = __uint_as_float(v[j]);
          if (g.bias) x += g.bias[n0 + cc + c0 + j];
          if (g.relu) x = fmaxf(x, 0.0f);
          stg[rl * kSP + c0 + j] = x;
        }
      }
      __syncthreads();
      const int rows = min(kTileM, g.M - m0);
      // row-major outputs: 8 consecutive columns per thread, coalesced
      const int c8 = cw >> 3;
      for (int i = tid; i < rows * c8; i += kThreads) {
        const int r = i / c8, c = (i - r * c8) * 8;
        float x[8];
#pragma unroll
        for (int j = 0; j < 8; j++) x[j] = stg[r * kSP + c + j];
        const size_t gc = (size_t)n0 + cc + c;
        if (g.mask) {
          const uint4 mv = *(const uint4 *)(g.mask + (size_t)(m0 + r) * g.ldm + gc);
          const bf16 *mb = (const bf16 *)&mv;
#pragma unroll
          for (int j = 0; j < 8; j++)
            if (!(__bfloat162float(mb[j]) > 0.0f)) x[j] = 0.0f;
#pragma unroll
          for (int j = 0; j < 8; j++) stg[r * kSP + c + j] = x[j];  // masked values for the transposed store
        }
        if (g.Cf) {
          float4 *dst = (float4 *)(g.Cf + (size_t)(m0 + r) * g.ldcf + gc);
          dst[0] = make_float4(x[0], x[1], x[2], x[3]);
          dst[1] = make_float4(x[4], x[5], x[6], x[7]);
        }
        if (g.Cb) {
          uint4 o;
          bf16 *ob = (bf16 *)&o;
#pragma unroll
          for (int j = 0; j < 8; j++) ob[j] = __float2bfloat16_rn(x[j]);
          *(uint4 *)(g.Cb + (size_t)(m0 + r) * g.ldcb + gc) = o;
        }
      }
      if (g.Ct) {
        __syncthreads();
        // transposed: consecutive threads take consecutive rows of one column
        for (int i = tid; i < rows * cw; i += kThreads) {
          const int c = i / rows, r = i - c * rows;
          g.Ct[((size_t)n0 + cc + c) * g.ldct + m0 + r] = __float2bfloat16_rn(stg[r * kSP + c]);
        }
      }
      __syncthreads();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols));
}

// ---- persistent GEMM for many row tiles --------------------------------------
// One CTA per SM walks row tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...
// W (the B operand) stays in shared memory; warp 4 (one lane) loads each
// tile's A by TMA into a single buffer and issues its MMAs into one of two
// TMEM accumulators, while warps 0-3 drain the other accumulator through the
// epilogue; so the next tile's loads and MMAs overlap the current epilogue.
constexpr int kPThreads = 160;

__device__ __forceinline__ bool epi_all(bool v) {  // uniform decision of the 128 epilogue threads
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, 1, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(out)
      : "r"((uint32_t)v)
      : "memory");
  return out != 0;
}

__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;\n" ::: "memory"); }

__global__ void __launch_bounds__(kPThreads) k_gemm_persist(const __grid_constant__ GemmArgs g,
                                                            const __grid_constant__ CUtensorMap ta,
                                                            const __grid_constant__ CUtensorMap tb) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int K = g.K, N = g.N, nkb = K >> 3;
  uint8_t *sB = smem;                                   // W: nkb boxes of N rows x 16 B
  uint8_t *sA = smem + (size_t)nkb * N * 16;            // A: nkb boxes of 128 rows x 16 B
  float *stg = (float *)(sA + (size_t)nkb * kTileM * 16);  // epilogue staging [128][kSP]
  uint64_t *bars = (uint64_t *)(stg + kTileM * kSP);    // w, a, full[2], empty[2]
  uint32_t *tslot = (uint32_t *)(bars + 6);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles = (g.M + kTileM - 1) / kTileM;
  uint32_t ncols = 32;
  while (ncols < (uint32_t)(2 * N)) ncols <<= 1;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int b = 0; b < 4; b++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bars + b)));
    for (int b = 4; b < 6; b++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;\n" ::"r"(smem_u32(bars + b)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t bw = smem_u32(bars), ba = smem_u32(bars + 1);
  if (warp == 4) {
    if (lane == 0) {
      bool ok = true;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bw),
                   "r"((uint32_t)(N * K * 2))
                   : "memory");
      for (int kb = 0; kb < nkb; kb++) tma_load_2d(smem_u32(sB + (size_t)kb * N * 16), &tb, kb * 8, 0, bw);
      const uint32_t id = idesc_bf16(kTileM, (uint32_t)N);
      int i = 0;
      for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, i++) {
        const int buf = i & 1;
        // the A buffer is free once the previous tile's MMAs completed
        if (i > 0) ok = mbar_wait(smem_u32(bars + 2 + ((i - 1) & 1)), ((i - 1) >> 1) & 1);
        if (!ok) break;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(ba),
                     "r"((uint32_t)(kTileM * K * 2))
                     : "memory");
        for (int kb = 0; kb < nkb; kb++)
          tma_load_2d(smem_u32(sA + (size_t)kb * kTileM * 16), &ta, kb * 8, t * kTileM, ba);
        // this accumulator is free once its tile from two rounds ago was drained
        if (i >= 2) ok = mbar_wait(smem_u32(bars + 4 + buf), ((i - 2) >> 1) & 1);
        if (ok) ok = mbar_wait(ba, i & 1);
        if (ok && i == 0) ok = mbar_wait(bw, 0);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        for (int sl = 0; sl < (K >> 4); sl++) {
          const uint64_t ad = sdesc(smem_u32(sA + (size_t)(2 * sl) * kTileM * 16), kTileM * 16, 128);
          const uint64_t bd = sdesc(smem_u32(sB + (size_t)(2 * sl) * N * 16), (uint32_t)N * 16, 128);
          mma_bf16(tmem + (uint32_t)(buf * N), ad, bd, id, sl > 0 ? 1u : 0u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         smem_u32(bars + 2 + buf))
                     : "memory");
      }
      if (!ok && g.err) atomicExch(g.err, 5);
    }
  } else {
    // epilogue warps 0-3: thread tid owns accumulator row tid
    int i = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, i++) {
      const int buf = i & 1;
      const bool ok = epi_all(mbar_wait(smem_u32(bars + 2 + buf), (i >> 1) & 1));
      if (!ok) {
        if (tid == 0 && g.err) atomicExch(g.err, 3);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int m0 = t * kTileM, rows = min(kTileM, g.M - m0);
      for (int cc = 0; cc < N; cc += kCW) {
        const int cw = min(kCW, N - cc);
        for (int c0 = 0; c0 < cw; c0 += 16) {
          uint32_t v[16];
          tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * N + cc + c0), v);
#pragma unroll
          for (int j = 0; j < 16; j++) {
            float x = __uint_as_float(v[j]);
            if (g.bias) x += g.bias[cc + c0 + j];
            if (g.relu) x = fmaxf(x, 0.0f);
            stg[tid * kSP + c0 + j] = x;
          }
        }
        epi_sync();
        const int c8 = cw >> 3;
        for (int k = tid; k < rows * c8; k += 128) {
          const int r = k / c8, c = (k - r * c8) * 8;
          float x[8];
#pragma unroll
          for (int j = 0; j < 8; j++) x[j] = stg[r * kSP + c + j];
          const size_t gc = (size_t)cc + c;
          if (g.Cf) {
            float4 *dst = (float4 *)(g.Cf + (size_t)(m0 + r) * g.ldcf + gc);
            dst[0] = make_float4(x[0], x[1], x[2], x[3]);
            dst[1] = make_float4(x[4], x[5], x[6], x[7]);
          }
          if (g.Cb) {
            uint4 o;
            bf16 *ob = (bf16 *)&o;
#pragma unroll
            for (int j = 0; j < 8; j++) ob[j] = __float2bfloat16_rn(x[j]);
            *(uint4 *)(g.Cb + (size_t)(m0 + r) * g.ldcb + gc) = o;
          }
        }
        epi_sync();
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bars + 4 + buf)) : "memory");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols));
}

size_t persist_smem(int N, int K) {
  return (size_t)(K / 8) * (N + kTileM) * 16 + (size_t)kTileM * kSP * 4 + 6 * 8 + 16;
}

size_t gemm_smem(int N, int K) {
  const size_t opnd = (size_t)(K / 8) * (kTileM + N) * 16, stage = (size_t)kTileM * kSP * 4;
  return (opnd > stage ? opnd : stage) + 8 * (1 + kMaxChunks) + 16;
}

// 2-D tensor map of a row-major BF16 matrix (rows x cols, leading dimension
// ld elements) read in boxes of box_rows rows x 8 columns (16 bytes)
typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_fn = nullptr;

int make_map(CUtensorMap *map, const bf16 *ptr, int rows, int cols, int ld, int box_rows, std::string &err) {
  if (!encode_fn) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
        q != cudaDriverEntryPointSuccess) {
      err = "gemm: cuTensorMapEncodeTiled is not available";
      return FS_ERR_CUDA;
    }
    encode_fn = (EncodeTiled)fn;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {8u, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = encode_fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)ptr, dims, strides, box, estr,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    err = "gemm: tensor map encoding failed (" + std::to_string((int)r) + ")";
    return FS_ERR_ARG;
  }
  return FS_OK;
}

bool gemm_attr_set = false;

// Checks the shape rules and launches one GEMM.
int gemm(const GemmArgs &g, cudaStream_t st, std::string &err) {
  if (g.N < 16 || g.N > 256 || g.N % 16 || g.K < 16 || g.K > 256 || g.K % 16 || g.M < 1 || g.lda % 8 ||
      g.ldb % 8 || ((uintptr_t)g.A & 15) || ((uintptr_t)g.B & 15) ||
      (g.Cf && (g.ldcf % 4 || ((uintptr_t)g.Cf & 15))) || (g.Cb && (g.ldcb % 8 || ((uintptr_t)g.Cb & 15))) ||
      (g.mask && (g.ldm % 8 || ((uintptr_t)g.mask & 15)))) {
    err = "gemm: N and K must be multiples of 16 in [16, 256], leading dimensions multiples of 8 (4 for "
          "FP32 output), operands and outputs 16-byte aligned";
    return FS_ERR_ARG;
  }
  if (!gemm_attr_set) {
    cudaFuncSetAttribute(k_gemm_tn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem(256, 256));
    gemm_attr_set = true;
  }
  // column tiles of 64 when there are few row tiles (training batches), so
  // that small-M GEMMs still spread over the SMs; one column tile otherwise
  const int tiles = (g.M + kTileM - 1) / kTileM;
  static int sms = 0;
  if (!sms && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0) != cudaSuccess) sms = 148;
  // many row tiles, plain outputs: the persistent kernel (W resident, the
  // next tile's loads and MMAs overlapping the current epilogue)
  if (!g.mask && !g.Ct && tiles >= 2 * sms && persist_smem(g.N, g.K) <= 232448) {
    static bool pattr = false;
    if (!pattr) {
      cudaFuncSetAttribute(k_gemm_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448);
      pattr = true;
    }
    CUtensorMap ta, tb;
    int rc = make_map(&ta, g.A, g.M, g.K, g.lda, kTileM, err);
    if (!rc) rc = make_map(&tb, g.B, g.N, g.K, g.ldb, g.N, err);
    if (rc) return rc;
    k_gemm_persist<<<std::min(tiles, sms), kPThreads, persist_smem(g.N, g.K), st>>>(g, ta, tb);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      err = std::string("gemm launch: ") + cudaGetErrorString(e);
      return FS_ERR_CUDA;
    }
    return FS_OK;
  }
  const int ny = (g.N % 64 == 0 && tiles < 296) ? g.N / 64 : 1;
  const dim3 grid((g.M + kTileM - 1) / kTileM, ny);
  CUtensorMap ta, tb;
  int rc = make_map(&ta, g.A, g.M, g.K, g.lda, kTileM, err);
  if (!rc) rc = make_map(&tb, g.B, g.N, g.K, g.ldb, g.N / ny, err);
  if (rc) return rc;
  k_gemm_tn<<<grid, kThreads, gemm_smem(g.N / ny, g.K), st>>>(g, ta, tb);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = std::string("gemm launch: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

// ---- element-wise kernels of the MLP -----------------------------------------

// rows of x (FP32, `cols` wide; row r taken from perm[ctr*rows + r] when
// perm is given) -> BF16 X [rows x pcols] and optionally X^T [pcols x ldt]
__global__ void k_stage_x(const float *x, int rows, int cols, int pcols, const int *perm, const int *ctr, bf16 *X,
                          bf16 *XT, int ldt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * pcols) return;
  const int r = i / pcols, c = i - r * pcols;
  const size_t src = perm ? (size_t)perm[(size_t)(*ctr) * rows + r] : (size_t)r;
  const float v = c < cols ? x[src * cols + c] : 0.0f;
  const bf16 b = __float2bfloat16_rn(v);
  X[(size_t)r * pcols + c] = b;
  if (XT) XT[(size_t)c * ldt + r] = b;
}

__global__ void k_stage_t(const float *t, int rows, int cols, int pcols, const int *perm, const int *ctr, float *T) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * pcols) return;
  const int r = i / pcols, c = i - r * pcols;
  const size_t src = perm ? (size_t)perm[(size_t)(*ctr) * rows + r] : (size_t)r;
  T[i] = c < cols ? t[src * cols + c] : 0.0f;
}

// Loss and output-layer gradient.  Columns [0, nr) regress log-rates (mean
// squared error averaged over nr columns and the rows), column nr is the
// hyperactivity logit (binary cross-entropy averaged over the rows); padded
// columns get zero gradient.
__global__ void k_loss(const float *Z, const float *T, int rows, int pcols, int nr, bf16 *dZ, bf16 *dZT, int ldt,
                       float *loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (i < rows * pcols) {
    const int r = i / pcols, c = i - r * pcols;
    const float y = Z[i], t = T[i];
    float d = 0.0f;
    if (c < nr) {
      const float e = y - t;
      d = 2.0f * e / (float)(nr * rows);
      l = e * e / (float)(nr * rows);
    } else if (c == nr) {
      const float p = 1.0f / (1.0f + expf(-y));
      d = (p - t) / (float)rows;
      l = (fmaxf(y, 0.0f) - y * t + log1pf(expf(-fabsf(y)))) / (float)rows;
    }
    const bf16 b = __float2bfloat16_rn(d);
    dZ[i] = b;
    dZT[(size_t)c * ldt + r] = b;
  }
  for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l);
}

// bias gradient: row sums of dZ^T, one warp per output unit
__global__ void k_bias_grad(const bf16 *dZT, int ldt, int rows, int n, float *gb) {
  const int c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (c >= n) return;
  float s = 0.0f;
  for (int r = lane; r < rows; r += 32) s += __bfloat162float(dZT[(size_t)c * ldt + r]);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) gb[c] = s;
}

// Adam on the FP32 master copy (step count from the device counter), then the
// BF16 copies W and W^T.
__global__ void k_adam(float *w, float *m, float *v, const float *g, int n, int rows, int cols, float lr,
                       const int *ctr, bf16 *Wb, bf16 *Wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float t = (float)(ctr[1] + 1);
  const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (Wb) {
    const bf16 b = __float2bfloat16_rn(wi);
    Wb[i] = b;
    const int r = i / cols, c = i - r * cols;
    Wt[(size_t)c * rows + r] = b;
  }
}

__global__ void k_step_end(int *ctr) {
  ctr[0] += 1;  // batch within the epoch
  ctr[1] += 1;  // Adam step
}

__global__ void k_refresh(const float *w, int rows, int cols, bf16 *Wb, bf16 *Wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const bf16 b = __float2bfloat16_rn(w[i]);
  Wb[i] = b;
  const int r = i / cols, c = i - r * cols;
  Wt[(size_t)c * rows + r] = b;
}

inline int pad16(int x) { return (x + 15) / 16 * 16; }

constexpr int kBatch = 256;     // training rows per step
constexpr int kChunk = 65536;   // inference rows per pass

struct Mlp {
  int device = 0;
  cudaStream_t st = nullptr;
  std::vector<int> dims, pd;  // logical and padded (multiple of 16) widths
  int L = 0;
  std::vector<float *> W, b, mW, vW, mb, vb, gW, gb;
  std::vector<bf16 *> Wb, Wt;
  // training buffers (kBatch rows)
  bf16 *X = nullptr, *XT = nullptr;
  std::vector<bf16 *> H, HT, dZ, dZT;
  float *Zo = nullptr, *T = nullptr, *loss = nullptr, *xs = nullptr, *ts = nullptr;
  int *ctr = nullptr, *err = nullptr;
  // inference buffers (kChunk rows, lazily)
  bf16 *PX = nullptr;
  std::vector<bf16 *> PH;
  float *PZ = nullptr, *px = nullptr;
  cudaGraphExec_t step_graph = nullptr;
  const float *graph_x = nullptr;
  std::vector<void *> allocs;
  float lr = 1e-3f;
};

template <class X>
int mal(Mlp *m, X **p, size_t n, std::string &err) {
  *p = nullptr;
  const size_t bytes = std::max<size_t>(n, 1) * sizeof(X);
  cudaError_t e = cudaMalloc((void **)p, bytes);
  if (e != cudaSuccess) {
    err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return FS_ERR_NOMEM;
  }
  m->allocs.push_back(*p);
  e = cudaMemsetAsync(*p, 0, bytes, m->st);
  if (e != cudaSuccess) {
    err = std::string("cudaMemset: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

void release(Mlp *m, void *p) {
  if (!p) return;
  auto it = std::find(m->allocs.begin(), m->allocs.end(), p);
  if (it != m->allocs.end()) m->allocs.erase(it);
  cudaFree(p);
}

int check(Mlp *m, std::string &err) {
  cudaError_t e = cudaStreamSynchronize(m->st);
  if (e != cudaSuccess) {
    err = std::string("mlp kernels: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  int h = 0;
  cudaMemcpy(&h, m->err, 4, cudaMemcpyDeviceToHost);
  if (h) {
    err = "mlp: tensor-core accumulator wait gave up (device error word set)";
    return FS_ERR_TIMEOUT;
  }
  return FS_OK;
}

void destroy(Mlp *m) {
  if (!m) return;
  cudaSetDevice(m->device);
  if (m->st) cudaStreamSynchronize(m->st);
  if (m->step_graph) cudaGraphExecDestroy(m->step_graph);
  for (void *p : m->allocs) cudaFree(p);
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
}

int create(const uint32_t *dims, uint32_t nd, int device, uint64_t seed, Mlp **out, std::string &err) {
  *out = nullptr;
  if (!dims || nd < 2) {
    err = "mlp: need at least an input and an output width";
    return FS_ERR_ARG;
  }
  for (uint32_t i = 0; i < nd; i++)
    if (dims[i] < 1 || dims[i] > 256) {
      err = "mlp: layer widths must be in [1, 256]";
      return FS_ERR_ARG;
    }
  if (dims[nd - 1] < 2) {
    err = "mlp: the output needs at least one rate and the hyperactivity logit";
    return FS_ERR_ARG;
  }
  Mlp *m = new Mlp();
  m->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    err = std::string("mlp: ") + cudaGetErrorString(e);
    delete m;
    return FS_ERR_CUDA;
  }
  if (!gemm_attr_set) {
    cudaFuncSetAttribute(k_gemm_tn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem(256, 256));
    gemm_attr_set = true;
  }
  for (uint32_t i = 0; i < nd; i++) {
    m->dims.push_back((int)dims[i]);
    m->pd.push_back(pad16((int)dims[i]));
  }
  m->L = (int)nd - 1;
  int rc = mal(m, &m->err, 1, err);
  if (!rc) rc = mal(m, &m->ctr, 2, err);
  std::mt19937_64 gen(seed ? seed : 1);
  std::normal_distribution<double> nrm(0.0, 1.0);
  for (int l = 0; l < m->L && !rc; l++) {
    const int pi = m->pd[l], po = m->pd[l + 1], n = pi * po;
    float *w, *bb, *mw, *vw, *mbb, *vbb, *gw, *gbb;
    bf16 *wb, *wt;
    if ((rc = mal(m, &w, n, err)) || (rc = mal(m, &bb, po, err)) || (rc = mal(m, &mw, n, err)) ||
        (rc = mal(m, &vw, n, err)) || (rc = mal(m, &mbb, po, err)) || (rc = mal(m, &vbb, po, err)) ||
        (rc = mal(m, &gw, n, err)) || (rc = mal(m, &gbb, po, err)) || (rc = mal(m, &wb, n, err)) ||
        (rc = mal(m, &wt, n, err)))
      break;
    m->W.push_back(w); m->b.push_back(bb); m->mW.push_back(mw); m->vW.push_back(vw);
    m->mb.push_back(mbb); m->vb.push_back(vbb); m->gW.push_back(gw); m->gb.push_back(gbb);
    m->Wb.push_back(wb); m->Wt.push_back(wt);
    // He initialisation of the logical block; padding stays zero
    std::vector<float> hw(n, 0.0f);
    const double sc = std::sqrt(2.0 / m->dims[l]);
    for (int r = 0; r < m->dims[l + 1]; r++)
      for (int c = 0; c < m->dims[l]; c++) hw[(size_t)r * pi + c] = (float)(sc * nrm(gen));
    cudaMemcpyAsync(w, hw.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->st);
    k_refresh<<<(n + 255) / 256, 256, 0, m->st>>>(w, po, pi, wb, wt);
    cudaStreamSynchronize(m->st);
  }
  if (!rc) rc = mal(m, &m->X, (size_t)kBatch * m->pd[0], err);
  if (!rc) rc = mal(m, &m->XT, (size_t)kBatch * m->pd[0], err);
  for (int l = 1; l <= m->L && !rc; l++) {
    bf16 *h, *ht, *dz, *dzt;
    const size_t n = (size_t)kBatch * m->pd[l];
    if ((rc = mal(m, &h, n, err)) || (rc = mal(m, &ht, n, err)) || (rc = mal(m, &dz, n, err)) ||
        (rc = mal(m, &dzt, n, err)))
      break;
    m->H.push_back(h); m->HT.push_back(ht); m->dZ.push_back(dz); m->dZT.push_back(dzt);
  }
  if (!rc) rc = mal(m, &m->Zo, (size_t)kBatch * m->pd[m->L], err);
  if (!rc) rc = mal(m, &m->T, (size_t)kBatch * m->pd[m->L], err);
  if (!rc) rc = mal(m, &m->loss, 1, err);
  if (!rc) rc = mal(m, &m->xs, (size_t)kBatch * m->dims[0], err);
  if (!rc) rc = mal(m, &m->ts, (size_t)kBatch * m->dims[m->L], err);
  if (!rc) rc = check(m, err);
  if (rc) {
    destroy(m);
    return rc;
  }
  *out = m;
  return FS_OK;
}

// forward over the `rows` staged rows of X (training buffers)
int forward_train(Mlp *m, int rows, std::string &err) {
  for (int l = 0; l < m->L; l++) {
    GemmArgs g{};
    g.A = l == 0 ? m->X : m->H[l - 1];
    g.lda = m->pd[l];
    g.B = m->Wb[l];
    g.ldb = m->pd[l];
    g.M = rows;
    g.N = m->pd[l + 1];
    g.K = m->pd[l];
    g.bias = m->b[l];
    g.err = m->err;
    if (l + 1 < m->L) {
      g.relu = 1;
      g.Cb = m->H[l];
      g.ldcb = m->pd[l + 1];
      g.Ct = m->HT[l];
      g.ldct = kBatch;
    } else {
      g.Cf = m->Zo;
      g.ldcf = m->pd[l + 1];
    }
    int rc = gemm(g, m->st, err);
    if (rc) return rc;
  }
  return FS_OK;
}

// loss and gradients of the staged batch; Adam step when `update`
int backward(Mlp *m, int rows, bool update, std::string &err) {
  const int L = m->L, po = m->pd[L];
  k_loss<<<(rows * po + 255) / 256, 256, 0, m->st>>>(m->Zo, m->T, rows, po, m->dims[L] - 1, m->dZ[L - 1],
                                                    m->dZT[L - 1], kBatch, m->loss);
  for (int l = L - 1; l >= 0; l--) {
    GemmArgs g{};  // dW_l = dZ_l^T . H_{l-1}
    g.A = m->dZT[l];
    g.lda = kBatch;
    g.B = l == 0 ? m->XT : m->HT[l - 1];
    g.ldb = kBatch;
    g.M = m->pd[l + 1];
    g.N = m->pd[l];
    g.K = rows;
    g.Cf = m->gW[l];
    g.ldcf = m->pd[l];
    g.err = m->err;
    int rc = gemm(g, m->st, err);
    if (rc) return rc;
    k_bias_grad<<<(m->pd[l + 1] + 7) / 8, 256, 0, m->st>>>(m->dZT[l], kBatch, rows, m->pd[l + 1], m->gb[l]);
    if (l > 0) {
      GemmArgs h{};  // dZ_{l-1} = (dZ_l . W_l) * (H_{l-1} > 0)
      h.A = m->dZ[l];
      h.lda = m->pd[l + 1];
      h.B = m->Wt[l];
      h.ldb = m->pd[l + 1];
      h.M = rows;
      h.N = m->pd[l];
      h.K = m->pd[l + 1];
      h.mask = m->H[l - 1];
      h.ldm = m->pd[l];
      h.Cb = m->dZ[l - 1];
      h.ldcb = m->pd[l];
      h.Ct = m->dZT[l - 1];
      h.ldct = kBatch;
      h.err = m->err;
      if ((rc = gemm(h, m->st, err))) return rc;
    }
  }
  if (update) {
    for (int l = 0; l < L; l++) {
      const int n = m->pd[l] * m->pd[l + 1];
      k_adam<<<(n + 255) / 256, 256, 0, m->st>>>(m->W[l], m->mW[l], m->vW[l], m->gW[l], n, m->pd[l + 1], m->pd[l],
                                                m->lr, m->ctr, m->Wb[l], m->Wt[l]);
      k_adam<<<(m->pd[l + 1] + 255) / 256, 256, 0, m->st>>>(m->b[l], m->mb[l], m->vb[l], m->gb[l], m->pd[l + 1], 1, 1,
                                                           m->lr, m->ctr, nullptr, nullptr);
    }
    k_step_end<<<1, 1, 0, m->st>>>(m->ctr);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = std::string("mlp backward: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

uint64_t param_count(const Mlp *m) {
  uint64_t n = 0;
  for (int l = 0; l < m->L; l++) n += (uint64_t)m->dims[l] * m->dims[l + 1] + m->dims[l + 1];
  return n;
}

// logical parameter vector (per layer: W [out x in] row-major, then b) <->
// padded device copies; `grads` reads the gradient buffers instead
int params_io(Mlp *m, float *out, const float *in, bool grads, std::string &err) {
  cudaStreamSynchronize(m->st);
  size_t o = 0;
  for (int l = 0; l < m->L; l++) {
    const int pi = m->pd[l], po = m->pd[l + 1], di = m->dims[l], dout = m->dims[l + 1];
    std::vector<float> w((size_t)pi * po, 0.0f), bb(po, 0.0f);
    float *dw = grads ? m->gW[l] : m->W[l], *db = grads ? m->gb[l] : m->b[l];
    if (!in) {
      cudaMemcpy(w.data(), dw, w.size() * 4, cudaMemcpyDeviceToHost);
      cudaMemcpy(bb.data(), db, bb.size() * 4, cudaMemcpyDeviceToHost);
    }
    for (int r = 0; r < dout; r++)
      for (int c = 0; c < di; c++) {
        if (in) w[(size_t)r * pi + c] = in[o + (size_t)r * di + c];
        else out[o + (size_t)r * di + c] = w[(size_t)r * pi + c];
      }
    o += (size_t)dout * di;
    for (int r = 0; r < dout; r++) {
      if (in) bb[r] = in[o + r];
      else out[o + r] = bb[r];
    }
    o += dout;
    if (in) {
      cudaMemcpy(dw, w.data(), w.size() * 4, cudaMemcpyHostToDevice);
      cudaMemcpy(db, bb.data(), bb.size() * 4, cudaMemcpyHostToDevice);
      k_refresh<<<(pi * po + 255) / 256, 256, 0, m->st>>>(m->W[l], po, pi, m->Wb[l], m->Wt[l]);
    }
  }
  return check(m, err);
}

// host rows -> the training buffers (X, X^T, T)
int stage_host(Mlp *m, const float *x, const float *t, int rows, std::string &err) {
  cudaMemcpyAsync(m->xs, x, (size_t)rows * m->dims[0] * 4, cudaMemcpyHostToDevice, m->st);
  k_stage_x<<<(rows * m->pd[0] + 255) / 256, 256, 0, m->st>>>(m->xs, rows, m->dims[0], m->pd[0], nullptr, nullptr,
                                                               m->X, m->XT, kBatch);
  if (t) {
    cudaMemcpyAsync(m->ts, t, (size_t)rows * m->dims[m->L] * 4, cudaMemcpyHostToDevice, m->st);
    k_stage_t<<<(rows * m->pd[m->L] + 255) / 256, 256, 0, m->st>>>(m->ts, rows, m->dims[m->L], m->pd[m->L], nullptr,
                                                                    nullptr, m->T);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = std::string("mlp staging: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

int grad(Mlp *m, const float *x, const float *t, int rows, float *g, float *loss, std::string &err) {
  if (rows < 16 || rows > kBatch || rows % 16) {
    err = "mlp grad: rows must be a multiple of 16 in [16, 256]";
    return FS_ERR_ARG;
  }
  int rc;
  cudaMemsetAsync(m->loss, 0, 4, m->st);
  if ((rc = stage_host(m, x, t, rows, err)) || (rc = forward_train(m, rows, err)) ||
      (rc = backward(m, rows, false, err)) || (rc = check(m, err)))
    return rc;
  if (loss) cudaMemcpy(loss, m->loss, 4, cudaMemcpyDeviceToHost);
  return params_io(m, g, nullptr, true, err);
}

int ensure_infer(Mlp *m, std::string &err) {
  if (m->PX) return FS_OK;
  int rc = mal(m, &m->PX, (size_t)kChunk * m->pd[0], err);
  for (int l = 1; l < m->L && !rc; l++) {
    bf16 *h;
    rc = mal(m, &h, (size_t)kChunk * m->pd[l], err);
    m->PH.push_back(h);
  }
  if (!rc) rc = mal(m, &m->PZ, (size_t)kChunk * m->pd[m->L], err);
  if (!rc) rc = mal(m, &m->px, (size_t)kChunk * m->dims[0], err);
  return rc;
}

int forward(Mlp *m, const float *x, uint64_t rows, float *y, double *device_ms, std::string &err) {
  int rc = ensure_infer(m, err);
  if (rc) return rc;
  const int L = m->L, no = m->dims[L], po = m->pd[L];
  std::vector<float> z((size_t)kChunk * po);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double ms_total = 0.0;
  for (uint64_t r0 = 0; r0 < rows; r0 += kChunk) {
    const int n = (int)std::min<uint64_t>(kChunk, rows - r0);
    cudaMemcpyAsync(m->px, x + r0 * m->dims[0], (size_t)n * m->dims[0] * 4, cudaMemcpyHostToDevice, m->st);
    cudaEventRecord(e0, m->st);
    k_stage_x<<<(n * m->pd[0] + 255) / 256, 256, 0, m->st>>>(m->px, n, m->dims[0], m->pd[0], nullptr, nullptr, m->PX,
                                                              nullptr, 0);
    for (int l = 0; l < L && !rc; l++) {
      GemmArgs g{};
      g.A = l == 0 ? m->PX : m->PH[l - 1];
      g.lda = m->pd[l];
      g.B = m->Wb[l];
      g.ldb = m->pd[l];
      g.M = n;
      g.N = m->pd[l + 1];
      g.K = m->pd[l];
      g.bias = m->b[l];
      g.err = m->err;
      if (l + 1 < L) {
        g.relu = 1;
        g.Cb = m->PH[l];
        g.ldcb = m->pd[l + 1];
      } else {
        g.Cf = m->PZ;
        g.ldcf = po;
      }
      rc = gemm(g, m->st, err);
    }
    cudaEventRecord(e1, m->st);
    if (rc) break;
    cudaMemcpyAsync(z.data(), m->PZ, (size_t)n * po * 4, cudaMemcpyDeviceToHost, m->st);
    if ((rc = check(m, err))) break;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    ms_total += ms;
    for (int r = 0; r < n; r++)
      std::memcpy(y + (r0 + r) * no, z.data() + (size_t)r * po, (size_t)no * 4);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (device_ms) *device_ms = ms_total;
  return rc;
}

int train(Mlp *m, const float *x, const float *t, uint64_t rows, uint32_t epochs, float lr, uint64_t seed,
          float *epoch_loss, double *device_ms, std::string &err) {
  const int steps = (int)(rows / kBatch);
  if (steps < 1) {
    err = "mlp train: need at least 256 rows";
    return FS_ERR_ARG;
  }
  m->lr = lr;
  float *xall = nullptr, *tall = nullptr;
  int *perm = nullptr;
  int rc;
  if ((rc = mal(m, &xall, rows * m->dims[0], err)) || (rc = mal(m, &tall, rows * m->dims[m->L], err)) ||
      (rc = mal(m, &perm, (size_t)steps * kBatch, err))) {
    release(m, xall);
    release(m, tall);
    release(m, perm);
    return rc;
  }
  cudaMemcpyAsync(xall, x, rows * m->dims[0] * 4, cudaMemcpyHostToDevice, m->st);
  cudaMemcpyAsync(tall, t, rows * m->dims[m->L] * 4, cudaMemcpyHostToDevice, m->st);
  // one training step, captured once and replayed
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaStreamBeginCapture(m->st, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    k_stage_x<<<(kBatch * m->pd[0] + 255) / 256, 256, 0, m->st>>>(xall, kBatch, m->dims[0], m->pd[0], perm, m->ctr,
                                                                   m->X, m->XT, kBatch);
    k_stage_t<<<(kBatch * m->pd[m->L] + 255) / 256, 256, 0, m->st>>>(tall, kBatch, m->dims[m->L], m->pd[m->L], perm,
                                                                      m->ctr, m->T);
    rc = forward_train(m, kBatch, err);
    if (!rc) rc = backward(m, kBatch, true, err);
    cudaError_t e2 = cudaStreamEndCapture(m->st, &graph);
    if (!rc && e2 != cudaSuccess) e = e2;
  }
  if (!rc && e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (!rc && e != cudaSuccess) {
    err = std::string("mlp train graph: ") + cudaGetErrorString(e);
    rc = FS_ERR_CUDA;
  }
  std::mt19937_64 gen(seed ? seed : 1);
  std::vector<int> order(rows);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double ms_total = 0.0;
  for (uint32_t ep = 0; ep < epochs && !rc; ep++) {
    std::iota(order.begin(), order.end(), 0);
    std::shuffle(order.begin(), order.end(), gen);
    cudaMemcpyAsync(perm, order.data(), (size_t)steps * kBatch * 4, cudaMemcpyHostToDevice, m->st);
    cudaMemsetAsync(m->ctr, 0, 4, m->st);  // batch index (the Adam count in ctr[1] runs on)
    cudaMemsetAsync(m->loss, 0, 4, m->st);
    cudaEventRecord(e0, m->st);
    for (int s = 0; s < steps; s++) {
      e = cudaGraphLaunch(exec, m->st);
      if (e != cudaSuccess) break;
    }
    cudaEventRecord(e1, m->st);
    if (e != cudaSuccess) {
      err = std::string("mlp train: ") + cudaGetErrorString(e);
      rc = FS_ERR_CUDA;
      break;
    }
    if ((rc = check(m, err))) break;
    float ms = 0, l = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    ms_total += ms;
    cudaMemcpy(&l, m->loss, 4, cudaMemcpyDeviceToHost);
    if (epoch_loss) epoch_loss[ep] = l / (float)steps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (exec) cudaGraphExecDestroy(exec);
  cudaStreamSynchronize(m->st);
  release(m, xall);
  release(m, tall);
  release(m, perm);
  if (device_ms) *device_ms = ms_total;
  return rc;
}

}  // namespace fsm

// ---- C ABI ---------------------------------------------------------------------
struct fs_mlp {
  fsm::Mlp *m;
};

namespace {
thread_local std::string g_mlp_err;
int mlp_fail(int rc, const std::string &msg) {
  g_mlp_err = msg;
  return rc;
}
}  // namespace

extern "C" {

const char *fs_mlp_error(void) { return g_mlp_err.c_str(); }

int fs_mlp_create(const uint32_t *dims, uint32_t ndims, int device, uint64_t seed, fs_mlp **out) {
  if (!out) return mlp_fail(FS_ERR_ARG, "fs_mlp_create: out is NULL");
  *out = nullptr;
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) return mlp_fail(FS_ERR_NODEVICE, "fs_mlp_create: no CUDA device");
  if (device < 0 || device >= nd) return mlp_fail(FS_ERR_ARG, "fs_mlp_create: bad device ordinal");
  std::string err;
  fsm::Mlp *m = nullptr;
  int rc = fsm::create(dims, ndims, device, seed, &m, err);
  if (rc) return mlp_fail(rc, err);
  *out = new fs_mlp{m};
  return FS_OK;
}

int fs_mlp_destroy(fs_mlp *h) {
  if (!h) return FS_OK;
  fsm::destroy(h->m);
  delete h;
  return FS_OK;
}

uint64_t fs_mlp_param_count(const fs_mlp *h) { return h ? fsm::param_count(h->m) : 0; }

int fs_mlp_get_params(fs_mlp *h, float *params) {
  if (!h || !params) return mlp_fail(FS_ERR_ARG, "fs_mlp_get_params: null argument");
  cudaSetDevice(h->m->device);
  std::string err;
  int rc = fsm::params_io(h->m, params, nullptr, false, err);
  return rc ? mlp_fail(rc, err) : FS_OK;
}

int fs_mlp_set_params(fs_mlp *h, const float *params) {
  if (!h || !params) return mlp_fail(FS_ERR_ARG, "fs_mlp_set_params: null argument");
  cudaSetDevice(h->m->device);
  std::string err;
  int rc = fsm::params_io(h->m, nullptr, params, false, err);
  return rc ? mlp_fail(rc, err) : FS_OK;
}

int fs_mlp_forward(fs_mlp *h, const float *x, uint64_t rows, float *y, double *device_ms) {
  if (!h || (rows && (!x || !y))) return mlp_fail(FS_ERR_ARG, "fs_mlp_forward: null argument");
  cudaSetDevice(h->m->device);
  std::string err;
  int rc = fsm::forward(h->m, x, rows, y, device_ms, err);
  return rc ? mlp_fail(rc, err) : FS_OK;
}

int fs_mlp_grad(fs_mlp *h, const float *x, const float *t, uint32_t rows, float *grads, float *loss) {
  if (!h || !x || !t || !grads) return mlp_fail(FS_ERR_ARG, "fs_mlp_grad: null argument");
  cudaSetDevice(h->m->device);
  std::string err;
  int rc = fsm::grad(h->m, x, t, (int)rows, grads, loss, err);
  return rc ? mlp_fail(rc, err) : FS_OK;
}

int fs_mlp_train(fs_mlp *h, const float *x, const float *t, uint64_t rows, uint32_t epochs, float lr, uint64_t seed,
                 float *epoch_loss, double *device_ms) {
  if (!h || !x || !t) return mlp_fail(FS_ERR_ARG, "fs_mlp_train: null argument");
  cudaSetDevice(h->m->device);
  std::string err;
  int rc = fsm::train(h->m, x, t, rows, epochs, lr, seed, epoch_loss, device_ms, err);
  return rc ? mlp_fail(rc, err) : FS_OK;
}

int fs_mlp_gemm(const uint16_t *a, const uint16_t *b, uint32_t m, uint32_t n, uint32_t k, const float *bias,
                int relu, float *c) {
  if (!a || !b || !c) return mlp_fail(FS_ERR_ARG, "fs_mlp_gemm: null argument");
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) return mlp_fail(FS_ERR_NODEVICE, "fs_mlp_gemm: no CUDA device");
  fsm::GemmArgs g{};
  g.M = (int)m;
  g.N = (int)n;
  g.K = (int)k;
  g.lda = (int)k;
  g.ldb = (int)k;
  g.relu = relu;
  g.ldcf = (int)n;
  void *da = nullptr, *db = nullptr, *dc = nullptr, *dbias = nullptr;
  int *derr = nullptr;
  cudaError_t e = cudaMalloc(&da, (size_t)m * k * 2);
  if (e == cudaSuccess) e = cudaMalloc(&db, (size_t)n * k * 2);
  if (e == cudaSuccess) e = cudaMalloc(&dc, (size_t)m * n * 4);
  if (e == cudaSuccess && bias) e = cudaMalloc(&dbias, (size_t)n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&derr, 4);
  int rc = FS_OK;
  std::string err;
  if (e == cudaSuccess) {
    cudaMemcpy(da, a, (size_t)m * k * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(db, b, (size_t)n * k * 2, cudaMemcpyHostToDevice);
    if (bias) cudaMemcpy(dbias, bias, (size_t)n * 4, cudaMemcpyHostToDevice);
    cudaMemset(derr, 0, 4);
    g.A = (const fsm::bf16 *)da;
    g.B = (const fsm::bf16 *)db;
    g.Cf = (float *)dc;
    g.bias = (const float *)dbias;
    g.err = derr;
    rc = fsm::gemm(g, nullptr, err);
    if (!rc) {
      e = cudaDeviceSynchronize();
      int h = 0;
      if (e == cudaSuccess) e = cudaMemcpy(&h, derr, 4, cudaMemcpyDeviceToHost);
      if (e == cudaSuccess && h) rc = mlp_fail(FS_ERR_TIMEOUT, "fs_mlp_gemm: accumulator wait gave up");
      if (e == cudaSuccess && !rc) e = cudaMemcpy(c, dc, (size_t)m * n * 4, cudaMemcpyDeviceToHost);
    }
  }
  if (e != cudaSuccess && !rc) rc = mlp_fail(FS_ERR_CUDA, std::string("fs_mlp_gemm: ") + cudaGetErrorString(e));
  else if (rc && !err.empty()) mlp_fail(rc, err);
  cudaFree(da);
  cudaFree(db);
  cudaFree(dc);
  cudaFree(dbias);
  cudaFree(derr);
  return rc;
}

}  // extern "C"
