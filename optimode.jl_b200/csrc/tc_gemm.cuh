// BF16 GEMM on the sm_100a tensor cores (tcgen05 + TMA), FP32 accumulation in tensor memory.
//
//   D[M×N] (=, +=) A[M×K] · B[N×K]ᵀ   (+ bias[N], ReLU), A and B row-major bf16 ("K-major")
//
// One CTA of 128 threads computes a 128×BN tile of D over a range of K (split-K CTAs add
// their partial tiles atomically into an FP32 D); two or more CTAs share an SM:
//   * warp 0, one lane: TMA producer.  Per 64-wide K step it loads the 128×64 A box and the
//     BN×64 B box (128-byte swizzle, the canonical K-major UMMA layout) into one stage of a
//     ring, completing on the stage's `full` mbarrier;
//   * warp 1, one lane: MMA issuer.  Four tcgen05.mma (M=128, N=BN, K=16 each) per stage;
//     tcgen05.commit releases the stage (`empty`) when the tensor core has read it, and a
//     last commit signals `done`;
//   * all four warps: epilogue.  Warp w reads TMEM lanes 32w..32w+31 (rows) with
//     tcgen05.ld, applies bias / ReLU, and stores (FP32, BF16 or FP32 atomics).
// Every mbarrier wait is bounded by the global timer (pipe.cuh); a wait that runs out
// records an error and the CTA leaves the pipeline only after its own TMA loads have landed
// and its MMAs have completed (both waited for with the same bound), then frees its TMEM.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "pipe.cuh"
#include "tc_gemm.h"

namespace omb {

constexpr int TC_BM = 128;       // rows per CTA tile (UMMA M)
constexpr int TC_BK = 64;        // K per stage: one 128-byte swizzle row of bf16
constexpr int TC_MAX_STAGES = 3;
constexpr int TC_THREADS = 128;
// Ring depth: two stages for the widest tiles and three otherwise, so that at least two CTAs
// fit an SM (≤ 97 KB of shared memory each, ≤ 256 TMEM columns each) and one CTA's epilogue
// overlaps another's main loop.
__host__ __device__ constexpr int tc_stages(int BN) { return BN >= 256 ? 2 : 3; }

struct TcGemmArgs {
  void* D;              // output, row-major, leading dimension ldd (elements)
  long long ldd;
  const float* bias;    // N values or NULL
  int M, N, K;          // K a multiple of 64
  int kt_per_split;     // K steps (of 64) per split-K CTA
  int relu;             // 1: max(0, ·) after the bias
  int epi;              // TcEpi
  int* err;             // pipeline error word (first error wins)
  uint64_t wait_ns;
};

// ---- PTX wrappers -------------------------------------------------------------------
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor of a K-major tile with the 128-byte swizzle: rows of 128 B,
// 8-row groups 1024 B apart (SBO), leading offset unused (1), descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M = 128, N = BN.
__host__ __device__ constexpr uint32_t tc_idesc(int BN) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}
__host__ __device__ constexpr uint32_t tc_tmem_cols(int BN) { return BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256; }
__host__ __device__ constexpr size_t tc_stage_bytes(int BN) { return (size_t)TC_BM * 128 + (size_t)BN * 128; }
__host__ __device__ constexpr size_t tc_smem_bytes(int BN) { return 1024 + tc_stages(BN) * tc_stage_bytes(BN) + 256; }

template <int BN>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_tc_gemm(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, TcGemmArgs g) {
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N for M = 128");
  constexpr int TC_STAGES = tc_stages(BN);
  static_assert(TC_STAGES <= TC_MAX_STAGES, "ring depth");
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  // 1024-byte aligned ring (the swizzle pattern repeats every 1024 B)
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + TC_STAGES * tc_stage_bytes(BN));
  uint64_t* empty = full + TC_STAGES;
  uint64_t* done = empty + TC_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * BN;
  const int ktiles = g.K / TC_BK;
  const int kt0 = blockIdx.z * g.kt_per_split;
  const int kt1 = min(ktiles, kt0 + g.kt_per_split);
  if (kt0 >= kt1) return;  // an empty split (uniform across the CTA)
  const int nk = kt1 - kt0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(done, 1);
    mbar_init_fence();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, tc_tmem_cols(BN));
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer
    int issued[TC_STAGES] = {};
    for (int i = 0; i < nk; ++i) {
      const int s = i % TC_STAGES;
      if (!mbar_wait(&empty[s], ((i / TC_STAGES) & 1) ^ 1, g.wait_ns)) { pipe_fail(g.err, PIPE_EMPTY_TIMEOUT); break; }
      unsigned char* sa = base + s * tc_stage_bytes(BN);
      unsigned char* sb = sa + TC_BM * 128;
      mbar_arrive_expect_tx(&full[s], (uint32_t)tc_stage_bytes(BN));
      const int kx = (kt0 + i) * TC_BK;
      tma_load_2d(sa, &ta, kx, m0, &full[s]);
      tma_load_2d(sb, &tb, kx, n0, &full[s]);
      issued[s] = i + 1;
    }
    // leave no load in flight
    for (int s = 0; s < TC_STAGES; ++s)
      if (issued[s] > 0 && !mbar_wait(&full[s], ((issued[s] - 1) / TC_STAGES) & 1, drain_limit(g.wait_ns)))
        pipe_fail(g.err, PIPE_DRAIN_TIMEOUT);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    constexpr uint32_t idesc = tc_idesc(BN);
    for (int i = 0; i < nk; ++i) {
      const int s = i % TC_STAGES;
      if (!mbar_wait(&full[s], (i / TC_STAGES) & 1, g.wait_ns)) { pipe_fail(g.err, PIPE_FULL_TIMEOUT); break; }
      tc_fence_after();
      const uint32_t sa = smem_u32(base + s * tc_stage_bytes(BN));
      const uint32_t sb = sa + TC_BM * 128;
#pragma unroll
      for (int kk = 0; kk < TC_BK / 16; ++kk)  // 16 bf16 = 32 bytes per MMA along K
        tc_mma_bf16(tmem, sw128_desc(sa + kk * 32), sw128_desc(sb + kk * 32), idesc, (i > 0 || kk > 0) ? 1u : 0u);
      tc_commit(&empty[s]);
    }
    tc_commit(done);  // arrives when every MMA issued above has completed
  }
  __syncwarp();
  // ---- epilogue: every thread owns one row of the tile
  const bool ok = mbar_wait(done, 0, drain_limit(g.wait_ns));
  if (!ok && lane == 0) pipe_fail(g.err, PIPE_DRAIN_TIMEOUT);
  tc_fence_after();
  const int row = m0 + warp * 32 + lane;
  const bool failed = !ok || *(volatile int*)g.err != 0;
#pragma unroll 1
  for (int c0 = 0; c0 < BN; c0 += 16) {
    float v[16];
    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);  // warp-collective
    if (failed || row >= g.M) continue;
    const int nb = n0 + c0;
    if (nb >= g.N) continue;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      float x = v[j];
      if (g.bias && nb + j < g.N) x += g.bias[nb + j];
      if (g.relu) x = fmaxf(x, 0.f);
      v[j] = x;
    }
    // a thread's 16 consecutive outputs of its row: whole 16-byte vectors when they are all in
    // range and aligned (full 32-byte sectors per thread instead of 16 scattered scalars)
    const size_t off = (size_t)row * g.ldd + nb;
    if (g.epi == TC_STORE_BF16) {
      __nv_bfloat16* dst = static_cast<__nv_bfloat16*>(g.D) + off;
      if (nb + 16 <= g.N && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
        uint4 q[2];
        uint32_t* w = reinterpret_cast<uint32_t*>(q);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
          w[j] = *reinterpret_cast<const uint32_t*>(&h);
        }
        reinterpret_cast<uint4*>(dst)[0] = q[0];
        reinterpret_cast<uint4*>(dst)[1] = q[1];
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (nb + j < g.N) dst[j] = __float2bfloat16_rn(v[j]);
      }
    } else {
      float* dst = static_cast<float*>(g.D) + off;
      const bool vec = nb + 16 <= g.N && (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
      if (g.epi == TC_STORE_F32) {
        if (vec) {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            reinterpret_cast<float4*>(dst)[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (nb + j < g.N) dst[j] = v[j];
        }
      } else {
        if (vec) {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            atomicAdd(reinterpret_cast<float4*>(dst) + j, make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]));
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (nb + j < g.N) atomicAdd(dst + j, v[j]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, tc_tmem_cols(BN));
}

}  // namespace omb
