// BF16 tensor-core GEMM (tcgen05 + TMA) used by the warm-start network.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace omb {

enum TcEpi : int { TC_STORE_F32 = 0, TC_STORE_BF16 = 1, TC_ATOMIC_F32 = 2 };

// D[M×N] = A[M×K]·B[N×K]ᵀ (+ bias[N], ReLU) with A, B row-major bf16 device matrices, K a
// multiple of 64, both 16-byte aligned.  epi: 0 store FP32, 1 store BF16, 2 FP32 atomic add
// (required when splits > 1: the K range is cut over `splits` CTAs per tile).  ldd is D's
// leading dimension in elements.  A pipeline wait that runs out sets *d_err.
int tc_gemm(cudaStream_t st, const void* A, const void* B, void* D, int M, int N, int K, long long ldd,
            const float* bias, int relu, int epi, int splits, int* d_err, uint64_t wait_ns);
// The tile width (UMMA N) chosen for N columns.
int tc_gemm_bn(int N);

}  // namespace omb
