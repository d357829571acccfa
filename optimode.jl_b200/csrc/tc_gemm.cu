// Host side of the tcgen05 BF16 GEMM (tc_gemm.cuh): TMA descriptors, tile choice, split-K.
#include <cuda.h>

#include <mutex>
#include <string>

#include "context.h"
#include "tc_gemm.h"
#include "tc_gemm.cuh"

namespace omb {

namespace {
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn g_encode = nullptr;
std::mutex g_encode_mu;

int encode_fn(EncodeTiledFn* out) {
  std::lock_guard<std::mutex> lk(g_encode_mu);
  if (!g_encode) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess || !p)
      return fail(OMB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    g_encode = reinterpret_cast<EncodeTiledFn>(p);
  }
  *out = g_encode;
  return OMB_OK;
}

// A row-major bf16 matrix [rows × K] (row pitch K·2 bytes) with boxes of 64 × box_rows and
// the 128-byte swizzle; out-of-range rows of a box read as zero.
int make_map(CUtensorMap* m, const void* base, long long rows, int K, int box_rows) {
  EncodeTiledFn enc = nullptr;
  int rc = encode_fn(&enc);
  if (rc) return rc;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
  const cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(OMB_ERR_CUDA, "cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")");
  return OMB_OK;
}

template <int BN>
cudaError_t launch_bn(const CUtensorMap& ta, const CUtensorMap& tb, const TcGemmArgs& g, dim3 grid, cudaStream_t st) {
  const size_t smem = tc_smem_bytes(BN);
  cudaError_t e = ensure_smem(reinterpret_cast<const void*>(k_tc_gemm<BN>), smem);
  if (e != cudaSuccess) return e;
  k_tc_gemm<BN><<<grid, TC_THREADS, smem, st>>>(ta, tb, g);
  return cudaGetLastError();
}
}  // namespace

int tc_gemm_bn(int N) { return N <= 16 ? 16 : N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256; }

int tc_gemm(cudaStream_t st, const void* A, const void* B, void* D, int M, int N, int K, long long ldd,
            const float* bias, int relu, int epi, int splits, int* d_err, uint64_t wait_ns) {
  if (M <= 0 || N <= 0 || K <= 0 || K % TC_BK != 0)
    return fail(OMB_ERR_INVALID_ARG, "tc_gemm: need M, N > 0 and K a positive multiple of 64");
  if (!A || !B || !D || !d_err) return fail(OMB_ERR_INVALID_ARG, "tc_gemm: NULL pointer");
  if ((reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15))
    return fail(OMB_ERR_INVALID_ARG, "tc_gemm: A and B must be 16-byte aligned");
  if (epi < TC_STORE_F32 || epi > TC_ATOMIC_F32) return fail(OMB_ERR_INVALID_ARG, "tc_gemm: bad epilogue");
  if (ldd < N) return fail(OMB_ERR_INVALID_ARG, "tc_gemm: ldd < N");
  const int BN = tc_gemm_bn(N);
  const int ktiles = K / TC_BK;
  if (splits < 1) splits = 1;
  if (splits > ktiles) splits = ktiles;
  if (splits > 1 && epi != TC_ATOMIC_F32)
    return fail(OMB_ERR_INVALID_ARG, "tc_gemm: split-K needs the atomic FP32 epilogue");
  const int per = (ktiles + splits - 1) / splits;
  splits = (ktiles + per - 1) / per;
  CUtensorMap ta, tb;
  int rc = make_map(&ta, A, M, K, TC_BM);
  if (rc) return rc;
  rc = make_map(&tb, B, N, K, BN);
  if (rc) return rc;
  TcGemmArgs g{};
  g.D = D; g.ldd = ldd; g.bias = bias; g.M = M; g.N = N; g.K = K;
  g.kt_per_split = per; g.relu = relu; g.epi = epi; g.err = d_err; g.wait_ns = wait_ns;
  const dim3 grid((M + TC_BM - 1) / TC_BM, (N + BN - 1) / BN, splits);
  cudaError_t e;
  switch (BN) {
    case 16: e = launch_bn<16>(ta, tb, g, grid, st); break;
    case 32: e = launch_bn<32>(ta, tb, g, grid, st); break;
    case 64: e = launch_bn<64>(ta, tb, g, grid, st); break;
    case 128: e = launch_bn<128>(ta, tb, g, grid, st); break;
    default: e = launch_bn<256>(ta, tb, g, grid, st); break;
  }
  if (e != cudaSuccess) return cuda_fail(e, "k_tc_gemm launch");
  return OMB_OK;
}

}  // namespace omb

extern "C" int omb_tc_gemm(omb_ctx* ctx, const void* d_A, const void* d_B, void* d_D, int32_t M, int32_t N, int32_t K,
                           int64_t ldd, const float* d_bias, int32_t relu, int32_t epi, int32_t splits) {
  using namespace omb;
  if (!ctx) return fail(OMB_ERR_INVALID_ARG, "ctx is NULL");
  OMB_CU(cudaSetDevice(ctx->device));
  int* d_err = nullptr;
  OMB_CU(cudaMallocAsync(reinterpret_cast<void**>(&d_err), sizeof(int), ctx->stream));
  cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(int), ctx->stream);
  if (e != cudaSuccess) { cudaFreeAsync(d_err, ctx->stream); return cuda_fail(e, "cudaMemsetAsync"); }
  int rc = tc_gemm(ctx->stream, d_A, d_B, d_D, M, N, K, ldd, d_bias, relu, epi, splits, d_err, ctx->wait_ns);
  int h = 0;
  e = cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFreeAsync(d_err, ctx->stream);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "omb_tc_gemm");
  if (h) return fail(OMB_ERR_TIMEOUT, "omb_tc_gemm: a pipeline wait ran out (code " + std::to_string(h) + ")");
  return OMB_OK;
}
