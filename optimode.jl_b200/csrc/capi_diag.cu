// Failure-detection controls of a context: the limit of the streaming kernels' bounded waits,
// and a self-test that makes one such wait run out.  No reference counterpart (the
// reference's solvers run on the host and have no device-side waits).
#include <cmath>

#include "context.h"
#include "pipe.cuh"

namespace omb {

// One CTA waits on an mbarrier phase that nothing completes (two arrivals expected, one
// made), with the same bounded wait the Gram and update pipelines use.  It records
// PIPE_FULL_TIMEOUT when the limit runs out and returns; no copy is ever issued, so nothing
// is in flight when it exits.
__global__ void k_selftest_wait(uint64_t wait_ns, int* err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 2);
    mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_arrive(&bar);
    if (!mbar_wait(&bar, 0, wait_ns)) pipe_fail(err, PIPE_FULL_TIMEOUT);
  }
}

}  // namespace omb

using namespace omb;

extern "C" {

int omb_ctx_set_wait_limit(omb_ctx* ctx, double seconds) {
  if (!ctx) return fail(OMB_ERR_INVALID_ARG, "ctx is NULL");
  if (!(seconds > 0) || !std::isfinite(seconds) || seconds > 60.0)
    return fail(OMB_ERR_INVALID_ARG, "wait limit must be in (0, 60] seconds");
  ctx->wait_ns = (uint64_t)std::llround(seconds * 1e9);
  if (ctx->wait_ns == 0) ctx->wait_ns = 1;
  return OMB_OK;
}

int omb_selftest_wait(omb_ctx* ctx, int32_t* code) {
  if (!ctx) return fail(OMB_ERR_INVALID_ARG, "ctx is NULL");
  OMB_CU(cudaSetDevice(ctx->device));
  int* d_err = nullptr;
  OMB_CU(cudaMallocAsync(reinterpret_cast<void**>(&d_err), sizeof(int), ctx->stream));
  cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(int), ctx->stream);
  if (e == cudaSuccess) {
    k_selftest_wait<<<1, 32, 0, ctx->stream>>>(ctx->wait_ns, d_err);
    e = cudaGetLastError();
  }
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFreeAsync(d_err, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "omb_selftest_wait");
  if (code) *code = h;
  if (h != PIPE_OK)
    return fail(OMB_ERR_TIMEOUT, "self-test wait ran out after " + std::to_string(ctx->wait_ns / 1e9) + " s (code " +
                                     std::to_string(h) + ")");
  return OMB_OK;
}

}  // extern "C"
