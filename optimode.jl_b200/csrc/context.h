// Context, error reporting, device buffers and problem upload for libomb200.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "omb200.h"
#include "ops.h"

struct omb_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  omb::TwTables tw{};
  void* tw_mem = nullptr;
  int num_sms = 0;
  // page-locked staging for result downloads (grown on demand, kept for the context's life)
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  // limit of every bounded wait in the streaming kernels (omb_ctx_set_wait_limit)
  uint64_t wait_ns = 1000000000ull;
  // learned warm-start network used by OMB_WARM_LEARNED (not owned)
  struct omb_warmstart* ws = nullptr;
  // every network created on this context: omb_ctx_destroy releases their device memory
  std::vector<struct omb_warmstart*> nets;
  // tune the FP32 operator tiles of a grid on its first batched solve (omb_ctx_set_autotune)
  int autotune = 1;
};

namespace omb {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define OMB_CU(x)                                            \
  do {                                                       \
    cudaError_t e__ = (x);                                   \
    if (e__ != cudaSuccess) return ::omb::cuda_fail(e__, #x); \
  } while (0)

// A device→host gather: every piece lands in the context's page-locked staging buffer at
// full link speed (one synchronisation), then host threads copy the pieces to the caller's
// (pageable) buffers in parallel.
struct D2HPiece {
  const void* src;  // device
  void* dst;        // host
  size_t bytes;
};
int gather_to_host(omb_ctx* ctx, const D2HPiece* pieces, size_t n);

// Large device blocks (≥ BIG_BLOCK bytes) come from a per-device cache of cudaMalloc'd
// blocks that are kept for the life of the process and handed out best-fit, so the
// multi-GB block buffers of consecutive phases, stages and batches reuse memory instead of
// growing the stream-ordered pool (which maps new pages, hundreds of ms per GB, whenever
// no free fragment fits).  A returned block records an event on the stream that last used
// it; a later user on another stream waits on that event first.
constexpr size_t BIG_BLOCK = (size_t)4 << 20;
cudaError_t big_alloc(void** p, size_t bytes, cudaStream_t st);
void big_free(void* p, cudaStream_t st);

// Stream-ordered device buffer: cudaMallocAsync from the device's pool for small buffers,
// the block cache above for large ones.
template <typename T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), st(o.st) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; st = o.st; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  cudaError_t alloc(size_t count, cudaStream_t stream) {
    release();
    st = stream;
    n = count;
    if (count == 0) return cudaSuccess;
    if (count * sizeof(T) >= BIG_BLOCK) return big_alloc(reinterpret_cast<void**>(&p), count * sizeof(T), stream);
    return cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), stream);
  }
  cudaError_t zero() { return n ? cudaMemsetAsync(p, 0, n * sizeof(T), st) : cudaSuccess; }
  void release() {
    if (p) {
      if (n * sizeof(T) >= BIG_BLOCK) big_free(p, st);
      else cudaFreeAsync(p, st);
    }
    p = nullptr;
    n = 0;
  }
};

// ε⁻¹ of one cell resident on the device in both precisions (6 unique entries per pixel)
// plus ε_ave = 3/tr(ε⁻¹) for the MPB-style preconditioner.
struct Problem {
  int Nx = 0, Ny = 0;
  int Nz = 1;       // z-periodic cells: Nz > 1 slabs over the period Dz
  double Dx = 0, Dy = 0, Dz = 0;
  double eps_mean = 0;  // cell mean of ε_ave (diagonal preconditioner scale)
  double min_diag = 0;  // min over pixels and a of ε⁻¹[a,a] (k_guess)
  double max_trace = 0; // max over pixels of tr ε⁻¹ (bounds the largest eigenvalue of ε⁻¹)
  DevBuf<float4> e32a;
  DevBuf<float2> e32b;
  DevBuf<double2> e64;
  DevBuf<float> eave32;
  DevBuf<double> eave64;
  size_t N() const { return (size_t)Nx * Ny * Nz; }
};

// Validate the grid and ε⁻¹ and upload them.  Returns OMB_OK or an error code.
int check_grid(const omb_grid* g);
// Nz > 1: a z-periodic cell, ε⁻¹ (3, 3, Nx, Ny, Nz) over the period Dz.
int upload_problem(omb_ctx* ctx, const omb_grid* g, const double* epsinv, Problem& P, int Nz = 1, double Dz = 0);

// Fill an OpUnit for one problem (pointers to block buffers set by the caller).
template <typename T> OpUnit<T> make_unit(const Problem& P);
// Autotuner (tune.cu): has (device, Nx, Ny) been tuned; tune it now (9 timed variants).
bool tune_known(int dev, int Nx, int Ny);
int autotune_grid(omb_ctx* ctx, const omb_grid* g, int ncol, int units, struct TileChoice* best, double* times);

// Release the device memory of every warm-start network created on `ctx` and detach them
// (warmstart.cu); omb_ctx_destroy calls it before the context's stream goes away.
void ws_release_all(omb_ctx* ctx);

}  // namespace omb
