// Allocation-free FP32 operator apply (omb_apply_M_noalloc).
//
// Some callers cannot allocate device memory at the moment they need the operator:
// host frameworks that own the whole device pool (a Julia or PyTorch caching allocator
// that forbids foreign cudaMalloc/cudaFree), callers with a fixed device-memory budget
// decided up front, and hot loops that must not pay the latency and the implicit device
// synchronisation of cudaMalloc/cudaFree.  This entry point takes every input and output as
// caller-owned device memory and allocates nothing itself: the intermediate 3-component
// field of the three FFT passes lives in a file-scope static device array of fixed size,
// and so do the small per-call parameter block and the twiddle tables.
//
// Limits and rules:
//  * Nx·Ny·ncol ≤ OMB_NOALLOC_MAX_PIXEL_COLUMNS (262144: e.g. 256×256 with 4 columns or
//    512×512 with 1); larger requests are rejected with OMB_ERR_INVALID_ARG.
//  * The array (6 MiB + 256 B) is held by every GPU that loads the library until exit.
//  * All calls share it, so calls that overlap on the GPU (different streams, or
//    different host threads) race; serialise them on one stream.
//  * The first call in a CUDA context does a one-time set-up with that context current
//    (it resolves the arrays' device addresses with cudaGetSymbolAddress and uploads the
//    twiddle tables with a blocking copy); make that first call before any stream capture
//    (a first call on a capturing stream is refused with OMB_ERR_INVALID_ARG).  The set-up
//    is keyed on the context, so a new primary context after cudaDeviceReset repeats it.
//  * Each call writes its parameter block (k and the pass descriptor) into the array with a
//    one-thread kernel that receives them by value, on the caller's stream, ahead of the
//    three passes; the field needs no clearing (the first pass writes every element the
//    later passes read).
//  * Lines that split into two register DFTs (every supported length up to 256) use the
//    two-level register-FFT passes of omb_apply; 320, 384 and 512 use the shared-memory
//    Stockham passes.  ε⁻¹ is read in the reference's (3, 3, Nx, Ny) layout.
#include <cuda.h>

#include <cmath>
#include <mutex>

#include "context.h"
#include "ops_impl.cuh"

namespace omb {

constexpr long long NOALLOC_MAX_PIXEL_COLUMNS = 262144;
constexpr size_t NOALLOC_PARAM_BYTES = 256;
constexpr size_t NOALLOC_FIELD_BYTES = 3 * (size_t)NOALLOC_MAX_PIXEL_COLUMNS * sizeof(float2);

// scratch: [0, 256) parameter block (k, then the pass descriptor), then the 3·N·ncol field
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_PARAM_BYTES + NOALLOC_FIELD_BYTES];

#define OMB_NOALLOC_LENS(X) X(8) X(12) X(16) X(20) X(24) X(32) X(40) X(48) X(64) X(80) X(96) \
  X(128) X(160) X(192) X(256) X(320) X(384) X(512)
#define OMB_LEN_SUM(n) +3 * n
// per length L: [exp(-2πi m/L), m < L | TW1 | TW3] (the layout of the context's tables)
constexpr int NOALLOC_TW_TOTAL = 0 OMB_NOALLOC_LENS(OMB_LEN_SUM);
#undef OMB_LEN_SUM
static __device__ __align__(16) float2 g_noalloc_tw[NOALLOC_TW_TOTAL];

struct NoallocDevice {
  unsigned long long ctx_id = 0;     // context the set-up was done in (0: none yet)
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  float2* tw = nullptr;              // device address of g_noalloc_tw
  int tw_off[513] = {};
};
static NoallocDevice g_noalloc_dev[64];
static std::mutex g_noalloc_mu;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (the runtime has made it current).
static int current_ctx_id(unsigned long long* id) {
  static CtxGetCurrentFn get_cur = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_cur || !get_id) {
    void* a = nullptr;
    void* b = nullptr;
    cudaDriverEntryPointQueryResult qa{}, qb{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess || !a ||
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess || !b)
      return fail(OMB_ERR_CUDA, "omb_apply_M_noalloc: cuCtxGetCurrent/cuCtxGetId not available from the driver");
    get_cur = reinterpret_cast<CtxGetCurrentFn>(a);
    get_id = reinterpret_cast<CtxGetIdFn>(b);
  }
  CUcontext c = nullptr;
  if (get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, id) != CUDA_SUCCESS)
    return fail(OMB_ERR_CUDA, "omb_apply_M_noalloc: no current CUDA context");
  return OMB_OK;
}

static int noalloc_setup(int dev, cudaStream_t st) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoallocDevice& D = g_noalloc_dev[dev];
  unsigned long long id = 0;
  int rc = current_ctx_id(&id);
  if (rc) return rc;
  if (D.ctx_id == id) return OMB_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(st, &cs);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamIsCapturing");
  if (cs != cudaStreamCaptureStatusNone)
    return fail(OMB_ERR_INVALID_ARG,
                "omb_apply_M_noalloc: the first call in a CUDA context does a blocking set-up; make one call "
                "outside any stream capture first");
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
  D.scratch = static_cast<unsigned char*>(p);
  e = cudaGetSymbolAddress(&p, g_noalloc_tw);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc twiddles)");
  D.tw = static_cast<float2*>(p);
  static float2 host_tw[NOALLOC_TW_TOTAL];  // fixed host table, no heap use
  const double two_pi = 6.283185307179586476925286766559;
  auto w_of = [&](int m, int L) {
    m %= L;
    double c = std::cos(-two_pi * (double)m / (double)L), s = std::sin(-two_pi * (double)m / (double)L);
    if (m == 0) { c = 1; s = 0; }
    if (4 * m == L) { c = 0; s = -1; }
    if (2 * m == L) { c = -1; s = 0; }
    if (4 * m == 3 * L) { c = 0; s = 1; }
    return make_float2((float)c, (float)s);
  };
  int off = 0;
  auto fill = [&](int L) {
    D.tw_off[L] = off;
    for (int m = 0; m < L; ++m) host_tw[off + m] = w_of(m, L);
    const int A = plan2_a(L), B = A ? L / A : 0;
    for (int k1 = 0; k1 < A; ++k1)
      for (int n2 = 0; n2 < B; ++n2) {
        host_tw[off + L + k1 * B + n2] = w_of(n2 * k1, L);
        host_tw[off + 2 * L + n2 * A + k1] = w_of(n2 * k1, L);
      }
    off += 3 * L;
  };
#define OMB_FILL(n) fill(n);
  OMB_NOALLOC_LENS(OMB_FILL)
#undef OMB_FILL
  e = cudaMemcpyToSymbol(g_noalloc_tw, host_tw, sizeof(host_tw));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyToSymbol(noalloc twiddles)");
  D.ctx_id = id;
  return OMB_OK;
}

// Writes the parameter block from kernel arguments, so no host memory is read later.
__global__ void k_noalloc_params(OpUnit<float> u, double k, OpUnit<float>* ud, double* kd) {
  *kd = k;
  *ud = u;
}

template <typename K> static cudaError_t noalloc_launch(K kern, dim3 g, int nt, size_t smem, cudaStream_t st,
                                                         const OpUnit<float>* u, const float2* tw) {
  if (smem > 32 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<g, nt, smem, st>>>(u, tw);
  return cudaGetLastError();
}

template <int NX> static cudaError_t noalloc_rows(bool in, int Ny, int ncol, const OpUnit<float>* u,
                                                  const float2* tw, cudaStream_t st) {
  if constexpr (plan2_a(NX) != 0) {  // two-level register FFT
    constexpr int G = l2_rows(NX), NT = l2_row_threads(NX);
    const size_t sm = (size_t)3 * G * l2_row_lstr<float2, NX>() * sizeof(float2);
    const dim3 g((Ny + G - 1) / G, ncol, 1);
    return in ? noalloc_launch(k_row_in2<float, NX, RI_KXTC, false>, g, NT, sm, st, u, tw)
              : noalloc_launch(k_row_out2<float, NX, RO_KXCT, true>, g, NT, sm, st, u, tw);
  } else {
    constexpr int ROWS = rows_for(NX);
    const size_t sm = (NX + 3 * ROWS * (NX + 1)) * sizeof(float2);
    const dim3 g((Ny + ROWS - 1) / ROWS, ncol, 1);
    return in ? noalloc_launch(k_row_in<float, NX, ROWS, NT_ROW, RI_KXTC, false>, g, NT_ROW, sm, st, u, tw)
              : noalloc_launch(k_row_out<float, NX, ROWS, NT_ROW, RO_KXCT, true>, g, NT_ROW, sm, st, u, tw);
  }
}
template <int NY> static cudaError_t noalloc_col(int Nx, int ncol, const OpUnit<float>* u, const float2* tw,
                                                 cudaStream_t st) {
  if constexpr (plan2_a(NY) != 0) {  // two-level register FFT
    constexpr int TX = l2_tx<float>(NY), NT = l2_col_threads<float>(NY);
    const size_t sm = (size_t)3 * TX * l2_col_lstr<float2, NY, TX>() * sizeof(float2);
    const dim3 g((Nx + TX - 1) / TX, ncol, 1);
    return noalloc_launch(k_col2<float, NY, CS_FWD, PW_EPS9, CS_INV>, g, NT, sm, st, u, tw);
  } else {
    constexpr int TX = tx_for<float>(NY);
    const size_t sm = (NY + 3 * TX * (NY + 1)) * sizeof(float2);
    const dim3 g((Nx + TX - 1) / TX, ncol, 1);
    return noalloc_launch(k_col<float, NY, TX, NT_COL, CS_FWD, PW_EPS9, CS_INV>, g, NT_COL, sm, st, u, tw);
  }
}

}  // namespace omb

using namespace omb;

extern "C" int omb_apply_M_noalloc(int32_t Nx, int32_t Ny, double Dx, double Dy, double k, const float* d_epsinv,
                                   int32_t ncol, const void* d_H_in, void* d_H_out, void* stream) {
  omb_grid g{Nx, Ny, Dx, Dy};
  int rc = check_grid(&g);
  if (rc) return rc;
  if (!(k > 0) || !std::isfinite(k)) return fail(OMB_ERR_INVALID_ARG, "k must be finite and positive");
  if (ncol <= 0 || !d_epsinv || !d_H_in || !d_H_out)
    return fail(OMB_ERR_INVALID_ARG, "need ncol > 0 and non-NULL device pointers");
  if ((long long)Nx * Ny * ncol > NOALLOC_MAX_PIXEL_COLUMNS)
    return fail(OMB_ERR_INVALID_ARG, "omb_apply_M_noalloc: Nx*Ny*ncol = " + std::to_string((long long)Nx * Ny * ncol) +
                                         " exceeds its fixed scratch of " + std::to_string(NOALLOC_MAX_PIXEL_COLUMNS) +
                                         " pixel-columns (use omb_apply for larger blocks)");
  int dev = 0;
  OMB_CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(OMB_ERR_UNSUPPORTED, "device index above 63");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  rc = noalloc_setup(dev, st);
  if (rc) return rc;
  const NoallocDevice& D = g_noalloc_dev[dev];
  const size_t N = (size_t)Nx * Ny;
  // parameter block: k at offset 0, the pass descriptor at offset 64
  double* kd = reinterpret_cast<double*>(D.scratch);
  OpUnit<float>* ud = reinterpret_cast<OpUnit<float>*>(D.scratch + 64);
  OpUnit<float> u{};
  u.in = static_cast<const float2*>(d_H_in);
  u.out = static_cast<float2*>(d_H_out);
  u.scr = reinterpret_cast<float2*>(D.scratch + NOALLOC_PARAM_BYTES);
  u.e9 = d_epsinv;
  u.k_dev = kd;
  u.in_cs = u.out_cs = (long long)(2 * N);
  u.scr_cs = (long long)(3 * N);
  u.Nx = Nx; u.Ny = Ny; u.ncol = ncol;
  u.part_stride = row_blocks(Nx, Ny);
  u.inv_dx = (float)(1.0 / Dx); u.inv_dy = (float)(1.0 / Dy);
  static_assert(sizeof(OpUnit<float>) + 64 <= NOALLOC_PARAM_BYTES, "parameter block too small");
  k_noalloc_params<<<1, 1, 0, st>>>(u, k, ud, kd);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "omb_apply_M_noalloc parameter block");
  switch (Nx) {
#define OMB_CASE(n) case n: e = noalloc_rows<n>(true, Ny, ncol, ud, D.tw + D.tw_off[n], st); break;
    OMB_NOALLOC_LENS(OMB_CASE)
#undef OMB_CASE
  }
  if (e != cudaSuccess) return cuda_fail(e, "omb_apply_M_noalloc row pass");
  switch (Ny) {
#define OMB_CASE(n) case n: e = noalloc_col<n>(Nx, ncol, ud, D.tw + D.tw_off[n], st); break;
    OMB_NOALLOC_LENS(OMB_CASE)
#undef OMB_CASE
  }
  if (e != cudaSuccess) return cuda_fail(e, "omb_apply_M_noalloc column pass");
  switch (Nx) {
#define OMB_CASE(n) case n: e = noalloc_rows<n>(false, Ny, ncol, ud, D.tw + D.tw_off[n], st); break;
    OMB_NOALLOC_LENS(OMB_CASE)
#undef OMB_CASE
  }
  if (e != cudaSuccess) return cuda_fail(e, "omb_apply_M_noalloc row pass");
  return OMB_OK;
}
