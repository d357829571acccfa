// Allocation-free FP32 operator apply (omb_apply_M_noalloc).
//
// Some callers cannot allocate device memory at the moment they need the operator: code
// running inside a CUDA stream capture (allocation calls are not capturable), host
// frameworks that own the whole device pool and forbid foreign cudaMalloc/cudaFree, or
// callers that must not add allocation latency to a hot loop.  This entry point takes
// every input and output as caller-owned device memory and allocates nothing itself:
// the intermediate 3-component field of the three FFT passes lives in a file-scope
// static device array of fixed size, and so do the small per-call parameter block and
// the twiddle tables.
//
// Limits and rules:
//  * Nx·Ny·ncol ≤ OMB_NOALLOC_MAX_PIXEL_COLUMNS (262144: e.g. 256×256 with 4 columns or
//    512×512 with 1); larger requests are rejected with OMB_ERR_INVALID_ARG.
//  * The array (6 MiB + 256 B) is held by every GPU that loads the library until exit.
//  * All calls share it, so calls that overlap on the GPU (different streams, or
//    different host threads) race; serialise them on one stream.
//  * The first call on a device does a one-time set-up (it resolves the array's device
//    address with cudaGetSymbolAddress and uploads the twiddle tables with a blocking
//    copy); make that first call before any stream capture.
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
#define OMB_LEN_SUM(n) +n
constexpr int NOALLOC_TW_TOTAL = 0 OMB_NOALLOC_LENS(OMB_LEN_SUM);
#undef OMB_LEN_SUM
static __device__ __align__(16) float2 g_noalloc_tw[NOALLOC_TW_TOTAL];

struct NoallocDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  float2* tw = nullptr;              // device address of g_noalloc_tw
  int tw_off[513] = {};
};
static NoallocDevice g_noalloc_dev[64];
static std::mutex g_noalloc_mu;

static int noalloc_setup(int dev) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoallocDevice& D = g_noalloc_dev[dev];
  if (D.ready) return OMB_OK;
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
  D.scratch = static_cast<unsigned char*>(p);
  e = cudaGetSymbolAddress(&p, g_noalloc_tw);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc twiddles)");
  D.tw = static_cast<float2*>(p);
  static float2 host_tw[NOALLOC_TW_TOTAL];  // fixed host table, no heap use
  const double two_pi = 6.283185307179586476925286766559;
  int off = 0;
#define OMB_FILL(n)                                                      \
  D.tw_off[n] = off;                                                     \
  for (int m = 0; m < n; ++m) {                                          \
    double c = std::cos(-two_pi * m / n), s = std::sin(-two_pi * m / n); \
    if (4 * m == n) { c = 0; s = -1; }                                   \
    if (2 * m == n) { c = -1; s = 0; }                                   \
    if (4 * m == 3 * n) { c = 0; s = 1; }                                \
    host_tw[off + m] = make_float2((float)c, (float)s);                  \
  }                                                                      \
  off += n;
  OMB_NOALLOC_LENS(OMB_FILL)
#undef OMB_FILL
  e = cudaMemcpyToSymbol(g_noalloc_tw, host_tw, sizeof(host_tw));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyToSymbol(noalloc twiddles)");
  D.ready = true;
  return OMB_OK;
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
  constexpr int ROWS = rows_for(NX);
  const size_t sm = (NX + 3 * ROWS * (NX + 1)) * sizeof(float2);
  const dim3 g((Ny + ROWS - 1) / ROWS, ncol, 1);
  return in ? noalloc_launch(k_row_in<float, NX, ROWS, NT_ROW, RI_KXTC, false>, g, NT_ROW, sm, st, u, tw)
            : noalloc_launch(k_row_out<float, NX, ROWS, NT_ROW, RO_KXCT, true>, g, NT_ROW, sm, st, u, tw);
}
template <int NY> static cudaError_t noalloc_col(int Nx, int ncol, const OpUnit<float>* u, const float2* tw,
                                                 cudaStream_t st) {
  constexpr int TX = tx_for<float>(NY);
  const size_t sm = (NY + 3 * TX * (NY + 1)) * sizeof(float2);
  const dim3 g((Nx + TX - 1) / TX, ncol, 1);
  return noalloc_launch(k_col<float, NY, TX, NT_COL, CS_FWD, PW_EPS9, CS_INV>, g, NT_COL, sm, st, u, tw);
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
  rc = noalloc_setup(dev);
  if (rc) return rc;
  const NoallocDevice& D = g_noalloc_dev[dev];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t N = (size_t)Nx * Ny;
  // parameter block: k at offset 0, the pass descriptor at offset 64 (both rewritten by
  // every call before the kernels read them; the field needs no clearing because the
  // first pass writes every element the later passes read)
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
  OMB_CU(cudaMemcpyAsync(kd, &k, sizeof(double), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaMemcpyAsync(ud, &u, sizeof(u), cudaMemcpyHostToDevice, st));
  cudaError_t e = cudaSuccess;
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
