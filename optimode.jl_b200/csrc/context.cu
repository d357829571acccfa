// Context lifetime, error reporting, twiddle tables and ε⁻¹ upload.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "context.h"
#include "ops_impl.cuh"

namespace omb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_last_error = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  return OMB_ERR_CUDA;
}

bool fft_size_supported(int L) {
  switch (L) {
#define OMB_CASE(n) case n:
    OMB_FFT_SIZES(OMB_CASE)
#undef OMB_CASE
    return true;
    default: return false;
  }
}

cudaError_t ensure_smem(const void* func, size_t bytes, bool max_shared) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  size_t& have = done[{func, dev}];
  if (have >= bytes && have > 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess && max_shared)
    e = cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess) have = bytes > 0 ? bytes : 1;
  return e;
}

int cluster_slots(const void* func, int cluster_ctas, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = done.find({func, dev});
  if (it != done.end()) return it->second;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster_ctas * (sms / cluster_ctas > 0 ? sms / cluster_ctas : 1), 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cluster_ctas;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, func, &cfg) != cudaSuccess || n < 1) {
    cudaGetLastError();  // a failed query leaves no sticky error; fall back to one per SM group
    n = sms / cluster_ctas > 0 ? sms / cluster_ctas : 1;
  }
  return done[{func, dev}] = n;
}

bool cluster_apply_available(int Nx, int Ny) { return Nx == 256 && Ny == 256; }

namespace {
struct BigBlock {
  void* p = nullptr;
  size_t bytes = 0;
  bool busy = false;
  cudaStream_t last = nullptr;
  cudaEvent_t done = nullptr;  // recorded on `last` when the block was returned
};
std::mutex g_big_mu;
std::map<int, std::vector<BigBlock>> g_big;  // per device
}  // namespace

cudaError_t big_alloc(void** p, size_t bytes, cudaStream_t st) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  bytes = (bytes + ((size_t)2 << 20) - 1) & ~(((size_t)2 << 20) - 1);  // 2 MiB granules
  std::lock_guard<std::mutex> lk(g_big_mu);
  std::vector<BigBlock>& v = g_big[dev];
  BigBlock* best = nullptr;
  for (BigBlock& b : v)
    if (!b.busy && b.bytes >= bytes && (!best || b.bytes < best->bytes)) best = &b;
  if (best) {
    if (best->last != st && best->done) {
      e = cudaStreamWaitEvent(st, best->done, 0);
      if (e != cudaSuccess) return e;
    }
    best->busy = true;
    best->last = st;
    *p = best->p;
    return cudaSuccess;
  }
  BigBlock b;
  e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    // release the idle cached blocks and try once more
    cudaDeviceSynchronize();
    for (auto it = v.begin(); it != v.end();) {
      if (!it->busy) {
        cudaFree(it->p);
        if (it->done) cudaEventDestroy(it->done);
        it = v.erase(it);
      } else {
        ++it;
      }
    }
    cudaGetLastError();
    e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) return e;
  }
  e = cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming);
  if (e != cudaSuccess) { cudaFree(b.p); return e; }
  b.bytes = bytes;
  b.busy = true;
  b.last = st;
  v.push_back(b);
  *p = b.p;
  return cudaSuccess;
}

void big_free(void* p, cudaStream_t st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  std::lock_guard<std::mutex> lk(g_big_mu);
  for (BigBlock& b : g_big[dev])
    if (b.p == p) {
      b.busy = false;
      b.last = st;
      cudaEventRecord(b.done, st);
      return;
    }
}

int row_blocks(int Nx, int Ny) {
  const int rows = plan2_a(Nx) ? l2_rows(Nx) : rows_for(Nx);
  return (Ny + rows - 1) / rows;
}

int check_grid(const omb_grid* g) {
  if (!g) return fail(OMB_ERR_INVALID_ARG, "grid is NULL");
  if (!fft_size_supported(g->Nx) || !fft_size_supported(g->Ny))
    return fail(OMB_ERR_UNSUPPORTED, "unsupported grid size " + std::to_string(g->Nx) + "x" +
                                         std::to_string(g->Ny) + " (see omb_fft_size_supported)");
  if (!(g->Dx > 0) || !(g->Dy > 0) || !std::isfinite(g->Dx) || !std::isfinite(g->Dy))
    return fail(OMB_ERR_INVALID_ARG, "cell sizes Dx, Dy must be finite and positive");
  return OMB_OK;
}

namespace {

constexpr size_t STAGE_CAP = (size_t)512 << 20;  // page-locked staging kept per context
inline size_t padded(size_t b) { return (b + 255) & ~(size_t)255; }

// One batch of pieces that fits the staging buffer: queue the copies, synchronise once,
// then copy out with a few host threads, each over a contiguous share of the bytes.
int gather_batch(omb_ctx* ctx, const D2HPiece* pieces, size_t n) {
  char* stage = static_cast<char*>(ctx->pinned);
  std::vector<size_t> off(n);
  size_t total = 0;
  for (size_t i = 0; i < n; ++i) {
    off[i] = total;
    if (pieces[i].bytes)
      OMB_CU(cudaMemcpyAsync(stage + total, pieces[i].src, pieces[i].bytes, cudaMemcpyDeviceToHost, ctx->stream));
    total += padded(pieces[i].bytes);
  }
  OMB_CU(cudaStreamSynchronize(ctx->stream));
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nth = (int)std::min<size_t>(std::min(8u, hw), std::max<size_t>(1, total >> 23));
  auto work = [&](int id) {
    const size_t lo = total * id / nth, hi = total * (id + 1) / nth;
    for (size_t i = 0; i < n; ++i) {
      const size_t a = std::max(lo, off[i]), b = std::min(hi, off[i] + pieces[i].bytes);
      if (a < b) std::memcpy(static_cast<char*>(pieces[i].dst) + (a - off[i]), stage + a, b - a);
    }
  };
  if (nth == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (int id = 1; id < nth; ++id) th.emplace_back(work, id);
    work(0);
    for (auto& t : th) t.join();
  }
  return OMB_OK;
}

}  // namespace

int gather_to_host(omb_ctx* ctx, const D2HPiece* pieces, size_t n) {
  size_t total = 0, largest = 0;
  for (size_t i = 0; i < n; ++i) {
    total += padded(pieces[i].bytes);
    largest = std::max(largest, padded(pieces[i].bytes));
  }
  if (total == 0) return OMB_OK;
  const size_t want = std::max(std::min(total, STAGE_CAP), largest);
  if (want > ctx->pinned_bytes) {
    OMB_CU(cudaStreamSynchronize(ctx->stream));
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
    if (cudaHostAlloc(&ctx->pinned, want, cudaHostAllocDefault) != cudaSuccess) {
      // no page-locked memory to be had: plain copies into the caller's buffers
      ctx->pinned = nullptr;
      cudaGetLastError();
      for (size_t i = 0; i < n; ++i)
        if (pieces[i].bytes)
          OMB_CU(cudaMemcpyAsync(pieces[i].dst, pieces[i].src, pieces[i].bytes, cudaMemcpyDeviceToHost, ctx->stream));
      OMB_CU(cudaStreamSynchronize(ctx->stream));
      return OMB_OK;
    }
    ctx->pinned_bytes = want;
  }
  // batches of pieces that fit the staging buffer
  size_t first = 0, bytes = 0;
  for (size_t i = 0; i <= n; ++i) {
    if (i == n || bytes + padded(pieces[i].bytes) > ctx->pinned_bytes) {
      if (i > first) {
        const int rc = gather_batch(ctx, pieces + first, i - first);
        if (rc) return rc;
      }
      first = i;
      bytes = 0;
    }
    if (i < n) bytes += padded(pieces[i].bytes);
  }
  return OMB_OK;
}

// ---- ε⁻¹ upload: validation and the per-precision layouts on the device ----------------
// The caller's (3, 3, Nx, Ny[, Nz]) FP64 array is copied once; one kernel finds the largest
// |entry| and the first non-finite one, a second checks symmetry (relative to that largest
// entry) and the trace pixel by pixel, writes the FP32 (float4 + float2) and FP64 (3 double2)
// unique entries and ε_ave = 3/tr, and reduces min diag, max trace and per-block sums of ε_ave
// (summed on the host in block order, so the mean does not depend on scheduling).
namespace {
constexpr int EPS_NT = 256;
constexpr unsigned long long NONE = ~0ull;
struct EpsStats {
  unsigned long long emax;      // bits of max |entry| (non-negative doubles order like their bits)
  unsigned long long bad_nan;   // first non-finite entry
  unsigned long long bad_asym;  // first pixel whose off-diagonal pairs differ by > 1e-9·max|entry|
  unsigned long long bad_trace; // first pixel with trace ≤ 0
  unsigned long long bad_diag;  // first pixel with a diagonal entry ≤ 0
  unsigned long long mind;      // bits of the least (positive) diagonal entry
  unsigned long long maxtr;     // bits of the largest (positive) trace
};

// Block-wide minimum (every thread calls it; the result is valid in thread 0).
__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long v, unsigned long long* sh) {
  for (int o = 16; o > 0; o >>= 1) { const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o); v = w < v ? w : v; }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < EPS_NT / 32 ? sh[threadIdx.x] : NONE;
    for (int o = 16; o > 0; o >>= 1) { const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o); v = w < v ? w : v; }
  }
  __syncthreads();
  return v;
}
__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long v, unsigned long long* sh) {
  return ~block_min_u64(~v, sh);
}

__global__ void __launch_bounds__(EPS_NT) k_eps_scan(const double* __restrict__ raw, size_t n, EpsStats* st) {
  __shared__ unsigned long long sh[EPS_NT / 32];
  unsigned long long mx = 0, bad = NONE;
  for (size_t i = (size_t)blockIdx.x * EPS_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * EPS_NT) {
    const double v = raw[i];
    if (!isfinite(v)) bad = i < bad ? i : bad;
    else { const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(v)); mx = b > mx ? b : mx; }
  }
  mx = block_max_u64(mx, sh);
  bad = block_min_u64(bad, sh);
  if (threadIdx.x == 0) {
    atomicMax(&st->emax, mx);
    if (bad != NONE) atomicMin(&st->bad_nan, bad);
  }
}

__global__ void __launch_bounds__(EPS_NT) k_eps_convert(const double* __restrict__ raw, size_t N, EpsStats* st,
                                                        float4* __restrict__ a32, float2* __restrict__ b32,
                                                        double2* __restrict__ e64, float* __restrict__ ea32,
                                                        double* __restrict__ ea64, double* __restrict__ part) {
  __shared__ unsigned long long sh[EPS_NT / 32];
  __shared__ double ssum[EPS_NT];
  const double emax = __longlong_as_double((long long)st->emax);
  const size_t p = (size_t)blockIdx.x * EPS_NT + threadIdx.x;
  unsigned long long basym = NONE, btr = NONE, bdiag = NONE, mind = NONE, maxtr = 0;
  double eave = 0;
  if (p < N) {
    const double* m = raw + 9 * p;  // column-major 3x3: m[a + 3b] = ε⁻¹[a,b]
    const double xx = m[0], yy = m[4], zz = m[8];
    const double xy = 0.5 * (m[1] + m[3]), xz = 0.5 * (m[2] + m[6]), yz = 0.5 * (m[5] + m[7]);
    const double asym = fmax(fabs(m[1] - m[3]), fmax(fabs(m[2] - m[6]), fabs(m[5] - m[7])));
    if (asym > 1e-9 * emax) basym = p;
    const double tr = xx + yy + zz;
    if (!(tr > 0)) btr = p;
    const double dmin = fmin(xx, fmin(yy, zz));
    if (!(dmin > 0)) bdiag = p;
    else mind = (unsigned long long)__double_as_longlong(dmin);
    if (tr > 0) maxtr = (unsigned long long)__double_as_longlong(tr);
    a32[p] = make_float4((float)xx, (float)yy, (float)zz, (float)xy);
    b32[p] = make_float2((float)xz, (float)yz);
    e64[3 * p] = make_double2(xx, yy);
    e64[3 * p + 1] = make_double2(zz, xy);
    e64[3 * p + 2] = make_double2(xz, yz);
    eave = 3.0 / tr;
    ea64[p] = eave;
    ea32[p] = (float)eave;
  }
  // per-block sum of ε_ave in a fixed order (pairwise tree)
  ssum[threadIdx.x] = eave;
  __syncthreads();
  for (int s = EPS_NT / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) ssum[threadIdx.x] += ssum[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = ssum[0];
  basym = block_min_u64(basym, sh);
  btr = block_min_u64(btr, sh);
  bdiag = block_min_u64(bdiag, sh);
  mind = block_min_u64(mind, sh);
  maxtr = block_max_u64(maxtr, sh);
  if (threadIdx.x == 0) {
    if (basym != NONE) atomicMin(&st->bad_asym, basym);
    if (btr != NONE) atomicMin(&st->bad_trace, btr);
    if (bdiag != NONE) atomicMin(&st->bad_diag, bdiag);
    if (mind != NONE) atomicMin(&st->mind, mind);
    atomicMax(&st->maxtr, maxtr);
  }
}
}  // namespace

int upload_problem(omb_ctx* ctx, const omb_grid* g, const double* epsinv, Problem& P, int Nz, double Dz) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!epsinv) return fail(OMB_ERR_INVALID_ARG, "epsinv is NULL");
  if (Nz > 1) {
    if (!fft_size_supported(Nz)) return fail(OMB_ERR_UNSUPPORTED, "unsupported Nz " + std::to_string(Nz));
    if (!(Dz > 0) || !std::isfinite(Dz)) return fail(OMB_ERR_INVALID_ARG, "the period Dz must be finite and positive");
    if ((long long)Nz * row_blocks(g->Nx, g->Ny) > 512)
      return fail(OMB_ERR_UNSUPPORTED, "Nz x row blocks of a slab above 512 (use fewer z slabs or rows)");
  } else if (Nz != 1) {
    return fail(OMB_ERR_INVALID_ARG, "Nz must be >= 1");
  }
  P.Nx = g->Nx; P.Ny = g->Ny; P.Dx = g->Dx; P.Dy = g->Dy;
  P.Nz = Nz; P.Dz = Nz > 1 ? Dz : 0;
  const size_t N = P.N();
  cudaStream_t st = ctx->stream;
  const unsigned nb = (unsigned)((N + EPS_NT - 1) / EPS_NT);
  DevBuf<double> raw, part;
  DevBuf<EpsStats> dst;
  OMB_CU(raw.alloc(9 * N, st));
  OMB_CU(part.alloc(nb, st));
  OMB_CU(dst.alloc(1, st));
  OMB_CU(P.e32a.alloc(N, st));
  OMB_CU(P.e32b.alloc(N, st));
  OMB_CU(P.e64.alloc(3 * N, st));
  OMB_CU(P.eave32.alloc(N, st));
  OMB_CU(P.eave64.alloc(N, st));
  const EpsStats init{0, NONE, NONE, NONE, NONE, NONE, 0};
  OMB_CU(cudaMemcpyAsync(dst.p, &init, sizeof(EpsStats), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaMemcpyAsync(raw.p, epsinv, 9 * N * sizeof(double), cudaMemcpyHostToDevice, st));
  const unsigned nscan = std::min<unsigned>(4 * (unsigned)std::max(ctx->num_sms, 1),
                                            (unsigned)((9 * N + EPS_NT - 1) / EPS_NT));
  k_eps_scan<<<nscan, EPS_NT, 0, st>>>(raw.p, 9 * N, dst.p);
  OMB_CU(cudaGetLastError());
  k_eps_convert<<<nb, EPS_NT, 0, st>>>(raw.p, N, dst.p, P.e32a.p, P.e32b.p, P.e64.p, P.eave32.p, P.eave64.p, part.p);
  OMB_CU(cudaGetLastError());
  EpsStats hs;
  std::vector<double> hp(nb);
  OMB_CU(cudaMemcpyAsync(&hs, dst.p, sizeof(EpsStats), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaMemcpyAsync(hp.data(), part.p, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaStreamSynchronize(st));
  if (hs.bad_nan != NONE) return fail(OMB_ERR_NAN, "epsinv holds a non-finite value");
  if (hs.bad_asym != NONE && hs.bad_asym <= hs.bad_trace)
    return fail(OMB_ERR_INVALID_ARG, "epsinv is not symmetric at pixel " + std::to_string(hs.bad_asym) +
                                         " (the Helmholtz operator needs a real symmetric ε⁻¹)");
  if (hs.bad_trace != NONE)
    return fail(OMB_ERR_INVALID_ARG, "epsinv has a non-positive trace at pixel " + std::to_string(hs.bad_trace));
  if (hs.bad_diag != NONE) return fail(OMB_ERR_INVALID_ARG, "epsinv has a non-positive diagonal entry");
  double mean = 0;
  for (unsigned b = 0; b < nb; ++b) mean += hp[b];
  P.eps_mean = mean / (double)N;
  double v;
  std::memcpy(&v, &hs.mind, sizeof v);
  P.min_diag = v;
  std::memcpy(&v, &hs.maxtr, sizeof v);
  P.max_trace = v;
  return OMB_OK;
}

template <> OpUnit<float> make_unit<float>(const Problem& P) {
  OpUnit<float> u{};
  u.e32a = P.e32a.p; u.e32b = P.e32b.p; u.e64 = P.e64.p; u.eave = P.eave32.p;
  u.Nx = P.Nx; u.Ny = P.Ny;
  u.inv_dx = (float)(1.0 / P.Dx); u.inv_dy = (float)(1.0 / P.Dy);
  u.part_stride = row_blocks(P.Nx, P.Ny) * P.Nz;
  u.inv_dz = P.Nz > 1 ? 1.0 / P.Dz : 0.0;
  return u;
}
template <> OpUnit<double> make_unit<double>(const Problem& P) {
  OpUnit<double> u{};
  u.e32a = P.e32a.p; u.e32b = P.e32b.p; u.e64 = P.e64.p; u.eave = P.eave64.p;
  u.Nx = P.Nx; u.Ny = P.Ny;
  u.inv_dx = 1.0 / P.Dx; u.inv_dy = 1.0 / P.Dy;
  u.part_stride = row_blocks(P.Nx, P.Ny) * P.Nz;
  u.inv_dz = P.Nz > 1 ? 1.0 / P.Dz : 0.0;
  return u;
}

static int make_twiddles(omb_ctx* ctx) {
  // one table per supported length, exp(-2πi m/L) for m < L, FP64 and FP32 copies
  std::vector<int> lens;
#define OMB_CASE(n) lens.push_back(n);
  OMB_FFT_SIZES(OMB_CASE)
#undef OMB_CASE
  // per length L: [exp(-2πi m/L), m < L | TW1 | TW3], the last two for the two-level plan
  // L = A·B: TW1[k1·B + n2] = W^{n2·k1}, TW3[m2·A + k1] = W^{m2·k1}
  size_t tot = 0;
  for (int L : lens) tot += 3 * (size_t)L;
  std::vector<double2> h64(tot);
  std::vector<float2> h32(tot);
  size_t off = 0;
  const double two_pi = 6.283185307179586476925286766559;
  auto w_of = [&](int m, int L) {
    m %= L;
    double c = std::cos(-two_pi * (double)m / (double)L), s = std::sin(-two_pi * (double)m / (double)L);
    if (m == 0) { c = 1; s = 0; }
    if (4 * m == L) { c = 0; s = -1; }
    if (2 * m == L) { c = -1; s = 0; }
    if (4 * m == 3 * L) { c = 0; s = 1; }
    return make_double2(c, s);
  };
  for (int L : lens) {
    for (int m = 0; m < L; ++m) h64[off + m] = w_of(m, L);
    const int A = plan2_a(L), B = A ? L / A : 0;
    for (int k1 = 0; k1 < A; ++k1)
      for (int n2 = 0; n2 < B; ++n2) {
        h64[off + L + k1 * B + n2] = w_of(n2 * k1, L);
        h64[off + 2 * L + n2 * A + k1] = w_of(n2 * k1, L);
      }
    for (int m = 0; m < 3 * L; ++m) h32[off + m] = make_float2((float)h64[off + m].x, (float)h64[off + m].y);
    off += 3 * (size_t)L;
  }
  void* mem = nullptr;
  OMB_CU(cudaMalloc(&mem, tot * (sizeof(double2) + sizeof(float2))));
  double2* d64 = reinterpret_cast<double2*>(mem);
  float2* d32 = reinterpret_cast<float2*>(d64 + tot);
  OMB_CU(cudaMemcpy(d64, h64.data(), tot * sizeof(double2), cudaMemcpyHostToDevice));
  OMB_CU(cudaMemcpy(d32, h32.data(), tot * sizeof(float2), cudaMemcpyHostToDevice));
  off = 0;
  for (int L : lens) {
    ctx->tw.f64[L] = d64 + off;
    ctx->tw.f32[L] = d32 + off;
    off += 3 * (size_t)L;
  }
  ctx->tw_mem = mem;
  return OMB_OK;
}

}  // namespace omb

using namespace omb;

extern "C" {

int omb_version(void) { return 100; }

int omb_fft_size_supported(int n) { return fft_size_supported(n) ? 1 : 0; }

const char* omb_last_error(void) { return g_last_error.c_str(); }

int omb_ctx_create(int device, omb_ctx** out) {
  if (!out) return fail(OMB_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  OMB_CU(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev)
    return fail(OMB_ERR_INVALID_ARG, "device " + std::to_string(device) + " out of range (found " +
                                         std::to_string(ndev) + ")");
  OMB_CU(cudaSetDevice(device));
  omb_ctx* c = new omb_ctx();
  c->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return cuda_fail(e, "cudaStreamCreate"); }
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  // keep freed blocks in the device pool between calls
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  int rc = make_twiddles(c);
  if (rc) { cudaStreamDestroy(c->stream); delete c; return rc; }
  *out = c;
  return OMB_OK;
}

int omb_ctx_destroy(omb_ctx* ctx) {
  if (!ctx) return OMB_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ws_release_all(ctx);
  if (ctx->tw_mem) cudaFree(ctx->tw_mem);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return OMB_OK;
}

}  // extern "C"
