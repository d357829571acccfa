// Size/mode dispatch for the fused operator passes.  Included once per precision.
#pragma once

#include <algorithm>
#include <mutex>

#include "op_cluster.cuh"
#include "op_kernels_2l.cuh"
#include "op_kernels_split.cuh"
#include "ops.h"

namespace omb {

#define OMB_FFT_SIZES(X) X(8) X(12) X(16) X(20) X(24) X(32) X(40) X(48) X(64) X(80) X(96) \
  X(128) X(160) X(192) X(256) X(320) X(384) X(512)

// Launch shape policy.  Row passes: NT_ROW threads, ROWS grid rows per CTA (≈512 pixels).
// Column pass: NT_COL threads, TX adjacent columns per CTA (8 for coalesced row segments,
// 4 for FP64 above 256 points to stay inside the shared-memory budget).
constexpr int NT_ROW = 128;
constexpr int NT_COL = 256;
__host__ __device__ constexpr int rows_for(int NX) { return NX >= 512 ? 1 : 512 / NX; }
template <typename T> __host__ __device__ constexpr int tx_for(int NY) {
  return (NY <= 256) ? 8 : (sizeof(T) == 4 ? 8 : 4);
}

template <typename T>
using PassKernel = void (*)(const OpUnit<T>*, const cplx<T>*);

template <typename T>
static cudaError_t launch_pass(PassKernel<T> kern, dim3 g, int nt, size_t smem, cudaStream_t st,
                               const OpUnit<T>* units, const cplx<T>* tw, bool max_shared = false) {
  if (smem > 32 * 1024 || max_shared) {  // the default limit counts static shared memory too
    cudaError_t e = ensure_smem(reinterpret_cast<const void*>(kern), smem, max_shared);
    if (e != cudaSuccess) return e;
  }
  kern<<<g, nt, smem, st>>>(units, tw);
  return cudaGetLastError();
}

// Tunable tiles (FP32, the eigensolver's M̂ passes): row passes with G/2, G or 2G rows per CTA,
// the column pass with TX/2, TX or 2·TX columns (variant 0, 1, 2; 1 is the default); row
// variant 3 runs row_in in the component-parallel form (op_kernels_split.cuh) and row_out in the
// default one, row variant 4 both passes in the component-parallel form; column variants 3 and
// 4 are the component-parallel column pass with a register budget for three or two CTAs per
// SM, and column variant 5 the default tile with a budget for four (and the whole
// shared-memory carve-out).
template <int NX> __host__ __device__ constexpr int row_g_variant(int v) {
  return v == 0 ? (l2_rows(NX) / 2 > 0 ? l2_rows(NX) / 2 : 1) : (v == 2 ? 2 * l2_rows(NX) : l2_rows(NX));
}
template <int NY> __host__ __device__ constexpr int col_tx_variant(int v) { return v == 0 ? 4 : (v == 2 ? 16 : 8); }

template <typename T, int NX, int G, int MODE, bool INV>
static cudaError_t row_in_g(const OpUnit<T>* u, int nunits, int Ny, int maxcol, const cplx<T>* tw, cudaStream_t st) {
  constexpr int NT = l2_row_threads(NX, G);
  const size_t sm = (size_t)3 * G * l2_row_lstr<cplx<T>, NX>() * sizeof(cplx<T>);
  const dim3 g((Ny + G - 1) / G, maxcol, nunits);
  return launch_pass<T>(k_row_in2<T, NX, MODE, INV, G>, g, NT, sm, st, u, tw);
}
template <typename T, int NX, int G, int MODE, bool INV>
static cudaError_t row_out_g(const OpUnit<T>* u, int nunits, int Ny, int maxcol, const cplx<T>* tw, cudaStream_t st) {
  constexpr int NT = l2_row_threads(NX, G);
  const size_t sm = (size_t)3 * G * l2_row_lstr<cplx<T>, NX>() * sizeof(cplx<T>);
  const dim3 g((Ny + G - 1) / G, maxcol, nunits);
  return launch_pass<T>(k_row_out2<T, NX, MODE, INV, G>, g, NT, sm, st, u, tw);
}
// the default tile with a register budget for four CTAs per SM and the whole shared-memory
// carve-out (four 53 KB blocks)
template <int NY, int S1, int PW, int S2>
static cudaError_t col_b4(const OpUnit<float>* u, int nunits, int Nx, int maxcol, const float2* tw, cudaStream_t st) {
  constexpr int TX = l2_tx<float>(NY), NT = l2_col_threads_tx(NY, TX);
  const size_t sm = (size_t)3 * TX * l2_col_lstr<float2, NY, TX>() * sizeof(float2);
  const dim3 g((Nx + TX - 1) / TX, maxcol, nunits);
  return launch_pass<float>(k_col2<float, NY, S1, PW, S2, TX, 4>, g, NT, sm, st, u, tw, true);
}
template <typename T, int NY, int TX, int S1, int PW, int S2>
static cudaError_t col_tx(const OpUnit<T>* u, int nunits, int Nx, int maxcol, const cplx<T>* tw, cudaStream_t st) {
  constexpr int NT = l2_col_threads_tx(NY, TX);
  const size_t sm = (size_t)3 * TX * l2_col_lstr<cplx<T>, NY, TX>() * sizeof(cplx<T>);
  const dim3 g((Nx + TX - 1) / TX, maxcol, nunits);
  return launch_pass<T>(k_col2<T, NY, S1, PW, S2, TX>, g, NT, sm, st, u, tw);
}

template <int NX, int MODE, bool INV, typename T = float>
static cudaError_t row_in_sp(const OpUnit<T>* u, int nunits, int Ny, int maxcol, const cplx<T>* tw, cudaStream_t st) {
  constexpr int G = l2_rows(NX), NT = sp_row_threads(NX, G);
  const size_t sm = (size_t)3 * G * l2_row_lstr<cplx<T>, NX>() * sizeof(cplx<T>);
  const dim3 g((Ny + G - 1) / G, maxcol, nunits);
  return launch_pass<T>(k_row_in_sp<T, NX, MODE, INV, G>, g, NT, sm, st, u, tw);
}
template <int NX, int MODE, bool INV, typename T = float>
static cudaError_t row_out_sp(const OpUnit<T>* u, int nunits, int Ny, int maxcol, const cplx<T>* tw, cudaStream_t st) {
  constexpr int G = l2_rows(NX), NT = sp_row_threads(NX, G);
  const size_t sm = (size_t)3 * G * l2_row_lstr<cplx<T>, NX>() * sizeof(cplx<T>);
  const dim3 g((Ny + G - 1) / G, maxcol, nunits);
  return launch_pass<T>(k_row_out_sp<T, NX, MODE, INV, G>, g, NT, sm, st, u, tw);
}
// FP64 M̂ row passes in the component-parallel form (one thread per line slot and component)
constexpr bool FP64_ROW_SPLIT = true;
template <int NY, int S1, int PW, int S2, int MINB>
static cudaError_t col_sp(const OpUnit<float>* u, int nunits, int Nx, int maxcol, const float2* tw, cudaStream_t st) {
  constexpr int TX = l2_tx<float>(NY), NT = sp_col_threads(NY, TX);
  const size_t sm = (size_t)3 * TX * l2_col_lstr<float2, NY, TX>() * sizeof(float2);
  const dim3 g((Nx + TX - 1) / TX, maxcol, nunits);
  return launch_pass<float>(k_col_sp<NY, S1, PW, S2, TX, MINB>, g, NT, sm, st, u, tw);
}

template <typename T, int NX>
static cudaError_t row_in_nx(int mode, const OpUnit<T>* u, int nunits, int Ny, int maxcol,
                             const cplx<T>* tw, cudaStream_t st, int gv = 1) {
  if constexpr (plan2_a(NX) != 0 && sizeof(T) == 4) {
    if (mode == RI_KXTC && (gv == 3 || gv == 4))
      return row_in_sp<NX, RI_KXTC, false>(reinterpret_cast<const OpUnit<float>*>(u), nunits, Ny, maxcol,
                                           reinterpret_cast<const float2*>(tw), st);
    if (mode == RI_KXTC && gv != 1)
      return gv == 0 ? row_in_g<T, NX, row_g_variant<NX>(0), RI_KXTC, false>(u, nunits, Ny, maxcol, tw, st)
                     : row_in_g<T, NX, row_g_variant<NX>(2), RI_KXTC, false>(u, nunits, Ny, maxcol, tw, st);
  }
  if constexpr (plan2_a(NX) != 0 && sizeof(T) == 8) {
    if (FP64_ROW_SPLIT && mode == RI_KXTC) return row_in_sp<NX, RI_KXTC, false, T>(u, nunits, Ny, maxcol, tw, st);
  }
  if constexpr (plan2_a(NX) != 0) {  // two-level register FFT
    constexpr int G = l2_rows(NX), NT = l2_row_threads(NX);
    const size_t sm = (size_t)3 * G * l2_row_lstr<cplx<T>, NX>() * sizeof(cplx<T>);
    const dim3 g((Ny + G - 1) / G, maxcol, nunits);
    switch (mode) {
      case RI_KXTC: return launch_pass<T>(k_row_in2<T, NX, RI_KXTC, false>, g, NT, sm, st, u, tw);
      case RI_KXINV: return launch_pass<T>(k_row_in2<T, NX, RI_KXINV, true>, g, NT, sm, st, u, tw);
      case RI_ZXTC: return launch_pass<T>(k_row_in2<T, NX, RI_ZXTC, false>, g, NT, sm, st, u, tw);
      case RI_HCART: return launch_pass<T>(k_row_in2<T, NX, RI_HCART, false>, g, NT, sm, st, u, tw);
      case RI_LOAD3: return launch_pass<T>(k_row_in2<T, NX, RI_LOAD3, true>, g, NT, sm, st, u, tw);
      default: return cudaErrorInvalidValue;
    }
  } else {
    constexpr int ROWS = rows_for(NX);
    const size_t sm = (NX + 3 * ROWS * (NX + 1)) * sizeof(cplx<T>);
    const dim3 g((Ny + ROWS - 1) / ROWS, maxcol, nunits);
    switch (mode) {
      case RI_KXTC: return launch_pass<T>(k_row_in<T, NX, ROWS, NT_ROW, RI_KXTC, false>, g, NT_ROW, sm, st, u, tw);
      case RI_KXINV: return launch_pass<T>(k_row_in<T, NX, ROWS, NT_ROW, RI_KXINV, true>, g, NT_ROW, sm, st, u, tw);
      case RI_ZXTC: return launch_pass<T>(k_row_in<T, NX, ROWS, NT_ROW, RI_ZXTC, false>, g, NT_ROW, sm, st, u, tw);
      case RI_HCART: return launch_pass<T>(k_row_in<T, NX, ROWS, NT_ROW, RI_HCART, false>, g, NT_ROW, sm, st, u, tw);
      case RI_LOAD3: return launch_pass<T>(k_row_in<T, NX, ROWS, NT_ROW, RI_LOAD3, true>, g, NT_ROW, sm, st, u, tw);
      default: return cudaErrorInvalidValue;
    }
  }
}

template <typename T, int NX>
static cudaError_t row_out_nx(int mode, const OpUnit<T>* u, int nunits, int Ny, int maxcol,
                              const cplx<T>* tw, cudaStream_t st, int gv = 1) {
  if constexpr (plan2_a(NX) != 0 && sizeof(T) == 4) {
    // (the dot-product mode keeps the default rows: its partial sums are laid out per row block)
    if (mode == RO_KXCT && gv == 3)
      return row_out_nx<T, NX>(mode, u, nunits, Ny, maxcol, tw, st, 1);
    if (mode == RO_KXCT && gv == 4)
      return row_out_sp<NX, RO_KXCT, true>(reinterpret_cast<const OpUnit<float>*>(u), nunits, Ny, maxcol,
                                           reinterpret_cast<const float2*>(tw), st);
    if (mode == RO_KXCT_DOT && gv == 4)
      return row_out_sp<NX, RO_KXCT_DOT, true>(reinterpret_cast<const OpUnit<float>*>(u), nunits, Ny, maxcol,
                                               reinterpret_cast<const float2*>(tw), st);
    if (mode == RO_KXCT && gv != 1)
      return gv == 0 ? row_out_g<T, NX, row_g_variant<NX>(0), RO_KXCT, true>(u, nunits, Ny, maxcol, tw, st)
                     : row_out_g<T, NX, row_g_variant<NX>(2), RO_KXCT, true>(u, nunits, Ny, maxcol, tw, st);
  }
  if constexpr (plan2_a(NX) != 0 && sizeof(T) == 8) {
    if (FP64_ROW_SPLIT && mode == RO_KXCT) return row_out_sp<NX, RO_KXCT, true, T>(u, nunits, Ny, maxcol, tw, st);
  }
  if constexpr (plan2_a(NX) != 0) {  // two-level register FFT
    constexpr int G = l2_rows(NX), NT = l2_row_threads(NX);
    const size_t sm = (size_t)3 * G * l2_row_lstr<cplx<T>, NX>() * sizeof(cplx<T>);
    const dim3 g((Ny + G - 1) / G, maxcol, nunits);
    switch (mode) {
      case RO_KXCT: return launch_pass<T>(k_row_out2<T, NX, RO_KXCT, true>, g, NT, sm, st, u, tw);
      case RO_KXINVCT: return launch_pass<T>(k_row_out2<T, NX, RO_KXINVCT, false>, g, NT, sm, st, u, tw);
      case RO_STORE3: return launch_pass<T>(k_row_out2<T, NX, RO_STORE3, true>, g, NT, sm, st, u, tw);
      case RO_KXCT_DOT: return launch_pass<T>(k_row_out2<T, NX, RO_KXCT_DOT, true>, g, NT, sm, st, u, tw);
      default: return cudaErrorInvalidValue;
    }
  } else {
    constexpr int ROWS = rows_for(NX);
    const size_t sm = (NX + 3 * ROWS * (NX + 1)) * sizeof(cplx<T>);
    const dim3 g((Ny + ROWS - 1) / ROWS, maxcol, nunits);
    switch (mode) {
      case RO_KXCT: return launch_pass<T>(k_row_out<T, NX, ROWS, NT_ROW, RO_KXCT, true>, g, NT_ROW, sm, st, u, tw);
      case RO_KXINVCT: return launch_pass<T>(k_row_out<T, NX, ROWS, NT_ROW, RO_KXINVCT, false>, g, NT_ROW, sm, st, u, tw);
      case RO_STORE3: return launch_pass<T>(k_row_out<T, NX, ROWS, NT_ROW, RO_STORE3, true>, g, NT_ROW, sm, st, u, tw);
      case RO_KXCT_DOT: return launch_pass<T>(k_row_out<T, NX, ROWS, NT_ROW, RO_KXCT_DOT, true>, g, NT_ROW, sm, st, u, tw);
      default: return cudaErrorInvalidValue;
    }
  }
}

// column-pass modes
enum ColMode : int { CM_M = 0, CM_P = 1, CM_E = 2, CM_FWD = 3, CM_EPSINV = 4, CM_BWD = 5 };

template <typename T, int NY>
static cudaError_t col_ny(int mode, const OpUnit<T>* u, int nunits, int Nx, int maxcol,
                          const cplx<T>* tw, cudaStream_t st, int tv = 1) {
  if constexpr (plan2_a(NY) != 0 && sizeof(T) == 4) {
    if (mode == CM_M && tv == 5)
      return col_b4<NY, CS_FWD, PW_EPS, CS_INV>(reinterpret_cast<const OpUnit<float>*>(u), nunits, Nx, maxcol,
                                                reinterpret_cast<const float2*>(tw), st);
    if (mode == CM_M && (tv == 3 || tv == 4)) {
      const auto* uf = reinterpret_cast<const OpUnit<float>*>(u);
      const auto* tf = reinterpret_cast<const float2*>(tw);
      return tv == 3 ? col_sp<NY, CS_FWD, PW_EPS, CS_INV, 3>(uf, nunits, Nx, maxcol, tf, st)
                     : col_sp<NY, CS_FWD, PW_EPS, CS_INV, 2>(uf, nunits, Nx, maxcol, tf, st);
    }
    if (mode == CM_M && tv != 1)
      return tv == 0 ? col_tx<T, NY, col_tx_variant<NY>(0), CS_FWD, PW_EPS, CS_INV>(u, nunits, Nx, maxcol, tw, st)
                     : col_tx<T, NY, col_tx_variant<NY>(2), CS_FWD, PW_EPS, CS_INV>(u, nunits, Nx, maxcol, tw, st);
  }
  if constexpr (plan2_a(NY) != 0) {  // two-level register FFT
    constexpr int TX = l2_tx<T>(NY), NT = l2_col_threads<T>(NY);
    const size_t sm = (size_t)3 * TX * l2_col_lstr<cplx<T>, NY, TX>() * sizeof(cplx<T>);
    const dim3 g((Nx + TX - 1) / TX, maxcol, nunits);
    switch (mode) {
      case CM_M: return launch_pass<T>(k_col2<T, NY, CS_FWD, PW_EPS, CS_INV>, g, NT, sm, st, u, tw);
      case CM_P: return launch_pass<T>(k_col2<T, NY, CS_INV, PW_EAVE, CS_FWD>, g, NT, sm, st, u, tw);
      case CM_E: return launch_pass<T>(k_col2<T, NY, CS_FWD, PW_EPS, CS_NONE>, g, NT, sm, st, u, tw);
      case CM_FWD: return launch_pass<T>(k_col2<T, NY, CS_FWD, PW_NONE, CS_NONE>, g, NT, sm, st, u, tw);
      case CM_EPSINV: return launch_pass<T>(k_col2<T, NY, CS_NONE, PW_EPS, CS_INV>, g, NT, sm, st, u, tw);
      case CM_BWD: return launch_pass<T>(k_col2<T, NY, CS_INV, PW_NONE, CS_NONE>, g, NT, sm, st, u, tw);
      default: return cudaErrorInvalidValue;
    }
  } else {
    constexpr int TX = tx_for<T>(NY);
    const size_t sm = (NY + 3 * TX * (NY + 1)) * sizeof(cplx<T>);
    const dim3 g((Nx + TX - 1) / TX, maxcol, nunits);
    switch (mode) {
      case CM_M: return launch_pass<T>(k_col<T, NY, TX, NT_COL, CS_FWD, PW_EPS, CS_INV>, g, NT_COL, sm, st, u, tw);
      case CM_P: return launch_pass<T>(k_col<T, NY, TX, NT_COL, CS_INV, PW_EAVE, CS_FWD>, g, NT_COL, sm, st, u, tw);
      case CM_E: return launch_pass<T>(k_col<T, NY, TX, NT_COL, CS_FWD, PW_EPS, CS_NONE>, g, NT_COL, sm, st, u, tw);
      case CM_FWD: return launch_pass<T>(k_col<T, NY, TX, NT_COL, CS_FWD, PW_NONE, CS_NONE>, g, NT_COL, sm, st, u, tw);
      case CM_EPSINV: return launch_pass<T>(k_col<T, NY, TX, NT_COL, CS_NONE, PW_EPS, CS_INV>, g, NT_COL, sm, st, u, tw);
      case CM_BWD: return launch_pass<T>(k_col<T, NY, TX, NT_COL, CS_INV, PW_NONE, CS_NONE>, g, NT_COL, sm, st, u, tw);
      default: return cudaErrorInvalidValue;
    }
  }
}

template <typename T> static const cplx<T>* tw_for(const TwTables& t, int L);
template <> const float2* tw_for<float>(const TwTables& t, int L) { return t.f32[L]; }
template <> const double2* tw_for<double>(const TwTables& t, int L) { return t.f64[L]; }

template <typename T>
static cudaError_t row_in(int mode, const OpUnit<T>* u, int nunits, int Nx, int Ny, int maxcol,
                          const TwTables& t, cudaStream_t st, int gv = 1) {
  switch (Nx) {
#define OMB_CASE(L) case L: return row_in_nx<T, L>(mode, u, nunits, Ny, maxcol, tw_for<T>(t, L), st, gv);
    OMB_FFT_SIZES(OMB_CASE)
#undef OMB_CASE
    default: return cudaErrorInvalidValue;
  }
}
template <typename T>
static cudaError_t row_out(int mode, const OpUnit<T>* u, int nunits, int Nx, int Ny, int maxcol,
                           const TwTables& t, cudaStream_t st, int gv = 1) {
  switch (Nx) {
#define OMB_CASE(L) case L: return row_out_nx<T, L>(mode, u, nunits, Ny, maxcol, tw_for<T>(t, L), st, gv);
    OMB_FFT_SIZES(OMB_CASE)
#undef OMB_CASE
    default: return cudaErrorInvalidValue;
  }
}
template <typename T>
static cudaError_t col(int mode, const OpUnit<T>* u, int nunits, int Nx, int Ny, int maxcol,
                       const TwTables& t, cudaStream_t st, int tv = 1) {
  switch (Ny) {
#define OMB_CASE(L) case L: return col_ny<T, L>(mode, u, nunits, Nx, maxcol, tw_for<T>(t, L), st, tv);
    OMB_FFT_SIZES(OMB_CASE)
#undef OMB_CASE
    default: return cudaErrorInvalidValue;
  }
}

#define OMB_TRY(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return e_; } while (0)

// The one-kernel cluster apply (op_cluster.cuh): a persistent grid of as many CTAS-CTA
// clusters as can be resident, never more than there are (unit, column) pairs.
template <int NX, int NY, int CTAS>
static cudaError_t cluster_apply(const OpUnit<float>* u, int nunits, int maxcol, const float2* twx,
                                 const float2* twy, cudaStream_t st) {
  using S = ClShape<NX, NY, CTAS>;
  auto kern = k_apply_cluster<NX, NY, CTAS>;
  const void* kp = reinterpret_cast<const void*>(kern);
  cudaError_t e = ensure_smem(kp, S::SMEM, true);
  if (e != cudaSuccess) return e;
  if (CTAS > 8) {  // above the portable cluster size (set once; later calls find it set)
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && !done[dev]) {
      e = cudaFuncSetAttribute(kp, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      if (e != cudaSuccess) return e;
      done[dev] = true;
    }
  }
  const long long total = (long long)nunits * maxcol;
  const long long ncl = std::min<long long>(cluster_slots(kp, CTAS, S::THREADS, S::SMEM), total);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(ncl * CTAS), 1, 1);
  cfg.blockDim = dim3(S::THREADS, 1, 1);
  cfg.dynamicSmemBytes = S::SMEM;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CTAS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, u, nunits, maxcol, twx, twy);
}

template <typename T>
cudaError_t launch_op(OpKind op, const OpUnit<T>* u, int nunits, int Nx, int Ny, int maxcol,
                      const TwTables& t, cudaStream_t st) {
  if (nunits <= 0 || maxcol <= 0) return cudaSuccess;
  TileChoice tc = sizeof(T) == 4 ? tiles_for(Nx, Ny) : TileChoice{};
  if (tc.row == ROW_CLUSTER || tc.row == ROW_CLUSTER16) {
    if constexpr (sizeof(T) == 4) {
      if (op == OP_M && Nx == 256 && Ny == 256) {
        const auto* uf = reinterpret_cast<const OpUnit<float>*>(u);
        return tc.row == ROW_CLUSTER ? cluster_apply<256, 256, 8>(uf, nunits, maxcol, t.f32[256], t.f32[256], st)
                                     : cluster_apply<256, 256, 16>(uf, nunits, maxcol, t.f32[256], t.f32[256], st);
      }
    }
    tc = TileChoice{};  // the other pipelines keep the default tiles
  }
  if (tc.wave > 0 && (op == OP_M || op == OP_MDOT)) {
    const int per = wave_columns(tc.wave) / maxcol > 0 ? wave_columns(tc.wave) / maxcol : 1;
    if (per < nunits) {
      for (int u0 = 0; u0 < nunits; u0 += per) {
        const int n = nunits - u0 < per ? nunits - u0 : per;
        OMB_TRY(row_in<T>(RI_KXTC, u + u0, n, Nx, Ny, maxcol, t, st, tc.row));
        OMB_TRY(col<T>(CM_M, u + u0, n, Nx, Ny, maxcol, t, st, tc.col));
        OMB_TRY(op == OP_M ? row_out<T>(RO_KXCT, u + u0, n, Nx, Ny, maxcol, t, st, tc.row)
                           : row_out<T>(RO_KXCT_DOT, u + u0, n, Nx, Ny, maxcol, t, st, tc.row == 4 ? 4 : 1));
      }
      return cudaSuccess;
    }
  }
  switch (op) {
    case OP_M:
      OMB_TRY(row_in<T>(RI_KXTC, u, nunits, Nx, Ny, maxcol, t, st, tc.row));
      OMB_TRY(col<T>(CM_M, u, nunits, Nx, Ny, maxcol, t, st, tc.col));
      return row_out<T>(RO_KXCT, u, nunits, Nx, Ny, maxcol, t, st, tc.row);
    case OP_MDOT:
      OMB_TRY(row_in<T>(RI_KXTC, u, nunits, Nx, Ny, maxcol, t, st, tc.row));
      OMB_TRY(col<T>(CM_M, u, nunits, Nx, Ny, maxcol, t, st, tc.col));
      return row_out<T>(RO_KXCT_DOT, u, nunits, Nx, Ny, maxcol, t, st, tc.row == 4 ? 4 : 1);
    case OP_P:
      OMB_TRY(row_in<T>(RI_KXINV, u, nunits, Nx, Ny, maxcol, t, st));
      OMB_TRY(col<T>(CM_P, u, nunits, Nx, Ny, maxcol, t, st));
      return row_out<T>(RO_KXINVCT, u, nunits, Nx, Ny, maxcol, t, st);
    case OP_HMKH:
      OMB_TRY(row_in<T>(RI_ZXTC, u, nunits, Nx, Ny, maxcol, t, st));
      OMB_TRY(col<T>(CM_M, u, nunits, Nx, Ny, maxcol, t, st));
      return row_out<T>(RO_KXCT_DOT, u, nunits, Nx, Ny, maxcol, t, st);
    case OP_EFIELD:
      OMB_TRY(row_in<T>(RI_KXTC, u, nunits, Nx, Ny, maxcol, t, st));
      return col<T>(CM_E, u, nunits, Nx, Ny, maxcol, t, st);
    case OP_H2D:
      OMB_TRY(row_in<T>(RI_KXTC, u, nunits, Nx, Ny, maxcol, t, st));
      return col<T>(CM_FWD, u, nunits, Nx, Ny, maxcol, t, st);
    case OP_D2E:
      OMB_TRY(col<T>(CM_EPSINV, u, nunits, Nx, Ny, maxcol, t, st));
      return row_out<T>(RO_STORE3, u, nunits, Nx, Ny, maxcol, t, st);
    case OP_HFIELD:
      OMB_TRY(row_in<T>(RI_HCART, u, nunits, Nx, Ny, maxcol, t, st));
      return col<T>(CM_FWD, u, nunits, Nx, Ny, maxcol, t, st);
    case OP_R2G:
      OMB_TRY(row_in<T>(RI_LOAD3, u, nunits, Nx, Ny, maxcol, t, st));
      return col<T>(CM_BWD, u, nunits, Nx, Ny, maxcol, t, st);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace omb
