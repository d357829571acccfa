// Entry points for single operator evaluations: omb_apply, omb_HMkH, omb_efield.
#include <cmath>
#include <vector>

#include "context.h"
#include "vec.cuh"

namespace omb {

static int grid_blocks(size_t n, int nt = 256) {
  size_t b = (n + nt - 1) / nt;
  return (int)(b > 65535 * 8 ? 65535 * 8 : (b ? b : 1));
}

// Device copies of a host block of `ncol` 2-component columns at precision T.

template <typename T>
static int to_device(omb_ctx* ctx, const double* h, size_t n, DevBuf<double2>& tmp64, DevBuf<cplx<T>>& out) {
  OMB_CU(tmp64.alloc(n, ctx->stream));
  OMB_CU(cudaMemcpyAsync(tmp64.p, h, n * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
  if constexpr (std::is_same<T, double>::value) {
    out = std::move(tmp64);
  } else {
    OMB_CU(out.alloc(n, ctx->stream));
    k_c64_to_c32<<<grid_blocks(n), 256, 0, ctx->stream>>>(tmp64.p, out.p, n);
    OMB_CU(cudaGetLastError());
  }
  return OMB_OK;
}

template <typename T>
static int to_host(omb_ctx* ctx, const cplx<T>* d, size_t n, double* h) {
  if constexpr (std::is_same<T, double>::value) {
    OMB_CU(cudaMemcpyAsync(h, d, n * sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream));
  } else {
    DevBuf<double2> t;
    OMB_CU(t.alloc(n, ctx->stream));
    k_c32_to_c64<<<grid_blocks(n), 256, 0, ctx->stream>>>(d, t.p, n);
    OMB_CU(cudaGetLastError());
    OMB_CU(cudaMemcpyAsync(h, t.p, n * sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream));
    OMB_CU(cudaStreamSynchronize(ctx->stream));
  }
  OMB_CU(cudaStreamSynchronize(ctx->stream));
  return OMB_OK;
}

template <typename T>
static int run_apply(omb_ctx* ctx, int op, const Problem& P, double k, int ncol, const double* Hin, double* Hout) {
  const size_t N = P.N(), n = 2 * N * (size_t)ncol;
  cudaStream_t st = ctx->stream;
  DevBuf<double2> tmp;
  DevBuf<cplx<T>> hin, hout, scr;
  int rc = to_device<T>(ctx, Hin, n, tmp, hin);
  if (rc) return rc;
  OMB_CU(hout.alloc(n, st));
  DevBuf<double> kd;
  OMB_CU(kd.alloc(1, st));
  OMB_CU(cudaMemcpyAsync(kd.p, &k, sizeof(double), cudaMemcpyHostToDevice, st));
  if (op == OMB_OP_P_DIAG) {
    k_prec_diag<T><<<grid_blocks(N * ncol), 256, 0, st>>>(hin.p, hout.p, P.Nx, P.Ny, (T)(1.0 / P.Dx),
                                                          (T)(1.0 / P.Dy), kd.p, P.eps_mean, ncol, (long long)(2 * N));
    OMB_CU(cudaGetLastError());
  } else {
    OMB_CU(scr.alloc(3 * N * (size_t)ncol, st));
    OpUnit<T> u = make_unit<T>(P);
    u.in = hin.p; u.out = hout.p; u.scr = scr.p; u.k_dev = kd.p;
    u.in_cs = u.out_cs = (long long)(2 * N); u.scr_cs = (long long)(3 * N); u.ncol = ncol;
    DevBuf<OpUnit<T>> du;
    OMB_CU(du.alloc(1, st));
    OMB_CU(cudaMemcpyAsync(du.p, &u, sizeof(u), cudaMemcpyHostToDevice, st));
    OMB_CU(launch_op<T>(op == OMB_OP_M ? OP_M : OP_P, du.p, 1, P.Nx, P.Ny, ncol, ctx->tw, st));
  }
  return to_host<T>(ctx, hout.p, n, Hout);
}

template <typename T>
static int run_hmkh(omb_ctx* ctx, const Problem& P, double k, int ncol, const double* H, double* out) {
  const size_t N = P.N(), n = 2 * N * (size_t)ncol;
  cudaStream_t st = ctx->stream;
  DevBuf<double2> tmp;
  DevBuf<cplx<T>> hin, scr;
  int rc = to_device<T>(ctx, H, n, tmp, hin);
  if (rc) return rc;
  OMB_CU(scr.alloc(3 * N * (size_t)ncol, st));
  DevBuf<double> kd, part, red;
  const int nb = row_blocks(P.Nx, P.Ny);
  OMB_CU(kd.alloc(1, st));
  OMB_CU(part.alloc(2 * (size_t)nb * ncol, st));
  OMB_CU(red.alloc(2 * (size_t)ncol, st));
  OMB_CU(cudaMemcpyAsync(kd.p, &k, sizeof(double), cudaMemcpyHostToDevice, st));
  OpUnit<T> u = make_unit<T>(P);
  u.in = hin.p; u.out = nullptr; u.scr = scr.p; u.k_dev = kd.p; u.partial = part.p;
  u.in_cs = (long long)(2 * N); u.scr_cs = (long long)(3 * N); u.ncol = ncol;
  DevBuf<OpUnit<T>> du;
  OMB_CU(du.alloc(1, st));
  OMB_CU(cudaMemcpyAsync(du.p, &u, sizeof(u), cudaMemcpyHostToDevice, st));
  OMB_CU(launch_op<T>(OP_HMKH, du.p, 1, P.Nx, P.Ny, ncol, ctx->tw, st));
  k_reduce_partials<<<ncol, 256, 0, st>>>(part.p, nb, ncol, red.p);
  OMB_CU(cudaGetLastError());
  std::vector<double> h(2 * (size_t)ncol);
  OMB_CU(cudaMemcpyAsync(h.data(), red.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaStreamSynchronize(st));
  for (int j = 0; j < ncol; ++j) out[j] = -h[2 * j];
  return OMB_OK;
}

template <typename T>
static int run_efield(omb_ctx* ctx, const Problem& P, double k, const double* H, double* E) {
  const size_t N = P.N(), n = 2 * N;
  cudaStream_t st = ctx->stream;
  DevBuf<double2> tmp;
  DevBuf<cplx<T>> hin, scr;
  int rc = to_device<T>(ctx, H, n, tmp, hin);
  if (rc) return rc;
  OMB_CU(scr.alloc(3 * N, st));
  DevBuf<double> kd;
  OMB_CU(kd.alloc(1, st));
  OMB_CU(cudaMemcpyAsync(kd.p, &k, sizeof(double), cudaMemcpyHostToDevice, st));
  OpUnit<T> u = make_unit<T>(P);
  u.in = hin.p; u.scr = scr.p; u.k_dev = kd.p;
  u.in_cs = (long long)(2 * N); u.scr_cs = (long long)(3 * N); u.ncol = 1;
  DevBuf<OpUnit<T>> du;
  OMB_CU(du.alloc(1, st));
  OMB_CU(cudaMemcpyAsync(du.p, &u, sizeof(u), cudaMemcpyHostToDevice, st));
  OMB_CU(launch_op<T>(OP_EFIELD, du.p, 1, P.Nx, P.Ny, 1, ctx->tw, st));
  // planar [c][p] → interleaved (3, Nx, Ny)
  std::vector<double2> h(3 * N);
  if constexpr (std::is_same<T, double>::value) {
    OMB_CU(cudaMemcpyAsync(h.data(), scr.p, 3 * N * sizeof(double2), cudaMemcpyDeviceToHost, st));
    OMB_CU(cudaStreamSynchronize(st));
  } else {
    DevBuf<double2> t;
    OMB_CU(t.alloc(3 * N, st));
    k_c32_to_c64<<<grid_blocks(3 * N), 256, 0, st>>>(scr.p, t.p, 3 * N);
    OMB_CU(cudaGetLastError());
    OMB_CU(cudaMemcpyAsync(h.data(), t.p, 3 * N * sizeof(double2), cudaMemcpyDeviceToHost, st));
    OMB_CU(cudaStreamSynchronize(st));
  }
  for (size_t p = 0; p < N; ++p)
    for (int c = 0; c < 3; ++c) {
      E[2 * (3 * p + c)] = h[c * N + p].x;
      E[2 * (3 * p + c) + 1] = h[c * N + p].y;
    }
  return OMB_OK;
}

static int check_common(omb_ctx* ctx, int precision, double k) {
  if (!ctx) return fail(OMB_ERR_INVALID_ARG, "ctx is NULL");
  if (precision != OMB_PREC_FP32 && precision != OMB_PREC_FP64)
    return fail(OMB_ERR_INVALID_ARG, "precision must be OMB_PREC_FP32 or OMB_PREC_FP64 for a single evaluation");
  if (!(k > 0) || !std::isfinite(k)) return fail(OMB_ERR_INVALID_ARG, "k must be finite and positive");
  OMB_CU(cudaSetDevice(ctx->device));
  return OMB_OK;
}

}  // namespace omb

using namespace omb;

extern "C" {

int omb_apply(omb_ctx* ctx, int op, int precision, const omb_grid* grid, double k,
              const double* epsinv, int ncol, const double* H_in, double* H_out) {
  int rc = check_common(ctx, precision, k);
  if (rc) return rc;
  if (op != OMB_OP_M && op != OMB_OP_P && op != OMB_OP_P_DIAG) return fail(OMB_ERR_INVALID_ARG, "unknown op");
  if (ncol <= 0 || !H_in || !H_out) return fail(OMB_ERR_INVALID_ARG, "need ncol > 0 and non-NULL H_in, H_out");
  Problem P;
  rc = upload_problem(ctx, grid, epsinv, P);
  if (rc) return rc;
  return precision == OMB_PREC_FP64 ? run_apply<double>(ctx, op, P, k, ncol, H_in, H_out)
                                    : run_apply<float>(ctx, op, P, k, ncol, H_in, H_out);
}

int omb_HMkH(omb_ctx* ctx, int precision, const omb_grid* grid, double k, const double* epsinv,
             int ncol, const double* H, double* out) {
  int rc = check_common(ctx, precision, k);
  if (rc) return rc;
  if (ncol <= 0 || !H || !out) return fail(OMB_ERR_INVALID_ARG, "need ncol > 0 and non-NULL H, out");
  Problem P;
  rc = upload_problem(ctx, grid, epsinv, P);
  if (rc) return rc;
  return precision == OMB_PREC_FP64 ? run_hmkh<double>(ctx, P, k, ncol, H, out)
                                    : run_hmkh<float>(ctx, P, k, ncol, H, out);
}

int omb_efield(omb_ctx* ctx, int precision, const omb_grid* grid, double k, const double* epsinv,
               const double* H, double* E) {
  int rc = check_common(ctx, precision, k);
  if (rc) return rc;
  if (!H || !E) return fail(OMB_ERR_INVALID_ARG, "need non-NULL H, E");
  Problem P;
  rc = upload_problem(ctx, grid, epsinv, P);
  if (rc) return rc;
  return precision == OMB_PREC_FP64 ? run_efield<double>(ctx, P, k, H, E) : run_efield<float>(ctx, P, k, H, E);
}

}  // extern "C"
