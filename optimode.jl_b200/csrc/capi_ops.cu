// Entry points for single operator evaluations: omb_apply, omb_HMkH, omb_efield.
#include <cmath>
#include <vector>

#include "context.h"
#include "lobpcg.cuh"
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

// One unit through a pipeline on a 2D or z-periodic cell.
template <typename T>
static int launch_cell(OpKind op, const OpUnit<T>* du, const Problem& P, int ncol, omb_ctx* ctx, cudaStream_t st) {
  if (P.Nz > 1) {
    DevBuf<OpUnit<T>> ex;
    OMB_CU(ex.alloc((size_t)P.Nz + 1, st));
    OMB_CU(launch_op3d<T>(op, du, 1, P.Nx, P.Ny, P.Nz, ncol, ctx->tw, ex.p, st));
    OMB_CU(cudaStreamSynchronize(st));  // ex is released at return
    return OMB_OK;
  }
  OMB_CU(launch_op<T>(op, du, 1, P.Nx, P.Ny, ncol, ctx->tw, st));
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
    rc = launch_cell<T>(op == OMB_OP_M ? OP_M : OP_P, du.p, P, ncol, ctx, st);
    if (rc) return rc;
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
  const int nb = row_blocks(P.Nx, P.Ny) * P.Nz;
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
  rc = launch_cell<T>(OP_HMKH, du.p, P, ncol, ctx, st);
  if (rc) return rc;
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

template <typename T>
static int run_profile(omb_ctx* ctx, int op, const Problem& P, double k, int ncol, int nbatch, int reps,
                       double* seconds) {
  const size_t N = P.N(), n2 = 2 * N;
  cudaStream_t st = ctx->stream;
  // nbatch private copies of the cell's ε⁻¹ so every copy streams its own tensor from HBM
  DevBuf<float4> a32;
  DevBuf<float2> b32;
  DevBuf<double2> e64;
  DevBuf<T> eave;
  OMB_CU(a32.alloc(N * nbatch, st));
  OMB_CU(b32.alloc(N * nbatch, st));
  OMB_CU(e64.alloc(3 * N * nbatch, st));
  OMB_CU(eave.alloc(N * nbatch, st));
  const T* eave_src = std::is_same<T, float>::value ? (const T*)P.eave32.p : (const T*)P.eave64.p;
  for (int c = 0; c < nbatch; ++c) {
    OMB_CU(cudaMemcpyAsync(a32.p + c * N, P.e32a.p, N * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    OMB_CU(cudaMemcpyAsync(b32.p + c * N, P.e32b.p, N * sizeof(float2), cudaMemcpyDeviceToDevice, st));
    OMB_CU(cudaMemcpyAsync(e64.p + 3 * c * N, P.e64.p, 3 * N * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    OMB_CU(cudaMemcpyAsync(eave.p + c * N, eave_src, N * sizeof(T), cudaMemcpyDeviceToDevice, st));
  }
  DevBuf<cplx<T>> hin, hout, scr;
  OMB_CU(hin.alloc(n2 * ncol * nbatch, st));
  OMB_CU(hout.alloc(n2 * ncol * nbatch, st));
  OMB_CU(scr.alloc(3 * N * ncol * nbatch, st));
  k_random_block<T><<<grid_blocks(n2 * ncol * nbatch), 256, 0, st>>>(hin.p, (long long)n2, ncol * nbatch, 99);
  OMB_CU(cudaGetLastError());
  DevBuf<double> kd;
  OMB_CU(kd.alloc(1, st));
  OMB_CU(cudaMemcpyAsync(kd.p, &k, sizeof(double), cudaMemcpyHostToDevice, st));
  std::vector<OpUnit<T>> units(nbatch);
  for (int c = 0; c < nbatch; ++c) {
    OpUnit<T> u = make_unit<T>(P);
    u.e32a = a32.p + c * N; u.e32b = b32.p + c * N; u.e64 = e64.p + 3 * c * N; u.eave = eave.p + c * N;
    u.in = hin.p + c * n2 * ncol; u.out = hout.p + c * n2 * ncol; u.scr = scr.p + c * 3 * N * ncol;
    u.k_dev = kd.p;
    u.in_cs = u.out_cs = (long long)n2; u.scr_cs = (long long)(3 * N); u.ncol = ncol;
    units[c] = u;
  }
  DevBuf<OpUnit<T>> du;
  OMB_CU(du.alloc(nbatch, st));
  OMB_CU(cudaMemcpyAsync(du.p, units.data(), nbatch * sizeof(OpUnit<T>), cudaMemcpyHostToDevice, st));
  const OpKind kind = op == OMB_OP_M ? OP_M : OP_P;
  for (int w = 0; w < 3; ++w) OMB_CU(launch_op<T>(kind, du.p, nbatch, P.Nx, P.Ny, ncol, ctx->tw, st));
  cudaEvent_t e0, e1;
  OMB_CU(cudaEventCreate(&e0));
  OMB_CU(cudaEventCreate(&e1));
  OMB_CU(cudaStreamSynchronize(st));
  OMB_CU(cudaEventRecord(e0, st));
  for (int r = 0; r < reps; ++r) OMB_CU(launch_op<T>(kind, du.p, nbatch, P.Nx, P.Ny, ncol, ctx->tw, st));
  OMB_CU(cudaEventRecord(e1, st));
  OMB_CU(cudaEventSynchronize(e1));
  float ms = 0;
  OMB_CU(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *seconds = (double)ms * 1e-3 / reps;
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

int omb_apply3(omb_ctx* ctx, int op, int precision, const omb_grid3* grid, double k, const double* epsinv, int ncol,
               const double* H_in, double* H_out) {
  int rc = check_common(ctx, precision, k);
  if (rc) return rc;
  if (!grid) return fail(OMB_ERR_INVALID_ARG, "grid is NULL");
  if (op != OMB_OP_M && op != OMB_OP_P) return fail(OMB_ERR_INVALID_ARG, "op must be OMB_OP_M or OMB_OP_P");
  if (ncol <= 0 || !H_in || !H_out) return fail(OMB_ERR_INVALID_ARG, "need ncol > 0 and non-NULL H_in, H_out");
  const omb_grid g2{grid->Nx, grid->Ny, grid->Dx, grid->Dy};
  Problem P;
  rc = upload_problem(ctx, &g2, epsinv, P, grid->Nz, grid->Dz);
  if (rc) return rc;
  return precision == OMB_PREC_FP64 ? run_apply<double>(ctx, op, P, k, ncol, H_in, H_out)
                                    : run_apply<float>(ctx, op, P, k, ncol, H_in, H_out);
}

int omb_HMkH3(omb_ctx* ctx, int precision, const omb_grid3* grid, double k, const double* epsinv, int ncol,
              const double* H, double* out) {
  int rc = check_common(ctx, precision, k);
  if (rc) return rc;
  if (!grid) return fail(OMB_ERR_INVALID_ARG, "grid is NULL");
  if (ncol <= 0 || !H || !out) return fail(OMB_ERR_INVALID_ARG, "need ncol > 0 and non-NULL H, out");
  const omb_grid g2{grid->Nx, grid->Ny, grid->Dx, grid->Dy};
  Problem P;
  rc = upload_problem(ctx, &g2, epsinv, P, grid->Nz, grid->Dz);
  if (rc) return rc;
  return precision == OMB_PREC_FP64 ? run_hmkh<double>(ctx, P, k, ncol, H, out)
                                    : run_hmkh<float>(ctx, P, k, ncol, H, out);
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

int omb_profile_apply(omb_ctx* ctx, int op, int precision, const omb_grid* grid, double k,
                      const double* epsinv, int ncol, int nbatch, int reps, double* seconds) {
  int rc = check_common(ctx, precision, k);
  if (rc) return rc;
  if (op != OMB_OP_M && op != OMB_OP_P) return fail(OMB_ERR_INVALID_ARG, "op must be OMB_OP_M or OMB_OP_P");
  if (ncol <= 0 || nbatch <= 0 || reps <= 0 || !seconds)
    return fail(OMB_ERR_INVALID_ARG, "need ncol, nbatch, reps > 0 and non-NULL seconds");
  Problem P;
  rc = upload_problem(ctx, grid, epsinv, P);
  if (rc) return rc;
  return precision == OMB_PREC_FP64 ? run_profile<double>(ctx, op, P, k, ncol, nbatch, reps, seconds)
                                    : run_profile<float>(ctx, op, P, k, ncol, nbatch, reps, seconds);
}

int omb_hfield(omb_ctx* ctx, const omb_grid* grid, double k, int ncol, const double* H, double* Hr) {
  int rc = check_common(ctx, OMB_PREC_FP64, k);
  if (rc) return rc;
  rc = check_grid(grid);
  if (rc) return rc;
  if (!H || !Hr || ncol <= 0) return fail(OMB_ERR_INVALID_ARG, "need ncol > 0 and non-NULL H, Hr");
  const size_t N = (size_t)grid->Nx * grid->Ny, n = 2 * N * (size_t)ncol;
  cudaStream_t st = ctx->stream;
  DevBuf<double2> hin, scr;
  OMB_CU(hin.alloc(n, st));
  OMB_CU(cudaMemcpyAsync(hin.p, H, n * sizeof(double2), cudaMemcpyHostToDevice, st));
  OMB_CU(scr.alloc(3 * N * (size_t)ncol, st));
  DevBuf<double> kd;
  OMB_CU(kd.alloc(1, st));
  OMB_CU(cudaMemcpyAsync(kd.p, &k, sizeof(double), cudaMemcpyHostToDevice, st));
  OpUnit<double> u{};
  u.in = hin.p; u.scr = scr.p; u.k_dev = kd.p;
  u.in_cs = (long long)(2 * N); u.scr_cs = (long long)(3 * N); u.ncol = ncol;
  u.Nx = grid->Nx; u.Ny = grid->Ny;
  u.inv_dx = 1.0 / grid->Dx; u.inv_dy = 1.0 / grid->Dy;
  u.part_stride = row_blocks(grid->Nx, grid->Ny);
  DevBuf<OpUnit<double>> du;
  OMB_CU(du.alloc(1, st));
  OMB_CU(cudaMemcpyAsync(du.p, &u, sizeof(u), cudaMemcpyHostToDevice, st));
  OMB_CU(launch_op<double>(OP_HFIELD, du.p, 1, grid->Nx, grid->Ny, ncol, ctx->tw, st));
  std::vector<double2> h(3 * N * (size_t)ncol);
  OMB_CU(cudaMemcpyAsync(h.data(), scr.p, h.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaStreamSynchronize(st));
  // planar [c][p] per column → interleaved (3, Nx, Ny) per column
  for (int j = 0; j < ncol; ++j)
    for (size_t p = 0; p < N; ++p)
      for (int c = 0; c < 3; ++c) {
        const double2 v = h[(size_t)j * 3 * N + c * N + p];
        Hr[2 * (3 * N * j + 3 * p + c)] = v.x;
        Hr[2 * (3 * N * j + 3 * p + c) + 1] = v.y;
      }
  return OMB_OK;
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
