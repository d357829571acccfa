/*
 * libomb200 — B200 (sm_100a) plane-wave Helmholtz eigensolver, C ABI.
 *
 * The drop-in boundary for OptiMode.jl's `solve_ω²` / `solve_k` hot path and its adjoint
 * pull-back.  Julia binds these with `ccall` from a new `B200Solver <: AbstractEigensolver`
 * (see INTEGRATION.md); Python binds them with ctypes.  Every symbol takes plain pointers
 * and sizes; no torch or CUDA types cross the boundary.
 *
 * Conventions
 *  - Host arrays are the reference's column-major Julia arrays, passed as raw memory:
 *      epsinv : Float64 (3, 3, Nx, Ny)          — 9·Nx·Ny doubles, symmetric per pixel
 *      H      : ComplexF64 (2, Nx, Ny) per column — 4·Nx·Ny doubles (re, im interleaved)
 *      E      : ComplexF64 (3, Nx, Ny)           — 6·Nx·Ny doubles
 *    Blocks of `ncol` columns are stored one column after another.
 *  - Units: cycles/μm (ω = 1/λ, k = n_eff/λ; no 2π), cell sizes in μm, c = 1.
 *  - Return value: OMB_OK (0) or one of the OMB_ERR_* codes; `omb_last_error()` then
 *    returns a thread-local message naming the failure.
 *  - A context is not thread-safe; use one per host thread.  Calls are synchronous: they
 *    return after the results are in the caller's host buffers.
 *  - Supported grid sizes: every Nx, Ny in {8, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96,
 *    128, 160, 192, 256, 320, 384, 512} (see omb_fft_size_supported).
 */
#ifndef OMB200_H
#define OMB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OMB_OK 0
#define OMB_ERR_INVALID_ARG 1
#define OMB_ERR_CUDA 2
#define OMB_ERR_NOT_CONVERGED 3
#define OMB_ERR_ORTHO_FAIL 4
#define OMB_ERR_TIMEOUT 5
#define OMB_ERR_UNSUPPORTED 6
#define OMB_ERR_NAN 7

/* arithmetic of a call */
#define OMB_PREC_FP32 0  /* FP32 operator, FP64 small dense algebra               */
#define OMB_PREC_FP64 1  /* FP64 everywhere                                       */
#define OMB_PREC_MIXED 2 /* FP32 iterations, then FP64 polish to the tolerance     */

/* operators for omb_apply */
#define OMB_OP_M 0      /* M̂(k)                                                   */
#define OMB_OP_P 1      /* MPB-style preconditioner P̂(k) (two FFT pairs)           */
#define OMB_OP_P_DIAG 2 /* diagonal preconditioner ⟨ε⟩/|k+G|²                      */

typedef struct omb_ctx omb_ctx;

/* A 2D periodic cell: Dx × Dy μm on Nx × Ny pixels (reference `Grid{2}`,
 * lib/DielectricSmoothing/src/grid.jl:46-76). */
typedef struct {
  int32_t Nx, Ny;
  double Dx, Dy;
} omb_grid;

/* Library version (major*10000 + minor*100 + patch). */
int omb_version(void);
/* 1 when n is a supported grid length, else 0. */
int omb_fft_size_supported(int n);
/* Message for the last failing call on this thread ("" when none). */
const char* omb_last_error(void);

/* Create / destroy a context on CUDA device `device`.  The context owns a stream,
 * device-resident twiddle tables and a stream-ordered memory pool. */
int omb_ctx_create(int device, omb_ctx** out);
int omb_ctx_destroy(omb_ctx* ctx);

/* Hout = op(k) Hin for `ncol` columns.
 * Replaces HelmholtzMap(Hout, Hin) / _M! (lib/MaxwellEigenmodes/src/maxwell.jl:471-481,
 * 1007-1025; device form _gpu_M!, src/solvers/gpu.jl:157-166) for OMB_OP_M, and
 * HelmholtzPreconditioner / _P! (maxwell.jl:459-469, 1027-1045) for OMB_OP_P. */
int omb_apply(omb_ctx* ctx, int op, int precision, const omb_grid* grid, double k,
              const double* epsinv, int ncol, const double* H_in, double* H_out);

/* out[j] = ⟨H_j|∂M̂/∂k|H_j⟩ for each column (∂ω²/∂k = 2·out for a unit eigenvector).
 * Replaces HMₖH (maxwell.jl:267-275) / _gpu_HMkH (gpu.jl:171-180). */
int omb_HMkH(omb_ctx* ctx, int precision, const omb_grid* grid, double k,
             const double* epsinv, int ncol, const double* H, double* out);

/* Un-normalised, un-canonicalised E = ε⁻¹·fft(kx_tc H) for one column.
 * Replaces E⃗(k, evec, ε⁻¹, ∂ε_∂ω, grid; canonicalize=false, normalized=false)
 * (lib/MaxwellEigenmodes/src/fields.jl:194-210). */
int omb_efield(omb_ctx* ctx, int precision, const omb_grid* grid, double k,
               const double* epsinv, const double* H, double* E);

#ifdef __cplusplus
}
#endif

#endif /* OMB200_H */
