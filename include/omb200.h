/*
 * libomb200 — B200 (sm_100a) plane-wave Helmholtz eigensolver, C ABI.
 *
 * The drop-in boundary for OptiMode.jl's `solve_ω²` / `solve_k` hot path and its adjoint
 * pull-back.  Julia binds these with `ccall` from a new `B200Solver <: AbstractEigensolver`;
 * Python binds them with ctypes.  Every symbol takes plain pointers and sizes; no torch or
 * CUDA types cross the boundary.
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

/* A 3D cell periodic along z (reference `Grid{3}`, grid.jl:46-76): Dx × Dy μm on Nx × Ny
 * pixels in the cross-section and Nz slabs over the period Dz = Λ (Nz a supported length, at
 * least 8). */
typedef struct {
  int32_t Nx, Ny, Nz;
  double Dx, Dy, Dz;
} omb_grid3;

/* Library version (major*10000 + minor*100 + patch). */
int omb_version(void);
/* 1 when n is a supported grid length, else 0. */
int omb_fft_size_supported(int n);
/* Message for the last failing call on this thread ("" when none). */
const char* omb_last_error(void);

/* Create / destroy a context on CUDA device `device`.  The context owns a stream,
 * device-resident twiddle tables and a stream-ordered memory pool.  Destroy the batches and
 * smoothing plans made on a context before the context; a warm-start network still alive
 * then is released with it (its handle then only goes to omb_warmstart_destroy). */
int omb_ctx_create(int device, omb_ctx** out);
int omb_ctx_destroy(omb_ctx* ctx);

/* Limit of every bounded wait in the context's streaming kernels (the Gram and update
 * pipelines: a wait for a bulk copy to land or a stage to be released), in seconds, (0, 60];
 * 1 s by default.  A wait that runs out makes its kernel record an error and return, and the
 * call that launched it returns OMB_ERR_TIMEOUT with the context still usable.  No reference
 * counterpart (its solvers have no device-side waits). */
int omb_ctx_set_wait_limit(omb_ctx* ctx, double seconds);
/* Self-test of that failure path: one kernel waits, with the context's limit, on a barrier
 * phase that nothing completes.  Returns OMB_ERR_TIMEOUT and the kernel's error code in
 * *code (1: a full-stage wait ran out); OMB_OK would mean the wait completed.  No reference
 * counterpart. */
int omb_selftest_wait(omb_ctx* ctx, int32_t* code);

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

/* The same on a z-periodic cell: epsinv (3, 3, Nx, Ny, Nz) Float64, columns ComplexF64
 * (2, Nx, Ny, Nz); w = k ẑ − G with G = (gx, gy, m/Λ) (the 3D forms of maxwell.jl's
 * kx_tc/kx_ct/mag_mn, 3D FFTs).  op: OMB_OP_M or OMB_OP_P. */
int omb_apply3(omb_ctx* ctx, int op, int precision, const omb_grid3* grid, double k, const double* epsinv, int ncol,
               const double* H_in, double* H_out);
int omb_HMkH3(omb_ctx* ctx, int precision, const omb_grid3* grid, double k, const double* epsinv, int ncol,
              const double* H, double* out);

/* Un-normalised, un-canonicalised E = ε⁻¹·fft(kx_tc H) for one column.
 * Replaces E⃗(k, evec, ε⁻¹, ∂ε_∂ω, grid; canonicalize=false, normalized=false)
 * (lib/MaxwellEigenmodes/src/fields.jl:194-210). */
int omb_efield(omb_ctx* ctx, int precision, const omb_grid* grid, double k,
               const double* epsinv, const double* H, double* E);

/* Real-space Cartesian magnetic field H(r) = fft(h1 m̂ + h2 n̂) of `ncol` columns (FP64), as
 * ComplexF64 (3, Nx, Ny) per column, un-normalised (the same transform as E).  Replaces
 * H⃗(ms; svecs=false) = fft(tc(H, mn)) (lib/MaxwellEigenmodes/src/fields.jl:125-126, tc at
 * src/maxwell.jl:184-186); builds the learned warm start's training targets. */
int omb_hfield(omb_ctx* ctx, const omb_grid* grid, double k, int ncol, const double* H, double* Hr);

/* Allocation-free FP32 Hout = M̂(k) Hin on caller-owned device memory.  No counterpart in
 * the reference: it exists for callers that cannot allocate device memory when they need
 * the operator — host frameworks that own the whole device pool and forbid foreign
 * cudaMalloc/cudaFree (a Julia or PyTorch caching allocator), callers whose device-memory
 * budget is fixed up front, and hot loops that must not pay the latency and implicit device
 * synchronisation of cudaMalloc/cudaFree.  It allocates nothing: its scratch is a fixed
 * static device array (6 MiB) held by every GPU that loads the library until exit.
 *   d_epsinv : device Float32 (3, 3, Nx, Ny), symmetric per pixel
 *   d_H_in, d_H_out : device ComplexF32 (2, Nx, Ny), ncol columns each
 *   stream   : a cudaStream_t, or NULL for the legacy default stream
 * Limit: Nx·Ny·ncol ≤ OMB_NOALLOC_MAX_PIXEL_COLUMNS, else OMB_ERR_INVALID_ARG.  All calls
 * share the scratch, so calls that overlap on the GPU race.  The first call in a CUDA
 * context sets up the scratch address and twiddle tables with a blocking copy; make it
 * before any stream capture (a first call on a capturing stream is refused). */
#define OMB_NOALLOC_MAX_PIXEL_COLUMNS 262144
int omb_apply_M_noalloc(int32_t Nx, int32_t Ny, double Dx, double Dy, double k, const float* d_epsinv,
                        int32_t ncol, const void* d_H_in, void* d_H_out, void* stream);

/* ---------------------------------------------------------------------------------
 * Autotuning of the FP32 operator passes (the counterpart of the reference's FFTW PATIENT
 * planning at ModeSolver construction, lib/MaxwellEigenmodes/src/maxwell.jl:940-943).
 * Per (device name, Nx, Ny) the combinations of row-pass variant (0, 1, 2: half, default,
 * double the grid rows per CTA; 3: default rows, row_in with one thread per line slot and field
 * component; 4: both row passes so; 5, 6: the whole application in one kernel on thread-block
 * clusters of 8 or 16 CTAs, the field held in distributed shared memory, where the grid has it:
 * 256 × 256 — each timed once, their column and wave slots report -1), column-pass variant (0, 1, 2: 4, 8, 16 columns per CTA;
 * 3, 4: 8 columns, one thread per slot and component, with a register budget for three or two
 * CTAs per SM; 5: 8 columns with a budget for four) and
 * wave variant (0: all columns in one launch per pass; 1, 2, 3: waves of 32, 64, 128 columns,
 * each wave's intermediate staying in L2) of an M̂ application are timed and the fastest is
 * kept in a process-wide table,
 * persisted in a text cache (OMB_TUNE_CACHE, else $XDG_CACHE_HOME/omb200/tiles.txt, else
 * ~/.cache/omb200/tiles.txt).  omb_batch_create tunes every grid it has not seen (unless
 * omb_ctx_set_autotune(ctx, 0)), outside the timed solve.
 * --------------------------------------------------------------------------------- */

/* Tune one grid now for `ncol`-column applications on 64 units; the chosen variants and, if
 * `seconds` is not NULL, the 168 timings (row-major over row, column, wave variant; -1 for
 * combinations not timed). */
int omb_autotune(omb_ctx* ctx, const omb_grid* grid, int32_t ncol, int32_t* row_variant, int32_t* col_variant,
                 int32_t* wave_variant, double* seconds);
int omb_ctx_set_autotune(omb_ctx* ctx, int32_t enabled);
/* Host-side table access (no device work). */
int omb_tune_set(const char* device_name, int32_t Nx, int32_t Ny, int32_t row_variant, int32_t col_variant,
                 int32_t wave_variant);
int omb_tune_get(const char* device_name, int32_t Nx, int32_t Ny, int32_t* row_variant, int32_t* col_variant,
                 int32_t* wave_variant);
int omb_tune_clear(void);
/* Write / merge the table to / from a cache file (NULL: the default path); malformed lines
 * are skipped; *entries (may be NULL) receives the number of lines read. */
int omb_tune_save(const char* path);
int omb_tune_load(const char* path, int32_t* entries);

/* ---------------------------------------------------------------------------------
 * Eigensolves
 * --------------------------------------------------------------------------------- */

/* Newton strategy for solve_k */
#define OMB_NEWTON_INNER 0 /* Newton steps inside the eigensolver iteration (default)     */
#define OMB_NEWTON_OUTER 1 /* the reference loop: bands one after another, a full block
                              eigensolve per Newton step (the plain baseline)            */

/* Warm starts across the instances of one batch (no counterpart in the reference, whose
 * callers pass each solve's result as the next one's kguess/Hguess by hand) */
#define OMB_WARM_NONE 0  /* every instance starts from its own guesses or at random      */
#define OMB_WARM_SWEEP 1 /* instances sharing one epsinv array (same pointer) and grid form
                            a frequency sweep: the one nearest the group's mean ω is solved
                            first, the others start from its eigenvectors (on the device)
                            with k_b + (ω − ω_a)·2ω_a/(∂ω²/∂k)_b per band; instances with
                            their own Hguess or kguess_bands keep them                  */
#define OMB_WARM_CELLS 2 /* instances with the same ω and grid form a stack of cells (an
                            eigenmode-expansion cross-section series): the middle one is
                            solved first and the others start from its eigenvectors and
                            per-band k — the batched form of the reference's per-cell warm
                            start (lib/EigenmodeExpansion/src/eme.jl:58-72)             */
#define OMB_WARM_LEARNED 3 /* instances without guesses of their own on 128², 256² or 512² grids start
                            from the learned network attached to the context
                            (omb_ctx_set_warmstart): its (Hx, Hy) fields of bands 0..3 projected
                            on the plane waves at k = n_eff·ω, and those k as Newton starts;
                            the solve itself is unchanged (same tolerances)            */
#define OMB_WARM_SWEEP_LEARNED 4 /* OMB_WARM_SWEEP whose first-solved instances (each sweep's
                            anchor, and instances in no sweep) start from the learned network
                            as with OMB_WARM_LEARNED                                    */

typedef struct {
  double k_tol;           /* Newton tolerance on |Δk|                       (1e-8) */
  double eig_tol;         /* residual ‖M̂h − ω²h‖ of a unit eigenvector       (1e-8) */
  int32_t max_eigsolves;  /* Newton steps per band                            (60)   */
  int32_t maxiter;        /* eigensolver iterations per band and phase       (1000)  */
  int32_t precision;      /* OMB_PREC_MIXED / OMB_PREC_FP64 / OMB_PREC_FP32   (MIXED)*/
  int32_t preconditioner; /* OMB_OP_P_DIAG or OMB_OP_P (MPB-style)          (DIAG) */
  int32_t newton;         /* OMB_NEWTON_INNER or OMB_NEWTON_OUTER             (INNER)*/
  int32_t canonicalize;   /* 1: rotate each eigenvector so the largest E component is
                             real and positive (fields.jl:258-260)           (1)    */
  uint64_t seed;          /* random start blocks                              (0)    */
  int32_t guard_bands;    /* extra block columns beyond the wanted bands of a
                             Newton track (OMB_NEWTON_INNER)                  (1)    */
  int32_t warm_start;     /* OMB_WARM_NONE / _SWEEP / _CELLS / _LEARNED /
                             _SWEEP_LEARNED                                   (NONE) */
} omb_options;

/* One solve_k problem: the lowest `nev` guided modes of one cell at frequency ω. */
typedef struct {
  omb_grid grid;
  double omega;            /* ω = 1/λ (μm⁻¹)                                         */
  const double* epsinv;    /* (3, 3, Nx, Ny) Float64                                 */
  int32_t nev;             /* bands (≤ 10)                                           */
  double kguess;           /* Newton start; ≤ 0 → k_guess(ω, ε⁻¹) = ω/√(min diag ε⁻¹) */
  const double* Hguess;    /* NULL or `nguess` warm-start columns (2, Nx, Ny)        */
  int32_t nguess;
  const double* kguess_bands; /* NULL or nev per-band Newton starts (override kguess) */
} omb_instance;

/* Caller-owned outputs of one instance; any pointer but kmags may be NULL. */
typedef struct {
  double* kmags;           /* nev                                                    */
  double* evecs;           /* nev columns ComplexF64 (2, Nx, Ny): 4·Nx·Ny·nev doubles */
  double* residuals;       /* nev: ‖M̂h − λh‖ at the last eigensolve                 */
  double* dw2dk;           /* nev: ∂ω²/∂k = 2⟨h|∂M̂/∂k|h⟩ (group index n_g = 2ω/dw2dk) */
  int32_t* status;         /* nev: OMB_OK or the band's error code                   */
  int32_t* iterations;     /* nev: eigensolver iterations                            */
  int32_t* newton_steps;   /* nev                                                    */
} omb_result;

/* Fill `opt` with the defaults shown above. */
int omb_options_default(omb_options* opt);

/* Solve `n_inst` independent problems in one batched device run.
 * Replaces solve_k(ω, ε⁻¹, grid, solver; nev, max_eigsolves, maxiter, k_tol, eig_tol,
 * kguess, Hguess) (lib/MaxwellEigenmodes/src/solve.jl:182-196; the GPU backend
 * src/solvers/gpu.jl:213-242).  kmags[b] is the band-b propagation constant after the
 * final Newton update; evecs are unit-norm and phase-canonicalised.  Returns OMB_OK when
 * every band converged, else OMB_ERR_NOT_CONVERGED (results are still written, per-band
 * status says which), or another error code. */
int omb_solve_k(omb_ctx* ctx, const omb_instance* inst, int n_inst, const omb_options* opt,
                omb_result* out);

/* Lowest `nev` eigenpairs (ω², h) of M̂(k) for one cell.
 * Replaces solve_ω²(ms, solver; nev, maxiter, tol) (src/solve.jl:38-63) and
 * solve_ω²(ms, ::GPUSolver) (src/solvers/gpu.jl:201-211).  evecs may be NULL; Hguess is
 * NULL or `nguess` warm-start columns. */
int omb_solve_omega2(omb_ctx* ctx, const omb_grid* grid, double k, const double* epsinv, int nev,
                     const double* Hguess, int nguess, const omb_options* opt, double* evals,
                     double* evecs, double* residuals, int32_t* status);

/* Propagation constants and Bloch modes of the lowest `nev` bands of a cell periodic along z
 * with period Λ = grid->Dz, at frequency ω.  Replaces solve_k_periodic(ω, ε⁻¹, Λ, grid,
 * solver; nev) (lib/MaxwellEigenmodes/src/grads/period.jl:108-112): solve_k on the grid whose
 * z-extent is Λ, here with the same device iteration as omb_solve_k (inner Newton, mixed /
 * FP64 precision, phase-canonicalised unit eigenvectors).  epsinv (3, 3, Nx, Ny, Nz), evecs
 * nev columns ComplexF64 (2, Nx, Ny, Nz); kguess ≤ 0 → ω/√(min diag ε⁻¹); any output but
 * kmags may be NULL. */
int omb_solve_k_periodic(omb_ctx* ctx, const omb_grid3* grid, double omega, const double* epsinv, int nev,
                         double kguess, const omb_options* opt, double* kmags, double* evecs, double* residuals,
                         double* dw2dk, int32_t* status, int32_t* iterations);

/* Adjoint pull-back of one solve_k result: cotangents (k̄, ē) of (kmags, evecs) → ω̄ and
 * ε̄⁻¹ (and optionally ε̄ = ∂/∂ε).  Replaces the pullback closure of
 * rrule(solve_k, ω, ε⁻¹, grid, solver) (lib/MaxwellEigenmodes/src/solve.jl:213-289; GPU
 * variant src/solvers/gpu.jl:292-365).  kmags/evecs are solve_k's outputs (nev values,
 * nev columns (2, Nx, Ny) ComplexF64); kbar is NULL (zero) or nev values; evbar is NULL
 * (zero) or nev columns, an all-zero column standing for an AbstractZero band.
 * epsinv_bar receives (3, 3, Nx, Ny) with the summed (i,j)+(j,i) off-diagonal sensitivity
 * mirrored into both slots (the ε⁻¹_bar convention, src/grads/solve.jl:490-515); eps_bar,
 * if non-NULL, receives the same pulled through ε⁻¹ = inv(ε) per pixel
 * (−Yᵀ ε̄⁻¹ Yᵀ, src/grads/linalg.jl:40-47).  iterations (NULL or nev) receives the adjoint
 * solver's iteration count per band. */
int omb_pullback(omb_ctx* ctx, const omb_grid* grid, double omega, const double* epsinv, int nev,
                 const double* kmags, const double* evecs, const double* kbar, const double* evbar,
                 const omb_options* opt, double* omega_bar, double* epsinv_bar, double* eps_bar,
                 int32_t* iterations);

/* The same pull-back for omb_solve_k_periodic's outputs on a z-periodic cell (Nz ≥ 8):
 * cotangents (k̄, ē) → ω̄, ε̄⁻¹ (3, 3, Nx, Ny, Nz) and the period cotangent Λ̄ (L_bar, may be
 * NULL).  Replaces _solve_k_period_grads (lib/MaxwellEigenmodes/src/grads/period.jl:136-200):
 * Λ̄ = Σ_bands [Λ̄ₕ + (k̄ + k̄ₕ)·(−∂ω²/∂Λ ÷ ∂ω²/∂k)], ∂ω²/∂Λ = 2⟨h|∂M̂/∂Λ|h⟩ with the ẑ× action
 * weighted by g_z/Λ per plane wave (HMₖH_weighted, period.jl:69-74), and Λ̄ₕ the same
 * per-plane-wave terms as the eigenvector channel's k̄ₕ weighted by g_z/Λ (period.jl:171-175). */
int omb_pullback_periodic(omb_ctx* ctx, const omb_grid3* grid, double omega, const double* epsinv, int nev,
                          const double* kmags, const double* evecs, const double* kbar, const double* evbar,
                          const omb_options* opt, double* omega_bar, double* epsinv_bar, double* L_bar,
                          int32_t* iterations);

/* ---------------------------------------------------------------------------------
 * Staged batches: the same solve as omb_solve_k split into its host→device, device and
 * device→host parts, so the device part can run (and be timed) with its inputs resident.
 * omb_solve_k(...) ≡ create + run + results + destroy.  No reference counterpart: the
 * reference has no batch call (its callers loop over solve_k).
 * --------------------------------------------------------------------------------- */

typedef struct omb_batch omb_batch;

typedef struct {
  int64_t graph_launches;  /* CUDA graph replays (two eigensolver iterations each)      */
  int64_t kernel_launches; /* library kernels launched (graph nodes counted per replay) */
  int64_t h2d_bytes;       /* host→device bytes of the inputs                           */
  int64_t d2h_bytes;       /* device→host bytes of the results                          */
  int32_t tracks;          /* Newton/eigensolve units                                   */
  int32_t max_iterations;  /* largest iteration count of any unit                      */
  double run_seconds;      /* device time of the last omb_batch_run (CUDA events)       */
} omb_stats;

/* Validate and upload `n_inst` problems (ε⁻¹ and any warm starts are copied). */
int omb_batch_create(omb_ctx* ctx, const omb_instance* inst, int n_inst, const omb_options* opt,
                     omb_batch** out);
/* Run the whole solve on the device (may be called again; each run starts afresh). */
int omb_batch_run(omb_batch* b);
/* Copy instance results to the caller's buffers (canonicalising if requested).  Returns
 * OMB_OK or OMB_ERR_NOT_CONVERGED like omb_solve_k. */
int omb_batch_results(omb_batch* b, omb_result* out);
int omb_batch_stats(const omb_batch* b, omb_stats* out);
int omb_batch_destroy(omb_batch* b);

/* Mean device seconds of one application of `op` to `ncol` columns on each of `nbatch`
 * copies of the cell, over `reps` back-to-back applications on device-resident data
 * (CUDA events on the library's stream, after 3 warm-up applications).  The inputs
 * (nbatch·ncol columns plus ε⁻¹ per copy) are allocated once, so choose nbatch to exceed
 * the 126 MB L2 when timing against HBM bandwidth.  No reference counterpart
 * (measurement support). */
int omb_profile_apply(omb_ctx* ctx, int op, int precision, const omb_grid* grid, double k,
                      const double* epsinv, int ncol, int nbatch, int reps, double* seconds);

/* The eigensolver's Gram products on caller blocks: G = ZᴴZ and S = ZᴴAZ of `n` columns
 * (≤ 36) of n2 complex rows (host ComplexF64, column after column), computed by the same
 * streaming kernel as a LOBPCG iteration (n2 even, as every solver vector is) in FP32
 * (operands rounded to FP32, products summed
 * over at most 16 rows per thread, or one tile's share, and those sums compensated by
 * two-sum) or FP64.  G and S receive n×n ComplexF64,
 * column-major.  No reference counterpart (accuracy check of the FP32 reductions; the
 * reference's products are BLAS calls, ME/src/solvers/dftk.jl:129-132). */
int omb_gram_blocks(omb_ctx* ctx, int precision, int64_t n2, int32_t n, const double* Z, const double* AZ,
                    double* G, double* S);

/* ---------------------------------------------------------------------------------
 * Kottke sub-pixel smoothing (the solver's input generator, lib/DielectricSmoothing)
 * --------------------------------------------------------------------------------- */

typedef struct omb_smoothing_plan omb_smoothing_plan;

/* fill fraction of an interface pixel */
#define OMB_FILL_PLANE 0 /* the reference's volfrac: the voxel's area on the inner side of the
                            tangent line through the nearest surface point              */
#define OMB_FILL_EXACT 1 /* the exact area of polygon ∩ voxel                            */

/* pixel kinds (SmoothingPlan's _PLAN_UNIFORM/_INTERFACE/_MULTI) */
#define OMB_PIXEL_UNIFORM 1
#define OMB_PIXEL_INTERFACE 2
#define OMB_PIXEL_MULTI 3

/* Frequency-independent geometry pass on the device.  Replaces
 * smoothing_plan(shapes, minds, grid) (lib/DielectricSmoothing/src/smoothing_plan.jl:70-100):
 * corners (src/grid.jl:271-312), corner_sinds/proc_sinds (src/smooth.jl:24-72) and the
 * interface geometry of smooth_ε_single! (src/smooth.jl:80-121).
 *   shapes : `nshapes` convex polygons in priority order (the first containing a point
 *            wins); polygon s has nverts[s] ∈ [3, 64] vertices, stored one polygon after
 *            another in `verts` as (x, y) pairs (either orientation)
 *   minds  : nshapes + 1 material columns in [0, 255] (0-based), the background last
 * Blocks until the plan is built. */
int omb_smoothing_plan_create(omb_ctx* ctx, const omb_grid* grid, int32_t nshapes, const int32_t* nverts,
                              const double* verts, const int32_t* minds, int32_t fill_rule,
                              omb_smoothing_plan** out);

/* Contents of a plan, pixels in corners(grid) order (x fastest); any pointer may be NULL.
 *   counts[3]      : uniform, interface and multi-material pixels
 *   kind[N]        : OMB_PIXEL_*
 *   mats[4N]       : material columns (uniform: [a]; interface: [a, b]; multi: the four
 *                    corners' columns; unused entries −1)
 *   rvol[N]        : fill fraction of material a (interface pixels; else 0)
 *   normal[2N]     : outward interface normal (nx, ny) of the higher-priority shape */
int omb_smoothing_plan_query(const omb_smoothing_plan* plan, int64_t* counts, uint8_t* kind, int32_t* mats,
                             double* rvol, double* normal);

/* Material pass for `nsets` material tables at once (e.g. one per frequency).  Replaces
 * smooth_ε(plan, mat_vals) (smoothing_plan.jl:120-140; per pixel the three branches of
 * smooth_ε_single!, with the dispersive Kottke kernel εₑ_∂ωεₑ_∂²ωεₑ of src/kottke.jl:218-268)
 * and, fused, sliceinv_3x3 of its ε slice (lib/MaxwellEigenmodes/src/linalg.jl:126-147).
 *   mat_vals : Float64 (27, nmat, nsets); column = vcat(vec(ε), vec(∂ωε), vec(∂²ωε))
 *   eps      : Float64 (3, 3, 3, Nx, Ny, nsets) or NULL
 *   epsinv   : Float64 (3, 3, Nx, Ny, nsets) or NULL — the solver's ε⁻¹ input */
int omb_smooth_eps(omb_smoothing_plan* plan, const double* mat_vals, int32_t nmat, int32_t nsets,
                   double* eps, double* epsinv);

/* As omb_smooth_eps with device outputs, stream-ordered on `stream` (a cudaStream_t, or
 * NULL for the context's stream); returns once the work is queued. */
int omb_smooth_eps_device(omb_smoothing_plan* plan, const double* mat_vals, int32_t nmat, int32_t nsets,
                          double* d_eps, double* d_epsinv, void* stream);

/* Material-data VJP of omb_smooth_eps's 27-value output: mat_vals_bar (27, nmat, nsets) =
 * ∂⟨eps_bar, smooth_ε(plan, mat_vals)⟩/∂mat_vals for eps_bar (3, 3, 3, Nx, Ny, nsets).
 * Replaces _plan_vjp / rrule(smooth_ε, plan, mat_vals) (smoothing_plan.jl:160-218): uniform
 * pixels pass their cotangent to their column, multi-material pixels a quarter to each corner
 * column, interface pixels Jᵀȳ of the Taylor-jet Kottke kernel (forward derivatives along
 * each of the two columns' 54 entries, one device thread each). */
int omb_smooth_eps_vjp(omb_smoothing_plan* plan, const double* mat_vals, int32_t nmat, int32_t nsets,
                       const double* eps_bar, double* mat_vals_bar);

/* Scalar material property (e.g. the Kerr coefficient n₂) on the plan's pixels: out (Nx, Ny)
 * from vals[nmat] — uniform pixels take their material's value, interface pixels
 * r·v_a + (1 − r)·v_b, multi-material pixels the mean of their four corners' values.
 * Replaces smooth_scalar / smooth_scalar_single (lib/DielectricSmoothing/src/smooth.jl:232-263)
 * on a plan's geometry. */
int omb_smooth_scalar(omb_smoothing_plan* plan, const double* vals, int32_t nmat, double* out);

/* Waits for the device, then frees the plan. */
int omb_smoothing_plan_destroy(omb_smoothing_plan* plan);

/* ---------------------------------------------------------------------------------
 * Learned warm start (no reference counterpart: the reference starts every solve from
 * random blocks or the caller's Hguess, lib/MaxwellEigenmodes/src/solve.jl:201-210).
 * A six-layer BF16 convolutional network on the tensor cores maps the ε⁻¹ map and ω of a
 * 128², 256² or 512² cross-section to initial (Hx, Hy) fields and effective indices of the four
 * lowest bands.  Device pointers throughout; calls are ordered on the context's stream.
 * --------------------------------------------------------------------------------- */

typedef struct omb_warmstart omb_warmstart;

/* The network's matrix product on the tensor cores (tcgen05.mma, TMA-loaded operands, FP32
 * accumulation in tensor memory): D[M×N] = A[M×K]·B[N×K]ᵀ (+ bias[N], then ReLU if relu),
 * A and B row-major BF16 device matrices (K a multiple of 64, 16-byte aligned), D row-major
 * with leading dimension ldd.  epi: 0 store FP32, 1 store BF16, 2 add atomically into FP32 D
 * (needed when splits > 1, the K range being cut over `splits` CTAs per tile).  Waits for
 * the context's stream. */
int omb_tc_gemm(omb_ctx* ctx, const void* d_A, const void* d_B, void* d_D, int32_t M, int32_t N, int32_t K,
                int64_t ldd, const float* d_bias, int32_t relu, int32_t epi, int32_t splits);

/* Network with He-initialised weights (seeded) and buffers for up to batch_cap images. */
int omb_warmstart_create(omb_ctx* ctx, int32_t batch_cap, uint64_t seed, omb_warmstart** out);
int omb_warmstart_destroy(omb_warmstart* ws);
/* Attach (or, with NULL, detach) the network OMB_WARM_LEARNED uses on this context; the
 * context does not own it (destroying the network detaches it). */
int omb_ctx_set_warmstart(omb_ctx* ctx, omb_warmstart* ws);
/* Number of parameters; get/set exchange them as FP32, layer by layer: the weights as
 * [cout × 9·cin] row-major (column = tap·cin + c, taps row-major over the 3×3 window),
 * then the cout biases. */
int64_t omb_warmstart_num_params(void);
int omb_warmstart_get_params(omb_warmstart* ws, float* host);
int omb_warmstart_set_params(omb_warmstart* ws, const float* host);
/* One input image (128×128×8 BF16, NHWC) from a device ε⁻¹ (3, 3, Nx, Ny) Float64 array of a
 * 128², 256² or 512² grid (pixels averaged down to 128²) and ω, on `stream` (NULL: the
 * context's stream). */
int omb_warmstart_features(omb_warmstart* ws, const double* d_epsinv, int32_t Nx, int32_t Ny, double omega,
                           void* d_feat, void* stream);
/* Network output for `batch` images: d_out [batch·64·64 × 16] FP32, channels 2b, 2b+1 the
 * (Hx, Hy) field of band b, 8+b its n_eff map (the band's n_eff is its mean). */
int omb_warmstart_forward(omb_warmstart* ws, const void* d_feat, int32_t batch, float* d_out);
/* One training step on `batch` images with targets d_tfield [batch·64·64 × 8] FP32 (the
 * bands' real-space (Hx, Hy), unit RMS per band) and d_tneff [batch × 4]: forward, loss,
 * backward and (update != 0) an Adam step with learning rate lr.  *loss (host, may be NULL)
 * receives the batch loss; grads (host, may be NULL) the parameter gradients in the
 * get_params layout. */
int omb_warmstart_train_step(omb_warmstart* ws, const void* d_feat, const float* d_tfield, const float* d_tneff,
                             int32_t batch, float lr, int32_t update, float* loss, float* grads);

#ifdef __cplusplus
}
#endif

#endif /* OMB200_H */
