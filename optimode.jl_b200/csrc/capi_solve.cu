// Entry points for eigensolves: omb_solve_k, omb_solve_omega2, the staged omb_batch_*
// calls and omb_options_default.
#include <cmath>
#include <complex>
#include <memory>
#include <vector>

#include "engine.h"

struct omb_batch {
  omb_ctx* ctx = nullptr;
  std::vector<omb_instance> inst;
  std::vector<std::vector<double>> guesses;  // copies of the warm starts
  std::vector<omb::Problem> probs;
  omb::SolveOptions so;
  bool canon = true;
  std::unique_ptr<omb::Engine> engine;
  std::vector<std::pair<int, int>> who;  // track → (instance, first band)
  int64_t h2d = 0, d2h = 0;
  double run_seconds = 0;
};

namespace omb {

static int options_from(const omb_options* o, SolveOptions& so) {
  omb_options d;
  omb_options_default(&d);
  if (!o) o = &d;
  if (!(o->k_tol > 0) || !(o->eig_tol > 0)) return fail(OMB_ERR_INVALID_ARG, "k_tol and eig_tol must be positive");
  if (o->max_eigsolves <= 0 || o->maxiter <= 0)
    return fail(OMB_ERR_INVALID_ARG, "max_eigsolves and maxiter must be positive");
  if (o->precision != OMB_PREC_FP32 && o->precision != OMB_PREC_FP64 && o->precision != OMB_PREC_MIXED)
    return fail(OMB_ERR_INVALID_ARG, "unknown precision");
  if (o->preconditioner != OMB_OP_P && o->preconditioner != OMB_OP_P_DIAG)
    return fail(OMB_ERR_INVALID_ARG, "preconditioner must be OMB_OP_P or OMB_OP_P_DIAG");
  if (o->newton != OMB_NEWTON_INNER && o->newton != OMB_NEWTON_OUTER)
    return fail(OMB_ERR_INVALID_ARG, "newton must be OMB_NEWTON_INNER or OMB_NEWTON_OUTER");
  so.tol = o->eig_tol;
  so.k_tol = o->k_tol;
  so.max_newton = o->max_eigsolves;
  so.maxiter = o->maxiter;
  so.precision = o->precision;
  so.prec_diag = o->preconditioner == OMB_OP_P_DIAG;
  so.newton_mode = o->newton == OMB_NEWTON_OUTER ? MODE_NEWTON_OUTER : MODE_NEWTON_INNER;
  so.seed = o->seed;
  if (o->guard_bands < 0 || o->guard_bands > 4) return fail(OMB_ERR_INVALID_ARG, "guard_bands must be in 0..4");
  so.guard = o->guard_bands;
  return OMB_OK;
}

static int status_code(int ts) {
  switch (ts) {
    case TS_CONVERGED: return OMB_OK;
    case TS_ORTHO: return OMB_ERR_ORTHO_FAIL;
    case TS_NAN: return OMB_ERR_NAN;
    default: return OMB_ERR_NOT_CONVERGED;
  }
}

// Bytes a Problem upload moves host→device (FP32 float4+float2, FP64 3×double2, ε_ave ×2).
static int64_t problem_bytes(const Problem& P) { return (int64_t)P.N() * (16 + 8 + 48 + 4 + 8); }

}  // namespace omb

using namespace omb;

extern "C" {

int omb_options_default(omb_options* o) {
  if (!o) return fail(OMB_ERR_INVALID_ARG, "opt is NULL");
  o->k_tol = 1e-8;
  o->eig_tol = 1e-8;
  o->max_eigsolves = 60;
  o->maxiter = 300;
  o->precision = OMB_PREC_MIXED;
  o->preconditioner = OMB_OP_P_DIAG;
  o->newton = OMB_NEWTON_INNER;
  o->canonicalize = 1;
  o->seed = 0;
  o->guard_bands = 1;
  return OMB_OK;
}

int omb_batch_create(omb_ctx* ctx, const omb_instance* inst, int n_inst, const omb_options* opt, omb_batch** out) {
  if (!out) return fail(OMB_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (!ctx) return fail(OMB_ERR_INVALID_ARG, "ctx is NULL");
  if (n_inst <= 0 || !inst) return fail(OMB_ERR_INVALID_ARG, "need n_inst > 0 and non-NULL inst");
  std::unique_ptr<omb_batch> b(new omb_batch());
  int rc = options_from(opt, b->so);
  if (rc) return rc;
  b->canon = opt ? opt->canonicalize != 0 : true;
  b->ctx = ctx;
  OMB_CU(cudaSetDevice(ctx->device));
  b->inst.assign(inst, inst + n_inst);
  b->probs.resize(n_inst);
  b->guesses.resize(n_inst);
  for (int i = 0; i < n_inst; ++i) {
    omb_instance& I = b->inst[i];
    if (I.nev <= 0 || I.nev + b->so.guard > MMAX)
      return fail(OMB_ERR_INVALID_ARG, "nev + guard_bands must be in 2..12");
    if (!(I.omega > 0) || !std::isfinite(I.omega)) return fail(OMB_ERR_INVALID_ARG, "omega must be finite and positive");
    if (I.nguess < 0 || (I.nguess > 0 && !I.Hguess)) return fail(OMB_ERR_INVALID_ARG, "bad Hguess/nguess");
    rc = upload_problem(ctx, &I.grid, I.epsinv, b->probs[i]);
    if (rc) return rc;
    b->h2d += problem_bytes(b->probs[i]);
    if (2 * (long long)b->probs[i].N() < 3 * (I.nev + 2))
      return fail(OMB_ERR_INVALID_ARG, "grid too small for the requested bands");
    if (I.nguess > 0) {
      const size_t n = 4 * b->probs[i].N() * (size_t)I.nguess;
      b->guesses[i].assign(I.Hguess, I.Hguess + n);
      I.Hguess = b->guesses[i].data();
      b->h2d += (int64_t)(n * sizeof(double));
    }
    I.epsinv = nullptr;  // uploaded; the caller's array is not kept
  }
  *out = b.release();
  return OMB_OK;
}

int omb_batch_run(omb_batch* b) {
  if (!b) return fail(OMB_ERR_INVALID_ARG, "batch is NULL");
  omb_ctx* ctx = b->ctx;
  OMB_CU(cudaSetDevice(ctx->device));
  std::vector<TrackSpec> tracks;
  b->who.clear();
  const int n_inst = (int)b->inst.size();
  for (int i = 0; i < n_inst; ++i) {
    const omb_instance& I = b->inst[i];
    const double k0 = I.kguess > 0 ? I.kguess : I.omega * std::sqrt(1.0 / b->probs[i].min_diag);
    if (b->so.newton_mode == MODE_NEWTON_INNER) {
      // one Newton track per band: block = bands 0..b plus one guard column
      for (int band = 0; band < I.nev; ++band) {
        TrackSpec ts;
        ts.prob = i; ts.band = band; ts.nbands = 1; ts.M = band + 1 + b->so.guard; ts.need = band + 1;
        ts.mode = MODE_NEWTON_INNER;
        ts.omega2 = I.omega * I.omega; ts.k0 = k0;
        ts.guess = I.Hguess; ts.nguess = I.nguess;
        tracks.push_back(ts);
        b->who.push_back({i, band});
      }
    } else {
      // the reference loop: bands in turn on one block of nev columns
      TrackSpec ts;
      ts.prob = i; ts.band = 0; ts.nbands = I.nev; ts.M = I.nev; ts.need = I.nev;
      ts.mode = MODE_NEWTON_OUTER;
      ts.omega2 = I.omega * I.omega; ts.k0 = k0;
      ts.guess = I.Hguess; ts.nguess = I.nguess;
      tracks.push_back(ts);
      b->who.push_back({i, 0});
    }
  }
  cudaEvent_t e0, e1;
  OMB_CU(cudaEventCreate(&e0));
  OMB_CU(cudaEventCreate(&e1));
  OMB_CU(cudaEventRecord(e0, ctx->stream));
  b->engine.reset(new Engine(ctx, &b->probs, tracks, b->so));
  int rc = b->engine->run();
  cudaEventRecord(e1, ctx->stream);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->run_seconds = ms * 1e-3;
  return rc;
}

int omb_batch_results(omb_batch* b, omb_result* out) {
  if (!b || !out) return fail(OMB_ERR_INVALID_ARG, "batch and out must be non-NULL");
  if (!b->engine) return fail(OMB_ERR_INVALID_ARG, "omb_batch_run has not been called");
  OMB_CU(cudaSetDevice(b->ctx->device));
  Engine& E = *b->engine;
  bool all_ok = true;
  b->d2h = 0;
  for (size_t t = 0; t < b->who.size(); ++t) {
    const int i = b->who[t].first, band0 = b->who[t].second;
    const omb_instance& I = b->inst[i];
    omb_result& r = out[i];
    if (!r.kmags) return fail(OMB_ERR_INVALID_ARG, "result kmags is NULL");
    const size_t n2 = 2 * b->probs[i].N();
    const int nb = b->so.newton_mode == MODE_NEWTON_INNER ? 1 : I.nev;
    for (int rb = 0; rb < nb; ++rb) {
      const int band = band0 + rb;
      const TrackState& s = E.result_state((int)t, rb);
      r.kmags[band] = s.k;
      if (r.residuals) r.residuals[band] = s.resid[band];
      if (r.dw2dk) r.dw2dk[band] = 2.0 * s.hmkh;
      if (r.status) r.status[band] = status_code(s.status);
      if (r.iterations) r.iterations[band] = s.iter;
      if (r.newton_steps) r.newton_steps[band] = s.newton_steps;
      b->d2h += 8 * 4 + 4 * 3;
      all_ok = all_ok && s.status == TS_CONVERGED;
      if (r.evecs) {
        double* v = r.evecs + 2 * n2 * band;
        int rc = E.fetch_result((int)t, rb, v);
        if (rc) return rc;
        b->d2h += (int64_t)(2 * n2 * sizeof(double));
        if (b->canon) {
          long long idx;
          double re, im;
          rc = E.result_efield_argmax((int)t, rb, &idx, &re, &im);
          if (rc) return rc;
          b->d2h += 24;
          const std::complex<double> ph = std::polar(1.0, -std::atan2(im, re));
          for (size_t q = 0; q < n2; ++q) {
            const std::complex<double> w = std::complex<double>(v[2 * q], v[2 * q + 1]) * ph;
            v[2 * q] = w.real();
            v[2 * q + 1] = w.imag();
          }
        }
      }
    }
  }
  if (!all_ok) return fail(OMB_ERR_NOT_CONVERGED, "one or more bands did not converge (see the per-band status)");
  return OMB_OK;
}

int omb_batch_stats(const omb_batch* b, omb_stats* out) {
  if (!b || !out) return fail(OMB_ERR_INVALID_ARG, "batch and out must be non-NULL");
  out->graph_launches = b->engine ? b->engine->graph_launches() : 0;
  out->kernel_launches = b->engine ? b->engine->kernel_launches() : 0;
  out->h2d_bytes = b->h2d;
  out->d2h_bytes = b->d2h;
  out->tracks = (int32_t)b->who.size();
  out->max_iterations = b->engine ? b->engine->max_iterations() : 0;
  out->run_seconds = b->run_seconds;
  return OMB_OK;
}

int omb_batch_destroy(omb_batch* b) {
  if (!b) return OMB_OK;
  cudaSetDevice(b->ctx->device);
  delete b;
  return OMB_OK;
}

int omb_solve_k(omb_ctx* ctx, const omb_instance* inst, int n_inst, const omb_options* opt, omb_result* out) {
  if (!out) return fail(OMB_ERR_INVALID_ARG, "out is NULL");
  omb_batch* b = nullptr;
  int rc = omb_batch_create(ctx, inst, n_inst, opt, &b);
  if (rc) return rc;
  rc = omb_batch_run(b);
  if (!rc) rc = omb_batch_results(b, out);
  const std::string msg = rc ? std::string(omb_last_error()) : std::string();
  omb_batch_destroy(b);
  if (rc) set_error(msg);
  return rc;
}

int omb_solve_omega2(omb_ctx* ctx, const omb_grid* grid, double k, const double* epsinv, int nev,
                     const double* Hguess, int nguess, const omb_options* opt, double* evals,
                     double* evecs, double* residuals, int32_t* status) {
  if (!ctx) return fail(OMB_ERR_INVALID_ARG, "ctx is NULL");
  if (nev <= 0 || nev > MMAX - 1) return fail(OMB_ERR_INVALID_ARG, "nev must be in 1..11");
  if (!(k > 0) || !std::isfinite(k)) return fail(OMB_ERR_INVALID_ARG, "k must be finite and positive");
  if (!evals) return fail(OMB_ERR_INVALID_ARG, "evals is NULL");
  if (nguess < 0 || (nguess > 0 && !Hguess)) return fail(OMB_ERR_INVALID_ARG, "bad Hguess/nguess");
  SolveOptions so;
  int rc = options_from(opt, so);
  if (rc) return rc;
  so.newton_mode = MODE_OMEGA2;
  OMB_CU(cudaSetDevice(ctx->device));
  std::vector<Problem> probs(1);
  rc = upload_problem(ctx, grid, epsinv, probs[0]);
  if (rc) return rc;
  TrackSpec ts;
  ts.prob = 0; ts.band = 0; ts.M = nev + 1; ts.need = nev; ts.mode = MODE_OMEGA2;
  ts.k0 = k; ts.guess = Hguess; ts.nguess = nguess;
  Engine E(ctx, &probs, {ts}, so);
  rc = E.run();
  if (rc) return rc;
  const TrackState& s = E.result_state(0, 0);
  const size_t n2 = 2 * probs[0].N();
  for (int b = 0; b < nev; ++b) {
    evals[b] = s.lam[b];
    if (residuals) residuals[b] = s.resid[b];
    if (status) status[b] = status_code(s.status);
    if (evecs) {
      rc = E.fetch_block_column(0, b, evecs + 2 * n2 * b);
      if (rc) return rc;
    }
  }
  if (s.status != TS_CONVERGED) return fail(OMB_ERR_NOT_CONVERGED, "solve_omega2 did not converge");
  return OMB_OK;
}

}  // extern "C"
