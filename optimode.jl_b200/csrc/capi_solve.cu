// Entry points for eigensolves: omb_solve_k, omb_solve_omega2, the staged omb_batch_*
// calls and omb_options_default.
#include <cmath>
#include <complex>
#include <memory>
#include <vector>

#include "engine.h"
#include "ops.h"
#include "warmstart.h"

struct omb_batch {
  struct Who { int inst, band0, eng, track; };  // a track's instance, first band, engine, index
  omb_ctx* ctx = nullptr;
  std::vector<omb_instance> inst;
  std::vector<const double*> src_eps;          // the caller's ε⁻¹ pointers (sweep groups)
  std::vector<std::vector<double>> guesses;    // copies of the warm starts
  std::vector<std::vector<double>> kbands;     // copies of the per-band k guesses
  std::vector<omb::Problem> probs;             // distinct uploaded cells
  std::vector<int> pidx;                        // instance → its cell in probs
  omb::SolveOptions so;
  bool canon = true;
  int warm = OMB_WARM_NONE;
  std::vector<std::unique_ptr<omb::Engine>> engines;  // one per stage
  omb::DevBuf<double2> learned;                      // learned starting columns (OMB_WARM_LEARNED)
  int learned_instances = 0;
  std::vector<Who> who;
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
  if (o->warm_start < OMB_WARM_NONE || o->warm_start > OMB_WARM_SWEEP_LEARNED)
    return fail(OMB_ERR_INVALID_ARG,
                "warm_start must be OMB_WARM_NONE, _SWEEP, _CELLS, _LEARNED or _SWEEP_LEARNED");
  return OMB_OK;
}

// Tracks of one instance.  k0[b] is band b's Newton start; gdev (optional) holds device
// FP64 start columns for the block (bands 0..ngdev−1 of a solved neighbour).
static void add_tracks(omb_batch* b, int i, const std::vector<double>& k0, const double2* const* gdev, int ngdev,
                       int eng, std::vector<TrackSpec>& tracks) {
  const omb_instance& I = b->inst[i];
  auto fill = [&](TrackSpec& ts) {
    ts.omega2 = I.omega * I.omega;
    ts.guess = I.Hguess; ts.nguess = I.nguess;
    if (!I.Hguess && gdev) {
      ts.nguess_dev = std::min(ngdev, MMAX);
      for (int c = 0; c < ts.nguess_dev; ++c) ts.guess_dev[c] = gdev[c];
    }
  };
  if (b->so.newton_mode == MODE_NEWTON_INNER) {
    // one Newton track per band: block = bands 0..b plus the guard columns
    for (int band = 0; band < I.nev; ++band) {
      TrackSpec ts;
      ts.prob = b->pidx[i]; ts.band = band; ts.nbands = 1; ts.M = band + 1 + b->so.guard; ts.need = band + 1;
      ts.mode = MODE_NEWTON_INNER;
      ts.k0 = k0[band];
      fill(ts);
      b->who.push_back({i, band, eng, (int)tracks.size()});
      tracks.push_back(ts);
    }
  } else {
    // the reference loop: bands in turn on one block of nev columns
    TrackSpec ts;
    ts.prob = b->pidx[i]; ts.band = 0; ts.nbands = I.nev; ts.M = I.nev; ts.need = I.nev;
    ts.mode = MODE_NEWTON_OUTER;
    ts.k0 = k0[0];
    fill(ts);
    b->who.push_back({i, 0, eng, (int)tracks.size()});
    tracks.push_back(ts);
  }
}

// Newton starts of instance i from its own guesses (kguess_bands, kguess) or k_guess(ω, ε⁻¹).
static std::vector<double> own_k0(const omb_batch* b, int i) {
  const omb_instance& I = b->inst[i];
  const double base = I.kguess > 0 ? I.kguess : I.omega * std::sqrt(1.0 / b->probs[b->pidx[i]].min_diag);
  std::vector<double> k0(I.nev, base);
  if (!b->kbands[i].empty())
    for (int j = 0; j < I.nev; ++j)
      if (b->kbands[i][j] > 0) k0[j] = b->kbands[i][j];
  return k0;
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
  o->maxiter = 1000;
  o->precision = OMB_PREC_MIXED;
  o->preconditioner = OMB_OP_P_DIAG;
  o->newton = OMB_NEWTON_INNER;
  o->canonicalize = 1;
  o->seed = 0;
  o->guard_bands = 1;
  o->warm_start = OMB_WARM_NONE;
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
  b->warm = opt ? opt->warm_start : OMB_WARM_NONE;
  b->probs.reserve(n_inst);
  b->pidx.assign(n_inst, -1);
  b->guesses.resize(n_inst);
  b->kbands.resize(n_inst);
  b->src_eps.resize(n_inst);
  for (int i = 0; i < n_inst; ++i) {
    omb_instance& I = b->inst[i];
    if (I.nev <= 0 || I.nev + b->so.guard > MMAX)
      return fail(OMB_ERR_INVALID_ARG, "nev + guard_bands must be in 2..12");
    if (!(I.omega > 0) || !std::isfinite(I.omega)) return fail(OMB_ERR_INVALID_ARG, "omega must be finite and positive");
    if (I.nguess < 0 || (I.nguess > 0 && !I.Hguess)) return fail(OMB_ERR_INVALID_ARG, "bad Hguess/nguess");
    // instances that pass the same ε⁻¹ array for the same grid share one uploaded cell
    for (int j = 0; j < i && b->pidx[i] < 0; ++j) {
      const omb_instance& J = b->inst[j];
      if (b->src_eps[j] == I.epsinv && J.grid.Nx == I.grid.Nx && J.grid.Ny == I.grid.Ny &&
          J.grid.Dx == I.grid.Dx && J.grid.Dy == I.grid.Dy)
        b->pidx[i] = b->pidx[j];
    }
    if (b->pidx[i] < 0) {
      b->probs.emplace_back();
      rc = upload_problem(ctx, &I.grid, I.epsinv, b->probs.back());
      if (rc) return rc;
      b->pidx[i] = (int)b->probs.size() - 1;
      b->h2d += problem_bytes(b->probs.back());
    }
    const Problem& Pi = b->probs[b->pidx[i]];
    if (2 * (long long)Pi.N() < 3 * (I.nev + 2))
      return fail(OMB_ERR_INVALID_ARG, "grid too small for the requested bands");
    if (I.nguess > 0) {
      const size_t n = 4 * Pi.N() * (size_t)I.nguess;
      b->guesses[i].assign(I.Hguess, I.Hguess + n);
      I.Hguess = b->guesses[i].data();
      b->h2d += (int64_t)(n * sizeof(double));
    }
    if (I.kguess_bands) {
      b->kbands[i].assign(I.kguess_bands, I.kguess_bands + I.nev);
      I.kguess_bands = b->kbands[i].data();
    }
    b->src_eps[i] = I.epsinv;
    I.epsinv = nullptr;  // uploaded; the caller's array is not kept
  }
  // the FP32 operator tiles of every grid not tuned yet on this device (once per process and
  // device, kept in the tuning cache), outside the timed solve like the reference's FFTW plans
  if (ctx->autotune && b->so.precision != OMB_PREC_FP64)
    for (const Problem& P : b->probs)
      if (!tune_known(ctx->device, P.Nx, P.Ny)) {
        const omb_grid g{P.Nx, P.Ny, P.Dx, P.Dy};
        rc = autotune_grid(ctx, &g, 4, 64, nullptr, nullptr);
        if (rc) return rc;
      }
  *out = b.release();
  return OMB_OK;
}

int omb_batch_run(omb_batch* b) {
  if (!b) return fail(OMB_ERR_INVALID_ARG, "batch is NULL");
  omb_ctx* ctx = b->ctx;
  OMB_CU(cudaSetDevice(ctx->device));
  b->who.clear();
  b->engines.clear();
  const int n_inst = (int)b->inst.size();
  // warm-start groups (no warm start of their own, same grid and band count): a frequency
  // sweep shares one ε⁻¹ pointer; a stack of cells shares one ω
  std::vector<int> anchor(n_inst, -1);  // stage-2 instance → its stage-1 neighbour
  const bool learned = b->warm == OMB_WARM_LEARNED || b->warm == OMB_WARM_SWEEP_LEARNED;
  if (b->warm == OMB_WARM_SWEEP || b->warm == OMB_WARM_CELLS || b->warm == OMB_WARM_SWEEP_LEARNED) {
    const bool cells = b->warm == OMB_WARM_CELLS;
    std::vector<std::vector<int>> groups;
    std::vector<int> gid(n_inst, -1);
    for (int i = 0; i < n_inst; ++i) {
      const omb_instance& I = b->inst[i];
      if (I.nguess > 0 || !b->kbands[i].empty()) continue;
      for (size_t g = 0; g < groups.size() && gid[i] < 0; ++g) {
        const omb_instance& J = b->inst[groups[g][0]];
        const bool same = cells ? J.omega == I.omega : b->src_eps[groups[g][0]] == b->src_eps[i];
        if (same && J.grid.Nx == I.grid.Nx && J.grid.Ny == I.grid.Ny && J.grid.Dx == I.grid.Dx &&
            J.grid.Dy == I.grid.Dy && J.nev == I.nev)
          gid[i] = (int)g;
      }
      if (gid[i] < 0) { gid[i] = (int)groups.size(); groups.push_back({i}); }
      else groups[gid[i]].push_back(i);
    }
    for (const auto& g : groups) {
      if (g.size() < 2) continue;
      // sweep: the member nearest the mean ω; cells: the middle of the stack
      int a = g[g.size() / 2];
      if (!cells) {
        double mean = 0;
        for (int i : g) mean += b->inst[i].omega;
        mean /= (double)g.size();
        a = g[0];
        for (int i : g)
          if (std::fabs(b->inst[i].omega - mean) < std::fabs(b->inst[a].omega - mean)) a = i;
      }
      for (int i : g)
        if (i != a) anchor[i] = a;
    }
  }
  cudaEvent_t e0, e1;
  OMB_CU(cudaEventCreate(&e0));
  OMB_CU(cudaEventCreate(&e1));
  OMB_CU(cudaEventRecord(e0, ctx->stream));
  // learned warm start: the network's starting block and per-band k for every first-stage
  // instance without guesses of its own on a grid the network reads
  std::vector<int> learned_of(n_inst, -1);
  std::vector<size_t> loff;
  std::vector<std::array<double, 4>> lk;
  b->learned_instances = 0;
  if (learned) {
    if (!ctx->ws) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return fail(OMB_ERR_INVALID_ARG, "a learned warm start needs a network attached with omb_ctx_set_warmstart");
    }
    std::vector<const Problem*> lp;
    std::vector<double> lw;
    for (int i = 0; i < n_inst; ++i) {
      const omb_instance& I = b->inst[i];
      const Problem& P = b->probs[b->pidx[i]];
      if (I.nguess > 0 || !b->kbands[i].empty() || anchor[i] >= 0) continue;
      if (!(P.Nx == P.Ny && (P.Nx == 128 || P.Nx == 256 || P.Nx == 512))) continue;
      learned_of[i] = (int)lp.size();
      lp.push_back(&P);
      lw.push_back(I.omega);
    }
    const int lrc = ws_guesses(ctx->ws, lp, lw, b->learned, loff, lk);
    if (lrc) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return lrc;
    }
    b->learned_instances = (int)lp.size();
  }
  // stage 1: every instance without a neighbour to start from
  std::vector<TrackSpec> tracks;
  for (int i = 0; i < n_inst; ++i) {
    if (anchor[i] >= 0) continue;
    if (learned_of[i] >= 0) {
      const int l = learned_of[i];
      const size_t n2 = 2 * b->probs[b->pidx[i]].N();
      std::vector<double> k0 = own_k0(b, i);
      const double2* gdev[4];
      for (int j = 0; j < 4; ++j) {
        if (j < (int)k0.size()) k0[j] = lk[l][j];
        gdev[j] = b->learned.p + loff[l] + (size_t)j * n2;
      }
      add_tracks(b, i, k0, gdev, 4, 0, tracks);
    } else {
      add_tracks(b, i, own_k0(b, i), nullptr, 0, 0, tracks);
    }
  }
  // Mixed precision with inner Newton: the rest of each group joins the same engine as a
  // second wave — its FP32 phase starts from the anchors' FP32 blocks once they finish theirs,
  // and all tracks share one FP64 phase (the anchors' polish overlaps the others' instead of
  // running alone).  Otherwise (FP64 or FP32 only, the reference loop) a second engine starts
  // from the anchors' converged FP64 vectors.
  const bool waves = b->so.precision == OMB_PREC_MIXED && b->so.newton_mode == MODE_NEWTON_INNER;
  if (waves) {
    std::vector<int> first_track(n_inst, -1);  // instance → its band-0 track (bands are consecutive)
    for (const auto& h : b->who)
      if (h.band0 == 0) first_track[h.inst] = h.track;
    for (int i = 0; i < n_inst; ++i) {
      const int a = anchor[i];
      if (a < 0) continue;
      const size_t t0 = tracks.size();
      add_tracks(b, i, own_k0(b, i), nullptr, 0, 0, tracks);
      for (size_t t = t0; t < tracks.size(); ++t) {
        tracks[t].wave = 1;
        tracks[t].src = first_track[a] >= 0 ? first_track[a] + tracks[t].band : -1;
        tracks[t].omega_src = b->inst[a].omega;
      }
    }
  }
  b->engines.emplace_back(new Engine(ctx, &b->probs, tracks, b->so));
  int rc = b->engines[0]->run();
  // stage 2: the rest of each sweep group, from its anchor's eigenvectors and k
  if (!rc && !waves) {
    std::vector<TrackSpec> tracks2;
    const Engine& E0 = *b->engines[0];
    std::vector<std::vector<int>> first(n_inst);  // anchor → stage-1 who entries per band
    for (size_t w = 0; w < b->who.size(); ++w) {
      const auto& h = b->who[w];
      auto& f = first[h.inst];
      if (f.empty()) f.assign(b->inst[h.inst].nev, -1);
      f[h.band0] = (int)w;
    }
    for (int i = 0; i < n_inst; ++i) {
      const int a = anchor[i];
      if (a < 0) continue;
      const omb_instance& I = b->inst[i];
      const double wa = b->inst[a].omega;
      std::vector<double> k0(I.nev);
      const double2* gdev[MMAX] = {};
      const bool inner = b->so.newton_mode == MODE_NEWTON_INNER;
      for (int j = 0; j < I.nev; ++j) {
        // band j of the anchor: its own track (inner) or result j of its single track
        const auto& h = b->who[first[a][inner ? j : 0]];
        const int rb = inner ? 0 : j;
        const TrackState& s = E0.result_state(h.track, rb);
        const double dw2dk = 2.0 * s.hmkh;
        double k = s.k * I.omega / wa;  // constant n_eff
        if (dw2dk > 0 && std::isfinite(dw2dk) && std::isfinite(s.k))
          k = s.k + (I.omega - wa) * 2.0 * wa / dw2dk;  // first order in ω: dk/dω = 2ω/(∂ω²/∂k)
        k0[j] = (k > 0 && std::isfinite(k)) ? k : own_k0(b, i)[j];
        if (j < MMAX) gdev[j] = E0.result_dev(h.track, rb);
      }
      add_tracks(b, i, k0, gdev, I.nev, 1, tracks2);
    }
    if (!tracks2.empty()) {
      b->engines.emplace_back(new Engine(ctx, &b->probs, tracks2, b->so));
      rc = b->engines[1]->run();
    }
  }
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
  if (b->engines.empty()) return fail(OMB_ERR_INVALID_ARG, "omb_batch_run has not been called");
  OMB_CU(cudaSetDevice(b->ctx->device));
  bool all_ok = true;
  b->d2h = 0;
  if (b->canon)
    for (auto& e : b->engines) {
      const int rc = e->canonicalize_results();
      if (rc) return rc;
    }
  std::vector<D2HPiece> pieces;
  for (size_t w = 0; w < b->who.size(); ++w) {
    const int i = b->who[w].inst, band0 = b->who[w].band0;
    Engine& E = *b->engines[b->who[w].eng];
    const int t = b->who[w].track;
    const omb_instance& I = b->inst[i];
    omb_result& r = out[i];
    if (!r.kmags) return fail(OMB_ERR_INVALID_ARG, "result kmags is NULL");
    const size_t n2 = 2 * b->probs[b->pidx[i]].N();
    const int nb = b->so.newton_mode == MODE_NEWTON_INNER ? 1 : I.nev;
    for (int rb = 0; rb < nb; ++rb) {
      const int band = band0 + rb;
      const TrackState& s = E.result_state(t, rb);
      r.kmags[band] = s.k;
      if (r.residuals) r.residuals[band] = s.resid[band];
      if (r.dw2dk) r.dw2dk[band] = 2.0 * s.hmkh;
      if (r.status) r.status[band] = status_code(s.status);
      if (r.iterations) r.iterations[band] = s.iter;
      if (r.newton_steps) r.newton_steps[band] = s.newton_steps;
      b->d2h += 8 * 4 + 4 * 3;
      all_ok = all_ok && s.status == TS_CONVERGED;
      if (r.evecs) {
        // (phase gauge already applied on the device above)
        pieces.push_back({E.result_dev(t, rb), r.evecs + 2 * n2 * band, n2 * sizeof(double2)});
        b->d2h += (int64_t)(2 * n2 * sizeof(double)) + (b->canon ? 24 : 0);
      }
    }
  }
  // the engines' work (canonicalisation) is on the context stream, ahead of the gather
  const int grc = gather_to_host(b->ctx, pieces.data(), pieces.size());
  if (grc) return grc;
  if (!all_ok) return fail(OMB_ERR_NOT_CONVERGED, "one or more bands did not converge (see the per-band status)");
  return OMB_OK;
}

int omb_batch_stats(const omb_batch* b, omb_stats* out) {
  if (!b || !out) return fail(OMB_ERR_INVALID_ARG, "batch and out must be non-NULL");
  out->graph_launches = 0;
  out->kernel_launches = 0;
  out->max_iterations = 0;
  for (const auto& e : b->engines) {
    out->graph_launches += e->graph_launches();
    out->kernel_launches += e->kernel_launches();
    out->max_iterations = std::max<int32_t>(out->max_iterations, e->max_iterations());
  }
  out->h2d_bytes = b->h2d;
  out->d2h_bytes = b->d2h;
  out->tracks = (int32_t)b->who.size();
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

int omb_solve_k_periodic(omb_ctx* ctx, const omb_grid3* grid, double omega, const double* epsinv, int nev,
                         double kguess, const omb_options* opt, double* kmags, double* evecs, double* residuals,
                         double* dw2dk, int32_t* status, int32_t* iterations) {
  if (!ctx || !grid) return fail(OMB_ERR_INVALID_ARG, "ctx and grid must be non-NULL");
  if (!kmags) return fail(OMB_ERR_INVALID_ARG, "kmags is NULL");
  if (!(omega > 0) || !std::isfinite(omega)) return fail(OMB_ERR_INVALID_ARG, "omega must be finite and positive");
  if (grid->Nz < 8) return fail(OMB_ERR_UNSUPPORTED, "a z-periodic cell needs Nz >= 8 slabs (a supported length)");
  SolveOptions so;
  int rc = options_from(opt, so);
  if (rc) return rc;
  if (so.newton_mode != MODE_NEWTON_INNER)
    return fail(OMB_ERR_UNSUPPORTED, "z-periodic cells use the inner Newton iteration (OMB_NEWTON_INNER)");
  if (nev <= 0 || nev + so.guard > MMAX) return fail(OMB_ERR_INVALID_ARG, "nev + guard_bands must be in 2..12");
  OMB_CU(cudaSetDevice(ctx->device));
  std::vector<Problem> probs(1);
  const omb_grid g2{grid->Nx, grid->Ny, grid->Dx, grid->Dy};
  rc = upload_problem(ctx, &g2, epsinv, probs[0], grid->Nz, grid->Dz);
  if (rc) return rc;
  const double k0 = kguess > 0 ? kguess : omega * std::sqrt(1.0 / probs[0].min_diag);
  std::vector<TrackSpec> tracks;
  for (int band = 0; band < nev; ++band) {
    TrackSpec ts;
    ts.prob = 0; ts.band = band; ts.nbands = 1; ts.M = band + 1 + so.guard; ts.need = band + 1;
    ts.mode = MODE_NEWTON_INNER; ts.k0 = k0; ts.omega2 = omega * omega;
    tracks.push_back(ts);
  }
  Engine E(ctx, &probs, tracks, so);
  rc = E.run();
  if (rc) return rc;
  if (!opt || opt->canonicalize) {
    rc = E.canonicalize_results();
    if (rc) return rc;
  }
  const size_t n2 = 2 * probs[0].N();
  bool all_ok = true;
  for (int b = 0; b < nev; ++b) {
    const TrackState& s = E.result_state(b, 0);
    kmags[b] = s.k;
    if (residuals) residuals[b] = s.resid[b];
    if (dw2dk) dw2dk[b] = 2.0 * s.hmkh;
    if (status) status[b] = status_code(s.status);
    if (iterations) iterations[b] = s.iter;
    all_ok = all_ok && s.status == TS_CONVERGED;
    if (evecs)
      OMB_CU(cudaMemcpyAsync(evecs + 2 * n2 * b, E.result_dev(b, 0), n2 * sizeof(double2), cudaMemcpyDeviceToHost,
                             ctx->stream));
  }
  OMB_CU(cudaStreamSynchronize(ctx->stream));
  if (!all_ok) return fail(OMB_ERR_NOT_CONVERGED, "one or more bands did not converge (see the per-band status)");
  return OMB_OK;
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
  if (s.status != TS_CONVERGED)
    return fail(status_code(s.status), s.status == TS_ORTHO ? "solve_omega2: the block lost rank (orthonormalisation failed)"
                                       : s.status == TS_NAN ? "solve_omega2: non-finite Ritz values"
                                                            : "solve_omega2 did not converge");
  return OMB_OK;
}

}  // extern "C"
