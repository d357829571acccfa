// Batched device LOBPCG/Newton engine: buffer management, graph capture, phase loop.
#include <algorithm>
#include <cmath>
#include <cstring>

#include <map>
#include <tuple>

#include "engine.h"
#include "vec.cuh"

namespace omb {

static int blocks_for(size_t n, int nt = 256) {
  size_t b = (n + nt - 1) / nt;
  return (int)std::max<size_t>(1, std::min<size_t>(b, 65535 * 4));
}

// Opt in to large dynamic shared memory.  The default limit covers static + dynamic, so
// opt in whenever the dynamic part alone comes near it.
template <typename K> static cudaError_t set_smem(K kern, size_t bytes) {
  if (bytes <= 32 * 1024) return cudaSuccess;
  return ensure_smem(reinterpret_cast<const void*>(kern), bytes);
}

Engine::Engine(omb_ctx* ctx, std::vector<Problem>* problems, std::vector<TrackSpec> tracks, SolveOptions opt)
    : ctx_(ctx), probs_(problems), tracks_(std::move(tracks)), opt_(opt) {
  nt_ = (int)tracks_.size();
  order_.resize(nt_);
  for (int i = 0; i < nt_; ++i) order_[i] = i;
  // by grid, and within a grid by wave, so that each wave of a grid group is one contiguous
  // range of positions (a phase of one wave launches the operator passes over that range only)
  std::stable_sort(order_.begin(), order_.end(), [&](int a, int b) {
    const Problem& pa = (*probs_)[tracks_[a].prob];
    const Problem& pb = (*probs_)[tracks_[b].prob];
    return std::make_tuple(pa.Nx, pa.Ny, pa.Nz, tracks_[a].wave) < std::make_tuple(pb.Nx, pb.Ny, pb.Nz, tracks_[b].wave);
  });
  for (int i = 0; i < nt_;) {
    const Problem& p = (*probs_)[tracks_[order_[i]].prob];
    Group g{i, 0, p.Nx, p.Ny, 0, p.Nz};
    while (i < nt_) {
      const Problem& q = (*probs_)[tracks_[order_[i]].prob];
      if (q.Nx != p.Nx || q.Ny != p.Ny || q.Nz != p.Nz) break;
      g.Mmax = std::max(g.Mmax, tracks_[order_[i]].M);
      ++g.n;
      ++i;
    }
    groups_.push_back(g);
  }
}

Engine::~Engine() { cudaStreamSynchronize(ctx_->stream); }

int Engine::upload_states() {
  OMB_CU(cudaMemcpyAsync(d_states_.p, host_states_.data(), nt_ * sizeof(TrackState), cudaMemcpyHostToDevice,
                         ctx_->stream));
  OMB_CU(cudaStreamSynchronize(ctx_->stream));
  return OMB_OK;
}
int Engine::download_states() {
  OMB_CU(cudaMemcpyAsync(host_states_.data(), d_states_.p, nt_ * sizeof(TrackState), cudaMemcpyDeviceToHost,
                         ctx_->stream));
  OMB_CU(cudaStreamSynchronize(ctx_->stream));
  return OMB_OK;
}

// Fill X (columns 0..M-1 of Y[0]) for the first phase: random, then the caller's guesses.
template <typename T> int Engine::init_block(int phase) {
  cudaStream_t st = ctx_->stream;
  DevBuf<cplx<T>>& Y = std::is_same<T, float>::value ? reinterpret_cast<DevBuf<cplx<T>>&>(y32_)
                                                      : reinterpret_cast<DevBuf<cplx<T>>&>(y64_);
  for (int t = 0; t < nt_; ++t) {
    const TrackSpec& ts = tracks_[t];
    const Problem& P = (*probs_)[ts.prob];
    const long long n2 = 2 * (long long)P.N();
    cplx<T>* X = Y.p + yoff_[t];
    if (phase == 0) {
      k_random_block<T><<<blocks_for(n2 * ts.M), 256, 0, st>>>(X, n2, ts.M, opt_.seed * 1000003ull + 7919ull * t + 1);
      OMB_CU(cudaGetLastError());
      const int ng = std::min(ts.nguess, ts.M);
      if (ng > 0 && ts.guess) {
        DevBuf<double2> g;
        OMB_CU(g.alloc(n2 * ng, st));
        OMB_CU(cudaMemcpyAsync(g.p, ts.guess, n2 * ng * sizeof(double2), cudaMemcpyHostToDevice, st));
        if constexpr (std::is_same<T, double>::value) {
          OMB_CU(cudaMemcpyAsync(X, g.p, n2 * ng * sizeof(double2), cudaMemcpyDeviceToDevice, st));
        } else {
          k_c64_to_c32<<<blocks_for(n2 * ng), 256, 0, st>>>(g.p, X, n2 * ng);
          OMB_CU(cudaGetLastError());
        }
        OMB_CU(cudaStreamSynchronize(st));
      } else if (ts.nguess_dev > 0) {
        // device-resident FP64 columns from an earlier engine
        for (int c = 0; c < std::min(ts.nguess_dev, ts.M); ++c) {
          if (!ts.guess_dev[c]) continue;
          if constexpr (std::is_same<T, double>::value) {
            OMB_CU(cudaMemcpyAsync(X + (size_t)c * n2, ts.guess_dev[c], n2 * sizeof(double2),
                                   cudaMemcpyDeviceToDevice, st));
          } else {
            k_c64_to_c32<<<blocks_for(n2), 256, 0, st>>>(ts.guess_dev[c], X + (size_t)c * n2, n2);
            OMB_CU(cudaGetLastError());
          }
        }
      }
    } else {
      // previous phase ran in FP32: promote its X
      if constexpr (std::is_same<T, double>::value) {
        const size_t src = yoff_[t] + (size_t)host_states_[t].cur_par * 3 * ts.M * n2;
        k_c32_to_c64<<<blocks_for(n2 * ts.M), 256, 0, st>>>(y32_.p + src, X, n2 * ts.M);
        OMB_CU(cudaGetLastError());
      }
    }
  }
  return OMB_OK;
}

template <typename T>
int Engine::run_phase(int phase, bool last, double tau, double lock_tol, int mode) {
  cudaStream_t st = ctx_->stream;
  DevBuf<cplx<T>>& Y = std::is_same<T, float>::value ? reinterpret_cast<DevBuf<cplx<T>>&>(y32_)
                                                      : reinterpret_cast<DevBuf<cplx<T>>&>(y64_);
  DevBuf<cplx<T>>& Sc = std::is_same<T, float>::value ? reinterpret_cast<DevBuf<cplx<T>>&>(s32_)
                                                       : reinterpret_cast<DevBuf<cplx<T>>&>(s64_);
  int rc = OMB_OK;
  auto active = [&](int t) { return wave_ < 0 || tracks_[t].wave == wave_; };
  if (mode == 0) {
    // ---- buffers: per track Y[2], AY[2] (3M columns each) and the operator scratch
    yoff_.assign(nt_, 0);
    soff_.assign(nt_, 0);
    size_t ytot = 0, stot = 0;
    for (int t = 0; t < nt_; ++t) {
      const Problem& P = (*probs_)[tracks_[t].prob];
      const size_t n2 = 2 * P.N();
      yoff_[t] = ytot;
      ytot += 12 * (size_t)tracks_[t].M * n2;
      soff_[t] = stot;
      // the A pass covers up to [X | W | P] (3M columns) right after a Newton step
      stot += 3 * (size_t)tracks_[t].M * 3 * P.N();
    }
    OMB_CU(Y.alloc(ytot, st));
    OMB_CU(Sc.alloc(stot, st));
    rc = init_block<T>(phase);
    if (rc) return rc;
    if (phase > 0 && std::is_same<T, double>::value) y32_.release(), s32_.release();
  } else if (mode == 1) {
    // continue from the current block: bring it to parity 0
    for (int t = 0; t < nt_; ++t) {
      if (host_states_[t].cur_par == 0) continue;
      const size_t n2 = 2 * (*probs_)[tracks_[t].prob].N();
      const size_t M = tracks_[t].M;
      OMB_CU(cudaMemcpyAsync(Y.p + yoff_[t], Y.p + yoff_[t] + 3 * M * n2, M * n2 * sizeof(cplx<T>),
                             cudaMemcpyDeviceToDevice, st));
    }
  }

  // ---- per-phase state (tracks outside the running wave sit this phase out, state kept)
  for (int t = 0; t < nt_; ++t) {
    TrackState& s = host_states_[t];
    if (!active(t)) {
      s.done = 1;
      s.op_ncol = 0; s.pw_ncol = 0; s.hmkh_ncol = 0;
      continue;
    }
    s.band = tracks_[t].band + round_;
    s.done = (round_ < tracks_[t].nbands) ? 0 : 1;
    s.status = s.done ? s.status : TS_RUNNING;
    s.nlocked = 0; s.nWa = 0; s.nP = 0; s.nP_next = 0;
    s.op_col0 = 0; s.op_ncol = s.M; s.pw_col0 = 0; s.pw_ncol = 0; s.hmkh_ncol = 0;
    s.iter_phase = 0; s.newton_phase = 0; s.since_newton = 0; s.stall = 0; s.resid_best = 1e300;
    s.phase = phase;
    s.cur_par = 0;
  }
  rc = upload_states();
  if (rc) return rc;

  // ---- descriptors
  std::vector<TrackDesc<T>> descs(nt_);
  std::vector<OpUnit<T>> uA[2], uP[2], uH[2];
  for (int par = 0; par < 2; ++par) { uA[par].resize(nt_); uP[par].resize(nt_); uH[par].resize(nt_); }
  for (int t = 0; t < nt_; ++t) {
    const TrackSpec& ts = tracks_[t];
    const Problem& P = (*probs_)[ts.prob];
    const long long n2 = 2 * (long long)P.N();
    const int M = ts.M;
    TrackDesc<T>& d = descs[t];
    cplx<T>* base = Y.p + yoff_[t];
    d.Y[0] = base;
    d.Y[1] = base + 3 * M * n2;
    d.AY[0] = base + 6 * M * n2;
    d.AY[1] = base + 9 * M * n2;
    d.st = d_states_.p + t;
    d.coef = coef_.p + (size_t)t * 2 * NMAX * MMAX;
    if constexpr (std::is_same<T, float>::value) d.coefT = coef32_.p + (size_t)t * 2 * NMAX * MMAX;
    else d.coefT = d.coef;
    d.gram_acc = gram_acc_.p + (size_t)t * 2 * NMAX * NMAX;
    d.res_acc = res_acc_.p + (size_t)t * MMAX;
    d.hmkh_part = hmkh_part_.p + (size_t)t * 2 * 512;
    d.n2 = n2; d.Nx = P.Nx; d.Ny = P.Ny; d.M = M;
    d.hmkh_nb = row_blocks(P.Nx, P.Ny) * P.Nz;
    d.inv_dx = 1.0 / P.Dx; d.inv_dy = 1.0 / P.Dy; d.eps_mean = P.eps_mean;
    d.Nz = P.Nz; d.inv_dz = P.Nz > 1 ? 1.0 / P.Dz : 0.0;
  }
  for (int gi = 0; gi < nt_; ++gi) {
    const int t = order_[gi];
    const TrackSpec& ts = tracks_[t];
    const Problem& P = (*probs_)[ts.prob];
    const long long n2 = 2 * (long long)P.N();
    const int M = ts.M;
    for (int par = 0; par < 2; ++par) {
      OpUnit<T> u = make_unit<T>(P);
      u.k_dev = &d_states_.p[t].k;
      u.scr = Sc.p + soff_[t];
      u.scr_cs = 3 * (long long)P.N();
      u.in_cs = u.out_cs = n2;
      // A pass over [X | W] of this parity
      OpUnit<T> a = u;
      a.in = descs[t].Y[par];
      a.out = descs[t].AY[par];
      a.ncol_dev = &d_states_.p[t].op_ncol;
      a.col0_dev = &d_states_.p[t].op_col0;
      uA[par][gi] = a;
      // MPB preconditioner in place on the W slot
      OpUnit<T> p = u;
      p.in = descs[t].Y[par] + M * n2;
      p.out = const_cast<cplx<T>*>(p.in);
      p.ncol_dev = &d_states_.p[t].pw_ncol;
      p.col0_dev = &d_states_.p[t].pw_col0;
      uP[par][gi] = p;
      // ⟨x_b|∂M̂/∂k|x_b⟩ on the Newton band
      OpUnit<T> h = u;
      h.in = descs[t].Y[par] + (long long)(ts.band + round_) * n2;
      h.ncol_dev = &d_states_.p[t].hmkh_ncol;
      h.partial = descs[t].hmkh_part;
      uH[par][gi] = h;
    }
  }
  DevBuf<TrackDesc<T>> d_descs;
  DevBuf<OpUnit<T>> d_uA[2], d_uP[2], d_uH[2];
  // device-side per-track arrays are in grid-sorted position order (order_), so every lane
  // below and every grid group is a contiguous range of positions
  std::vector<TrackDesc<T>> sdescs(nt_);
  for (int gi = 0; gi < nt_; ++gi) sdescs[gi] = descs[order_[gi]];
  OMB_CU(d_descs.alloc(nt_, st));
  OMB_CU(cudaMemcpyAsync(d_descs.p, sdescs.data(), nt_ * sizeof(TrackDesc<T>), cudaMemcpyHostToDevice, st));
  for (int par = 0; par < 2; ++par) {
    OMB_CU(d_uA[par].alloc(nt_, st));
    OMB_CU(d_uP[par].alloc(nt_, st));
    OMB_CU(d_uH[par].alloc(nt_, st));
    OMB_CU(cudaMemcpyAsync(d_uA[par].p, uA[par].data(), nt_ * sizeof(OpUnit<T>), cudaMemcpyHostToDevice, st));
    OMB_CU(cudaMemcpyAsync(d_uP[par].p, uP[par].data(), nt_ * sizeof(OpUnit<T>), cudaMemcpyHostToDevice, st));
    OMB_CU(cudaMemcpyAsync(d_uH[par].p, uH[par].data(), nt_ * sizeof(OpUnit<T>), cudaMemcpyHostToDevice, st));
  }
  OMB_CU(cudaStreamSynchronize(st));

  IterParams prm{};
  prm.tol = opt_.tol;
  prm.k_tol = opt_.k_tol;
  prm.lock_tol = lock_tol;
  prm.tau_phase = tau;
  prm.dk_phase = 1e-6;
  prm.gram_drop = std::is_same<T, float>::value ? 1e-6 : 1e-12;
  // an FP32 block's Gram matrices carry FP32 products: rotating below 1e-9 of ‖A‖ buys nothing
  prm.jacobi_tol2 = std::is_same<T, float>::value ? 1e-18 : 1e-26;
  prm.maxiter = opt_.maxiter;
  prm.max_newton = opt_.max_newton;
  prm.last_phase = last ? 1 : 0;
  prm.prec_diag = opt_.prec_diag ? 1 : 0;

  int Mmax = 1;
  for (const auto& ts : tracks_) Mmax = std::max(Mmax, ts.M);
  const int nmax = 3 * Mmax;
  // Gram: as many ring stages as fit in ≈200 KB (2..8); update: a fixed ring
  const int rg = GramCfg<T>::rows(nmax);
  const size_t gstage = GramCfg<T>::stage_elems(nmax, rg) * sizeof(cplx<T>);
  const size_t gred = GramCfg<T>::red_entries(nmax) * sizeof(double2);
  const int gstages = (int)std::max<size_t>(2, std::min<size_t>(8, (200 * 1024 - 128 - gred) / gstage));
  const size_t sm_gram = 128 + gstages * gstage + gred;
  const size_t sm_upd = UpdCfg<T>::smem;
  const size_t sm_rr = 4 * (size_t)NMAX * NMAX * sizeof(double2);
  OMB_CU(set_smem(k_gram<T>, sm_gram));
  auto update_kernel = Mmax <= 2 ? k_update<T, 2>
                       : Mmax <= 4 ? k_update<T, 4>
                       : Mmax <= 6 ? k_update<T, 6>
                       : Mmax <= 8 ? k_update<T, 8> : k_update<T, MMAX>;
  OMB_CU(set_smem(update_kernel, sm_upd));
  OMB_CU(set_smem(k_rr, sm_rr));
  int occ_g = 0, occ_u = 0;
  OMB_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_g, k_gram<T>, GramCfg<T>::NT, sm_gram));
  OMB_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_u, update_kernel, UpdCfg<T>::NT, sm_upd));
  const int grid_g = std::max(1, occ_g) * ctx_->num_sms;
  const int grid_u = std::max(1, occ_u) * ctx_->num_sms;
  OMB_CU(gram_acc_.zero());
  OMB_CU(res_acc_.zero());
  // Lanes of tracks (split by Σ M², the Gram cost) run their iterations on separate streams,
  // so one lane's latency-bound kernels (k_rr, k_control, k_newton, the prefix) overlap the
  // other lanes' streaming kernels.
  const int nl = std::max(1, std::min(LANES, nt_));
  int lane_lo[LANES], lane_hi[LANES];
  {
    // (tracks sitting the phase out weigh nothing)
    auto w2 = [&](int gi) { const int t = order_[gi]; return active(t) ? (double)tracks_[t].M * tracks_[t].M : 0.0; };
    double tot = 0, acc = 0;
    for (int gi = 0; gi < nt_; ++gi) tot += w2(gi);
    int gi = 0;
    for (int L = 0; L < nl; ++L) {
      lane_lo[L] = gi;
      if (L == nl - 1) { gi = nt_; }
      else {
        // at least one track per lane, and leave one for each later lane
        do { acc += w2(gi); ++gi; }
        while (gi < nt_ - (nl - 1 - L) && acc < tot * (L + 1) / nl);
      }
      lane_hi[L] = gi;
    }
  }
  // per grid group, the positions of the tracks taking part in this phase (contiguous: the
  // positions of a group are sorted by wave)
  std::vector<int> act_lo(groups_.size()), act_hi(groups_.size());
  for (size_t gi = 0; gi < groups_.size(); ++gi) {
    const Group& g = groups_[gi];
    int lo = g.off + g.n, hi = g.off;
    for (int p = g.off; p < g.off + g.n; ++p)
      if (active(order_[p])) { lo = std::min(lo, p); hi = std::max(hi, p + 1); }
    act_lo[gi] = lo;
    act_hi[gi] = std::max(lo, hi);
  }
  OMB_CU(d_pre_.alloc(2 * (size_t)LANES * ((size_t)nt_ + 1), st));
  OMB_CU(d_wpre_.alloc(2 * (size_t)LANES * ((size_t)nt_ + 1), st));
  // z-periodic groups: per-lane room for the slab and line units of launch_op3d
  int maxNz = 1;
  for (const Group& g : groups_) maxNz = std::max(maxNz, g.Nz);
  DevBuf<OpUnit<T>> d_exp[LANES];
  if (maxNz > 1)
    for (int L = 0; L < LANES; ++L) OMB_CU(d_exp[L].alloc((size_t)(maxNz + 1) * nt_, st));

  const char* step = "";
  auto iteration = [&](int par, int L, cudaStream_t s) -> cudaError_t {
    cudaError_t e = cudaSuccess;
    auto ok = [&](const char* name, cudaError_t r) { step = name; e = r; return r == cudaSuccess; };
    const int a = lane_lo[L], n = lane_hi[L] - lane_lo[L];
    if (n <= 0) return e;
    int* preg = d_pre_.p + (size_t)L * 2 * (nt_ + 1);
    int* preu = preg + nt_ + 1;
    long long* wpreg = d_wpre_.p + (size_t)L * 2 * (nt_ + 1);
    long long* wpreu = wpreg + nt_ + 1;
    auto op = [&](OpKind kind, const OpUnit<T>* u, int cnt, const Group& g, int maxcol) -> cudaError_t {
      return g.Nz > 1 ? launch_op3d<T>(kind, u, cnt, g.Nx, g.Ny, g.Nz, maxcol, ctx_->tw, d_exp[L].p, s)
                      : launch_op<T>(kind, u, cnt, g.Nx, g.Ny, maxcol, ctx_->tw, s);
    };
    // the lane's part of every grid group (its positions of the running wave)
    auto for_groups = [&](auto&& f) -> bool {
      for (size_t gi = 0; gi < groups_.size(); ++gi) {
        const Group& g = groups_[gi];
        const int lo = std::max(act_lo[gi], a), hi = std::min(act_hi[gi], a + n);
        if (hi > lo && !f(g, lo, hi - lo)) return false;
      }
      return true;
    };
    if (!opt_.prec_diag &&
        !for_groups([&](const Group& g, int off, int cnt) {
          return ok("preconditioner pass", op(OP_P, d_uP[par].p + off, cnt, g, g.Mmax));
        }))
      return e;
    if (!for_groups([&](const Group& g, int off, int cnt) {
          return ok("HMkH pass", op(OP_HMKH, d_uH[par].p + off, cnt, g, 1));
        }))
      return e;
    k_newton<<<(n + 127) / 128, 128, 0, s>>>(d_state_ptrs_.p + a, d_hmkh_ptrs_.p + a, d_hmkh_nb_.p + a, n, prm);
    if (!ok("k_newton", cudaGetLastError())) return e;
    if (!for_groups([&](const Group& g, int off, int cnt) {
          return ok("operator pass", op(OP_M, d_uA[par].p + off, cnt, g, 3 * g.Mmax));
        }))
      return e;
    k_live_prefix<<<1, 1024, 0, s>>>(d_state_ptrs_.p + a, d_n2_.p + a, n, rg, UpdCfg<T>::R, preg, preu, wpreg,
                                     wpreu);
    if (!ok("k_live_prefix", cudaGetLastError())) return e;
    k_gram<T><<<grid_g, GramCfg<T>::NT, sm_gram, s>>>(d_descs.p + a, preg, wpreg, n, par, nmax, rg, gstages,
                                                       d_err_.p, ctx_->wait_ns);
    if (!ok("k_gram", cudaGetLastError())) return e;
    k_rr<<<n, RR_NT, sm_rr, s>>>(d_state_ptrs_.p + a, d_gram_ptrs_.p + a, d_coef_ptrs_.p + a, d_coef32_ptrs_.p + a, n,
                                 prm);
    if (!ok("k_rr", cudaGetLastError())) return e;
    update_kernel<<<grid_u, UpdCfg<T>::NT, sm_upd, s>>>(d_descs.p + a, preu, wpreu, n, par, prm.prec_diag,
                                                        d_err_.p, ctx_->wait_ns);
    if (!ok("k_update", cudaGetLastError())) return e;
    k_control<<<(n + 3) / 4, 128, 0, s>>>(d_state_ptrs_.p + a, d_res_ptrs_.p + a, n, prm);
    ok("k_control", cudaGetLastError());
    return e;
  };

  // two eager iterations (they also size the kernels' shared memory), then the graph
  for (int par = 0; par < 2; ++par)
    for (int L = 0; L < nl; ++L) {
      const cudaError_t e = iteration(par, L, st);
      if (e != cudaSuccess) return cuda_fail(e, step);
    }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t lst[LANES] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[LANES] = {};
  lst[0] = st;
  auto release = [&]() {
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (int L = 1; L < LANES; ++L) {
      if (ev_join[L]) cudaEventDestroy(ev_join[L]);
      if (lst[L]) cudaStreamDestroy(lst[L]);
    }
  };
  {
    cudaError_t ce0 = cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming);
    for (int L = 1; L < nl && ce0 == cudaSuccess; ++L) {
      ce0 = cudaStreamCreateWithFlags(&lst[L], cudaStreamNonBlocking);
      if (ce0 == cudaSuccess) ce0 = cudaEventCreateWithFlags(&ev_join[L], cudaEventDisableTiming);
    }
    if (ce0 != cudaSuccess) { release(); return cuda_fail(ce0, "lane streams"); }
  }
  OMB_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaError_t ce = cudaSuccess;
  if (nl > 1) {
    ce = cudaEventRecord(ev_fork, st);
    for (int L = 1; L < nl && ce == cudaSuccess; ++L) ce = cudaStreamWaitEvent(lst[L], ev_fork, 0);
  }
  for (int par = 0; par < 2 && ce == cudaSuccess; ++par)
    for (int L = 0; L < nl && ce == cudaSuccess; ++L) ce = iteration(par, L, lst[L]);
  for (int L = 1; L < nl; ++L) {
    const cudaError_t j1 = cudaEventRecord(ev_join[L], lst[L]);
    const cudaError_t j2 = cudaStreamWaitEvent(st, ev_join[L], 0);
    if (ce == cudaSuccess) ce = j1 != cudaSuccess ? j1 : j2;
  }
  cudaError_t ee = cudaStreamEndCapture(st, &graph);
  release();
  if (ce != cudaSuccess) { if (graph) cudaGraphDestroy(graph); return cuda_fail(ce, step); }
  OMB_CU(ee);
  OMB_CU(cudaGraphInstantiate(&exec, graph, 0));
  size_t nodes = 0;
  OMB_CU(cudaGraphGetNodes(graph, nullptr, &nodes));
  kernels_ += (int64_t)nodes;  // the two eager iterations
  // every track ends a phase within maxiter (+2) iterations, per Newton step in the
  // reference loop; two iterations per graph launch
  const int per = opt_.maxiter / 2 + 4;
  const int cap = per * (opt_.newton_mode == MODE_NEWTON_OUTER ? opt_.max_newton + 1 : 1) + 4;
  int rc_out = OMB_OK;
  for (int it = 0; it < cap; ++it) {
    cudaError_t e = cudaGraphLaunch(exec, st);
    if (e != cudaSuccess) { rc_out = cuda_fail(e, "cudaGraphLaunch"); break; }
    launches_++;
    kernels_ += (int64_t)nodes;
    if ((it & 3) == 3 || it < 4) {
      rc_out = download_states();
      if (rc_out) break;
      int perr = 0;  // a streaming kernel gave up on a wait: stop replaying
      if (cudaMemcpy(&perr, d_err_.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess || perr != PIPE_OK) break;
      bool all = true;
      for (const TrackState& s : host_states_) all = all && s.done;
      if (all) break;
    }
  }
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  if (rc_out) return rc_out;
  rc_out = download_states();
  if (rc_out) return rc_out;
  int perr = 0;
  OMB_CU(cudaMemcpy(&perr, d_err_.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (perr != PIPE_OK)
    return fail(OMB_ERR_TIMEOUT, "a streaming kernel's pipeline wait ran out after " +
                                     std::to_string(ctx_->wait_ns / 1e9) + " s (code " + std::to_string(perr) + ")");
  last_prec_ = std::is_same<T, float>::value ? 0 : 1;
  return rc_out;
}

int Engine::run() {
  cudaStream_t st = ctx_->stream;
  OMB_CU(cudaSetDevice(ctx_->device));
  // ---- per-track FP64 state and small buffers
  host_states_.assign(nt_, TrackState{});
  double normA = 0;
  for (int t = 0; t < nt_; ++t) {
    const TrackSpec& ts = tracks_[t];
    const Problem& P = (*probs_)[ts.prob];
    TrackState& s = host_states_[t];
    std::memset(&s, 0, sizeof(s));
    s.k = ts.k0; s.k_eig = ts.k0; s.omega2 = ts.omega2;
    s.M = ts.M; s.band = ts.band; s.need = ts.need; s.mode = ts.mode;
    s.dk_last = 1e300;
    const double gx = 0.5 * P.Nx / P.Dx, gy = 0.5 * P.Ny / P.Dy;
    const double kz = std::fabs(ts.k0) + (P.Nz > 1 ? 0.5 * P.Nz / P.Dz : 0.0);
    normA = std::max(normA, (gx * gx + gy * gy + kz * kz) * P.max_trace);
  }
  OMB_CU(d_states_.alloc(nt_, st));
  OMB_CU(coef_.alloc((size_t)nt_ * 2 * NMAX * MMAX, st));
  OMB_CU(coef32_.alloc((size_t)nt_ * 2 * NMAX * MMAX, st));
  OMB_CU(gram_acc_.alloc((size_t)nt_ * 2 * NMAX * NMAX, st));
  OMB_CU(res_acc_.alloc((size_t)nt_ * MMAX, st));
  OMB_CU(hmkh_part_.alloc((size_t)nt_ * 2 * 512, st));
  OMB_CU(coef_.zero());
  OMB_CU(coef32_.zero());
  OMB_CU(d_err_.alloc(1, st));
  OMB_CU(d_err_.zero());
  std::vector<TrackState*> sp(nt_);
  std::vector<double2*> gp(nt_), cp(nt_);
  std::vector<float2*> cp32(nt_);
  std::vector<double*> rp(nt_), hp(nt_);
  std::vector<int> hnb(nt_);
  std::vector<long long> n2s(nt_);
  for (int gi = 0; gi < nt_; ++gi) {  // position gi holds track order_[gi]
    const int t = order_[gi];
    const Problem& P = (*probs_)[tracks_[t].prob];
    sp[gi] = d_states_.p + t;
    gp[gi] = gram_acc_.p + (size_t)t * 2 * NMAX * NMAX;
    cp[gi] = coef_.p + (size_t)t * 2 * NMAX * MMAX;
    cp32[gi] = coef32_.p + (size_t)t * 2 * NMAX * MMAX;
    rp[gi] = res_acc_.p + (size_t)t * MMAX;
    hp[gi] = hmkh_part_.p + (size_t)t * 2 * 512;
    hnb[gi] = row_blocks(P.Nx, P.Ny) * P.Nz;
    n2s[gi] = 2 * (long long)P.N();
  }
  OMB_CU(d_state_ptrs_.alloc(nt_, st));
  OMB_CU(d_gram_ptrs_.alloc(nt_, st));
  OMB_CU(d_coef_ptrs_.alloc(nt_, st));
  OMB_CU(d_coef32_ptrs_.alloc(nt_, st));
  OMB_CU(d_n2_.alloc(nt_, st));
  OMB_CU(cudaMemcpyAsync(d_coef32_ptrs_.p, cp32.data(), nt_ * sizeof(void*), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaMemcpyAsync(d_n2_.p, n2s.data(), nt_ * sizeof(long long), cudaMemcpyHostToDevice, st));
  OMB_CU(d_res_ptrs_.alloc(nt_, st));
  OMB_CU(d_hmkh_ptrs_.alloc(nt_, st));
  OMB_CU(d_hmkh_nb_.alloc(nt_, st));
  OMB_CU(cudaMemcpyAsync(d_state_ptrs_.p, sp.data(), nt_ * sizeof(void*), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaMemcpyAsync(d_gram_ptrs_.p, gp.data(), nt_ * sizeof(void*), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaMemcpyAsync(d_coef_ptrs_.p, cp.data(), nt_ * sizeof(void*), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaMemcpyAsync(d_res_ptrs_.p, rp.data(), nt_ * sizeof(void*), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaMemcpyAsync(d_hmkh_ptrs_.p, hp.data(), nt_ * sizeof(void*), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaMemcpyAsync(d_hmkh_nb_.p, hnb.data(), nt_ * sizeof(int), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaStreamSynchronize(st));

  // FP32 noise floor of the residual of a unit vector: ~ ε₃₂·√‖M̂‖ (FFT round-off scales
  // with the field's norm, the curl epilogue with |k+G|)
  const double tauA = std::max(opt_.tol, 16.0 * 5.96e-8 * std::sqrt(normA));
  // result store: one FP64 vector per finished band
  store_off_.assign(nt_, 0);
  snaps_.assign(nt_, {});
  size_t tot = 0;
  for (int t = 0; t < nt_; ++t) {
    store_off_[t] = tot;
    const int nb = tracks_[t].mode == MODE_OMEGA2 ? 1 : tracks_[t].nbands;
    tot += (size_t)nb * 2 * (*probs_)[tracks_[t].prob].N();
    snaps_[t].resize(nb);
  }
  OMB_CU(store_.alloc(tot, st));
  round_ = 0;
  int rc = OMB_OK;
  if (opt_.precision == OMB_PREC_FP64) {
    rc = run_phase<double>(0, true, opt_.tol, opt_.tol, 0);
  } else if (opt_.precision == OMB_PREC_FP32) {
    // tolerances clamped to what FP32 can resolve (the reference clamps to 50·eps(T),
    // src/solvers/gpu.jl:58)
    opt_.tol = std::max(opt_.tol, tauA);
    opt_.k_tol = std::max(opt_.k_tol, 50 * 1.1920929e-7);
    rc = run_phase<float>(0, true, opt_.tol, opt_.tol, 0);
  } else {
    bool waves = false;
    for (const auto& ts : tracks_) waves = waves || ts.wave == 1;
    if (waves) {
      // wave 0's FP32 phase, then wave 1's from wave 0's blocks, then one FP64 phase for all
      wave_ = 0;
      rc = run_phase<float>(0, false, tauA, tauA, 0);
      if (!rc) rc = start_wave(1);
      wave_ = 1;
      if (!rc) rc = run_phase<float>(0, false, tauA, tauA, 2);
      wave_ = -1;
    } else {
      rc = run_phase<float>(0, false, tauA, tauA, 0);
    }
    if (!rc) rc = run_phase<double>(1, true, opt_.tol, opt_.tol, 0);
  }
  if (!rc) rc = snapshot(0);
  int maxb = 1;
  for (const auto& ts : tracks_) maxb = std::max(maxb, ts.mode == MODE_NEWTON_OUTER ? ts.nbands : 1);
  for (round_ = 1; round_ < maxb && !rc; ++round_) {
    rc = last_prec_ == 1 ? run_phase<double>(2, true, opt_.tol, opt_.tol, 1)
                         : run_phase<float>(2, true, opt_.tol, opt_.tol, 1);
    if (!rc) rc = snapshot(round_);
  }
  round_ = 0;
  return rc;
}

// Set up the tracks of `wave` after the FP32 phase of the tracks before it: each starts from
// the FP32 block of its source track (all M columns, at that track's current parity) with the
// source's k carried to first order in ω, k + (ω − ω_src)·2ω_src/(∂ω²/∂k).  A source that
// did not end its phase normally leaves the track at its own start (random block, own k).
int Engine::start_wave(int wave) {
  cudaStream_t st = ctx_->stream;
  int rc = download_states();
  if (rc) return rc;
  for (int t = 0; t < nt_; ++t) {
    const TrackSpec& ts = tracks_[t];
    if (ts.wave != wave || ts.src < 0 || ts.src >= nt_) continue;
    const TrackState& sa = host_states_[ts.src];
    if (sa.status != TS_PHASE_DONE || !std::isfinite(sa.k) || !(sa.k > 0)) continue;
    const double w = std::sqrt(ts.omega2), wa = ts.omega_src;
    double k = sa.k * w / wa;  // constant n_eff
    const double dw2dk = 2.0 * sa.hmkh;
    if (dw2dk > 0 && std::isfinite(dw2dk)) k = sa.k + (w - wa) * 2.0 * wa / dw2dk;
    if (!(k > 0 && std::isfinite(k))) k = ts.k0;
    TrackState& s = host_states_[t];
    s.k = k;
    s.k_eig = k;
    const size_t n2 = 2 * (*probs_)[ts.prob].N();
    const int Ma = tracks_[ts.src].M;
    const int ncol = std::min(ts.M, Ma);
    const float2* from = y32_.p + yoff_[ts.src] + (size_t)sa.cur_par * 3 * Ma * n2;
    OMB_CU(cudaMemcpyAsync(y32_.p + yoff_[t], from, ncol * n2 * sizeof(float2), cudaMemcpyDeviceToDevice, st));
  }
  return OMB_OK;
}

int Engine::snapshot(int round) {
  cudaStream_t st = ctx_->stream;
  int rc = download_states();
  if (rc) return rc;
  for (int t = 0; t < nt_; ++t) {
    const TrackSpec& ts = tracks_[t];
    const int nb = ts.mode == MODE_OMEGA2 ? 1 : ts.nbands;
    if (round >= nb) continue;
    snaps_[t][round] = host_states_[t];
    if (ts.mode == MODE_OMEGA2) continue;  // solve_ω² reads the block itself
    const size_t n2 = 2 * (*probs_)[ts.prob].N();
    double2* dst = store_.p + store_off_[t] + (size_t)round * n2;
    const size_t src = col_offset(t, ts.band + round);
    if (last_prec_ == 1) {
      OMB_CU(cudaMemcpyAsync(dst, y64_.p + src, n2 * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    } else {
      k_c32_to_c64<<<blocks_for(n2), 256, 0, st>>>(y32_.p + src, dst, n2);
      OMB_CU(cudaGetLastError());
    }
  }
  return OMB_OK;
}

int Engine::max_iterations() const {
  int m = 0;
  for (const auto& v : snaps_)
    for (const auto& s : v) m = std::max(m, s.iter);
  return m;
}

size_t Engine::col_offset(int t, int col) const {
  const Problem& P = (*probs_)[tracks_[t].prob];
  const size_t n2 = 2 * P.N();
  return yoff_[t] + ((size_t)host_states_[t].cur_par * 3 * tracks_[t].M + col) * n2;
}

int Engine::fetch_result(int t, int b, double* out) {
  const size_t n2 = 2 * (*probs_)[tracks_[t].prob].N();
  OMB_CU(cudaMemcpyAsync(out, store_.p + store_off_[t] + (size_t)b * n2, n2 * sizeof(double2),
                         cudaMemcpyDeviceToHost, ctx_->stream));
  OMB_CU(cudaStreamSynchronize(ctx_->stream));
  return OMB_OK;
}

int Engine::fetch_block_column(int t, int col, double* out) {
  const Problem& P = (*probs_)[tracks_[t].prob];
  const size_t n2 = 2 * P.N();
  cudaStream_t st = ctx_->stream;
  if (last_prec_ == 1) {
    OMB_CU(cudaMemcpyAsync(out, y64_.p + col_offset(t, col), n2 * sizeof(double2), cudaMemcpyDeviceToHost, st));
  } else {
    DevBuf<double2> tmp;
    OMB_CU(tmp.alloc(n2, st));
    k_c32_to_c64<<<blocks_for(n2), 256, 0, st>>>(y32_.p + col_offset(t, col), tmp.p, n2);
    OMB_CU(cudaGetLastError());
    OMB_CU(cudaMemcpyAsync(out, tmp.p, n2 * sizeof(double2), cudaMemcpyDeviceToHost, st));
    OMB_CU(cudaStreamSynchronize(st));
  }
  OMB_CU(cudaStreamSynchronize(st));
  return OMB_OK;
}

int Engine::canonicalize_results() {
  cudaStream_t st = ctx_->stream;
  // finished results (track, band), grouped by grid
  std::map<std::tuple<int, int, int>, std::vector<std::pair<int, int>>> groups;
  for (int t = 0; t < nt_; ++t) {
    const Problem& P = (*probs_)[tracks_[t].prob];
    for (int b = 0; b < (int)snaps_[t].size(); ++b) groups[{P.Nx, P.Ny, P.Nz}].push_back({t, b});
  }
  constexpr int CHUNK = 64;
  for (const auto& kv : groups) {
    const int Nx = std::get<0>(kv.first), Ny = std::get<1>(kv.first), Nz = std::get<2>(kv.first);
    const size_t N = (size_t)Nx * Ny * Nz, n2 = 2 * N;
    const auto& all = kv.second;
    for (size_t c0 = 0; c0 < all.size(); c0 += CHUNK) {
      const int cnt = (int)std::min<size_t>(CHUNK, all.size() - c0);
      DevBuf<double> kd, red;
      DevBuf<double2> scr;
      DevBuf<OpUnit<double>> du;
      OMB_CU(kd.alloc(cnt, st));
      OMB_CU(red.alloc(3 * (size_t)cnt, st));
      OMB_CU(scr.alloc(3 * N * (size_t)cnt, st));
      OMB_CU(du.alloc(cnt, st));
      std::vector<double> kh(cnt);
      std::vector<OpUnit<double>> uh(cnt);
      for (int j = 0; j < cnt; ++j) {
        const int t = all[c0 + j].first, b = all[c0 + j].second;
        kh[j] = snaps_[t][b].k;
        OpUnit<double> u = make_unit<double>((*probs_)[tracks_[t].prob]);
        u.in = store_.p + store_off_[t] + (size_t)b * n2;
        u.scr = scr.p + (size_t)j * 3 * N;
        u.k_dev = kd.p + j;
        u.in_cs = (long long)n2; u.scr_cs = 3 * (long long)N; u.ncol = 1;
        uh[j] = u;
      }
      OMB_CU(cudaMemcpyAsync(kd.p, kh.data(), cnt * sizeof(double), cudaMemcpyHostToDevice, st));
      OMB_CU(cudaMemcpyAsync(du.p, uh.data(), cnt * sizeof(OpUnit<double>), cudaMemcpyHostToDevice, st));
      DevBuf<OpUnit<double>> ex;
      if (Nz > 1) {
        OMB_CU(ex.alloc((size_t)(Nz + 1) * cnt, st));
        OMB_CU(launch_op3d<double>(OP_EFIELD, du.p, cnt, Nx, Ny, Nz, 1, ctx_->tw, ex.p, st));
      } else {
        OMB_CU(launch_op<double>(OP_EFIELD, du.p, cnt, Nx, Ny, 1, ctx_->tw, st));
      }
      k_argmax_abs2<double><<<cnt, 1024, 0, st>>>(scr.p, (long long)N, 3 * (long long)N, cnt, red.p);
      OMB_CU(cudaGetLastError());
      std::vector<double> h(3 * (size_t)cnt);
      OMB_CU(cudaMemcpyAsync(h.data(), red.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
      OMB_CU(cudaStreamSynchronize(st));  // also keeps kh/uh alive until the uploads are done
      for (int j = 0; j < cnt; ++j) {
        const double re = h[3 * j + 1], im = h[3 * j + 2], a = std::hypot(re, im);
        if (a > 0) {
          const int rc = rotate_result(all[c0 + j].first, all[c0 + j].second, re / a, -im / a);
          if (rc) return rc;
        }
      }
    }
  }
  return OMB_OK;
}

int Engine::rotate_result(int t, int b, double c, double s) {
  const size_t n2 = 2 * (*probs_)[tracks_[t].prob].N();
  k_rotate_c64<<<blocks_for(n2), 256, 0, ctx_->stream>>>(store_.p + store_off_[t] + (size_t)b * n2, n2, c, s);
  OMB_CU(cudaGetLastError());
  return OMB_OK;
}

int Engine::result_efield_argmax(int t, int b, long long* idx, double* re, double* im) {
  const TrackSpec& ts = tracks_[t];
  const Problem& P = (*probs_)[ts.prob];
  const size_t N = P.N(), n2 = 2 * N;
  cudaStream_t st = ctx_->stream;
  DevBuf<double> red, kd;
  DevBuf<double2> scr;
  OMB_CU(red.alloc(3, st));
  OMB_CU(kd.alloc(1, st));
  OMB_CU(scr.alloc(3 * N, st));
  const double k = snaps_[t][b].k;
  OMB_CU(cudaMemcpyAsync(kd.p, &k, sizeof(double), cudaMemcpyHostToDevice, st));
  OpUnit<double> u = make_unit<double>(P);
  u.in = store_.p + store_off_[t] + (size_t)b * n2;
  u.scr = scr.p;
  u.k_dev = kd.p;
  u.in_cs = n2; u.scr_cs = 3 * N; u.ncol = 1;
  DevBuf<OpUnit<double>> du;
  OMB_CU(du.alloc(1, st));
  OMB_CU(cudaMemcpyAsync(du.p, &u, sizeof(u), cudaMemcpyHostToDevice, st));
  DevBuf<OpUnit<double>> ex;
  if (P.Nz > 1) {
    OMB_CU(ex.alloc((size_t)(P.Nz + 1), st));
    OMB_CU(launch_op3d<double>(OP_EFIELD, du.p, 1, P.Nx, P.Ny, P.Nz, 1, ctx_->tw, ex.p, st));
  } else {
    OMB_CU(launch_op<double>(OP_EFIELD, du.p, 1, P.Nx, P.Ny, 1, ctx_->tw, st));
  }
  k_argmax_abs2<double><<<1, 1024, 0, st>>>(scr.p, (long long)N, 3 * (long long)N, 1, red.p);
  OMB_CU(cudaGetLastError());
  double h[3];
  OMB_CU(cudaMemcpyAsync(h, red.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaStreamSynchronize(st));
  *idx = (long long)h[0];
  *re = h[1];
  *im = h[2];
  return OMB_OK;
}

}  // namespace omb
