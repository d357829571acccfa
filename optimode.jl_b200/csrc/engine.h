// Batched device LOBPCG/Newton engine: host side.
#pragma once

#include <memory>
#include <vector>

#include "context.h"
#include "lobpcg.cuh"

namespace omb {

struct SolveOptions {
  double tol = 1e-8;
  double k_tol = 1e-8;
  int max_newton = 60;
  int maxiter = 1000;
  int precision = OMB_PREC_MIXED;
  bool prec_diag = false;
  int newton_mode = MODE_NEWTON_INNER;
  uint64_t seed = 0;
  int guard = 1;  // extra block columns of a Newton track
};

// One eigensolve unit: a Newton band track (solve_k) or a fixed-k block (solve_ω²).
// In the reference-loop mode a unit runs `nbands` bands one after another (band b+1
// continues from band b's block and k).
struct TrackSpec {
  int prob = 0;             // index into the problem list
  int band = 0;             // (first) Newton band
  int nbands = 1;           // bands run in turn (MODE_NEWTON_OUTER)
  int M = 1;                // block columns
  int need = 1;             // leading columns that must converge
  int mode = MODE_NEWTON_INNER;
  double omega2 = 0, k0 = 0;
  const double* guess = nullptr;  // host, interleaved complex, nguess columns of length n2
  int nguess = 0;
  const double2* guess_dev[MMAX] = {};  // or device FP64 columns (another engine's results)
  int nguess_dev = 0;
  // Two-wave runs (mixed precision, inner Newton): a wave-1 track starts its FP32 phase once
  // the wave-0 tracks have finished theirs, from the FP32 block of wave-0 track `src` (the
  // same band of a solved neighbour at ω_src) with k extrapolated to first order in ω; both
  // waves then share one FP64 phase.
  int wave = 0;
  int src = -1;
  double omega_src = 0;
};

class Engine {
 public:
  Engine(omb_ctx* ctx, std::vector<Problem>* problems, std::vector<TrackSpec> tracks, SolveOptions opt);
  ~Engine();
  // Run all phases (and, in the reference-loop mode, all bands) to completion.
  int run();
  // Result b of track t: its state when the band finished, the FP64 eigenvector (band
  // column of the block, or block column b for solve_ω²) and the argmax of its E field.
  const TrackState& result_state(int t, int b) const { return snaps_[t][b]; }
  int fetch_result(int t, int b, double* out);
  // device address of result b of track t (FP64, n2 complex); valid while the engine lives
  const double2* result_dev(int t, int b) const {
    return store_.p + store_off_[t] + (size_t)b * 2 * (*probs_)[tracks_[t].prob].N();
  }
  int fetch_block_column(int t, int col, double* out);
  int result_efield_argmax(int t, int b, long long* idx, double* re, double* im);
  // multiply result b of track t by the unit phase c + i s on the device
  int rotate_result(int t, int b, double c, double s);
  // phase gauge of every finished result on the device: the largest E component of each
  // becomes real and positive (batched per grid: one E-field pass, one argmax, one sync)
  int canonicalize_results();
  int64_t graph_launches() const { return launches_; }
  int64_t kernel_launches() const { return kernels_; }
  int max_iterations() const;

 private:
  // mode: 0 fresh buffers and blocks, 1 continue from the current block (next reference-loop
  // band), 2 keep buffers and blocks (the tracks of wave_ were set up by start_wave)
  template <typename T> int run_phase(int phase, bool last, double tau, double lock_tol, int mode);
  int start_wave(int wave);
  template <typename T> int init_block(int phase);
  int upload_states();
  int download_states();
  int snapshot(int round);
  size_t col_offset(int t, int col) const;  // complex offset of a column of the current block

  omb_ctx* ctx_;
  std::vector<Problem>* probs_;
  std::vector<TrackSpec> tracks_;
  SolveOptions opt_;
  int nt_ = 0;
  int round_ = 0;
  int wave_ = -1;  // the wave a phase runs (-1: every track)
  int last_prec_ = 1;  // precision of the buffers holding the final block (0 fp32, 1 fp64)
  int64_t launches_ = 0, kernels_ = 0;

  struct Group { int off, n, Nx, Ny, Mmax, Nz; };
  std::vector<Group> groups_;
  std::vector<int> order_;  // tracks sorted by grid size

  DevBuf<TrackState> d_states_;
  std::vector<TrackState> host_states_;
  DevBuf<double2> coef_, gram_acc_;
  DevBuf<float2> coef32_;
  DevBuf<double> res_acc_, hmkh_part_;
  DevBuf<TrackState*> d_state_ptrs_;
  DevBuf<double2*> d_gram_ptrs_, d_coef_ptrs_;
  DevBuf<float2*> d_coef32_ptrs_;
  DevBuf<double*> d_res_ptrs_, d_hmkh_ptrs_;
  DevBuf<int> d_hmkh_nb_;
  DevBuf<long long> d_n2_;
  DevBuf<int> d_pre_;   // live-tile prefixes: Gram tiles [0, nt], update tiles [nt+1, 2nt+1]
  DevBuf<long long> d_wpre_;  // the same prefixes weighted by each tile's cost
  DevBuf<int> d_err_;   // first pipeline error of the streaming kernels (0: none)

  // block buffers of the current precision (Y/AY per parity, scratch)
  DevBuf<float2> y32_, s32_;
  DevBuf<double2> y64_, s64_;
  std::vector<size_t> yoff_, soff_;  // per-track offsets (complex elements) into the pools

  // finished bands: FP64 vectors on the device and the state at the end of each band
  DevBuf<double2> store_;
  std::vector<size_t> store_off_;  // per track; band b at store_off_[t] + b·n2
  std::vector<std::vector<TrackState>> snaps_;
};

}  // namespace omb
