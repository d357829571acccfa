// Device-resident block LOBPCG with an inner Newton iteration on k (sm_100a).
//
// Every piece of per-track state (k, Ritz values, residual norms, locking, Newton
// bookkeeping, the column ranges the operator passes act on) lives in device memory, so
// one iteration is a fixed sequence of kernel launches that is captured once in a CUDA
// graph and replayed; tracks that finished (or whose phase finished) make every kernel
// return at once.
//
// Method.  LOBPCG (Knyazev 2001) with the basis Z = [X | W | P], W = P̂(AX − XΛ) and
// P = W C_W + P C_P.  Rayleigh–Ritz is solved in the Gram metric G = ZᴴZ (FP64):
// G is scaled to unit diagonal, eigen-decomposed, directions with relative Gram
// eigenvalue below a floor are dropped (SVQB, Stathopoulos & Wu 2002), and the projected
// S = ZᴴAZ is eigen-decomposed in the kept basis.  Locking is "soft" and in order:
// converged columns stop receiving W directions but stay in the Rayleigh–Ritz basis.
//
// Newton on k (reference: the per-band loop of ME/src/solve.jl:77-115 and
// ME/src/solvers/gpu.jl:222-237): instead of converging a full eigensolve at every k, a
// Newton step k ← k − (λ_b − ω²)/(2⟨x_b|∂M̂/∂k|x_b⟩) is taken inside the iteration as soon
// as the Ritz value of band b is trustworthy; after a step AX is recomputed at the new k
// and P is dropped.  The final step is only taken from an eigenpair converged to the
// tolerance, and the track stops when that step is below k_tol (the returned k is the
// updated one, as in gpu.jl).  OUTER mode reproduces the reference loop exactly: a step
// only after all block columns converged.
#pragma once

#include "op_kernels.cuh"
#include "pipe.cuh"
#include "smallmat.cuh"

namespace omb {

constexpr int MMAX = 12;         // block columns per track
constexpr int NMAX = 3 * MMAX;   // Rayleigh–Ritz basis size
constexpr int LANES = 2;         // track lanes (streams) of an engine's iteration graph
constexpr int RR_NT = 128;

enum TrackStatus : int {
  TS_RUNNING = 0, TS_CONVERGED = 1, TS_MAXITER = 2, TS_ORTHO = 3, TS_NAN = 4, TS_PHASE_DONE = 5,
};
enum TrackMode : int { MODE_OMEGA2 = 0, MODE_NEWTON_INNER = 1, MODE_NEWTON_OUTER = 2 };

struct TrackState {
  double k;            // current wavevector (the operator passes read it here)
  double k_eig;        // k of the last Newton evaluation (where the returned vector lives)
  double omega2;       // target ω² (Newton modes)
  double dk_last;      // last Newton step
  double hmkh;         // last ⟨x_b|∂M̂/∂k|x_b⟩
  double resid_best;   // stall detection
  double lam[MMAX];
  double resid[MMAX];
  int M, band, need;   // block size, Newton band, bands that must converge
  int nlocked, nWa, nP, nP_next;
  int op_col0, op_ncol;    // A pass over [X | W] columns [col0, col0+ncol)
  int pw_col0, pw_ncol;    // MPB preconditioner pass over W slot columns
  int hmkh_ncol;           // 1 when a Newton step is pending
  int iter, iter_phase, newton_steps, newton_phase, since_newton, stall;
  int status, done, mode, phase;
  int rr_n, rr_rank;
  int cur_par;          // parity of the Y/AY buffers holding the current block
};

template <typename T> struct TrackDesc {
  cplx<T>* Y[2];        // [X | W | P], 3M columns of n2 complex, per parity
  cplx<T>* AY[2];       // [AX | AW | AP]
  TrackState* st;
  double2* coef;        // C (NMAX×MMAX) then CP (NMAX×MMAX), row-major [l][m]
  const cplx<T>* coefT; // the same coefficients in the block's precision
  double2* gram_acc;    // G then S (NMAX×NMAX each, upper triangles), summed by k_gram
  double* res_acc;      // ‖R‖² per block column, summed by k_update
  double* hmkh_part;    // row_out partial sums of the HMkH pass
  long long n2;         // vector length (2·Nx·Ny complex)
  int Nx, Ny, M, hmkh_nb;
  double inv_dx, inv_dy, eps_mean;
  int Nz;                // z-periodic cells: slabs (1 for a 2D cell)
  double inv_dz;
};

struct IterParams {
  double tol, k_tol;
  double lock_tol;     // locking threshold of this phase
  double tau_phase;    // phase-A exit residual (FP32 floor) — equals tol in the last phase
  double dk_phase;     // phase-A exit Newton step
  double gram_drop;    // relative Gram eigenvalue floor
  double jacobi_tol2;  // k_rr's Jacobi stops at ‖offdiag‖²_F ≤ jacobi_tol2·‖A‖²_F
  int maxiter, max_newton, last_phase, prec_diag;
};

__device__ __forceinline__ int z_phys(const TrackState& s, int M, int l) {
  if (l < M) return l;
  l -= M;
  if (l < s.nWa) return M + s.nlocked + l;
  return 2 * M + (l - s.nWa);
}

// ---------------------------------------------------------------------------------
// Streaming kernels: the tall-skinny Gram products and the Rayleigh–Ritz update.
//
// Both stream the row tiles of the live tracks through shared memory with bulk copies
// (one producer warp, a ring of `stages` buffers guarded by full/empty mbarriers) while
// the consumer warps compute.  The rows of all live tracks form one sequence of tiles
// (k_live_prefix counts them after the Newton step of the iteration); CTA b of a 1D grid
// of X takes the tiles that start in [b·W/X, (b+1)·W/X) of the tiles' summed cost W (a
// tile of a wide track costs several times one of a narrow track), so the work stays
// spread evenly over every SM however few tracks are left.  Per-track sums leave each CTA through FP64 atomics into the
// track's accumulators, which k_rr (Gram) and k_control (‖R‖²) read and clear.

// Tile sequence of one CTA: tiles of R rows of the live tracks, in track order.
struct TileWalk {
  const int* pre;      // prefix of tile counts over tracks (pre[t+1] − pre[t] tiles of track t)
  int ntracks, t;      // current track
  long long i, end;    // current global tile, one past the last
  int R;
  // first global tile whose cost-weighted start is ≥ x (wpre: prefix of the tracks' costs,
  // each a fixed F followed by its tiles, the tiles of one track costing the same; a point
  // inside a track's F maps to its first tile)
  __device__ __forceinline__ long long tile_at(const long long* wpre, long long F, long long x) const {
    if (x >= wpre[ntracks]) return pre[ntracks];
    int lo = 0, hi = ntracks - 1;  // first track with wpre[t+1] > x
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (wpre[mid + 1] > x) hi = mid; else lo = mid + 1;
    }
    const long long nt = pre[lo + 1] - pre[lo];
    const long long wt = (wpre[lo + 1] - wpre[lo] - F) / nt;
    const long long xr = x - wpre[lo] - F;
    const long long j = xr > 0 ? (xr + wt - 1) / wt : 0;
    return pre[lo] + (j < nt ? j : nt);
  }
  // wpre == nullptr: every tile costs the same; F: the fixed cost per live track in wpre
  __device__ __forceinline__ void start(const int* pre_, const long long* wpre, int ntracks_, int R_,
                                        long long F = 0) {
    pre = pre_; ntracks = ntracks_; R = R_;
    if (wpre && wpre[ntracks] > 0) {
      const long long W = wpre[ntracks];
      i = tile_at(wpre, F, (long long)blockIdx.x * W / gridDim.x);
      end = tile_at(wpre, F, (long long)(blockIdx.x + 1) * W / gridDim.x);
    } else {
      const long long T = pre[ntracks];
      i = (long long)blockIdx.x * T / gridDim.x;
      end = (long long)(blockIdx.x + 1) * T / gridDim.x;
    }
    // first track whose tile range contains i (skips tracks with no tiles)
    int lo = 0, hi = ntracks - 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (pre[mid + 1] > i) hi = mid; else lo = mid + 1;
    }
    t = lo;
  }
  __device__ __forceinline__ bool valid() const { return i < end; }
  __device__ __forceinline__ long long row0() const { return (i - pre[t]) * (long long)R; }
  __device__ __forceinline__ void next() {
    ++i;
    while (t < ntracks - 1 && pre[t + 1] <= i) ++t;
  }
  // is the current tile the last of its track within this CTA's range?
  __device__ __forceinline__ bool last_of_track() const { return i + 1 >= end || pre[t + 1] <= i + 1; }
};

// Live-tile prefixes for the Gram (rows per tile rg) and update (ru) kernels, and the
// prefixes of their cost-weighted tile counts (wpre_g, wpre_u).
__global__ void k_live_prefix(TrackState* const* __restrict__ states, const long long* __restrict__ n2,
                              int ntracks, int rg, int ru, int* __restrict__ pre_g, int* __restrict__ pre_u,
                              long long* __restrict__ wpre_g, long long* __restrict__ wpre_u);
// Relative cost of one tile of a track with n block columns of which M are X: the Gram's 4×4
// items (each 16 complex products per row) plus its loads plus a fixed GRAM_TILE_FIXED, and
// GRAM_TRACK_COST once per track for the flush of its sums (each CTA that takes part in a
// track adds its partial sums to the track's Gram); the update's n·M products per row of X,
// AX, P, AP plus its 4M stores plus a fixed 16 per tile (pipeline round trips and bulk-copy
// set-up: per-CTA times on B200 fit 1.25 µs per tile + 0.08 µs per unit of n·M + 4M to 5 %).
constexpr long long GRAM_TILE_FIXED = 48;
constexpr long long GRAM_TRACK_COST = 390;
__host__ __device__ __forceinline__ long long gram_tile_cost(int n) {
  const int nb4 = (n + 3) / 4;
  return 8LL * nb4 * (nb4 + 1) + n + GRAM_TILE_FIXED;
}
__host__ __device__ __forceinline__ long long update_tile_cost(int n, int M) { return (long long)n * M + 4LL * M + 16; }

// ---- Gram ---------------------------------------------------------------------------
// G = ZᴴZ and S = ZᴴAZ (upper triangles).  The outputs are cut into 4×4 blocks (items);
// items·SPLIT ≤ 512 consumer threads, each thread owns one item and every SPLIT-th row of
// a tile (16 complex accumulators), and the SPLIT threads of an item are adjacent lanes,
// so their partial sums meet in a shuffle reduction (FP64) before the atomics.
template <typename T> struct GramCfg {
  static constexpr int NCW = 15;                                 // consumer warps
  static constexpr int NT = (NCW + 1) * 32;                      // + the producer warp (16 warps: 128 regs;
                                                                 // FP32 keeps its compensation terms in local memory)
  static constexpr int PAD = 16 / (int)sizeof(cplx<T>);          // column pad: 16 bytes
  // Z columns at [0, n), AZ columns at [n4, n4 + n) with n4 = 4·⌈n/4⌉: the 4×4 blocks read
  // up to column 2·n4 − 1, so a stage holds 2·4·⌈nmax/4⌉ columns of R + PAD elements
  static __host__ __device__ constexpr int n4(int n) { return (n + 3) / 4 * 4; }
  static __host__ __device__ constexpr size_t stage_elems(int nmax, int R) { return (size_t)2 * n4(nmax) * (R + PAD); }
  // rows per tile: the largest multiple of 64 (≤ 256 FP32, ≤ 128 FP64) whose stage fits in ≈95 KB
  static __host__ int rows(int nmax) {
    const int cap = sizeof(T) == 4 ? 256 : 128;
    int R = (int)(95 * 1024 / (2 * n4(nmax) * sizeof(cplx<T>))) - PAD;
    R = R / 64 * 64;
    return R < 64 ? 64 : (R > cap ? cap : R);
  }
  // FP64 reduction buffer after the ring: 16 entries per item
  static __host__ __device__ constexpr int red_entries(int nmax) {
    return 2 * ((nmax + 3) / 4) * ((nmax + 3) / 4 + 1) / 2 * 16;
  }
};

// Named barrier over the first `count` threads of the CTA (the consumer warps).
__device__ __forceinline__ void bar_sync_count(int id, int count) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(count) : "memory");
}
// Item q of a track with nb4 column blocks: matrix (0: G, 1: S) and block (bi ≤ bj).
__device__ __forceinline__ void gram_item(int q, int nblk, int nb4, int& which, int& bi, int& bj) {
  which = q / nblk;
  int r = q - which * nblk;
  bi = 0;
  while (r >= nb4 - bi) { r -= nb4 - bi; ++bi; }
  bj = bi + r;
}

// s + lo += x with the rounding error of the FP32 addition carried in lo (two-sum: Knuth,
// TAOCP vol. 2, 4.2.2; the error of s + x is exact in FP32).
__device__ __forceinline__ void two_sum_acc(float& s, float& lo, float x) {
  const float t = s + x;
  const float xp = t - s, sp = t - xp;
  lo += (s - sp) + (x - xp);
  s = t;
}

// (acc, lo) += t entry by entry with two-sum; t is cleared.
__device__ __forceinline__ void gram_fold(float2 (&acc)[4][4], float2 (&lo)[4][4], float2 (&t)[4][4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      two_sum_acc(acc[i][j].x, lo[i][j].x, t[i][j].x);
      two_sum_acc(acc[i][j].y, lo[i][j].y, t[i][j].y);
      t[i][j] = make_float2(0.f, 0.f);
    }
}

template <typename T>
__global__ void __launch_bounds__(GramCfg<T>::NT, 1)
    k_gram(const TrackDesc<T>* __restrict__ D, const int* __restrict__ pre, const long long* __restrict__ wpre,
           int ntracks, int par, int nmax, int R, int stages, int* __restrict__ err, uint64_t wait_ns) {
  using C = cplx<T>;
  using Cfg = GramCfg<T>;
  const int CS = R + Cfg::PAD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
  uint64_t* empty = full + 8;
  C* stage0 = reinterpret_cast<C*>(smem_raw + 128);
  const size_t sel = Cfg::stage_elems(nmax, R);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int q = 0; q < stages; ++q) { mbar_init(&full[q], 1); mbar_init(&empty[q], Cfg::NCW); }
    mbar_init_fence();
  }
  __syncthreads();
  TileWalk w;
  w.start(pre, wpre, ntracks, R, GRAM_TRACK_COST);
  if (warp == Cfg::NCW) {
    // ---- producer: one bulk copy per column segment of the tile
    int q = 0, fills[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t ph = 0;
    bool ok = true;
    for (; w.valid() && ok; w.next()) {
      const TrackDesc<T>& d = D[w.t];
      const TrackState& s = *d.st;
      const int M = d.M, n = M + s.nWa + s.nP;
      const long long r0 = w.row0();
      const int rows = (int)min((long long)R, d.n2 - r0);
      if (lane == 0) {
        ok = mbar_wait(&empty[q], ph ^ 1, wait_ns);
        if (ok) mbar_arrive_expect_tx(&full[q], (uint32_t)(2 * n * rows * sizeof(C)));
        else pipe_fail(err, PIPE_EMPTY_TIMEOUT);
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      C* st = stage0 + (size_t)q * sel;
      const int nz = Cfg::n4(n);
      for (int c = lane; c < 2 * n; c += 32) {
        const int l = c < n ? c : c - n;
        const C* src = (c < n ? d.Y[par] : d.AY[par]) + (size_t)z_phys(s, M, l) * d.n2 + r0;
        bulk_g2s(st + (size_t)(c < n ? c : nz + l) * CS, src, (uint32_t)(rows * sizeof(C)), &full[q]);
      }
      fills[q]++;
      if (++q == stages) { q = 0; ph ^= 1; }
    }
    // leave no copy in flight: the last fill of every stage has landed
    if (lane == 0)
      for (int k = 0; k < stages; ++k)
        if (fills[k] > 0 && !mbar_wait(&full[k], (uint32_t)((fills[k] - 1) & 1), drain_limit(wait_ns)))
          pipe_fail(err, PIPE_DRAIN_TIMEOUT);
    return;
  }
  // ---- consumers: thread (item, sub) accumulates one 4×4 block over rows sub, sub+split, …
  constexpr int NC = Cfg::NCW * 32;
  const int tid = threadIdx.x;
  double2* red = reinterpret_cast<double2*>(smem_raw + 128 + (size_t)stages * sel * sizeof(C));
  for (int e = tid; e < Cfg::red_entries(nmax); e += NC) red[e] = make_double2(0, 0);
  bar_sync_count(1, NC);
  int q = 0;
  uint32_t ph = 0;
  bool failed = false;
  // FP32: a thread's rows are summed into t, and t into the compensated pair (acc, lo) by
  // two-sum (Knuth) once the thread has summed GRAM_FOLD_ROWS rows (or a whole tile's share,
  // when that is more), so the rounding error of the track's sum stays at the FP32 level of
  // that many rows instead of growing with the number of tiles; FP64 sums directly.  Folding
  // by rows rather than every tile keeps the fold (32 two-sums, the compensation terms in
  // local memory) off the tiles of narrow tracks, whose items are split over ≈240 threads
  // with one or two rows each.
  constexpr bool COMP = sizeof(T) == 4;
  constexpr int GRAM_FOLD_ROWS = 16;
  C acc[4][4], lo[COMP ? 4 : 1][COMP ? 4 : 1], t[COMP ? 4 : 1][COMP ? 4 : 1];
  int tcnt = 0;
  int cur = -1, items = 0, split = 1, nblk = 0, nb4 = 1, n = 0, item = 0, sub = 0, which = 0, bi = 0, bj = 0;
  bool active = false;
  for (; w.valid(); w.next()) {
    const TrackDesc<T>& d = D[w.t];
    if (w.t != cur) {  // new track: its item layout
      cur = w.t;
      const TrackState& s = *d.st;
      n = d.M + s.nWa + s.nP;
      nb4 = (n + 3) / 4;
      nblk = nb4 * (nb4 + 1) / 2;
      items = 2 * nblk;
      split = max(1, NC / items);
      item = tid / split;
      sub = tid - item * split;
      active = item < items;
      gram_item(active ? item : 0, nblk, nb4, which, bi, bj);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = mk<C>(0, 0);
      if constexpr (COMP) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) { lo[i][j] = mk<C>(0, 0); t[i][j] = mk<C>(0, 0); }
        tcnt = 0;
      }
    }
    const int rows = (int)min((long long)R, d.n2 - w.row0());
    bool ok = failed ? false : mbar_wait(&full[q], ph, wait_ns);
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && !failed) { pipe_fail(err, PIPE_FULL_TIMEOUT); failed = true; }
    if (!failed) {
      if (active) {
        const C* st = stage0 + (size_t)q * sel;
        const C* za = st + (size_t)(4 * bi) * CS;
        const C* zb = st + (size_t)((which ? Cfg::n4(n) : 0) + 4 * bj) * CS;
        if constexpr (COMP) {
          const int mine = rows > sub ? (rows - sub + split - 1) / split : 0;
          if (tcnt > 0 && tcnt + mine > GRAM_FOLD_ROWS) {
            gram_fold(acc, lo, t);
            tcnt = 0;
          }
          tcnt += mine;
#pragma unroll 2
          for (int r = sub; r < rows; r += split) {
            C a[4], b[4], bs[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) { a[i] = za[i * CS + r]; b[i] = zb[i * CS + r]; }
#pragma unroll
            for (int j = 0; j < 4; ++j) bs[j] = make_float2(b[j].y, b[j].x);
            // conj(a)·b = a.x·(b.x, b.y) + a.y·(b.y, −b.x): two packed FP32x2 FMAs per product
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const float2 ax = make_float2(a[i].x, a[i].x), ay = make_float2(a[i].y, -a[i].y);
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                t[i][j] = __ffma2_rn(ax, b[j], t[i][j]);
                t[i][j] = __ffma2_rn(ay, bs[j], t[i][j]);
              }
            }
          }
        } else {
#pragma unroll 2
          for (int r = sub; r < rows; r += split) {
            C a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) { a[i] = za[i * CS + r]; b[i] = zb[i * CS + r]; }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
              for (int j = 0; j < 4; ++j) {  // conj(a)·b
                acc[i][j].x += a[i].x * b[j].x + a[i].y * b[j].y;
                acc[i][j].y += a[i].x * b[j].y - a[i].y * b[j].x;
              }
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[q]);
    }
    if (++q == stages) { q = 0; ph ^= 1; }
    if (w.last_of_track()) {
      // the split partial sums of each item meet in shared memory (FP64), then one global
      // atomic per matrix entry.  The split threads of an item are a contiguous run of lanes
      // (item = tid / split), so each warp first sums its part of every run with a segmented
      // shuffle (suffix sums toward the run's first lane; every lane of the warp takes part,
      // idle ones with zeros) and only that first lane adds to shared memory: a few adds per
      // entry instead of `split` (up to 80) contending ones.
      if constexpr (COMP) {
        if (active && tcnt > 0) gram_fold(acc, lo, t);
      }
      {
        const int key = active ? item : -1;
        const unsigned seg = __match_any_sync(0xffffffffu, key);
        const int head = __ffs(seg) - 1;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            double vx = 0.0, vy = 0.0;
            if (active) {
              vx = (double)acc[i][j].x;
              vy = (double)acc[i][j].y;
              if constexpr (COMP) { vx += (double)lo[i][j].x; vy += (double)lo[i][j].y; }
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
              const double tx = __shfl_down_sync(0xffffffffu, vx, o), ty = __shfl_down_sync(0xffffffffu, vy, o);
              if (lane + o < 32 && ((seg >> (lane + o)) & 1u)) { vx += tx; vy += ty; }
            }
            if (active && lane == head) {
              atomicAdd(&red[item * 16 + i * 4 + j].x, vx);
              atomicAdd(&red[item * 16 + i * 4 + j].y, vy);
            }
          }
      }
      bar_sync_count(1, NC);
      for (int e = tid; e < items * 16; e += NC) {
        int wh, ei, ej;
        gram_item(e >> 4, nblk, nb4, wh, ei, ej);
        const int a = 4 * ei + ((e >> 2) & 3), b = 4 * ej + (e & 3);
        const double2 v = red[e];
        if (!failed && a < n && b < n && a <= b) {
          double2* g = d.gram_acc + (size_t)wh * NMAX * NMAX + (size_t)a * NMAX + b;
          atomicAdd(&g->x, v.x);
          atomicAdd(&g->y, v.y);
        }
        red[e] = make_double2(0, 0);
      }
      bar_sync_count(1, NC);
      cur = -1;
    }
  }
}

// ---- Update -----------------------------------------------------------------------
// X ← ZC, AX ← AZC, P ← ZCP, AP ← AZCP into the other parity, then R = AX − XΛ,
// W = P̂_diag R (or R when the MPB preconditioner follows) and ‖R‖².  One consumer thread
// per tile row; a stage holds LG columns of Z and AZ for the tile plus the matching rows
// of C and CP (in the block's precision), so the coefficients follow the tile's track.
static_assert(MMAX == 12, "k_update dispatches M = 1..12");
template <typename T> struct UpdCfg {
  // rows per tile = consumer threads; with the producer warp 16 warps (FP32, 128 registers)
  // or 9 warps (FP64, whose M ≤ 6 tile bodies need ≈170 registers)
  static constexpr int R = sizeof(T) == 4 ? 480 : 256;
  static constexpr int LG = sizeof(T) == 4 ? 4 : 2;      // columns per stage
  static constexpr int NCW = R / 32;
  static constexpr int NT = (NCW + 1) * 32;
  static constexpr int STAGES = 6;
  // stage: Z[LG][R], AZ[LG][R], C[LG][MMAX], CP[LG][MMAX]
  static constexpr size_t stage_elems = (size_t)2 * LG * R + (size_t)2 * LG * MMAX;
  static constexpr size_t smem = 128 + STAGES * stage_elems * sizeof(cplx<T>);
};

// One tile of the update for a track with M block columns (compile-time, so the column
// loops unroll without per-column branches).  Entries of CP beyond nP_next may be stale;
// they only reach P columns that are not stored.
template <typename T, int M, int MB>
__device__ __forceinline__ void update_tile(const TrackDesc<T>& d, const TrackState& s, long long r0, int rows,
                                            int par, int prec_diag, const cplx<T>* stage0, uint64_t* full,
                                            uint64_t* empty, int& q, uint32_t& ph, bool& failed,
                                            double (&racc)[MB], int* err, uint64_t wait_ns) {
  using C = cplx<T>;
  using Cfg = UpdCfg<T>;
  constexpr int R = Cfg::R, LG = Cfg::LG, S = Cfg::STAGES;
  const int r = threadIdx.x, lane = r & 31;
  const int n = M + s.nWa + s.nP, nPn = s.nP_next;
  C x[M], ax[M], p[M], ap[M];
#pragma unroll
  for (int m = 0; m < M; ++m) x[m] = ax[m] = p[m] = ap[m] = mk<C>(0, 0);
  for (int l0 = 0; l0 < n; l0 += LG) {
    bool ok = failed ? false : mbar_wait(&full[q], ph, wait_ns);
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && !failed) { pipe_fail(err, PIPE_FULL_TIMEOUT); failed = true; }
    if (!failed) {
      const C* st = stage0 + (size_t)q * Cfg::stage_elems;
      const C* Cs = st + 2 * LG * R;
      const C* CPs = Cs + LG * MMAX;
      if (r < rows) {
#pragma unroll
        for (int j = 0; j < LG; ++j) {
          if (l0 + j < n) {
            const C z = st[j * R + r], az = st[(LG + j) * R + r];
#pragma unroll
            for (int m = 0; m < M; ++m) {
              const C c = Cs[j * MMAX + m];
              x[m] = cmac(x[m], z, c);
              ax[m] = cmac(ax[m], az, c);
            }
            if (l0 + j >= M) {  // the X rows of CP are zero
#pragma unroll
              for (int m = 0; m < M; ++m) {
                const C c = CPs[j * MMAX + m];
                p[m] = cmac(p[m], z, c);
                ap[m] = cmac(ap[m], az, c);
              }
            }
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[q]);
    }
    if (++q == S) { q = 0; ph ^= 1; }
  }
  if (failed) return;
  if (r0 == 0 && r == 0) d.st->cur_par = par ^ 1;
  if (r < rows) {
    const long long row = r0 + r, n2 = d.n2;
    C* __restrict__ Yo = d.Y[par ^ 1];
    C* __restrict__ AYo = d.AY[par ^ 1];
    T pscale = T(1);
    if (prec_diag) {
      const long long pix = row >> 1;
      const int ix = (int)(pix % d.Nx);
      const long long rest = pix / d.Nx;
      const int iy = (int)(rest % d.Ny), iz = (int)(rest / d.Ny);
      const T k = (T)(s.k - freq_index(iz, d.Nz) * d.inv_dz);  // w_z = k − g_z
      const T gx = T(freq_index(ix, d.Nx)) * (T)d.inv_dx, gy = T(freq_index(iy, d.Ny)) * (T)d.inv_dy;
      pscale = T(d.eps_mean) / (gx * gx + gy * gy + k * k);
    }
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const C res = ax[m] - x[m] * (T)s.lam[m];
      racc[m] += (double)res.x * res.x + (double)res.y * res.y;
      Yo[(size_t)m * n2 + row] = x[m];
      AYo[(size_t)m * n2 + row] = ax[m];
      Yo[(size_t)(M + m) * n2 + row] = res * pscale;
    }
#pragma unroll
    for (int m = 0; m < M; ++m) {
      if (m < nPn) {
        Yo[(size_t)(2 * M + m) * n2 + row] = p[m];
        AYo[(size_t)(2 * M + m) * n2 + row] = ap[m];
      }
    }
  }
}

// MB: the largest block size of the launch (the tile bodies for M ≤ MB are compiled in).
template <typename T, int MB>
__global__ void __launch_bounds__(UpdCfg<T>::NT, 1)
    k_update(const TrackDesc<T>* __restrict__ D, const int* __restrict__ pre, const long long* __restrict__ wpre,
             int ntracks, int par, int prec_diag, int* __restrict__ err, uint64_t wait_ns) {
  using C = cplx<T>;
  using Cfg = UpdCfg<T>;
  constexpr int R = Cfg::R, LG = Cfg::LG, S = Cfg::STAGES;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
  uint64_t* empty = full + 8;
  C* stage0 = reinterpret_cast<C*>(smem_raw + 128);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int q = 0; q < S; ++q) { mbar_init(&full[q], 1); mbar_init(&empty[q], Cfg::NCW); }
    mbar_init_fence();
  }
  __syncthreads();
  TileWalk w;
  w.start(pre, wpre, ntracks, R);
  if (warp == Cfg::NCW) {
    // ---- producer
    int q = 0, fills[S] = {};
    uint32_t ph = 0;
    bool ok = true;
    for (; w.valid() && ok; w.next()) {
      const TrackDesc<T>& d = D[w.t];
      const TrackState& s = *d.st;
      if (s.done) continue;  // finished in k_rr after the tiles were counted
      const int M = d.M, n = M + s.nWa + s.nP;
      const long long r0 = w.row0();
      const int rows = (int)min((long long)R, d.n2 - r0);
      for (int l0 = 0; l0 < n && ok; l0 += LG) {
        const int nl = min(LG, n - l0);
        if (lane == 0) {
          ok = mbar_wait(&empty[q], ph ^ 1, wait_ns);
          if (ok)
            mbar_arrive_expect_tx(&full[q], (uint32_t)((2 * nl * rows + 2 * nl * MMAX) * sizeof(C)));
          else
            pipe_fail(err, PIPE_EMPTY_TIMEOUT);
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) break;
        C* st = stage0 + (size_t)q * Cfg::stage_elems;
        if (lane < 2 * nl) {
          const int j = lane % nl, l = l0 + j;
          const C* src = (lane < nl ? d.Y[par] : d.AY[par]) + (size_t)z_phys(s, M, l) * d.n2 + r0;
          bulk_g2s(st + (size_t)(lane < nl ? j : LG + j) * R, src, (uint32_t)(rows * sizeof(C)), &full[q]);
        } else if (lane == 2 * LG) {
          bulk_g2s(st + 2 * LG * R, d.coefT + (size_t)l0 * MMAX, (uint32_t)(nl * MMAX * sizeof(C)), &full[q]);
        } else if (lane == 2 * LG + 1) {
          bulk_g2s(st + 2 * LG * R + LG * MMAX, d.coefT + (size_t)NMAX * MMAX + (size_t)l0 * MMAX,
                   (uint32_t)(nl * MMAX * sizeof(C)), &full[q]);
        }
        fills[q]++;
        if (++q == S) { q = 0; ph ^= 1; }
      }
    }
    if (lane == 0)
      for (int k = 0; k < S; ++k)
        if (fills[k] > 0 && !mbar_wait(&full[k], (uint32_t)((fills[k] - 1) & 1), drain_limit(wait_ns)))
          pipe_fail(err, PIPE_DRAIN_TIMEOUT);
    return;
  }
  // ---- consumers: thread r owns row row0 + r of each tile
  int q = 0;
  uint32_t ph = 0;
  bool failed = false;
  double racc[MB];
#pragma unroll
  for (int m = 0; m < MB; ++m) racc[m] = 0;
  for (; w.valid(); w.next()) {
    const TrackDesc<T>& d = D[w.t];
    const TrackState& s = *d.st;
    if (s.done) continue;
    const long long r0 = w.row0();
    const int rows = (int)min((long long)R, d.n2 - r0);
    switch (d.M) {
#define OMB_UPD_CASE(MM)                                                                                \
  case MM:                                                                                              \
    if constexpr (MM <= MB)                                                                             \
      update_tile<T, (MM <= MB ? MM : 1), MB>(d, s, r0, rows, par, prec_diag, stage0, full, empty, q, ph, \
                                              failed, racc, err, wait_ns);                              \
    break;
      OMB_UPD_CASE(1) OMB_UPD_CASE(2) OMB_UPD_CASE(3) OMB_UPD_CASE(4) OMB_UPD_CASE(5) OMB_UPD_CASE(6)
      OMB_UPD_CASE(7) OMB_UPD_CASE(8) OMB_UPD_CASE(9) OMB_UPD_CASE(10) OMB_UPD_CASE(11) OMB_UPD_CASE(12)
#undef OMB_UPD_CASE
      default: break;
    }
    if (w.last_of_track()) {
#pragma unroll
      for (int m = 0; m < MB; ++m) {
        double v = racc[m];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && m < d.M && !failed) atomicAdd(d.res_acc + m, v);
        racc[m] = 0;
      }
    }
  }
}

// ---------------------------------------------------------------------------------
// Rayleigh–Ritz: one CTA per track.  Reads the track's Gram accumulators (and clears
// them for the next iteration); writes C, CP in FP64 and in FP32 (coef32).
__global__ void __launch_bounds__(RR_NT) k_rr(TrackState* const* __restrict__ states,
                                               double2* const* __restrict__ gram_accs,
                                               double2* const* __restrict__ coefs,
                                               float2* const* __restrict__ coefs32, int ntracks,
                                               IterParams prm);

// ---------------------------------------------------------------------------------
// Control (after the update; one warp per track) and Newton (after the HMkH pass; one
// thread per track).
__global__ void k_control(TrackState* const* __restrict__ states, double* const* __restrict__ res_accs,
                          int ntracks, IterParams prm);
__global__ void k_newton(TrackState* const* __restrict__ states, double* const* __restrict__ hmkh_parts,
                         const int* __restrict__ hmkh_nb, int ntracks, IterParams prm);

// Random start block (uniform in [-1,1]² per entry from a counter-based hash).
template <typename T>
__global__ void k_random_block(cplx<T>* X, long long n2, int ncol, unsigned long long seed) {
  const size_t tot = (size_t)n2 * ncol;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double a = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    z = z * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double b = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    X[i] = mk<cplx<T>>((T)(2 * a - 1), (T)(2 * b - 1));
  }
}

}  // namespace omb
