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
#include "smallmat.cuh"

namespace omb {

constexpr int MMAX = 12;         // block columns per track
constexpr int NMAX = 3 * MMAX;   // Rayleigh–Ritz basis size
constexpr int GRAM_ROWS = 64;    // rows per Gram tile
constexpr int UPD_ROWS = 64;     // rows per update tile
constexpr int GRAM_NT = 256;
constexpr int UPD_NT = 256;
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
  double2* gram_part;   // [gram_chunks][2·NMAX·NMAX]
  double* res_part;     // [upd_chunks][MMAX]
  double* hmkh_part;    // row_out partial sums of the HMkH pass
  long long n2;         // vector length (2·Nx·Ny complex)
  int Nx, Ny, M, hmkh_nb;
  double inv_dx, inv_dy, eps_mean;
};

struct IterParams {
  double tol, k_tol;
  double lock_tol;     // locking threshold of this phase
  double tau_phase;    // phase-A exit residual (FP32 floor) — equals tol in the last phase
  double dk_phase;     // phase-A exit Newton step
  double gram_drop;    // relative Gram eigenvalue floor
  int maxiter, max_newton, last_phase, prec_diag, gram_chunks, upd_chunks;
};

__device__ __forceinline__ int z_phys(const TrackState& s, int M, int l) {
  if (l < M) return l;
  l -= M;
  if (l < s.nWa) return M + s.nlocked + l;
  return 2 * M + (l - s.nWa);
}

// ---------------------------------------------------------------------------------
// Gram: partial G = ZᴴZ and S = ZᴴAZ over row tiles (FP64 accumulation).
template <typename T>
__global__ void __launch_bounds__(GRAM_NT) k_gram(const TrackDesc<T>* __restrict__ D, int par, int nchunk) {
  using C = cplx<T>;
  const TrackDesc<T>& d = D[blockIdx.y];
  const TrackState& s = *d.st;
  if (s.done) return;
  const int M = d.M;
  const int n = M + s.nWa + s.nP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Zs = reinterpret_cast<C*>(smem_raw);      // [l][r]
  C* AZs = Zs + (size_t)n * GRAM_ROWS;
  __shared__ int phys[NMAX];
  for (int l = threadIdx.x; l < n; l += GRAM_NT) phys[l] = z_phys(s, M, l);
  constexpr int QMAX = (2 * NMAX * NMAX + GRAM_NT - 1) / GRAM_NT;
  double2 acc[QMAX];
#pragma unroll
  for (int i = 0; i < QMAX; ++i) acc[i] = make_double2(0, 0);
  const int nq = 2 * n * n;
  const long long n2 = d.n2;
  const C* Y = d.Y[par];
  const C* AY = d.AY[par];
  const long long ntile = (n2 + GRAM_ROWS - 1) / GRAM_ROWS;
  __syncthreads();
  for (long long tile = blockIdx.x; tile < ntile; tile += nchunk) {
    const long long r0 = tile * GRAM_ROWS;
    for (int e = threadIdx.x; e < n * GRAM_ROWS; e += GRAM_NT) {
      const int l = e / GRAM_ROWS, r = e % GRAM_ROWS;
      const long long row = r0 + r;
      const size_t off = (size_t)phys[l] * n2 + row;
      const bool ok = row < n2;
      Zs[l * GRAM_ROWS + r] = ok ? Y[off] : mk<C>(0, 0);
      AZs[l * GRAM_ROWS + r] = ok ? AY[off] : mk<C>(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < QMAX; ++i) {
      const int q = threadIdx.x + i * GRAM_NT;
      if (q < nq) {
        const int which = q / (n * n), ab = q % (n * n), a = ab / n, b = ab % n;
        const C* za = Zs + a * GRAM_ROWS;
        const C* zb = (which ? AZs : Zs) + b * GRAM_ROWS;
        double sr = 0, si = 0;
#pragma unroll 8
        for (int r = 0; r < GRAM_ROWS; ++r) {
          const C x = za[r], y = zb[r];
          // conj(x)·y
          sr += (double)x.x * y.x + (double)x.y * y.y;
          si += (double)x.x * y.y - (double)x.y * y.x;
        }
        acc[i].x += sr;
        acc[i].y += si;
      }
    }
    __syncthreads();
  }
  double2* out = d.gram_part + (size_t)blockIdx.x * (2 * NMAX * NMAX);
#pragma unroll
  for (int i = 0; i < QMAX; ++i) {
    const int q = threadIdx.x + i * GRAM_NT;
    if (q < nq) {
      const int which = q / (n * n), ab = q % (n * n), a = ab / n, b = ab % n;
      out[which * NMAX * NMAX + a * NMAX + b] = acc[i];
    }
  }
}

// ---------------------------------------------------------------------------------
// Rayleigh–Ritz: one CTA per track.
__global__ void __launch_bounds__(RR_NT) k_rr(TrackState* const* __restrict__ states,
                                               double2* const* __restrict__ gram_parts,
                                               double2* const* __restrict__ coefs, int ntracks,
                                               IterParams prm);

// ---------------------------------------------------------------------------------
// Update: X ← ZC, AX ← AZC, P ← ZCP, AP ← AZCP into the other parity, then
// R = AX − XΛ, W = P̂_diag R (or R when the MPB preconditioner follows), ‖R‖² partials.
template <typename T>
__global__ void __launch_bounds__(UPD_NT) k_update(const TrackDesc<T>* __restrict__ D, int par, int nchunk,
                                                   int prec_diag) {
  using C = cplx<T>;
  const TrackDesc<T>& d = D[blockIdx.y];
  const TrackState& s = *d.st;
  if (s.done) return;
  const int M = d.M;
  const int n = M + s.nWa + s.nP;
  const int nPn = s.nP_next;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Zs = reinterpret_cast<C*>(smem_raw);          // [l][r]
  C* AZs = Zs + (size_t)n * UPD_ROWS;
  C* Cs = AZs + (size_t)n * UPD_ROWS;               // [l][m], m < M
  C* CPs = Cs + (size_t)n * MMAX;                   // [l][m], m < nPn
  __shared__ int phys[NMAX];
  __shared__ T lam[MMAX];
  __shared__ double rsum[UPD_NT / 32][MMAX];
  for (int l = threadIdx.x; l < n; l += UPD_NT) phys[l] = z_phys(s, M, l);
  for (int e = threadIdx.x; e < n * M; e += UPD_NT) {
    const int l = e / M, m = e % M;
    const double2 c = d.coef[l * MMAX + m];
    Cs[l * MMAX + m] = mk<C>((T)c.x, (T)c.y);
  }
  for (int e = threadIdx.x; e < n * nPn; e += UPD_NT) {
    const int l = e / nPn, m = e % nPn;
    const double2 c = d.coef[NMAX * MMAX + l * MMAX + m];
    CPs[l * MMAX + m] = mk<C>((T)c.x, (T)c.y);
  }
  for (int m = threadIdx.x; m < M; m += UPD_NT) lam[m] = (T)s.lam[m];
  if (blockIdx.x == 0 && threadIdx.x == 0) d.st->cur_par = par ^ 1;
  const long long n2 = d.n2;
  const C* Y = d.Y[par];
  const C* AY = d.AY[par];
  C* Yo = d.Y[par ^ 1];
  C* AYo = d.AY[par ^ 1];
  const T k = (T)s.k;
  // each thread owns fixed (row-in-tile, column) slots: e = tid + j·NT → r = e % ROWS
  constexpr int SLOTS = (MMAX * UPD_ROWS + UPD_NT - 1) / UPD_NT;
  double racc[SLOTS];
#pragma unroll
  for (int i = 0; i < SLOTS; ++i) racc[i] = 0;
  const long long ntile = (n2 + UPD_ROWS - 1) / UPD_ROWS;
  __syncthreads();
  for (long long tile = blockIdx.x; tile < ntile; tile += nchunk) {
    const long long r0 = tile * UPD_ROWS;
    for (int e = threadIdx.x; e < n * UPD_ROWS; e += UPD_NT) {
      const int l = e / UPD_ROWS, r = e % UPD_ROWS;
      const long long row = r0 + r;
      const size_t off = (size_t)phys[l] * n2 + row;
      const bool ok = row < n2;
      Zs[l * UPD_ROWS + r] = ok ? Y[off] : mk<C>(0, 0);
      AZs[l * UPD_ROWS + r] = ok ? AY[off] : mk<C>(0, 0);
    }
    __syncthreads();
    // X, AX, W and ‖R‖²
#pragma unroll
    for (int i = 0; i < SLOTS; ++i) {
      const int e = threadIdx.x + i * UPD_NT;
      if (e < M * UPD_ROWS) {
        const int r = e % UPD_ROWS, m = e / UPD_ROWS;
        const long long row = r0 + r;
        if (row < n2) {
          C x = mk<C>(0, 0), ax = mk<C>(0, 0);
          for (int l = 0; l < n; ++l) {
            const C c = Cs[l * MMAX + m];
            x = x + cmul(Zs[l * UPD_ROWS + r], c);
            ax = ax + cmul(AZs[l * UPD_ROWS + r], c);
          }
          const C res = ax - x * lam[m];
          racc[i] += (double)res.x * res.x + (double)res.y * res.y;
          C w = res;
          if (prec_diag) {
            const long long p = row >> 1;
            const int ix = (int)(p % d.Nx), iy = (int)(p / d.Nx);
            const T gx = T(freq_index(ix, d.Nx)) * (T)d.inv_dx, gy = T(freq_index(iy, d.Ny)) * (T)d.inv_dy;
            w = res * (T(d.eps_mean) / (gx * gx + gy * gy + k * k));
          }
          Yo[(size_t)m * n2 + row] = x;
          AYo[(size_t)m * n2 + row] = ax;
          Yo[(size_t)(M + m) * n2 + row] = w;
        }
      }
    }
    // P, AP
    for (int e = threadIdx.x; e < nPn * UPD_ROWS; e += UPD_NT) {
      const int r = e % UPD_ROWS, m = e / UPD_ROWS;
      const long long row = r0 + r;
      if (row < n2) {
        C p = mk<C>(0, 0), ap = mk<C>(0, 0);
        for (int l = 0; l < n; ++l) {
          const C c = CPs[l * MMAX + m];
          p = p + cmul(Zs[l * UPD_ROWS + r], c);
          ap = ap + cmul(AZs[l * UPD_ROWS + r], c);
        }
        Yo[(size_t)(2 * M + m) * n2 + row] = p;
        AYo[(size_t)(2 * M + m) * n2 + row] = ap;
      }
    }
    __syncthreads();
  }
  // reduce ‖R‖² per column: slots of a thread share m = (tid + i·NT)/ROWS
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int m = 0; m < M; ++m) {
    double v = 0;
#pragma unroll
    for (int i = 0; i < SLOTS; ++i) {
      const int e = threadIdx.x + i * UPD_NT;
      if (e < M * UPD_ROWS && e / UPD_ROWS == m) v += racc[i];
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (l == 0) rsum[w][m] = v;
  }
  __syncthreads();
  if (threadIdx.x < M) {
    double v = 0;
    for (int i = 0; i < UPD_NT / 32; ++i) v += rsum[i][threadIdx.x];
    d.res_part[(size_t)blockIdx.x * MMAX + threadIdx.x] = v;
  }
}

// ---------------------------------------------------------------------------------
// Control (after the update) and Newton (after the HMkH pass): one thread per track.
__global__ void k_control(TrackState* const* __restrict__ states, double* const* __restrict__ res_parts,
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
