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
// Gram: partial G = ZᴴZ and S = ZᴴAZ, upper triangles only, per CTA row slice.
// The n columns (padded to even) are cut into 2×2 output blocks; each warp owns
// gram_ipw blocks and its lanes stride the rows of a staged tile, so shared-memory reads
// are consecutive (conflict-free) and every lane keeps 4 complex accumulators per block.
// Tiles are staged with double-buffered cp.async copies (the next tile's loads are in
// flight while the current one is reduced).  Lane partials are reduced in FP64 at the end.
// Grid: (row chunks, tracks, block chunks).
template <typename T> __host__ __device__ constexpr int gram_ipw() { return sizeof(T) == 4 ? 6 : 4; }
template <typename T> __host__ __device__ constexpr int gram_ipc() { return (GRAM_NT / 32) * gram_ipw<T>(); }
template <typename T> __host__ __device__ constexpr int gram_rows() { return sizeof(T) == 4 ? 128 : 64; }
template <typename T> __host__ __device__ constexpr size_t gram_smem(int nbmax) {
  return 2 /*buffers*/ * 2 /*Z, AZ*/ * (size_t)(2 * nbmax) * gram_rows<T>() * sizeof(cplx<T>);
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::); }

template <typename T>
__global__ void __launch_bounds__(GRAM_NT) k_gram(const TrackDesc<T>* __restrict__ D, int par, int nchunk) {
  using C = cplx<T>;
  constexpr int IPW = gram_ipw<T>();
  constexpr int ROWS = gram_rows<T>();
  const TrackDesc<T>& d = D[blockIdx.y];
  const TrackState& s = *d.st;
  if (s.done) return;
  const int M = d.M;
  const int n = M + s.nWa + s.nP;
  const int nb = (n + 1) / 2;
  const int nblk = nb * (nb + 1) / 2;
  const int item0 = blockIdx.z * gram_ipc<T>();
  if (item0 >= 2 * nblk) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);  // [2 buffers][Z, AZ][2nb columns][ROWS]
  const int tsz = 2 * nb * ROWS;            // one matrix of one buffer
  __shared__ int phys[NMAX + 1];
  __shared__ unsigned char bi_of[NMAX * NMAX / 4 + NMAX], bj_of[NMAX * NMAX / 4 + NMAX];
  for (int l = threadIdx.x; l < 2 * nb; l += GRAM_NT) phys[l] = l < n ? z_phys(s, M, l) : -1;
  if (threadIdx.x == 0) {
    int q = 0;
    for (int i = 0; i < nb; ++i)
      for (int j = i; j < nb; ++j) { bi_of[q] = (unsigned char)i; bj_of[q] = (unsigned char)j; ++q; }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C acc[IPW][4];
#pragma unroll
  for (int i = 0; i < IPW; ++i)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[i][e] = mk<C>(0, 0);
  const long long n2 = d.n2;
  const C* __restrict__ Y = d.Y[par];
  const C* __restrict__ AY = d.AY[par];
  const long long ntile = (n2 + ROWS - 1) / ROWS;
  __syncthreads();
  auto stage = [&](long long tile, int b) {
    C* Zs = buf + (size_t)b * 2 * tsz;
    C* AZs = Zs + tsz;
    const long long r0 = tile * ROWS;
    for (int e = threadIdx.x; e < tsz; e += GRAM_NT) {
      const int l = e / ROWS, r = e % ROWS;
      const long long row = r0 + r;
      if (row < n2 && phys[l] >= 0) {
        const size_t off = (size_t)phys[l] * n2 + row;
        if constexpr (sizeof(C) == 16) { cp_async16(Zs + e, Y + off); cp_async16(AZs + e, AY + off); }
        else { cp_async8(Zs + e, Y + off); cp_async8(AZs + e, AY + off); }
      } else {
        Zs[e] = mk<C>(0, 0);
        AZs[e] = mk<C>(0, 0);
      }
    }
    cp_async_commit();
  };
  int it = 0;
  if (blockIdx.x < ntile) stage(blockIdx.x, 0);
  for (long long tile = blockIdx.x; tile < ntile; tile += nchunk, ++it) {
    if (tile + nchunk < ntile) stage(tile + nchunk, (it + 1) & 1);
    else cp_async_commit();  // empty group keeps the wait count uniform
    cp_async_wait_prev();
    __syncthreads();
    const C* Zs = buf + (size_t)(it & 1) * 2 * tsz;
    const C* AZs = Zs + tsz;
#pragma unroll
    for (int i = 0; i < IPW; ++i) {
      const int itm = item0 + warp * IPW + i;
      if (itm < 2 * nblk) {
        const int which = itm / nblk, q = itm % nblk;
        const C* za = Zs + 2 * bi_of[q] * ROWS;
        const C* zb = (which ? AZs : Zs) + 2 * bj_of[q] * ROWS;
#pragma unroll
        for (int k = 0; k < ROWS / 32; ++k) {
          const int r = lane + 32 * k;
          const C a0 = za[r], a1 = za[ROWS + r], b0 = zb[r], b1 = zb[ROWS + r];
          // conj(a)·b
          acc[i][0] = acc[i][0] + cmul(cconj(a0), b0);
          acc[i][1] = acc[i][1] + cmul(cconj(a0), b1);
          acc[i][2] = acc[i][2] + cmul(cconj(a1), b0);
          acc[i][3] = acc[i][3] + cmul(cconj(a1), b1);
        }
      }
    }
    __syncthreads();
  }
  double2* out = d.gram_part + (size_t)blockIdx.x * (2 * NMAX * NMAX);
#pragma unroll
  for (int i = 0; i < IPW; ++i) {
    const int itm = item0 + warp * IPW + i;
    if (itm >= 2 * nblk) continue;  // warp-uniform
    const int which = itm / nblk, q = itm % nblk;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      double re = (double)acc[i][e].x, im = (double)acc[i][e].y;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
      }
      const int a = 2 * bi_of[q] + (e >> 1), bcol = 2 * bj_of[q] + (e & 1);
      if (lane == 0 && a < n && bcol < n) out[which * NMAX * NMAX + a * NMAX + bcol] = make_double2(re, im);
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
// One thread per vector row (coalesced column reads straight from global memory), the
// coefficients broadcast from shared memory, MB ≥ M register accumulators per output.
template <typename T, int MB>
__global__ void __launch_bounds__(UPD_NT) k_update(const TrackDesc<T>* __restrict__ D, int par, int nchunk,
                                                   int prec_diag) {
  using C = cplx<T>;
  const TrackDesc<T>& d = D[blockIdx.y];
  const TrackState& s = *d.st;
  if (s.done) return;
  const int M = d.M;
  const int n = M + s.nWa + s.nP;
  const int nPn = s.nP_next;
  __shared__ C Cs[NMAX][MB];
  __shared__ C CPs[NMAX][MB];
  __shared__ int phys[NMAX];
  __shared__ T lam[MB];
  __shared__ double rsum[UPD_NT / 32][MB];
  for (int l = threadIdx.x; l < n; l += UPD_NT) phys[l] = z_phys(s, M, l);
  for (int e = threadIdx.x; e < n * MB; e += UPD_NT) {
    const int l = e / MB, m = e % MB;
    const double2 c = m < M ? d.coef[l * MMAX + m] : make_double2(0, 0);
    const double2 cp = m < nPn ? d.coef[NMAX * MMAX + l * MMAX + m] : make_double2(0, 0);
    Cs[l][m] = mk<C>((T)c.x, (T)c.y);
    CPs[l][m] = mk<C>((T)cp.x, (T)cp.y);
  }
  for (int m = threadIdx.x; m < MB; m += UPD_NT) lam[m] = m < M ? (T)s.lam[m] : T(0);
  if (blockIdx.x == 0 && threadIdx.x == 0) d.st->cur_par = par ^ 1;
  __syncthreads();
  const long long n2 = d.n2;
  const C* __restrict__ Y = d.Y[par];
  const C* __restrict__ AY = d.AY[par];
  C* __restrict__ Yo = d.Y[par ^ 1];
  C* __restrict__ AYo = d.AY[par ^ 1];
  const T k = (T)s.k;
  double racc[MB];
#pragma unroll
  for (int m = 0; m < MB; ++m) racc[m] = 0;
  for (long long row = (long long)blockIdx.x * UPD_NT + threadIdx.x; row < n2; row += (long long)nchunk * UPD_NT) {
    C x[MB], ax[MB];
#pragma unroll
    for (int m = 0; m < MB; ++m) { x[m] = mk<C>(0, 0); ax[m] = mk<C>(0, 0); }
#pragma unroll 4
    for (int l = 0; l < n; ++l) {
      const size_t off = (size_t)phys[l] * n2 + row;
      const C z = Y[off], az = AY[off];
#pragma unroll
      for (int m = 0; m < MB; ++m) {
        if (m < M) {
          const C c = Cs[l][m];
          x[m] = x[m] + cmul(z, c);
          ax[m] = ax[m] + cmul(az, c);
        }
      }
    }
    T pscale = T(1);
    if (prec_diag) {
      const long long p = row >> 1;
      const int ix = (int)(p % d.Nx), iy = (int)(p / d.Nx);
      const T gx = T(freq_index(ix, d.Nx)) * (T)d.inv_dx, gy = T(freq_index(iy, d.Ny)) * (T)d.inv_dy;
      pscale = T(d.eps_mean) / (gx * gx + gy * gy + k * k);
    }
#pragma unroll
    for (int m = 0; m < MB; ++m) {
      if (m < M) {
        const C res = ax[m] - x[m] * lam[m];
        racc[m] += (double)res.x * res.x + (double)res.y * res.y;
        Yo[(size_t)m * n2 + row] = x[m];
        AYo[(size_t)m * n2 + row] = ax[m];
        Yo[(size_t)(M + m) * n2 + row] = res * pscale;
      }
    }
    if (nPn > 0) {
#pragma unroll
      for (int m = 0; m < MB; ++m) { x[m] = mk<C>(0, 0); ax[m] = mk<C>(0, 0); }
#pragma unroll 4
      for (int l = M; l < n; ++l) {  // the X rows of CP are zero
        const size_t off = (size_t)phys[l] * n2 + row;
        const C z = Y[off], az = AY[off];
#pragma unroll
        for (int m = 0; m < MB; ++m) {
          if (m < nPn) {
            const C c = CPs[l][m];
            x[m] = x[m] + cmul(z, c);
            ax[m] = ax[m] + cmul(az, c);
          }
        }
      }
#pragma unroll
      for (int m = 0; m < MB; ++m) {
        if (m < nPn) {
          Yo[(size_t)(2 * M + m) * n2 + row] = x[m];
          AYo[(size_t)(2 * M + m) * n2 + row] = ax[m];
        }
      }
    }
  }
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
#pragma unroll
  for (int m = 0; m < MB; ++m) {
    double v = racc[m];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (ln == 0) rsum[w][m] = v;
  }
  __syncthreads();
  if (threadIdx.x < M) {
    double v = 0;
    for (int i = 0; i < UPD_NT / 32; ++i) v += rsum[i][threadIdx.x];
    d.res_part[(size_t)blockIdx.x * MMAX + threadIdx.x] = v;
  }
}

// ---------------------------------------------------------------------------------
// Control (after the update; one warp per track) and Newton (after the HMkH pass; one
// thread per track).
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
