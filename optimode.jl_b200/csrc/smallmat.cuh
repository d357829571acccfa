// Small dense Hermitian algebra for the Rayleigh–Ritz step, one CTA per problem (FP64).
//
// Matrices live in shared memory, row-major with leading dimension `ld`, complex double.
// The eigensolver is the cyclic Jacobi method for complex Hermitian matrices with the
// round-robin (tournament) ordering of Brent & Luk, so the n/2 rotations of a round act on
// disjoint index pairs.  Each 2×2 rotation first removes the phase of A_pq
// (D = diag(1, e^{-iφ})) and then applies the real symmetric Jacobi rotation with
// t = sign(ζ)/(|ζ| + √(1+ζ²)), ζ = (A_qq − A_pp)/(2|A_pq|) (Golub & Van Loan, Matrix
// Computations, §8.5).  A round is two barriers: one thread per pair computes its rotation
// (reciprocal square roots only, no divisions by |A_pq|), then every element of the new
// matrix is formed from the four old elements it depends on, A' = JᴴAJ, into a second
// buffer, while V ← VJ is updated in place by column pairs.  Sweeps stop when the
// off-diagonal Frobenius norm falls below 1e-13·‖A‖_F (eigenvalue perturbation
// ≲ 1e-26‖A‖²/gap; rounding keeps the off-diagonal near n·1e-16‖A‖, so a tighter test
// would never pass) or after `max_sweeps`.
#pragma once

#include "omb_common.cuh"

namespace omb {

// Per index a of a round: partner pa and the coefficients of the two-sided update,
// (JᴴA)_a· = α_a A_a· + β_a A_pa·  and  (AJ)_·a = γ_a A_·a + δ_a A_·pa.
struct RotIdx { double2 al, be, ga, de; int pa; };

// Round-robin pairing: players 0..ne-1 (ne even); player 0 fixed, the rest rotate.
__device__ __forceinline__ void rr_pair(int round, int i, int ne, int& p, int& q) {
  auto pos = [&](int k) { return k == 0 ? 0 : 1 + ((k - 1 + round) % (ne - 1)); };
  int a = pos(i), b = pos(ne - 1 - i);
  p = a < b ? a : b;
  q = a < b ? b : a;
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Jacobi eigen-decomposition of the n×n Hermitian matrix A (overwritten with its
// eigenvalues on the diagonal); V (n×n) receives the eigenvectors as columns.
// `A2` is n×n scratch (leading dimension ld), `ri` ≥ n entries, `red` ≥ 2·(warps) doubles.
// Sweeps stop once ‖offdiag‖²_F ≤ tol2·‖A‖²_F.
__device__ inline void jacobi_eigh(double2* A, double2* V, int n, int ld, double2* A2, RotIdx* ri, double* red,
                                   double tol2 = 1e-26, int max_sweeps = 20) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < n * n; e += nt) {
    const int r = e / n, c = e % n;
    V[r * ld + c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
    if (r == c) A[r * ld + c].y = 0.0;
  }
  __syncthreads();
  if (n <= 1) return;
  double2* cur = A;
  double2* nxt = A2;
  const int ne = n + (n & 1);
  const int npair = ne / 2;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    // convergence check: off-diagonal vs total Frobenius norm
    double off = 0, tot = 0;
    for (int e = tid; e < n * n; e += nt) {
      const int r = e / n, c = e % n;
      const double2 v = cur[r * ld + c];
      const double a2 = v.x * v.x + v.y * v.y;
      tot += a2;
      if (r != c) off += a2;
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      tot += __shfl_xor_sync(0xffffffffu, tot, o);
    }
    if ((tid & 31) == 0) { red[2 * (tid >> 5)] = off; red[2 * (tid >> 5) + 1] = tot; }
    __syncthreads();
    double so = 0, st = 0;
    for (int w = 0; w < (nt + 31) / 32; ++w) { so += red[2 * w]; st += red[2 * w + 1]; }
    __syncthreads();
    if (so <= tol2 * st || so == 0.0) break;
    for (int round = 0; round < ne - 1; ++round) {
      // 1. rotations of this round (identity for the odd player out and settled pairs)
      for (int i = tid; i < npair; i += nt) {
        int p, q;
        rr_pair(round, i, ne, p, q);
        const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
        RotIdx rp{one, zero, one, zero, q}, rq{one, zero, one, zero, p};
        if (q < n) {
          const double2 apq = cur[p * ld + q];
          const double g2 = apq.x * apq.x + apq.y * apq.y;
          const double app = cur[p * ld + p].x, aqq = cur[q * ld + q].x;
          if (g2 > 1e-300 && g2 > 1e-36 * fabs(app * aqq)) {
            const double rg = rsqrt(g2);                    // 1/|A_pq|
            const double er = apq.x * rg, ei = apq.y * rg;  // e^{iφ}
            const double zeta = 0.5 * (aqq - app) * rg;
            const double h = 1.0 + zeta * zeta;
            const double t = (zeta >= 0 ? 1.0 : -1.0) * __drcp_rn(fabs(zeta) + h * rsqrt(h));
            const double c = rsqrt(1.0 + t * t), sn = t * c;
            // rows:    A_p· ← c A_p· − s e A_q·,    A_q· ← s A_p· + c e A_q·
            // columns: A_·p ← c A_·p − s ē A_·q,    A_·q ← s A_·p + c ē A_·q
            rp.al = make_double2(c, 0.0);         rp.be = make_double2(-sn * er, -sn * ei);
            rq.al = make_double2(c * er, c * ei); rq.be = make_double2(sn, 0.0);
            rp.ga = make_double2(c, 0.0);         rp.de = make_double2(-sn * er, sn * ei);
            rq.ga = make_double2(c * er, -c * ei); rq.de = make_double2(sn, 0.0);
          }
          ri[q] = rq;
        }
        ri[p] = rp;
      }
      __syncthreads();
      // 2. A' = JᴴAJ element by element into the other buffer; V ← VJ by column pairs
      for (int e = tid; e < n * n; e += nt) {
        const int i = e / n, j = e % n;
        const RotIdx a = ri[i], b = ri[j];
        double2 v = zmul(zmul(a.al, cur[i * ld + j]), b.ga);
        if (b.pa < n) v = v + zmul(zmul(a.al, cur[i * ld + b.pa]), b.de);
        if (a.pa < n) {
          v = v + zmul(zmul(a.be, cur[a.pa * ld + j]), b.ga);
          if (b.pa < n) v = v + zmul(zmul(a.be, cur[a.pa * ld + b.pa]), b.de);
        }
        nxt[i * ld + j] = v;
      }
      for (int e = tid; e < n * npair; e += nt) {
        const int i = e / npair, k = e % npair;
        int p, q;
        rr_pair(round, k, ne, p, q);
        if (q >= n) continue;
        const RotIdx rp = ri[p], rq = ri[q];
        const double2 vp = V[i * ld + p], vq = V[i * ld + q];
        V[i * ld + p] = zmul(rp.ga, vp) + zmul(rp.de, vq);
        V[i * ld + q] = zmul(rq.ga, vq) + zmul(rq.de, vp);
      }
      __syncthreads();
      double2* tmp = cur; cur = nxt; nxt = tmp;
    }
  }
  if (cur != A) {
    for (int e = tid; e < n * n; e += nt) A[(e / n) * ld + e % n] = cur[(e / n) * ld + e % n];
    __syncthreads();
  }
  for (int e = tid; e < n; e += nt) A[e * ld + e].y = 0.0;
  __syncthreads();
}

// Indices of the eigenvalues (diagonal of A) in ascending order → order[0..n).
__device__ inline void sort_diag(const double2* A, int n, int ld, int* order) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < n; ++i) order[i] = i;
    for (int i = 1; i < n; ++i) {
      int v = order[i], j = i - 1;
      while (j >= 0 && A[order[j] * ld + order[j]].x > A[v * ld + v].x) { order[j + 1] = order[j]; --j; }
      order[j + 1] = v;
    }
  }
  __syncthreads();
}

}  // namespace omb
