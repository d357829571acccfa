// Small dense Hermitian algebra for the Rayleigh–Ritz step, one CTA per problem (FP64).
//
// Matrices live in shared memory, row-major with leading dimension `ld`, complex double.
// The eigensolver is the cyclic Jacobi method for complex Hermitian matrices with the
// round-robin (tournament) ordering of Brent & Luk, so the n/2 rotations of a round act on
// disjoint index pairs and are applied together: all row rotations (A ← JᴴA), then all
// column rotations (A ← AJ, V ← VJ).  Each 2×2 rotation first removes the phase of A_pq
// (D = diag(1, e^{-iφ})) and then applies the real symmetric Jacobi rotation with
// t = sign(ζ)/(|ζ| + √(1+ζ²)), ζ = (A_qq − A_pp)/(2|A_pq|) (Golub & Van Loan, Matrix
// Computations, §8.5).  Sweeps stop when the off-diagonal Frobenius norm falls below
// 1e-13·‖A‖_F (eigenvalue perturbation ≲ 1e-26‖A‖²/gap; rounding keeps the off-diagonal
// near n·1e-16‖A‖, so a tighter test would never pass) or after `max_sweeps`.
#pragma once

#include "omb_common.cuh"

namespace omb {

struct Rot { double c, s, er, ei; int p, q; };

// Round-robin pairing: players 0..ne-1 (ne even); player 0 fixed, the rest rotate.
__device__ __forceinline__ void rr_pair(int round, int i, int ne, int& p, int& q) {
  auto pos = [&](int k) { return k == 0 ? 0 : 1 + ((k - 1 + round) % (ne - 1)); };
  int a = pos(i), b = pos(ne - 1 - i);
  p = a < b ? a : b;
  q = a < b ? b : a;
}

// Jacobi eigen-decomposition of the n×n Hermitian matrix A (overwritten with its
// eigenvalues on the diagonal); V (n×n) receives the eigenvectors as columns.
// `rot` needs ≥ n/2+1 entries of shared scratch, `red` ≥ 32 doubles.
__device__ inline void jacobi_eigh(double2* A, double2* V, int n, int ld, Rot* rot, double* red,
                                   int max_sweeps = 20) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < n * n; e += nt) {
    const int r = e / n, c = e % n;
    V[r * ld + c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
    if (r == c) A[r * ld + c].y = 0.0;
  }
  __syncthreads();
  if (n <= 1) return;
  const int ne = n + (n & 1);
  const int npair = ne / 2;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    // convergence check: off-diagonal vs total Frobenius norm
    double off = 0, tot = 0;
    for (int e = tid; e < n * n; e += nt) {
      const int r = e / n, c = e % n;
      const double2 v = A[r * ld + c];
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
    if (so <= 1e-26 * st || so == 0.0) break;
    for (int round = 0; round < ne - 1; ++round) {
      for (int i = tid; i < npair; i += nt) {
        int p, q;
        rr_pair(round, i, ne, p, q);
        Rot R{1.0, 0.0, 1.0, 0.0, p, q};
        if (q < n) {
          const double2 apq = A[p * ld + q];
          const double g = sqrt(apq.x * apq.x + apq.y * apq.y);
          const double app = A[p * ld + p].x, aqq = A[q * ld + q].x;
          if (g > 1e-300 && g > 1e-18 * sqrt(fabs(app * aqq))) {
            const double zeta = (aqq - app) / (2.0 * g);
            const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            R.c = 1.0 / sqrt(1.0 + t * t);
            R.s = t * R.c;
            R.er = apq.x / g;  // e^{iφ}
            R.ei = apq.y / g;
          } else {
            R.q = n;  // no-op
          }
        }
        rot[i] = R;
      }
      __syncthreads();
      // rows: A_p· ← c A_p· − s e^{iφ} A_q· ;  A_q· ← s A_p· + c e^{iφ} A_q·
      for (int e = tid; e < npair * n; e += nt) {
        const Rot R = rot[e / n];
        if (R.q >= n) continue;
        const int col = e % n;
        const double2 ap = A[R.p * ld + col], aq = A[R.q * ld + col];
        const double2 eaq = make_double2(R.er * aq.x - R.ei * aq.y, R.er * aq.y + R.ei * aq.x);
        A[R.p * ld + col] = make_double2(R.c * ap.x - R.s * eaq.x, R.c * ap.y - R.s * eaq.y);
        A[R.q * ld + col] = make_double2(R.s * ap.x + R.c * eaq.x, R.s * ap.y + R.c * eaq.y);
      }
      __syncthreads();
      // columns: A_·p ← c A_·p − s e^{-iφ} A_·q ;  A_·q ← s A_·p + c e^{-iφ} A_·q   (and V)
      for (int e = tid; e < 2 * npair * n; e += nt) {
        const int which = e / (npair * n);
        const int ee = e % (npair * n);
        const Rot R = rot[ee / n];
        if (R.q >= n) continue;
        const int row = ee % n;
        double2* M = which ? V : A;
        const double2 ap = M[row * ld + R.p], aq = M[row * ld + R.q];
        const double2 eaq = make_double2(R.er * aq.x + R.ei * aq.y, R.er * aq.y - R.ei * aq.x);
        M[row * ld + R.p] = make_double2(R.c * ap.x - R.s * eaq.x, R.c * ap.y - R.s * eaq.y);
        M[row * ld + R.q] = make_double2(R.s * ap.x + R.c * eaq.x, R.s * ap.y + R.c * eaq.y);
      }
      __syncthreads();
    }
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
