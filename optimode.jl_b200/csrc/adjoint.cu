// Adjoint pull-back of solve_k on the device (omb_pullback).
//
// Per band b with mode (k_b, h_b) and cotangents (k̄_b, ē_b) (reference:
// rrule(solve_k), lib/MaxwellEigenmodes/src/solve.jl:213-289; GPU variant
// src/solvers/gpu.jl:292-365):
//   ∂ω²/∂k = 2⟨h|∂M̂/∂k|h⟩                                   (HMₖH pass)
//   (M̂ − ω²) λ = ē − h⟨h,ē⟩,  λ ⟂ h                         (deflated, preconditioned MINRES)
//   D0 = fft(kx_tc h),  Λd = fft(kx_tc λ)                   (H2D passes)
//   ẽ = bfft(ε⁻¹ D0)/N,  λ̃e = bfft(ε⁻¹ Λd)/N                (D2E passes)
//   k̄ₕ = −∇ₖ(mag, m̂, n̂) · (m̄, n̄, māg) from ẽ, λ̃e, h, λ     (one reduction kernel)
//   s = (k̄ + k̄ₕ)/(∂ω²/∂k),  ω̄ += 2ωs
//   ε̄⁻¹ += ε⁻¹_bar(D0/N, Λd + s·D0)                          (one pointwise kernel: the
//          eigenvalue-path term ε⁻¹_bar(d, fft(kx_tc(s h))) is bilinear in D0, so it folds
//          into the same pass)
//
// MINRES (C. C. Paige & M. A. Saunders, SIAM J. Numer. Anal. 12 (1975)) with a symmetric
// positive-definite preconditioner: for a Hermitian operator the Lanczos coefficients and
// Givens rotations are real, only the vectors are complex.  Every vector stays orthogonal to
// h (the right-hand side is, and the preconditioned vector is projected), which deflates the
// eigenvalue ω² of the operator.  All recurrence scalars live in device memory; one
// iteration is a fixed launch sequence replayed from a CUDA graph.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "context.h"
#include "vec.cuh"

namespace omb {

constexpr int ADJ_NT = 256;
constexpr int ADJ_BLOCKS = 296;  // 2 × 148 SMs for the streaming vector kernels

struct MinresState {
  double shift;          // ω²
  double beta1, beta, oldb, alfa, dbar, epsln, oldeps, phibar, cs, sn, gamma, delta, phi;
  double dot_ey_r, dot_ey_i, dot_ez_r, dot_ez_i;
  double rtol;
  double phibar_mark;  // phibar at itn_mark (stagnation test)
  int itn, maxit, done, status;  // status: 0 running, 1 converged, 2 maxiter, 3 breakdown,
                                 // 4 maxiter with the residual below LOOSE_TOL
  int itn_mark;
  int flat_windows;  // consecutive windows in which phibar did not halve
};

// Below rtol the recurrence residual phibar can flatten at the rounding floor of the FP64
// operator (≈1e-12 of β₁ for right-hand sides dominated by modes near the deflated
// eigenvalue), while the iterate has long converged.  The solve also ends, converged, when
// phibar ≤ STALL_TOL·β₁ and did not halve over the last STALL_WINDOW iterations.
constexpr double STALL_TOL = 1e-10;
constexpr int STALL_WINDOW = 50;
// A solve that reaches its iteration cap is still accepted when its relative residual is
// below √ε₆₄ ≈ 1.5e-8, the default relative tolerance of the reference's GMRES
// (IterativeSolvers `gmres`, lib/MaxwellEigenmodes/src/grads/solve.jl:56-66, which returns
// whatever it reached after maxiter = 1000).
constexpr double LOOSE_TOL = 1.4901161193847656e-08;
// Near-degenerate bands make (M̂ − ω²) ill-conditioned on the complement of the deflated
// eigenvector, and the FP64 recurrence then flattens at ≈ε₆₄·cond above LOOSE_TOL.  A solve
// whose phibar has not halved over FLAT_WINDOWS consecutive windows while below FLAT_TOL·β₁
// ends there, accepted (status 4): more iterations would not lower it.
constexpr double FLAT_TOL = 1e-6;
constexpr int FLAT_WINDOWS = 4;

// block-reduce two complex partial sums (4 doubles) into part[blockIdx.x*4 + 0..3]
__device__ __forceinline__ void block_reduce4(double a, double b, double c, double d, double* part) {
  __shared__ double sm[4][ADJ_NT / 32];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
    d += __shfl_xor_sync(0xffffffffu, d, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { sm[0][w] = a; sm[1][w] = b; sm[2][w] = c; sm[3][w] = d; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int i = 0; i < ADJ_NT / 32; ++i) { s0 += sm[0][i]; s1 += sm[1][i]; s2 += sm[2][i]; s3 += sm[3][i]; }
    part[4 * blockIdx.x + 0] = s0;
    part[4 * blockIdx.x + 1] = s1;
    part[4 * blockIdx.x + 2] = s2;
    part[4 * blockIdx.x + 3] = s3;
  }
}

struct AdjVecs {
  double2 *x, *v, *w, *w2, *r1, *r2, *y, *Av;
  const double2* e;  // unit eigenvector (deflation direction)
  long long n2;
  int Nx, Ny;
  double inv_dx, inv_dy, k, eps_mean;
  int Nz;            // z-periodic cells (1 for a 2D cell)
  double inv_dz;
};

// Diagonal preconditioner ⟨ε⟩/|w|² at row `row` (w = k ẑ − G; g_z of the row's slab)
__device__ __forceinline__ double prec_scale(long long row, const AdjVecs& V) {
  const long long p = row >> 1;
  const int ix = (int)(p % V.Nx);
  const long long rest = p / V.Nx;
  const int iy = (int)(rest % V.Ny), iz = (int)(rest / V.Ny);
  const double gx = freq_index(ix, V.Nx) * V.inv_dx, gy = freq_index(iy, V.Ny) * V.inv_dy;
  const double wz = V.k - freq_index(iz, V.Nz) * V.inv_dz;
  return V.eps_mean / (gx * gx + gy * gy + wz * wz);
}

// init: r1 = r2 = b, z = P b, partials ⟨e,z⟩, ⟨b,z⟩ (y holds z)
__global__ void __launch_bounds__(ADJ_NT) k_minres_init(AdjVecs V, const double2* __restrict__ b, double* part) {
  double er = 0, ei = 0, br = 0, bi = 0;
  for (long long i = blockIdx.x * (long long)ADJ_NT + threadIdx.x; i < V.n2; i += (long long)gridDim.x * ADJ_NT) {
    const double2 bb = b[i];
    const double s = prec_scale(i, V);
    const double2 z = make_double2(bb.x * s, bb.y * s);
    V.r1[i] = bb; V.r2[i] = bb; V.y[i] = z;
    V.x[i] = make_double2(0, 0); V.w[i] = make_double2(0, 0); V.w2[i] = make_double2(0, 0);
    const double2 e = V.e[i];
    er += e.x * z.x + e.y * z.y; ei += e.x * z.y - e.y * z.x;   // conj(e)·z
    br += bb.x * z.x + bb.y * z.y; bi += bb.x * z.y - bb.y * z.x;
  }
  block_reduce4(er, ei, br, bi, part);
}

__global__ void k_minres_init_scalar(MinresState* S, const double* part, int nb) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double er = 0, ei = 0, br = 0;
  for (int i = 0; i < nb; ++i) { er += part[4 * i]; ei += part[4 * i + 1]; br += part[4 * i + 2]; }
  S->dot_ez_r = er; S->dot_ez_i = ei;
  const double b2 = br;
  S->itn = 0; S->done = 0; S->status = 0;
  S->oldb = 0; S->dbar = 0; S->epsln = 0; S->oldeps = 0; S->cs = -1; S->sn = 0;
  if (!(b2 > 0) || !isfinite(b2)) {  // zero right-hand side: λ = 0
    S->beta1 = S->beta = 0; S->phibar = 0; S->done = 1; S->status = 1;
    return;
  }
  S->beta1 = S->beta = sqrt(b2);
  S->phibar = S->beta1;
  S->phibar_mark = S->beta1;
  S->itn_mark = 0;
  S->flat_windows = 0;
}

// v = (z − ⟨e,z⟩e)/beta  (start of the first iteration)
__global__ void __launch_bounds__(ADJ_NT) k_minres_first_v(AdjVecs V, const MinresState* S) {
  if (S->done) return;
  const double inv = 1.0 / S->beta, er = S->dot_ez_r, ei = S->dot_ez_i;
  for (long long i = blockIdx.x * (long long)ADJ_NT + threadIdx.x; i < V.n2; i += (long long)gridDim.x * ADJ_NT) {
    const double2 z = V.y[i], e = V.e[i];
    V.v[i] = make_double2((z.x - (er * e.x - ei * e.y)) * inv, (z.y - (er * e.y + ei * e.x)) * inv);
  }
}

// y = Av − shift·v − (beta/oldb)·r1 ; partials ⟨e,y⟩, ⟨v,y⟩
__global__ void __launch_bounds__(ADJ_NT) k_minres_a(AdjVecs V, const MinresState* S, double* part) {
  if (S->done) return;
  const double sh = S->shift;
  const double c1 = S->itn >= 1 ? S->beta / S->oldb : 0.0;
  double er = 0, ei = 0, vr = 0, vi = 0;
  for (long long i = blockIdx.x * (long long)ADJ_NT + threadIdx.x; i < V.n2; i += (long long)gridDim.x * ADJ_NT) {
    const double2 av = V.Av[i], v = V.v[i], r1 = V.r1[i], e = V.e[i];
    const double2 y = make_double2(av.x - sh * v.x - c1 * r1.x, av.y - sh * v.y - c1 * r1.y);
    V.y[i] = y;
    er += e.x * y.x + e.y * y.y; ei += e.x * y.y - e.y * y.x;
    vr += v.x * y.x + v.y * y.y; vi += v.x * y.y - v.y * y.x;
  }
  block_reduce4(er, ei, vr, vi, part);
}

__global__ void k_minres_a_scalar(MinresState* S, const double* part, int nb) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || S->done) return;
  double er = 0, ei = 0, vr = 0;
  for (int i = 0; i < nb; ++i) { er += part[4 * i]; ei += part[4 * i + 1]; vr += part[4 * i + 2]; }
  S->dot_ey_r = er; S->dot_ey_i = ei;
  S->alfa = vr;  // ⟨v, y⟩ is real for a Hermitian operator (v ⟂ e)
}

// y ← y − ⟨e,y⟩e − (alfa/beta) r2 ; r1 ← r2 ; r2 ← y ; z = P r2 (into y) ; partials ⟨e,z⟩, ⟨r2,z⟩
__global__ void __launch_bounds__(ADJ_NT) k_minres_b(AdjVecs V, const MinresState* S, double* part) {
  if (S->done) return;
  const double c2 = S->alfa / S->beta, er0 = S->dot_ey_r, ei0 = S->dot_ey_i;
  double er = 0, ei = 0, rr = 0, ri = 0;
  for (long long i = blockIdx.x * (long long)ADJ_NT + threadIdx.x; i < V.n2; i += (long long)gridDim.x * ADJ_NT) {
    const double2 y = V.y[i], e = V.e[i], r2 = V.r2[i];
    const double2 yn = make_double2(y.x - (er0 * e.x - ei0 * e.y) - c2 * r2.x, y.y - (er0 * e.y + ei0 * e.x) - c2 * r2.y);
    V.r1[i] = r2;
    V.r2[i] = yn;
    const double s = prec_scale(i, V);
    const double2 z = make_double2(yn.x * s, yn.y * s);
    V.y[i] = z;
    er += e.x * z.x + e.y * z.y; ei += e.x * z.y - e.y * z.x;
    rr += yn.x * z.x + yn.y * z.y; ri += yn.x * z.y - yn.y * z.x;
  }
  block_reduce4(er, ei, rr, ri, part);
}

// Lanczos coefficient β_{k+1} and the Givens rotation of MINRES (all real)
__global__ void k_minres_b_scalar(MinresState* S, const double* part, int nb) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || S->done) return;
  double er = 0, ei = 0, rr = 0;
  for (int i = 0; i < nb; ++i) { er += part[4 * i]; ei += part[4 * i + 1]; rr += part[4 * i + 2]; }
  S->dot_ez_r = er; S->dot_ez_i = ei;
  const double b2 = rr;  // ⟨r2, z − e⟨e,z⟩⟩ = ⟨r2, z⟩ since r2 ⟂ e
  S->oldb = S->beta;
  S->beta = b2 > 0 ? sqrt(b2) : 0.0;
  S->oldeps = S->epsln;
  const double alfa = S->alfa;
  S->delta = S->cs * S->dbar + S->sn * alfa;
  const double gbar = S->sn * S->dbar - S->cs * alfa;
  S->epsln = S->sn * S->beta;
  S->dbar = -S->cs * S->beta;
  double gamma = sqrt(gbar * gbar + S->beta * S->beta);
  if (gamma < 1e-300) gamma = 1e-300;
  S->gamma = gamma;
  S->cs = gbar / gamma;
  S->sn = S->beta / gamma;
  S->phi = S->cs * S->phibar;
  S->phibar = S->sn * S->phibar;
  S->itn++;
  if (!isfinite(S->phibar) || !isfinite(S->phi)) { S->done = 1; S->status = 3; return; }
  if (S->phibar <= S->rtol * S->beta1) { S->done = 2; S->status = 1; return; }  // finish this update
  if (S->itn - S->itn_mark >= STALL_WINDOW) {
    const bool flat = S->phibar > 0.5 * S->phibar_mark;
    if (S->phibar <= STALL_TOL * S->beta1 && flat) {
      S->done = 2; S->status = 1; return;
    }
    S->flat_windows = flat ? S->flat_windows + 1 : 0;
    if (S->flat_windows >= FLAT_WINDOWS && S->phibar <= FLAT_TOL * S->beta1) {
      S->done = 2; S->status = 4; return;
    }
    S->phibar_mark = S->phibar;
    S->itn_mark = S->itn;
  }
  if (S->beta == 0.0) { S->done = 2; S->status = 1; return; }                   // invariant subspace
  if (S->itn >= S->maxit) { S->done = 2; S->status = S->phibar <= LOOSE_TOL * S->beta1 ? 4 : 2; }
}

// w_k = (v − oldeps·w_{k−2} − delta·w_{k−1})/gamma ; x += phi·w_k ; v ← (z − ⟨e,z⟩e)/β_{k+1}
__global__ void __launch_bounds__(ADJ_NT) k_minres_c(AdjVecs V, MinresState* S) {
  if (S->done == 1) return;
  const double ig = 1.0 / S->gamma, oe = S->oldeps, de = S->delta, ph = S->phi;
  const bool next = S->done == 0 && S->beta > 0;
  const double ib = next ? 1.0 / S->beta : 0.0, er = S->dot_ez_r, ei = S->dot_ez_i;
  for (long long i = blockIdx.x * (long long)ADJ_NT + threadIdx.x; i < V.n2; i += (long long)gridDim.x * ADJ_NT) {
    const double2 v = V.v[i], wa = V.w2[i], wb = V.w[i];
    const double2 wn = make_double2((v.x - oe * wa.x - de * wb.x) * ig, (v.y - oe * wa.y - de * wb.y) * ig);
    V.w2[i] = wb;
    V.w[i] = wn;
    double2 x = V.x[i];
    x.x += ph * wn.x; x.y += ph * wn.y;
    V.x[i] = x;
    if (next) {
      const double2 z = V.y[i], e = V.e[i];
      V.v[i] = make_double2((z.x - (er * e.x - ei * e.y)) * ib, (z.y - (er * e.y + ei * e.x)) * ib);
    }
  }
}
__global__ void k_minres_finish(MinresState* S) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && S->done == 2) S->done = 1;
}

// λ ← λ − ⟨e,λ⟩e (two passes: partial dot, then update with the reduced value)
__global__ void __launch_bounds__(ADJ_NT) k_dot_e(const double2* __restrict__ e, const double2* __restrict__ x,
                                                  long long n, double* part) {
  double r = 0, im = 0;
  for (long long i = blockIdx.x * (long long)ADJ_NT + threadIdx.x; i < n; i += (long long)gridDim.x * ADJ_NT) {
    const double2 a = e[i], b = x[i];
    r += a.x * b.x + a.y * b.y; im += a.x * b.y - a.y * b.x;
  }
  block_reduce4(r, im, 0, 0, part);
}
__global__ void __launch_bounds__(ADJ_NT) k_sub_proj(const double2* __restrict__ e, double2* __restrict__ x, long long n,
                                                     const double* part, int nb) {
  __shared__ double cr, ci;
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int i = 0; i < nb; ++i) { a += part[4 * i]; b += part[4 * i + 1]; }
    cr = a; ci = b;
  }
  __syncthreads();
  for (long long i = blockIdx.x * (long long)ADJ_NT + threadIdx.x; i < n; i += (long long)gridDim.x * ADJ_NT) {
    const double2 a = e[i];
    double2 b = x[i];
    b.x -= cr * a.x - ci * a.y;
    b.y -= cr * a.y + ci * a.x;
    x[i] = b;
  }
}

// k̄ₕ partials from ẽ = EC/N, λ̃e = ED/N (planar), h and λ (interleaved), basis at k
// (z-periodic cells: the basis at k − g_z, and beside k̄ₕ's sum the same per-plane-wave terms
// weighted by g_z/Λ, whose negative is the eigenvector channel's period cotangent Λ̄_H,
// lib/MaxwellEigenmodes/src/grads/period.jl:113-117, 171-175)
__global__ void __launch_bounds__(ADJ_NT) k_adj_kbar(const double2* __restrict__ EC, const double2* __restrict__ ED,
                                                     const double2* __restrict__ h, const double2* __restrict__ lam,
                                                     int Nx, int Ny, int Nz, double inv_dx, double inv_dy,
                                                     double inv_dz, double k, double* part) {
  const long long N = (long long)Nx * Ny * Nz;
  const double sN = 1.0 / (double)N;
  double acc = 0, accL = 0;
  for (long long p = blockIdx.x * (long long)ADJ_NT + threadIdx.x; p < N; p += (long long)gridDim.x * ADJ_NT) {
    const int ix = (int)(p % Nx);
    const long long rest = p / Nx;
    const int iy = (int)(rest % Ny), iz = (int)(rest / Ny);
    const double gz = freq_index(iz, Nz) * inv_dz;
    const Basis<double> B = basis_at<double>(k - gz, freq_index(ix, Nx) * inv_dx, freq_index(iy, Ny) * inv_dy);
    const double m[3] = {B.mx, B.my, B.mz}, n[3] = {B.nx, B.ny, 0.0};
    const double2 h1 = h[2 * p], h2 = h[2 * p + 1], l1 = lam[2 * p], l2 = lam[2 * p + 1];
    double km[3], kn[3];
    for (int c = 0; c < 3; ++c) {
      const double2 le = ED[c * N + p], ee = EC[c * N + p];
      // Re(λ̃e·conj(h₂) + ẽ·conj(λ₂)) and −Re(λ̃e·conj(h₁) + ẽ·conj(λ₁)), with the 1/N scale
      km[c] = (le.x * h2.x + le.y * h2.y + ee.x * l2.x + ee.y * l2.y) * sN;
      kn[c] = -(le.x * h1.x + le.y * h1.y + ee.x * l1.x + ee.y * l1.y) * sN;
    }
    const double magbar = n[0] * kn[0] + n[1] * kn[1] + n[2] * kn[2] + m[0] * km[0] + m[1] * km[1] + m[2] * km[2];
    // ∇ₖmag_m_n (ME/src/maxwell.jl:560-566) with dk̂ = ẑ: u = (m × n)/mag, q = u × ẑ
    const double u[3] = {(m[1] * n[2] - m[2] * n[1]) / B.mag, (m[2] * n[0] - m[0] * n[2]) / B.mag,
                         (m[0] * n[1] - m[1] * n[0]) / B.mag};
    const double q[3] = {u[1], -u[0], 0.0};
    const double mq[3] = {m[1] * q[2] - m[2] * q[1], m[2] * q[0] - m[0] * q[2], m[0] * q[1] - m[1] * q[0]};
    const double nq[3] = {n[1] * q[2] - n[2] * q[1], n[2] * q[0] - n[0] * q[2], n[0] * q[1] - n[1] * q[0]};
    const double kmag = magbar * u[2] * B.mag;
    const double kmm = -(km[0] * mq[0] + km[1] * mq[1] + km[2] * mq[2]) * B.mag;  // m̄ = kx̄_m·mag
    const double knn = -(kn[0] * nq[0] + kn[1] * nq[1] + kn[2] * nq[2]) * B.mag;
    acc += kmag + kmm + knn;
    accL += (kmag + kmm + knn) * gz * inv_dz;
  }
  block_reduce4(acc, accL, 0, 0, part);
}

// ε̄⁻¹ (6 unique entries) += ε⁻¹_bar(d, lt), d = D0/N, lt = Λd + s·D0
__global__ void __launch_bounds__(ADJ_NT) k_adj_eibar(const double2* __restrict__ D0, const double2* __restrict__ LD,
                                                      long long N, double s, double* __restrict__ eib) {
  const double sN = 1.0 / (double)N;
  for (long long p = blockIdx.x * (long long)ADJ_NT + threadIdx.x; p < N; p += (long long)gridDim.x * ADJ_NT) {
    double2 d[3], l[3];
    for (int c = 0; c < 3; ++c) {
      const double2 a = D0[c * N + p], b = LD[c * N + p];
      d[c] = make_double2(a.x * sN, a.y * sN);
      l[c] = make_double2(b.x + s * a.x, b.y + s * a.y);
    }
    auto re = [](double2 a, double2 b) { return a.x * b.x + a.y * b.y; };  // Re(a·conj(b))
    double* o = eib + 6 * p;
    o[0] -= re(l[0], d[0]);                 // xx
    o[1] -= re(l[1], d[1]);                 // yy
    o[2] -= re(l[2], d[2]);                 // zz
    o[3] -= re(l[1], d[0]) + re(l[0], d[1]);  // xy (summed (x,y)+(y,x), mirrored)
    o[4] -= re(l[2], d[0]) + re(l[0], d[2]);  // xz
    o[5] -= re(l[2], d[1]) + re(l[1], d[2]);  // yz
  }
}

// expand to (3,3,Nx,Ny) and, if requested, ε̄ = −Y ε̄⁻¹ Y with Y = ε⁻¹ (sliceinv_3x3 pull-back,
// ME/src/grads/linalg.jl:40-47; Y is symmetric so Yᵀ = Y)
__global__ void __launch_bounds__(ADJ_NT) k_adj_expand(const double* __restrict__ eib, const double2* __restrict__ e64,
                                                       long long N, double* __restrict__ out_ei, double* __restrict__ out_e) {
  for (long long p = blockIdx.x * (long long)ADJ_NT + threadIdx.x; p < N; p += (long long)gridDim.x * ADJ_NT) {
    const double* o = eib + 6 * p;
    const double Gb[3][3] = {{o[0], o[3], o[4]}, {o[3], o[1], o[5]}, {o[4], o[5], o[2]}};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) out_ei[9 * p + a + 3 * b] = Gb[a][b];
    if (out_e) {
      const double2 y0 = e64[3 * p], y1 = e64[3 * p + 1], y2 = e64[3 * p + 2];
      const double Y[3][3] = {{y0.x, y1.y, y2.x}, {y1.y, y0.y, y2.y}, {y2.x, y2.y, y1.x}};
      double T[3][3];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) T[a][b] = Y[a][0] * Gb[0][b] + Y[a][1] * Gb[1][b] + Y[a][2] * Gb[2][b];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          out_e[9 * p + a + 3 * b] = -(T[a][0] * Y[0][b] + T[a][1] * Y[1][b] + T[a][2] * Y[2][b]);
    }
  }
}

}  // namespace omb

using namespace omb;

// The pull-back on an uploaded problem; Nz > 1 is a z-periodic cell, for which L_bar (when
// non-NULL) receives the period cotangent Λ̄ (lib/MaxwellEigenmodes/src/grads/period.jl:136-200).
static int pullback_impl(omb_ctx* ctx, Problem& P, double omega, int nev, const double* kmags, const double* evecs,
                         const double* kbar, const double* evbar, const omb_options& O, double* omega_bar,
                         double* epsinv_bar, double* eps_bar, double* L_bar, int32_t* iterations) {
  cudaStream_t st = ctx->stream;
  const long long N = (long long)P.N(), n2 = 2 * N;
  const bool periodic = P.Nz > 1;
  const double inv_dz = periodic ? 1.0 / P.Dz : 0.0;  // (a 2D cell has Dz = 0)
  // device buffers
  DevBuf<double2> vecs, scr, ev, eb, lamv;
  OMB_CU(vecs.alloc(8 * n2, st));   // x v w w2 r1 r2 y Av
  OMB_CU(scr.alloc(6 * 3 * N, st)); // operator scratch ×2, copies ×2, E fields ×2
  OMB_CU(ev.alloc(n2, st));
  OMB_CU(eb.alloc(n2, st));
  DevBuf<double> part, eib, kd, hpart, hred;
  const int nb = ADJ_BLOCKS;
  OMB_CU(part.alloc(4 * nb, st));
  OMB_CU(eib.alloc(6 * N, st));
  OMB_CU(eib.zero());
  OMB_CU(kd.alloc(1, st));
  const int rb = row_blocks(P.Nx, P.Ny) * P.Nz;  // HMₖH partials: row blocks of every slab
  OMB_CU(hpart.alloc(2 * rb, st));
  OMB_CU(hred.alloc(2, st));
  DevBuf<MinresState> S;
  OMB_CU(S.alloc(1, st));
  double2* vb = vecs.p;
  AdjVecs V{vb, vb + n2, vb + 2 * n2, vb + 3 * n2, vb + 4 * n2, vb + 5 * n2, vb + 6 * n2, vb + 7 * n2, ev.p,
            n2, P.Nx, P.Ny, 1.0 / P.Dx, 1.0 / P.Dy, 0.0, P.eps_mean, P.Nz, inv_dz};
  double2* SA = scr.p;              // D0 = fft(kx_tc h)
  double2* SB = SA + 3 * N;         // Λd = fft(kx_tc λ)
  double2* SC = SB + 3 * N;         // copies consumed by the D2E passes
  double2* SD = SC + 3 * N;
  double2* EC = SD + 3 * N;         // N·ẽ
  double2* ED = EC + 3 * N;         // N·λ̃e
  // operator units (FP64): M on v → Av; HMkH on h; H2D on h and λ; D2E on the copies
  auto unit = [&](const double2* in, double2* out, double2* s) {
    OpUnit<double> u = make_unit<double>(P);
    u.in = in; u.out = out; u.scr = s; u.k_dev = kd.p; u.partial = hpart.p;
    u.in_cs = n2; u.out_cs = n2; u.scr_cs = 3 * N; u.ncol = 1;
    return u;
  };
  // (unit 6: HMₖH with the ẑ× action weighted by g_z/Λ, for ∂ω²/∂Λ)
  OpUnit<double> hu[7] = {unit(V.v, V.Av, SC),   unit(ev.p, nullptr, SC), unit(ev.p, nullptr, SA),
                          unit(V.x, nullptr, SB), unit(nullptr, EC, SC),   unit(nullptr, ED, SD),
                          unit(ev.p, nullptr, SC)};
  hu[4].out_cs = 3 * N;
  hu[5].out_cs = 3 * N;
  hu[6].zx_weight_gz = 1;
  DevBuf<OpUnit<double>> du, dexp;
  OMB_CU(du.alloc(7, st));
  OMB_CU(cudaMemcpyAsync(du.p, hu, 7 * sizeof(OpUnit<double>), cudaMemcpyHostToDevice, st));
  if (periodic) OMB_CU(dexp.alloc(P.Nz + 1, st));
  const TwTables& tw = ctx->tw;
  auto run = [&](OpKind kind, int u) -> cudaError_t {
    return periodic ? launch_op3d<double>(kind, du.p + u, 1, P.Nx, P.Ny, P.Nz, 1, tw, dexp.p, st)
                    : launch_op<double>(kind, du.p + u, 1, P.Nx, P.Ny, 1, tw, st);
  };
  // ⟨h|∂M̂|h⟩ with unit u (the device partials hold Re⟨h|kx_ct(…)⟩ = −HMₖH)
  auto hmkh = [&](int u, double& out) -> cudaError_t {
    cudaError_t e = run(OP_HMKH, u);
    if (e != cudaSuccess) return e;
    k_reduce_partials<<<1, 256, 0, st>>>(hpart.p, rb, 1, hred.p);
    e = cudaGetLastError();
    double hh[2];
    if (e == cudaSuccess) e = cudaMemcpyAsync(hh, hred.p, sizeof(hh), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    out = -hh[0];
    return e;
  };
  double wbar = 0.0, Lbar = 0.0;
  for (int b = 0; b < nev; ++b) {
    const double kb = kmags[b];
    if (!(kb > 0) || !std::isfinite(kb)) return fail(OMB_ERR_INVALID_ARG, "kmags must be finite and positive");
    V.k = kb;
    OMB_CU(cudaMemcpyAsync(kd.p, &kb, sizeof(double), cudaMemcpyHostToDevice, st));
    OMB_CU(cudaMemcpyAsync(ev.p, evecs + 4 * N * (size_t)b, n2 * sizeof(double2), cudaMemcpyHostToDevice, st));
    // ∂ω²/∂k = 2⟨h|∂M̂/∂k|h⟩ and, on a periodic cell, ∂ω²/∂Λ = 2⟨h|∂M̂/∂Λ|h⟩ (period.jl:150-151)
    double hk = 0, hL = 0;
    OMB_CU(hmkh(1, hk));
    const double dw2dk = 2.0 * hk;
    if (!(dw2dk > 0) || !std::isfinite(dw2dk)) return fail(OMB_ERR_NAN, "non-positive ∂ω²/∂k in the pull-back");
    if (periodic && L_bar) OMB_CU(hmkh(6, hL));
    const double dw2dL = 2.0 * hL;
    double Lbar_h = 0.0;
    const double kb_bar = kbar ? kbar[b] : 0.0;
    double kbar_h = 0.0;
    const double* eb_host = evbar ? evbar + 4 * N * (size_t)b : nullptr;
    bool have_eb = false;
    if (eb_host)
      for (long long i = 0; i < 2 * n2 && !have_eb; ++i) have_eb = eb_host[i] != 0.0;
    // D0 = fft(kx_tc h) into SA
    OMB_CU(run(OP_H2D, 2));
    if (have_eb) {
      // b = ē − h⟨h,ē⟩
      OMB_CU(cudaMemcpyAsync(eb.p, eb_host, n2 * sizeof(double2), cudaMemcpyHostToDevice, st));
      k_dot_e<<<nb, ADJ_NT, 0, st>>>(ev.p, eb.p, n2, part.p);
      k_sub_proj<<<nb, ADJ_NT, 0, st>>>(ev.p, eb.p, n2, part.p, nb);
      OMB_CU(cudaGetLastError());
      MinresState s0{};
      s0.shift = omega * omega;
      s0.rtol = 1e-12;
      s0.maxit = std::max(4 * O.maxiter, 3000);
      OMB_CU(cudaMemcpyAsync(S.p, &s0, sizeof(s0), cudaMemcpyHostToDevice, st));
      k_minres_init<<<nb, ADJ_NT, 0, st>>>(V, eb.p, part.p);
      k_minres_init_scalar<<<1, 32, 0, st>>>(S.p, part.p, nb);
      k_minres_first_v<<<nb, ADJ_NT, 0, st>>>(V, S.p);
      OMB_CU(cudaGetLastError());
      // one MINRES iteration; 8 per graph replay, host checks the flag between replays
      auto iter = [&]() -> cudaError_t {
        cudaError_t e = run(OP_M, 0);
        if (e != cudaSuccess) return e;
        k_minres_a<<<nb, ADJ_NT, 0, st>>>(V, S.p, part.p);
        k_minres_a_scalar<<<1, 32, 0, st>>>(S.p, part.p, nb);
        k_minres_b<<<nb, ADJ_NT, 0, st>>>(V, S.p, part.p);
        k_minres_b_scalar<<<1, 32, 0, st>>>(S.p, part.p, nb);
        k_minres_c<<<nb, ADJ_NT, 0, st>>>(V, S.p);
        k_minres_finish<<<1, 32, 0, st>>>(S.p);
        return cudaGetLastError();
      };
      OMB_CU(iter());  // eager once (sets kernel attributes outside the capture)
      cudaGraph_t graph = nullptr;
      cudaGraphExec_t exec = nullptr;
      OMB_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      cudaError_t ce = cudaSuccess;
      for (int i = 0; i < 8 && ce == cudaSuccess; ++i) ce = iter();
      cudaError_t ee = cudaStreamEndCapture(st, &graph);
      if (ce != cudaSuccess) { if (graph) cudaGraphDestroy(graph); return cuda_fail(ce, "MINRES capture"); }
      OMB_CU(ee);
      OMB_CU(cudaGraphInstantiate(&exec, graph, 0));
      MinresState sh{};
      const int cap = s0.maxit / 8 + 2;
      for (int it = 0; it < cap; ++it) {
        cudaError_t e = cudaGraphLaunch(exec, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&sh, S.p, sizeof(sh), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { cudaGraphExecDestroy(exec); cudaGraphDestroy(graph); return cuda_fail(e, "MINRES"); }
        if (sh.done) break;
      }
      cudaGraphExecDestroy(exec);
      cudaGraphDestroy(graph);
      if (iterations) iterations[b] = sh.itn;
      if (sh.status == 3) return fail(OMB_ERR_NAN, "MINRES breakdown in the adjoint solve");
      if (sh.status != 1 && sh.status != 4) {
        char msg[160];
        snprintf(msg, sizeof msg, "adjoint MINRES did not converge (band %d: relative residual %.3g after %d iterations)",
                 b, sh.beta1 > 0 ? sh.phibar / sh.beta1 : 0.0, sh.itn);
        return fail(OMB_ERR_NOT_CONVERGED, msg);
      }
      // λ ⟂ h (re-projection against round-off), then Λd = fft(kx_tc λ) into SB
      k_dot_e<<<nb, ADJ_NT, 0, st>>>(ev.p, V.x, n2, part.p);
      k_sub_proj<<<nb, ADJ_NT, 0, st>>>(ev.p, V.x, n2, part.p, nb);
      OMB_CU(cudaGetLastError());
      OMB_CU(run(OP_H2D, 3));
      // ẽ·N and λ̃e·N through the D2E passes on copies (the passes work in place)
      OMB_CU(cudaMemcpyAsync(SC, SA, 3 * N * sizeof(double2), cudaMemcpyDeviceToDevice, st));
      OMB_CU(cudaMemcpyAsync(SD, SB, 3 * N * sizeof(double2), cudaMemcpyDeviceToDevice, st));
      OMB_CU(run(OP_D2E, 4));
      OMB_CU(run(OP_D2E, 5));
      k_adj_kbar<<<nb, ADJ_NT, 0, st>>>(EC, ED, ev.p, V.x, P.Nx, P.Ny, P.Nz, 1.0 / P.Dx, 1.0 / P.Dy, inv_dz, kb,
                                        part.p);
      OMB_CU(cudaGetLastError());
      std::vector<double> hp(4 * nb);
      OMB_CU(cudaMemcpyAsync(hp.data(), part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
      OMB_CU(cudaStreamSynchronize(st));
      double acc = 0, accL = 0;
      for (int i = 0; i < nb; ++i) {
        acc += hp[4 * i];
        accL += hp[4 * i + 1];
      }
      kbar_h = -acc;
      Lbar_h = -accL;
    } else {
      if (iterations) iterations[b] = 0;
      OMB_CU(cudaMemsetAsync(SB, 0, 3 * N * sizeof(double2), st));
    }
    const double s = (kb_bar + kbar_h) / dw2dk;
    k_adj_eibar<<<nb, ADJ_NT, 0, st>>>(SA, SB, N, s, eib.p);
    OMB_CU(cudaGetLastError());
    wbar += 2.0 * omega * s;
    Lbar += Lbar_h + (kb_bar + kbar_h) * (-dw2dL / dw2dk);
  }
  DevBuf<double> oei, oe;
  OMB_CU(oei.alloc(9 * N, st));
  if (eps_bar) OMB_CU(oe.alloc(9 * N, st));
  k_adj_expand<<<nb, ADJ_NT, 0, st>>>(eib.p, P.e64.p, N, oei.p, eps_bar ? oe.p : nullptr);
  OMB_CU(cudaGetLastError());
  OMB_CU(cudaMemcpyAsync(epsinv_bar, oei.p, 9 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (eps_bar) OMB_CU(cudaMemcpyAsync(eps_bar, oe.p, 9 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaStreamSynchronize(st));
  *omega_bar = wbar;
  if (L_bar) *L_bar = Lbar;
  return OMB_OK;
}

static int pullback_args(omb_ctx* ctx, double omega, int nev, const double* kmags, const double* evecs,
                         double* omega_bar, double* epsinv_bar) {
  if (!ctx) return fail(OMB_ERR_INVALID_ARG, "ctx is NULL");
  if (nev <= 0 || !kmags || !evecs || !omega_bar || !epsinv_bar)
    return fail(OMB_ERR_INVALID_ARG, "need nev > 0 and non-NULL kmags, evecs, omega_bar, epsinv_bar");
  if (!(omega > 0) || !std::isfinite(omega)) return fail(OMB_ERR_INVALID_ARG, "omega must be finite and positive");
  return OMB_OK;
}

extern "C" int omb_pullback(omb_ctx* ctx, const omb_grid* grid, double omega, const double* epsinv, int nev,
                            const double* kmags, const double* evecs, const double* kbar, const double* evbar,
                            const omb_options* opt, double* omega_bar, double* epsinv_bar, double* eps_bar,
                            int32_t* iterations) {
  int rc = pullback_args(ctx, omega, nev, kmags, evecs, omega_bar, epsinv_bar);
  if (rc) return rc;
  omb_options dflt;
  omb_options_default(&dflt);
  OMB_CU(cudaSetDevice(ctx->device));
  Problem P;
  rc = upload_problem(ctx, grid, epsinv, P);
  if (rc) return rc;
  return pullback_impl(ctx, P, omega, nev, kmags, evecs, kbar, evbar, opt ? *opt : dflt, omega_bar, epsinv_bar,
                       eps_bar, nullptr, iterations);
}

extern "C" int omb_pullback_periodic(omb_ctx* ctx, const omb_grid3* grid, double omega, const double* epsinv,
                                     int nev, const double* kmags, const double* evecs, const double* kbar,
                                     const double* evbar, const omb_options* opt, double* omega_bar,
                                     double* epsinv_bar, double* L_bar, int32_t* iterations) {
  int rc = pullback_args(ctx, omega, nev, kmags, evecs, omega_bar, epsinv_bar);
  if (rc) return rc;
  if (!grid) return fail(OMB_ERR_INVALID_ARG, "grid is NULL");
  if (grid->Nz < 8) return fail(OMB_ERR_UNSUPPORTED, "a z-periodic cell needs Nz >= 8 slabs (a supported length)");
  omb_options dflt;
  omb_options_default(&dflt);
  OMB_CU(cudaSetDevice(ctx->device));
  Problem P;
  const omb_grid g2{grid->Nx, grid->Ny, grid->Dx, grid->Dy};
  rc = upload_problem(ctx, &g2, epsinv, P, grid->Nz, grid->Dz);
  if (rc) return rc;
  return pullback_impl(ctx, P, omega, nev, kmags, evecs, kbar, evbar, opt ? *opt : dflt, omega_bar, epsinv_bar,
                       nullptr, L_bar, iterations);
}
