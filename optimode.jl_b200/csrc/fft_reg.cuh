// Register-resident DFTs and the two-level line transform plan (sm_100a).
//
// A line of length L = A·B is transformed with one shared-memory transpose (the
// "four-step" factorisation of Bailey, "FFTs in external or hierarchical memory",
// J. Supercomputing 4, 1990):
//
//   X[k1 + A·k2] = Σ_{n2<B} W_B^{n2·k2} · W_L^{n2·k1} · Σ_{n1<A} x[B·n1 + n2] · W_A^{n1·k1}
//
// step 1: a thread per n2 holds the A inputs x[B·n1 + n2] in registers, does the A-point
//         DFT, multiplies by W_L^{n2·k1} and writes row k1, column n2 of a padded
//         A×(B+1) block in shared memory;
// step 2: a thread per k1 reads row k1 (B values), does the B-point DFT and holds the
//         outputs X[k1 + A·k2], k2 < B.
// The reverse order (natural-order output from the k1-strided layout) uses
//   y[m2 + B·m1] = Σ_{k1<A} W_A^{m1·k1} · W_L^{m2·k1} · Σ_{k2<B} V[k1 + A·k2] · W_B^{m2·k2}.
// Rows of the block are B+1 elements apart, so the column writes of step 1 and the row
// reads of step 2 are both free of bank conflicts.
//
// The A- and B-point DFTs run entirely in registers: radix 2, 3, 4, 5, 8 butterflies
// (fft_smem.cuh) and composites R = R1·R2 of them (the same factorisation with
// compile-time indices and twiddle constants).  Twiddle constants are evaluated at
// compile time from a Taylor series after reduction of the angle to [0, π/4].
#pragma once

#include <type_traits>
#include <utility>

#include "fft_smem.cuh"

namespace omb {

// ---- compile-time cos/sin of 2π·m/R --------------------------------------------------
constexpr double kPi = 3.141592653589793238462643383279502884;

__host__ __device__ constexpr double taylor_sin(double x) {
  double t = x, s = x;
  for (int i = 1; i < 14; ++i) { t *= -x * x / ((2.0 * i) * (2.0 * i + 1.0)); s += t; }
  return s;
}
__host__ __device__ constexpr double taylor_cos(double x) {
  double t = 1.0, s = 1.0;
  for (int i = 1; i < 14; ++i) { t *= -x * x / ((2.0 * i - 1.0) * (2.0 * i)); s += t; }
  return s;
}
// cos and sin of π·num/den for 0 ≤ num/den ≤ 2, by exact rational reduction.
__host__ __device__ constexpr double trig_pi(long num, long den, bool want_sin) {
  double sgn = 1.0;
  if (num > den) {  // θ ∈ (π, 2π]: θ → 2π − θ, sin flips
    num = 2 * den - num;
    if (want_sin) sgn = -sgn;
  }
  if (2 * num > den) {  // θ ∈ (π/2, π]: θ → π − θ, cos flips
    num = den - num;
    if (!want_sin) sgn = -sgn;
  }
  if (4 * num > den) {  // θ ∈ (π/4, π/2]: θ → π/2 − θ, cos ↔ sin
    num = den - 2 * num;
    den = 2 * den;
    want_sin = !want_sin;
  }
  const double x = kPi * (double)num / (double)den;
  return sgn * (want_sin ? taylor_sin(x) : taylor_cos(x));
}
__host__ __device__ constexpr double tw_cos(int m, int R) { return trig_pi(2L * (((m % R) + R) % R), R, false); }
__host__ __device__ constexpr double tw_sin(int m, int R) { return trig_pi(2L * (((m % R) + R) % R), R, true); }

// Compile-time loop: f(std::integral_constant<int, I>) for I in [I0, N).
template <int I, int N> struct Unroll {
  template <typename F> __device__ __forceinline__ static void run(F&& f) {
    if constexpr (I < N) {
      f(std::integral_constant<int, I>{});
      Unroll<I + 1, N>::run(f);
    }
  }
};

// a · W_R^{E}, W_R = exp(∓2πi/R) (− forward, + inverse), E a compile-time exponent.
template <int R, int E, bool INV, typename C> __device__ __forceinline__ C twc(C a) {
  using T = decltype(C::x);
  constexpr int e = ((E % R) + R) % R;
  if constexpr (e == 0) {
    return a;
  } else if constexpr (2 * e == R) {
    return mk<C>(-a.x, -a.y);
  } else if constexpr (4 * e == R) {
    return mul_mi<INV>(a);
  } else if constexpr (4 * e == 3 * R) {
    return mul_mi<!INV>(a);
  } else {
    constexpr double c = tw_cos(e, R), s = tw_sin(e, R);
    const T wc = (T)c, ws = INV ? (T)s : (T)(-s);  // W = c ∓ i s
    return mk<C>(a.x * wc - a.y * ws, a.x * ws + a.y * wc);
  }
}

__host__ __device__ constexpr bool reg_dft_base(int R) { return R == 2 || R == 3 || R == 4 || R == 5 || R == 8; }
__host__ __device__ constexpr bool reg_dft_ok(int R) {
  return R == 1 || reg_dft_base(R) || R == 6 || R == 10 || R == 12 || R == 16;
}
// first factor of a composite register DFT
__host__ __device__ constexpr int reg_split(int R) { return R == 16 ? 4 : R == 12 ? 4 : R == 10 ? 5 : 3; }

// In-place DFT of R values held in registers, natural order in and out.
template <int R, bool INV, typename C> __device__ __forceinline__ void dft_reg(C* v) {
  if constexpr (R == 1) {
  } else if constexpr (reg_dft_base(R)) {
    dftR<R, INV>(v);
  } else {
    constexpr int R1 = reg_split(R), R2 = R / R1;
    C y[R1][R2];
    Unroll<0, R2>::run([&](auto n2c) {
      constexpr int N2 = decltype(n2c)::value;
      C u[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) u[n1] = v[R2 * n1 + N2];
      dft_reg<R1, INV>(u);
      Unroll<0, R1>::run([&](auto k1c) {
        constexpr int K1 = decltype(k1c)::value;
        y[K1][N2] = twc<R, N2 * K1, INV>(u[K1]);
      });
    });
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      C w[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) w[n2] = y[k1][n2];
      dft_reg<R2, INV>(w);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = w[k2];
    }
  }
}

// ---- two-level plan ---------------------------------------------------------------------
// A (first factor) for a line of length L, or 0 when L has no split into two register
// DFT lengths ≤ 16.  Among valid splits the one with the smallest max(A, B) wins (fewest
// idle threads), ties going to the larger A.
__host__ __device__ constexpr int plan2_a(int L) {
  int best = 0, bestmax = 1 << 30;
  for (int a = 16; a >= 2; --a) {
    if (L % a != 0) continue;
    const int b = L / a;
    if (!reg_dft_ok(a) || !reg_dft_ok(b) || b < 2) continue;
    const int mx = a > b ? a : b;
    if (mx < bestmax) { bestmax = mx; best = a; }
  }
  return best;
}
__host__ __device__ constexpr int plan2_b(int L) { return plan2_a(L) ? L / plan2_a(L) : 0; }
__host__ __device__ constexpr int plan2_max(int L) {
  return plan2_a(L) > plan2_b(L) ? plan2_a(L) : plan2_b(L);
}

// Step 1 (natural-order input): v[n1] = x[B·n1 + n2] → line[k1·(B+1) + n2] = (DFT_A v)[k1]·W_L^{n2·k1}.
// tw1[k1·B + n2] = W_L^{n2·k1} (forward sign; conjugated for the inverse).
template <int L, bool INV, typename C>
__device__ __forceinline__ void l2_first(C* v, int n2, C* line, const C* __restrict__ tw1) {
  constexpr int A = plan2_a(L), B = L / A;
  dft_reg<A, INV>(v);
  line[n2] = v[0];
#pragma unroll
  for (int k1 = 1; k1 < A; ++k1) {
    const C w = __ldg(tw1 + k1 * B + n2);
    line[k1 * (B + 1) + n2] = INV ? cmulc(v[k1], w) : cmul(v[k1], w);
  }
}
// Step 2: w[k2] ← X[k1 + A·k2] from row k1 of the block.
template <int L, bool INV, typename C>
__device__ __forceinline__ void l2_second(const C* line, int k1, C* w) {
  constexpr int A = plan2_a(L), B = L / A;
#pragma unroll
  for (int n2 = 0; n2 < B; ++n2) w[n2] = line[k1 * (B + 1) + n2];
  dft_reg<B, INV>(w);
}
// Reverse step 1 (k1-strided input): w[k2] = V[k1 + A·k2] → line[k1·(B+1) + m2] =
// (DFT_B w)[m2]·W_L^{m2·k1}.  tw3[m2·A + k1] = W_L^{m2·k1}.
template <int L, bool INV, typename C>
__device__ __forceinline__ void l2_rfirst(C* w, int k1, C* line, const C* __restrict__ tw3) {
  constexpr int A = plan2_a(L), B = L / A;
  dft_reg<B, INV>(w);
  line[k1 * (B + 1)] = w[0];
#pragma unroll
  for (int m2 = 1; m2 < B; ++m2) {
    const C t = __ldg(tw3 + m2 * A + k1);
    line[k1 * (B + 1) + m2] = INV ? cmulc(w[m2], t) : cmul(w[m2], t);
  }
}
// Reverse step 2: v[m1] ← y[m2 + B·m1] from column m2 of the block.
template <int L, bool INV, typename C>
__device__ __forceinline__ void l2_rsecond(const C* line, int m2, C* v) {
  constexpr int A = plan2_a(L), B = L / A;
#pragma unroll
  for (int k1 = 0; k1 < A; ++k1) v[k1] = line[k1 * (B + 1) + m2];
  dft_reg<A, INV>(v);
}

}  // namespace omb
