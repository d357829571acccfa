// Batched 1D FFTs of many lines held in shared memory (sm_100a).
//
// Mixed-radix (8, 4, 2, 3, 5) Stockham auto-sort formulation (N. K. Govindaraju et al.,
// "High performance discrete Fourier transforms on graphics processors", SC 2008): stage
// s with radix R combines R inputs at stride L/R, multiplies by the twiddles
// W_L^{r·(j mod Ns)·L/(Ns·R)} and writes the R outputs at stride Ns into sorted order, so
// no bit-reversal pass is needed.  The line length L and the number of lines per CTA are
// compile-time constants, so every stage unrolls; each thread keeps its butterflies in
// registers across the one barrier that separates a stage's reads from its writes, which
// makes the transform in place in a single shared buffer.
//
// Twiddles come from a table tw[m] = exp(-2πi m/L), m < L, computed on the host in
// double precision and staged into shared memory; the inverse transform (unnormalised,
// sign +1, FFTW's "bfft") uses their conjugates.
#pragma once

#include "omb_common.cuh"

namespace omb {

__host__ __device__ constexpr int radix_for(int rem) {
  return (rem % 8 == 0) ? 8 : (rem % 4 == 0) ? 4 : (rem % 2 == 0) ? 2 : (rem % 3 == 0) ? 3 : 5;
}
__host__ __device__ constexpr bool fft_len_ok(int L) {
  while (L % 2 == 0) L /= 2;
  while (L % 3 == 0) L /= 3;
  while (L % 5 == 0) L /= 5;
  return L == 1;
}

// ---- small DFTs on register arrays -------------------------------------------------
template <bool INV, typename C> __device__ __forceinline__ void dft2(C& a, C& b) {
  C t = a; a = t + b; b = t - b;
}
template <bool INV, typename C> __device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3) {
  C t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = mul_mi<INV>(a1 - a3);
  a0 = t0 + t2; a2 = t0 - t2; a1 = t1 + t3; a3 = t1 - t3;
}
template <bool INV, typename C> __device__ __forceinline__ void dft8(C* v) {
  using T = decltype(C::x);
  const T h = T(0.70710678118654752440);  // 1/sqrt(2)
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  // o_k *= W8^k (W8 = exp(∓iπ/4))
  C w1 = INV ? mk<C>(h * (o1.x - o1.y), h * (o1.x + o1.y)) : mk<C>(h * (o1.x + o1.y), h * (o1.y - o1.x));
  C w2 = mul_mi<INV>(o2);
  C w3 = INV ? mk<C>(-h * (o3.x + o3.y), h * (o3.x - o3.y)) : mk<C>(h * (o3.y - o3.x), -h * (o3.x + o3.y));
  v[0] = e0 + o0; v[4] = e0 - o0;
  v[1] = e1 + w1; v[5] = e1 - w1;
  v[2] = e2 + w2; v[6] = e2 - w2;
  v[3] = e3 + w3; v[7] = e3 - w3;
}
template <bool INV, typename C> __device__ __forceinline__ void dft3(C* v) {
  using T = decltype(C::x);
  const T s3 = T(0.86602540378443864676);  // sqrt(3)/2
  C s = v[1] + v[2], d = v[1] - v[2];
  C m = v[0] - s * T(0.5);
  v[0] = v[0] + s;
  // (∓i·sqrt(3)/2)·d
  C t = INV ? mk<C>(-s3 * d.y, s3 * d.x) : mk<C>(s3 * d.y, -s3 * d.x);
  v[1] = m + t; v[2] = m - t;
}
template <bool INV, typename C> __device__ __forceinline__ void dft5(C* v) {
  using T = decltype(C::x);
  // cos/sin of 2π/5 and 4π/5
  const T c1 = T(0.30901699437494742410), c2 = T(-0.80901699437494742410);
  const T s1 = T(0.95105651629515357212), s2 = T(0.58778525229247312917);
  const T sg = INV ? T(1) : T(-1);
  C a = v[1] + v[4], b = v[1] - v[4], c = v[2] + v[3], d = v[2] - v[3];
  C x0 = v[0];
  v[0] = x0 + a + c;
  C r1 = x0 + a * c1 + c * c2, r2 = x0 + a * c2 + c * c1;
  // i·sg·(s1 b + s2 d), i·sg·(s2 b − s1 d)
  C u1 = b * s1 + d * s2, u2 = b * s2 - d * s1;
  C i1 = mk<C>(-sg * u1.y, sg * u1.x), i2 = mk<C>(-sg * u2.y, sg * u2.x);
  v[1] = r1 + i1; v[4] = r1 - i1;
  v[2] = r2 + i2; v[3] = r2 - i2;
}
template <int R, bool INV, typename C> __device__ __forceinline__ void dftR(C* v) {
  if constexpr (R == 2) dft2<INV>(v[0], v[1]);
  else if constexpr (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 8) dft8<INV>(v);
  else if constexpr (R == 3) dft3<INV>(v);
  else dft5<INV>(v);
}

// ---- Stockham stages over NL lines of length L (line stride LS) -------------------
// Lines start at s + line*LS.  NT threads cooperate (all of them must call).
template <typename C, int L, int NS, bool INV, int NL, int NT>
__device__ __forceinline__ void stockham_stages(C* __restrict__ s, int LS, const C* __restrict__ tw) {
  if constexpr (NS < L) {
    constexpr int R = radix_for(L / NS);
    constexpr int NB = L / R;
    constexpr int TOT = NB * NL;
    constexpr int PER = (TOT + NT - 1) / NT;
    C v[PER][R];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int q = threadIdx.x + p * NT;
      if ((TOT % NT == 0) || q < TOT) {
        const int line = q / NB, j = q - line * NB;
        const C* b = s + line * LS;
        const int kk = j % NS;
#pragma unroll
        for (int r = 0; r < R; ++r) v[p][r] = b[j + r * NB];
        if constexpr (NS > 1) {
#pragma unroll
          for (int r = 1; r < R; ++r) {
            C w = tw[(r * kk) * (L / (NS * R))];
            if (INV) w.y = -w.y;
            v[p][r] = cmul(v[p][r], w);
          }
        }
        dftR<R, INV>(v[p]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int q = threadIdx.x + p * NT;
      if ((TOT % NT == 0) || q < TOT) {
        const int line = q / NB, j = q - line * NB;
        C* b = s + line * LS;
        const int kk = j % NS;
        const int o = (j - kk) * R + kk;
#pragma unroll
        for (int r = 0; r < R; ++r) b[o + r * NS] = v[p][r];
      }
    }
    __syncthreads();
    stockham_stages<C, L, NS * R, INV, NL, NT>(s, LS, tw);
  }
}

// Transform NL lines in place.  Requires a __syncthreads() between the last write of the
// input and this call (the first stage reads right away).
template <typename C, int L, bool INV, int NL, int NT>
__device__ __forceinline__ void fft_lines(C* s, int LS, const C* tw) {
  static_assert(fft_len_ok(L), "FFT length must factor into 2, 3 and 5");
  stockham_stages<C, L, 1, INV, NL, NT>(s, LS, tw);
}

}  // namespace omb
