// Common device/host helpers for libomb200 (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace omb {

template <typename T> struct cplx_t;
template <> struct cplx_t<float> { using type = float2; };
template <> struct cplx_t<double> { using type = double2; };
template <typename T> using cplx = typename cplx_t<T>::type;

template <typename C> __host__ __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) {
  C r; r.x = a; r.y = b; return r;
}
// FP32 complex arithmetic: on the device the sm_100 packed two-lane instructions (one issue
// slot for both halves, each half rounded like the scalar operation).
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) {
#ifdef __CUDA_ARCH__
  return __fadd2_rn(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) {
#ifdef __CUDA_ARCH__
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
__host__ __device__ __forceinline__ float2 operator*(float2 a, float s) {
#ifdef __CUDA_ARCH__
  return __fmul2_rn(a, make_float2(s, s));
#else
  return make_float2(a.x * s, a.y * s);
#endif
}
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) { return a * s; }
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(a.x * s, a.y * s); }

template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// acc + a·b; in FP32 two packed FP32x2 FMAs: acc + (a.x, a.x)·(b.x, b.y) + (a.y, a.y)·(−b.y, b.x)
__device__ __forceinline__ float2 cmac(float2 acc, float2 a, float2 b) {
  acc = __ffma2_rn(make_float2(a.x, a.x), b, acc);
  return __ffma2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x), acc);
}
__device__ __forceinline__ double2 cmac(double2 acc, double2 a, double2 b) {
  return make_double2(acc.x + (a.x * b.x - a.y * b.y), acc.y + (a.x * b.y + a.y * b.x));
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { C r; r.x = a.x; r.y = -a.y; return r; }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C> __host__ __device__ __forceinline__ C mul_mi(C a) {
  C r;
  if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

// Signed FFT-order frequency index of bin i on an n-point axis (fftfreq order).
__host__ __device__ __forceinline__ int freq_index(int i, int n) { return (i < (n + 1) / 2) ? i : i - n; }

// Transverse polarisation basis at one plane wave, kpg = k ẑ − G with G = (gx, gy, 0):
// mag = |kpg|, n̂ = ẑ×kpg/|ẑ×kpg| (ŷ when kpg ∥ ẑ), m̂ = n̂×kpg/|n̂×kpg|.
template <typename T> struct Basis { T mag, imag, mx, my, mz, nx, ny; };  // imag = 1/mag

template <typename T>
__host__ __device__ __forceinline__ Basis<T> basis_at(T k, T gx, T gy) {
  Basis<T> b;
  T p2 = gx * gx + gy * gy;
  b.mag = sqrt(p2 + k * k);
  const T im = T(1) / b.mag;
  b.imag = im;
  if (p2 > T(0)) {
    T ip = T(1) / sqrt(p2);
    b.nx = gy * ip; b.ny = -gx * ip;
    b.mx = -gx * k * ip * im; b.my = -gy * k * ip * im; b.mz = -p2 * ip * im;
  } else {
    b.nx = T(0); b.ny = T(1);
    b.mx = (k >= T(0)) ? T(1) : T(-1); b.my = T(0); b.mz = T(0);
  }
  return b;
}

}  // namespace omb
