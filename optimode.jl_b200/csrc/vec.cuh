// Pointwise and reduction helpers shared by the entry points.
#pragma once

#include "op_kernels.cuh"

namespace omb {

// Precision conversion of complex arrays (n elements).
__global__ void k_c64_to_c32(const double2* __restrict__ a, float2* __restrict__ b, size_t n);
__global__ void k_c32_to_c64(const float2* __restrict__ a, double2* __restrict__ b, size_t n);
// v ← v·(c + i s) (a unit phase), n elements
__global__ void k_rotate_c64(double2* __restrict__ v, size_t n, double c, double s);

// Diagonal preconditioner on a 2-component block: H ← H · eps_mean / |k+G|².
template <typename T>
__global__ void k_prec_diag(const cplx<T>* __restrict__ in, cplx<T>* __restrict__ out, int Nx, int Ny,
                            T inv_dx, T inv_dy, const double* __restrict__ k_dev, double eps_mean,
                            int ncol, long long cs) {
  const size_t N = (size_t)Nx * Ny;
  const T k = (T)(*k_dev);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N * ncol; i += (size_t)gridDim.x * blockDim.x) {
    const size_t col = i / N, p = i - col * N;
    const int ix = (int)(p % Nx), iy = (int)(p / Nx);
    const T gx = T(freq_index(ix, Nx)) * inv_dx, gy = T(freq_index(iy, Ny)) * inv_dy;
    const T s = T(eps_mean) / (gx * gx + gy * gy + k * k);
    const cplx<T>* a = in + col * cs + 2 * p;
    cplx<T>* b = out + col * cs + 2 * p;
    b[0] = a[0] * s;
    b[1] = a[1] * s;
  }
}

// Sum per-column partials (2 doubles each, `nb` per column) → out[2·col] (re, im).
__global__ void k_reduce_partials(const double* __restrict__ partial, int nb, int ncol,
                                  double* __restrict__ out);

// argmax of |E|² over a planar 3-component field (first index in the reference's
// column-major (3, Nx, Ny) order on ties); writes (index, E re, E im) per column.
template <typename T>
__global__ void k_argmax_abs2(const cplx<T>* __restrict__ E, long long N, long long cs, int ncol,
                              double* __restrict__ out) {
  const int col = blockIdx.x;
  if (col >= ncol) return;
  const cplx<T>* e = E + col * cs;
  double best = -1.0;
  long long bidx = 0;  // index in column-major (3, Nx, Ny) order: c + 3p
  for (long long p = threadIdx.x; p < N; p += blockDim.x) {
    for (int c = 0; c < 3; ++c) {
      const cplx<T> v = e[c * N + p];
      const double a = (double)v.x * v.x + (double)v.y * v.y;
      const long long li = c + 3 * p;
      if (a > best || (a == best && li < bidx)) { best = a; bidx = li; }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const long long oi = __shfl_xor_sync(0xffffffffu, bidx, o);
    if (ob > best || (ob == best && oi < bidx)) { best = ob; bidx = oi; }
  }
  __shared__ double sb[32];
  __shared__ long long si[32];
  if ((threadIdx.x & 31) == 0) { sb[threadIdx.x >> 5] = best; si[threadIdx.x >> 5] = bidx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (sb[w] > best || (sb[w] == best && si[w] < bidx)) { best = sb[w]; bidx = si[w]; }
    const long long c = bidx % 3, p = bidx / 3;
    const cplx<T> v = e[c * N + p];
    out[3 * col] = (double)bidx;
    out[3 * col + 1] = (double)v.x;
    out[3 * col + 2] = (double)v.y;
  }
}

}  // namespace omb
