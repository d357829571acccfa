// Pointwise and reduction helpers shared by the entry points.
#include "vec.cuh"

namespace omb {

__global__ void k_c64_to_c32(const double2* __restrict__ a, float2* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = make_float2((float)a[i].x, (float)a[i].y);
}
__global__ void k_c32_to_c64(const float2* __restrict__ a, double2* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = make_double2((double)a[i].x, (double)a[i].y);
}
__global__ void k_rotate_c64(double2* __restrict__ v, size_t n, double c, double s) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 a = v[i];
    v[i] = make_double2(a.x * c - a.y * s, a.x * s + a.y * c);
  }
}

__global__ void k_reduce_partials(const double* __restrict__ partial, int nb, int ncol, double* __restrict__ out) {
  const int col = blockIdx.x;
  if (col >= ncol) return;
  __shared__ double sr[32], si[32];
  double r = 0, i = 0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    r += partial[2 * ((size_t)col * nb + b)];
    i += partial[2 * ((size_t)col * nb + b) + 1];
  }
  for (int o = 16; o > 0; o >>= 1) {
    r += __shfl_xor_sync(0xffffffffu, r, o);
    i += __shfl_xor_sync(0xffffffffu, i, o);
  }
  if ((threadIdx.x & 31) == 0) { sr[threadIdx.x >> 5] = r; si[threadIdx.x >> 5] = i; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += sr[w]; b += si[w]; }
    out[2 * col] = a;
    out[2 * col + 1] = b;
  }
}

}  // namespace omb
