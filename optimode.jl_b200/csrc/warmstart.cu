// Learned warm start: a six-layer BF16 convolutional network on the tensor cores that maps
// the smoothed ε⁻¹ map and ω of a cross-section to initial real-space transverse fields
// (Hx, Hy) and effective indices of the lowest four bands, with its training kernels.
//
// Network (activations NHWC, BF16 between layers, FP32 accumulation in TMEM):
//   input  128×128×8  : ε⁻¹ xx, yy, zz, xy, xz, yz (averaged over 2×2 / 4×4 pixels of 256² / 512²
//                       grids), ω, 0
//   L1 3×3/2   8 →  64, ReLU    64×64
//   L2 3×3/1  64 → 128, ReLU    64×64
//   L3 3×3/2 128 → 256, ReLU    32×32
//   L4 3×3/1 256 → 256, ReLU    32×32
//   L5 3×3/1 256 → 128, ReLU    32×32, then nearest ×2 → 64×64
//   L6 3×3/1 128 →  12          64×64: channels 2b, 2b+1 = (Hx, Hy) of band b, 8+b its n_eff map
// ≈1.28 M parameters.  Every convolution is an explicit im2col (k = tap·C + c, taps
// row-major, zero padding 1) followed by the tcgen05 GEMM (tc_gemm.cuh); the backward pass
// is the same GEMM on transposed operands (dW = dZᵀ·A, dA = dZ·W) and a col2im gather.
// Loss per (sample, band): the sign-invariant field misfit (‖p‖² + ‖t‖² − 2|⟨p, t⟩|)/‖t‖²
// plus λ_n·(n̄ − n)² with n̄ the band's n_eff map averaged over the pixels.  Adam on FP32
// master weights, BF16 copies (and their transposes) for the GEMMs.
#include <cuda_bf16.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "context.h"
#include "ops.h"
#include "tc_gemm.h"
#include "warmstart.h"

namespace omb {

using bf16 = __nv_bfloat16;

namespace {

constexpr int WS_IN = 128;     // input image side
constexpr int WS_CIN = 8;      // input channels
constexpr int WS_OUT = 64;     // output image side
constexpr int WS_OUT_LD = 16;  // output row pitch (floats)
constexpr float WS_LAMBDA_N = 100.f;

__host__ __device__ constexpr int rup(int x, int m) { return (x + m - 1) / m * m; }

struct LayerSpec { int cin, cout, stride, relu, up_after, H; };
constexpr LayerSpec kLayers[WS_LAYERS] = {
    {8, 64, 2, 1, 0, 128}, {64, 128, 1, 1, 0, 64}, {128, 256, 2, 1, 0, 64},
    {256, 256, 1, 1, 0, 32}, {256, 128, 1, 1, 1, 32}, {128, 12, 1, 0, 0, 64},
};

// ---- kernels ---------------------------------------------------------------------------
__global__ void k_im2col(const bf16* __restrict__ X, int B, int H, int W, int C, int stride, bf16* __restrict__ A,
                         int Kp) {
  const int Ho = H / stride, Wo = W / stride;
  const long long total = (long long)B * Ho * Wo * Kp;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i % Kp);
    const long long m = i / Kp;
    bf16 v = __float2bfloat16_rn(0.f);
    if (k < 9 * C) {
      const int tap = k / C, c = k - tap * C, ky = tap / 3, kx = tap - 3 * ky;
      const int ox = (int)(m % Wo), oy = (int)((m / Wo) % Ho), b = (int)(m / ((long long)Wo * Ho));
      const int y = oy * stride + ky - 1, x = ox * stride + kx - 1;
      if (y >= 0 && y < H && x >= 0 && x < W) v = X[(((long long)b * H + y) * W + x) * C + c];
    }
    A[i] = v;
  }
}

// dX[b, y, x, c] = Σ over the taps that read (y, x) of dA[(b, oy, ox), tap·C + c]
__global__ void k_col2im(const float* __restrict__ dA, int B, int H, int W, int C, int stride, int Kp,
                         float* __restrict__ dX) {
  const int Ho = H / stride, Wo = W / stride;
  const long long total = (long long)B * H * W * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int x = (int)((i / C) % W), y = (int)((i / ((long long)C * W)) % H), b = (int)(i / ((long long)C * W * H));
    float s = 0.f;
    for (int ky = 0; ky < 3; ++ky) {
      const int ty = y + 1 - ky;
      if (ty < 0 || ty % stride) continue;
      const int oy = ty / stride;
      if (oy >= Ho) continue;
      for (int kx = 0; kx < 3; ++kx) {
        const int tx = x + 1 - kx;
        if (tx < 0 || tx % stride) continue;
        const int ox = tx / stride;
        if (ox >= Wo) continue;
        s += dA[(((long long)b * Ho + oy) * Wo + ox) * Kp + (ky * 3 + kx) * C + c];
      }
    }
    dX[i] = s;
  }
}

// dst[c, r] = src[r, c] for r < R, c < C (bf16 or fp32 source), dst row pitch ldd ≥ R;
// rows c in [C, Cp) of dst are written as zeros.
template <typename S>
__global__ void k_transpose(const S* __restrict__ src, long long R, int C, long long lds, bf16* __restrict__ dst,
                            int Cp, long long ldd) {
  __shared__ float tile[32][33];
  const long long r0 = (long long)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const long long r = r0 + j;
    const int c = c0 + threadIdx.x;
    float v = 0.f;
    if (r < R && c < C) {
      if constexpr (sizeof(S) == 2) v = __bfloat162float(src[r * lds + c]);
      else v = (float)src[r * lds + c];
    }
    tile[j][threadIdx.x] = v;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j;
    const long long r = r0 + threadIdx.x;
    if (c < Cp && r < R) dst[(long long)c * ldd + r] = __float2bfloat16_rn(tile[threadIdx.x][j]);
  }
}

// dZ (bf16, [M × ldz], columns ≥ C zero) = dY masked by the ReLU (Y > 0) when relu != 0
__global__ void k_relu_bwd(const float* __restrict__ dY, int ldy, const bf16* __restrict__ Y, int ly, long long M,
                           int C, int relu, bf16* __restrict__ dZ, int ldz, float* __restrict__ dYm) {
  const long long total = M * ldz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % ldz);
    const long long m = i / ldz;
    float v = 0.f;
    if (c < C) {
      v = dY[m * ldy + c];
      if (relu && !(__bfloat162float(Y[m * ly + c]) > 0.f)) v = 0.f;
      dYm[m * C + c] = v;
    }
    dZ[i] = __float2bfloat16_rn(v);
  }
}

// db[c] += Σ_m dZ[m, c] (FP32, dZ as masked FP32 [M × C])
__global__ void k_colsum(const float* __restrict__ Z, long long M, int C, float* __restrict__ db) {
  const int c = blockIdx.x * 32 + (threadIdx.x & 31);
  const int part = threadIdx.x >> 5, nparts = blockDim.x >> 5;
  float s = 0.f;
  if (c < C)
    for (long long m = (long long)blockIdx.y * nparts + part; m < M; m += (long long)gridDim.y * nparts) s += Z[m * C + c];
  __shared__ float red[32][33];
  red[part][threadIdx.x & 31] = s;
  __syncthreads();
  if (part == 0 && c < C) {
    float t = 0.f;
    for (int p = 0; p < nparts; ++p) t += red[p][threadIdx.x & 31];
    atomicAdd(db + c, t);
  }
}

__global__ void k_upsample2(const bf16* __restrict__ X, int B, int H, int W, int C, bf16* __restrict__ Y) {
  const long long total = (long long)B * 2 * H * 2 * W * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int x = (int)((i / C) % (2 * W)), y = (int)((i / ((long long)C * 2 * W)) % (2 * H));
    const int b = (int)(i / ((long long)C * 4 * W * H));
    Y[i] = X[(((long long)b * H + y / 2) * W + x / 2) * C + c];
  }
}
__global__ void k_upsample2_bwd(const float* __restrict__ dY, int B, int H, int W, int C, float* __restrict__ dX) {
  const long long total = (long long)B * H * W * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int x = (int)((i / C) % W), y = (int)((i / ((long long)C * W)) % H), b = (int)(i / ((long long)C * W * H));
    float s = 0.f;
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) s += dY[(((long long)b * 2 * H + 2 * y + dy) * 2 * W + 2 * x + dx) * C + c];
    dX[i] = s;
  }
}

// One block per (sample, band): loss terms and the gradient of the network output.
__global__ void k_loss(const float* __restrict__ out, const float* __restrict__ tf, const float* __restrict__ tn,
                       int B, float* __restrict__ dout, float* __restrict__ loss) {
  constexpr int NPIX = WS_OUT * WS_OUT;
  const int s = blockIdx.x, b = blockIdx.y;
  __shared__ double red[4][8];
  double dot = 0, pp = 0, tt = 0, nm = 0;
  for (int p = threadIdx.x; p < NPIX; p += blockDim.x) {
    const float* o = out + ((size_t)s * NPIX + p) * WS_OUT_LD;
    const float* t = tf + ((size_t)s * NPIX + p) * 8;
    for (int q = 0; q < 2; ++q) {
      dot += (double)o[2 * b + q] * t[2 * b + q];
      pp += (double)o[2 * b + q] * o[2 * b + q];
      tt += (double)t[2 * b + q] * t[2 * b + q];
    }
    nm += o[8 + b];
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int o = 16; o > 0; o >>= 1) {
    dot += __shfl_xor_sync(0xffffffffu, dot, o);
    pp += __shfl_xor_sync(0xffffffffu, pp, o);
    tt += __shfl_xor_sync(0xffffffffu, tt, o);
    nm += __shfl_xor_sync(0xffffffffu, nm, o);
  }
  if (l == 0) { red[0][w] = dot; red[1][w] = pp; red[2][w] = tt; red[3][w] = nm; }
  __syncthreads();
  __shared__ float coef[4];
  if (threadIdx.x == 0) {
    double D = 0, P = 0, T = 0, Nm = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { D += red[0][i]; P += red[1][i]; T += red[2][i]; Nm += red[3][i]; }
    if (!(T > 0)) T = 1;
    const double nbar = Nm / NPIX, dn = nbar - tn[s * 4 + b];
    const double scale = 1.0 / (4.0 * B);
    atomicAdd(loss, (float)(((P + T - 2 * fabs(D)) / T + WS_LAMBDA_N * dn * dn) * scale));
    coef[0] = (float)(2.0 / T * scale);                     // ∂/∂p = coef0·(p − sgn·t)
    coef[1] = D >= 0 ? 1.f : -1.f;
    coef[2] = (float)(2.0 * WS_LAMBDA_N * dn / NPIX * scale);  // ∂/∂o[8+b]
  }
  __syncthreads();
  for (int p = threadIdx.x; p < NPIX; p += blockDim.x) {
    const float* o = out + ((size_t)s * NPIX + p) * WS_OUT_LD;
    const float* t = tf + ((size_t)s * NPIX + p) * 8;
    float* d = dout + ((size_t)s * NPIX + p) * WS_OUT_LD;
    for (int q = 0; q < 2; ++q) d[2 * b + q] = coef[0] * (o[2 * b + q] - coef[1] * t[2 * b + q]);
    d[8 + b] = coef[2];
  }
}

__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g,
                       long long n, float lr, float b1, float b2, float c1, float c2, float eps) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1 - b1) * gi, vi = b2 * v[i] + (1 - b2) * gi * gi;
    m[i] = mi; v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}
// BF16 weights [rows_p × Kp] from FP32 masters [cout × Kp] (rows ≥ cout zero)
__global__ void k_w_to_bf16(const float* __restrict__ w, int cout, int rows_p, int Kp, bf16* __restrict__ w16) {
  const long long total = (long long)rows_p * Kp;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / Kp);
    w16[i] = __float2bfloat16_rn(r < cout ? w[i] : 0.f);
  }
}

// Input features from a device ε⁻¹ (3, 3, Nx, Ny) FP64 array: 128×128×8 BF16, 2×2 averaged
// for 256² grids (pixel (x, y) of the image is grid pixel (x, y), x along Nx).
__global__ void k_features(const double* __restrict__ ei, int Nx, int Ny, double omega, bf16* __restrict__ F) {
  const int f = Nx / WS_IN;  // 1 or 2
  const int total = WS_IN * WS_IN;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int x = i % WS_IN, y = i / WS_IN;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int dy = 0; dy < f; ++dy)
      for (int dx = 0; dx < f; ++dx) {
        const double* e = ei + 9 * ((size_t)(x * f + dx) + (size_t)Nx * (y * f + dy));
        acc[0] += e[0]; acc[1] += e[4]; acc[2] += e[8];
        acc[3] += 0.5 * (e[1] + e[3]); acc[4] += 0.5 * (e[2] + e[6]); acc[5] += 0.5 * (e[5] + e[7]);
      }
    bf16* o = F + (size_t)i * WS_CIN;
    for (int c = 0; c < 6; ++c) o[c] = __float2bfloat16_rn((float)(acc[c] / (f * f)));
    o[6] = __float2bfloat16_rn((float)omega);
    o[7] = __float2bfloat16_rn(0.f);
  }
}

// Input image from an uploaded cell (FP64 ε⁻¹ as 3 double2 per pixel: (xx, yy), (zz, xy),
// (xz, yz)), the same features as k_features.
__global__ void k_features_cell(const double2* __restrict__ e64, int Nx, int Ny, double omega, bf16* __restrict__ F) {
  const int f = Nx / WS_IN;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < WS_IN * WS_IN; i += gridDim.x * blockDim.x) {
    const int x = i % WS_IN, y = i / WS_IN;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int dy = 0; dy < f; ++dy)
      for (int dx = 0; dx < f; ++dx) {
        const size_t p = (size_t)(x * f + dx) + (size_t)Nx * (y * f + dy);
        const double2 a = e64[3 * p], b = e64[3 * p + 1], c = e64[3 * p + 2];
        acc[0] += a.x; acc[1] += a.y; acc[2] += b.x; acc[3] += b.y; acc[4] += c.x; acc[5] += c.y;
      }
    bf16* o = F + (size_t)i * WS_CIN;
    for (int c = 0; c < 6; ++c) o[c] = __float2bfloat16_rn((float)(acc[c] / (f * f)));
    o[6] = __float2bfloat16_rn((float)omega);
    o[7] = __float2bfloat16_rn(0.f);
  }
  (void)Ny;
}

// Per (image, band): the mean of the band's n_eff channel.
__global__ void k_neff_mean(const float* __restrict__ out, double* __restrict__ neff) {
  const int s = blockIdx.x, b = blockIdx.y;
  double acc = 0;
  for (int p = threadIdx.x; p < WS_OUT * WS_OUT; p += blockDim.x) acc += out[((size_t)s * WS_OUT * WS_OUT + p) * WS_OUT_LD + 8 + b];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    neff[s * 4 + b] = t / (WS_OUT * WS_OUT);
  }
}

// Bilinear resampling of the bands' (Hx, Hy) from the 64×64 output to the Nx×Ny grid (pixel
// centres aligned, edge values held), as planar complex (Hx, Hy, 0) per band: dst[b][c][p].
__global__ void k_fields_to_grid(const float* __restrict__ out, int Nx, int Ny, double2* __restrict__ dst) {
  const size_t N = (size_t)Nx * Ny;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 4 * N; i += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / N);
    const size_t p = i - (size_t)b * N;
    const int ix = (int)(p % Nx), iy = (int)(p / Nx);
    const float u = fminf(fmaxf((ix + 0.5f) * WS_OUT / Nx - 0.5f, 0.f), WS_OUT - 1.f);
    const float v = fminf(fmaxf((iy + 0.5f) * WS_OUT / Ny - 0.5f, 0.f), WS_OUT - 1.f);
    const int x0 = min((int)u, WS_OUT - 2), y0 = min((int)v, WS_OUT - 2);
    const float fx = u - x0, fy = v - y0;
    float h[2];
    for (int c = 0; c < 2; ++c) {
      auto at = [&](int x, int y) { return out[((size_t)y * WS_OUT + x) * WS_OUT_LD + 2 * b + c]; };
      h[c] = (1 - fy) * ((1 - fx) * at(x0, y0) + fx * at(x0 + 1, y0)) + fy * ((1 - fx) * at(x0, y0 + 1) + fx * at(x0 + 1, y0 + 1));
    }
    double2* d = dst + (size_t)b * 3 * N;
    d[p] = make_double2(h[0], 0);
    d[N + p] = make_double2(h[1], 0);
    d[2 * N + p] = make_double2(0, 0);
  }
}

// Plane-wave coefficients of a band from its transformed Cartesian field G (planar, 3
// components): H_z replaced by the transverse value (g·H_t)/k' (w·H = 0 with w = (−gx, −gy, k')),
// then h1 = m̂·H, h2 = n̂·H at the band's k.
__global__ void k_project_guess(const double2* __restrict__ G, int Nx, int Ny, double inv_dx, double inv_dy,
                                const double* __restrict__ kb, double2* __restrict__ cols) {
  const size_t N = (size_t)Nx * Ny;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 4 * N; i += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / N);
    const size_t p = i - (size_t)b * N;
    const int ix = (int)(p % Nx), iy = (int)(p / Nx);
    const double k = kb[b];
    const double gx = freq_index(ix, Nx) * inv_dx, gy = freq_index(iy, Ny) * inv_dy;
    const Basis<double> bs = basis_at<double>(k, gx, gy);
    const double2 hx = G[(size_t)b * 3 * N + p], hy = G[(size_t)b * 3 * N + N + p];
    const double2 hz = make_double2((gx * hx.x + gy * hy.x) / k, (gx * hx.y + gy * hy.y) / k);
    double2* c = cols + (size_t)b * 2 * N;
    c[2 * p] = make_double2(bs.mx * hx.x + bs.my * hy.x + bs.mz * hz.x, bs.mx * hx.y + bs.my * hy.y + bs.mz * hz.y);
    c[2 * p + 1] = make_double2(bs.nx * hx.x + bs.ny * hy.x, bs.nx * hx.y + bs.ny * hy.y);
  }
}

inline int blocks_for_n(long long n) { long long b = (n + 255) / 256; return (int)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b)); }

}  // namespace

// ---- the network object ------------------------------------------------------------------
struct WsLayer {
  LayerSpec s;
  int Ho, Kp, K9, cout_p64, cout_rows;  // cout_rows: rows of the forward B operand (≥ 16)
  DevBuf<float> w, b, mw, vw, mb, vb, gw, gb;
  DevBuf<bf16> w16, wt16;  // [cout_rows × Kp], [Kp × cout_p64]
  DevBuf<bf16> acol;       // [M × Kp] of the last forward
  DevBuf<bf16> y;          // [M × cout] output (bf16; the last layer writes FP32 `out`)
  long long M(int B) const { return (long long)B * Ho * Ho; }
};

}  // namespace omb

struct omb_warmstart {
  omb_ctx* ctx = nullptr;  // null once the context was destroyed (device memory released)
  int device = 0;
  int cap = 0;
  omb::WsLayer L[omb::WS_LAYERS];
  omb::DevBuf<omb::bf16> up;          // L5 output upsampled [B·64·64 × 128]
  omb::DevBuf<float> out, dout;       // [B·4096 × 16]
  omb::DevBuf<float> dy, dx;          // gradient buffers (FP32, largest activation)
  omb::DevBuf<float> dym;             // masked dY (FP32)
  omb::DevBuf<omb::bf16> dz, dzt, at; // dZ [M × cout_p64], dZᵀ [cout_rows × M], Aᵀ [Kp × M]
  omb::DevBuf<float> da;              // [M × Kp]
  omb::DevBuf<float> loss;
  omb::DevBuf<int> err;
  int step = 0;
};

namespace omb {

namespace {
#define WS_TRY(x) do { int rc_ = (x); if (rc_) return rc_; } while (0)
#define WS_CU(x) OMB_CU(x)

int ws_alloc(omb_warmstart* W, int cap) {
  cudaStream_t st = W->ctx->stream;
  size_t max_act = 0, max_acol_t = 0, max_da = 0, max_dz = 0, max_dzt = 0;
  for (int l = 0; l < WS_LAYERS; ++l) {
    WsLayer& L = W->L[l];
    const long long M = L.M(cap);
    WS_CU(L.acol.alloc((size_t)M * L.Kp, st));
    if (l < WS_LAYERS - 1) WS_CU(L.y.alloc((size_t)M * L.s.cout, st));
    max_acol_t = std::max(max_acol_t, (size_t)M * L.Kp);
    max_da = std::max(max_da, (size_t)M * L.Kp);
    max_dz = std::max(max_dz, (size_t)M * L.cout_p64);
    max_dzt = std::max(max_dzt, (size_t)M * L.cout_rows);
    // output gradients (M × cout) and input gradients (B·H²·cin, the upsampled size included)
    max_act = std::max(max_act, std::max((size_t)M * L.s.cout, (size_t)cap * L.s.H * L.s.H * L.s.cin));
  }
  WS_CU(W->up.alloc((size_t)cap * 64 * 64 * 128, st));
  WS_CU(W->out.alloc((size_t)cap * 4096 * WS_OUT_LD, st));
  WS_CU(W->dout.alloc((size_t)cap * 4096 * WS_OUT_LD, st));
  WS_CU(W->dy.alloc(max_act, st));
  WS_CU(W->dx.alloc(max_act, st));
  WS_CU(W->dym.alloc(max_act, st));
  WS_CU(W->dz.alloc(max_dz, st));
  WS_CU(W->dzt.alloc(max_dzt, st));
  WS_CU(W->at.alloc(max_acol_t, st));
  WS_CU(W->da.alloc(max_da, st));
  WS_CU(W->loss.alloc(1, st));
  WS_CU(W->err.alloc(1, st));
  WS_CU(W->err.zero());
  return OMB_OK;
}

int ws_refresh_bf16(omb_warmstart* W, int l) {
  cudaStream_t st = W->ctx->stream;
  WsLayer& L = W->L[l];
  k_w_to_bf16<<<blocks_for_n((long long)L.cout_rows * L.Kp), 256, 0, st>>>(L.w.p, L.s.cout, L.cout_rows, L.Kp, L.w16.p);
  // Wᵀ [Kp × cout_p64]: transpose of the FP32 master (rows ≥ cout zero)
  k_transpose<float><<<dim3((L.s.cout + 31) / 32, (L.Kp + 31) / 32), dim3(32, 8), 0, st>>>(
      L.w.p, L.s.cout, L.Kp, L.Kp, L.wt16.p, L.Kp, L.cout_p64);
  WS_CU(cudaGetLastError());
  // columns cout..cout_p64 of Wᵀ must be zero: cleared once at creation, never written
  return OMB_OK;
}

int gemm(omb_warmstart* W, const void* A, const void* B, void* D, long long M, int N, int K, long long ldd,
         const float* bias, int relu, int epi, int splits) {
  return tc_gemm(W->ctx->stream, A, B, D, (int)M, N, K, ldd, bias, relu, epi, splits, W->err.p, W->ctx->wait_ns);
}

int ws_forward(omb_warmstart* W, const bf16* feat, int B) {
  cudaStream_t st = W->ctx->stream;
  const bf16* x = feat;
  for (int l = 0; l < WS_LAYERS; ++l) {
    WsLayer& L = W->L[l];
    const long long M = L.M(B);
    k_im2col<<<blocks_for_n(M * L.Kp), 256, 0, st>>>(x, B, L.s.H, L.s.H, L.s.cin, L.s.stride, L.acol.p, L.Kp);
    WS_CU(cudaGetLastError());
    if (l == WS_LAYERS - 1) {
      WS_TRY(gemm(W, L.acol.p, L.w16.p, W->out.p, M, L.s.cout, L.Kp, WS_OUT_LD, L.b.p, 0, TC_STORE_F32, 1));
    } else {
      WS_TRY(gemm(W, L.acol.p, L.w16.p, L.y.p, M, L.s.cout, L.Kp, L.s.cout, L.b.p, L.s.relu, TC_STORE_BF16, 1));
      x = L.y.p;
      if (L.s.up_after) {
        k_upsample2<<<blocks_for_n(M * 4 * L.s.cout), 256, 0, st>>>(L.y.p, B, L.Ho, L.Ho, L.s.cout, W->up.p);
        WS_CU(cudaGetLastError());
        x = W->up.p;
      }
    }
  }
  return OMB_OK;
}

// splits for a weight-gradient GEMM (reduction over M)
int wgrad_splits(long long M, int cout, int Kp) {
  const long long tiles = (long long)((cout + 127) / 128) * ((Kp + tc_gemm_bn(Kp) - 1) / tc_gemm_bn(Kp));
  const long long kt = M / 64;
  long long s = (2 * 148 + tiles - 1) / tiles;
  if (s > kt) s = kt;
  return (int)std::max(1LL, s);
}

int ws_backward(omb_warmstart* W, const bf16* feat, int B) {
  cudaStream_t st = W->ctx->stream;
  // gradient w.r.t. the current layer's output (FP32): starts as dout of the last layer
  const float* dY = W->dout.p;
  int ldy = WS_OUT_LD;
  for (int l = WS_LAYERS - 1; l >= 0; --l) {
    WsLayer& L = W->L[l];
    const long long M = L.M(B);
    const int C = L.s.cout;
    // dZ = dY ⊙ ReLU'(Y): bf16 [M × cout_p64] (zero padded) and FP32 [M × C]
    k_relu_bwd<<<blocks_for_n(M * L.cout_p64), 256, 0, st>>>(dY, ldy, L.s.relu ? L.y.p : nullptr, C, M, C, L.s.relu,
                                                              W->dz.p, L.cout_p64, W->dym.p);
    WS_CU(cudaGetLastError());
    // db = Σ_m dZ
    WS_CU(cudaMemsetAsync(L.gb.p, 0, C * sizeof(float), st));
    k_colsum<<<dim3((C + 31) / 32, 64), 256, 0, st>>>(W->dym.p, M, C, L.gb.p);
    WS_CU(cudaGetLastError());
    // dW = dZᵀ · A: transposes dZᵀ [cout_rows × M] and Aᵀ [Kp × M]
    k_transpose<float><<<dim3((unsigned)((M + 31) / 32), (L.cout_rows + 31) / 32), dim3(32, 8), 0, st>>>(
        W->dym.p, M, C, C, W->dzt.p, L.cout_rows, M);
    k_transpose<bf16><<<dim3((unsigned)((M + 31) / 32), (L.Kp + 31) / 32), dim3(32, 8), 0, st>>>(
        L.acol.p, M, L.Kp, L.Kp, W->at.p, L.Kp, M);
    WS_CU(cudaGetLastError());
    WS_CU(cudaMemsetAsync(L.gw.p, 0, (size_t)C * L.Kp * sizeof(float), st));
    WS_TRY(gemm(W, W->dzt.p, W->at.p, L.gw.p, C, L.Kp, (int)M, L.Kp, nullptr, 0, TC_ATOMIC_F32,
                wgrad_splits(M, C, L.Kp)));
    if (l == 0) break;
    // dA = dZ · W  ([M × Kp], FP32), then col2im to the layer input
    WS_TRY(gemm(W, W->dz.p, L.wt16.p, W->da.p, M, L.Kp, L.cout_p64, L.Kp, nullptr, 0, TC_STORE_F32, 1));
    const int Hin = L.s.H, Cin = L.s.cin;
    const long long nin = (long long)B * Hin * Hin * Cin;
    k_col2im<<<blocks_for_n(nin), 256, 0, st>>>(W->da.p, B, Hin, Hin, Cin, L.s.stride, L.Kp, W->dx.p);
    WS_CU(cudaGetLastError());
    const WsLayer& P = W->L[l - 1];
    if (P.s.up_after) {  // the input was the ×2 upsampled output of the previous layer
      k_upsample2_bwd<<<blocks_for_n((long long)B * P.Ho * P.Ho * P.s.cout), 256, 0, st>>>(W->dx.p, B, P.Ho, P.Ho,
                                                                                         P.s.cout, W->dy.p);
      WS_CU(cudaGetLastError());
    } else {
      WS_CU(cudaMemcpyAsync(W->dy.p, W->dx.p, nin * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    dY = W->dy.p;
    ldy = P.s.cout;
  }
  (void)feat;
  return OMB_OK;
}

int ws_check_err(omb_warmstart* W) {
  int h = 0;
  WS_CU(cudaMemcpyAsync(&h, W->err.p, sizeof(int), cudaMemcpyDeviceToHost, W->ctx->stream));
  WS_CU(cudaStreamSynchronize(W->ctx->stream));
  if (h) {
    WS_CU(cudaMemsetAsync(W->err.p, 0, sizeof(int), W->ctx->stream));
    return fail(OMB_ERR_TIMEOUT, "warm-start network: a tensor-core pipeline wait ran out (code " + std::to_string(h) + ")");
  }
  return OMB_OK;
}

}  // namespace

int64_t ws_num_params() {
  int64_t n = 0;
  for (int l = 0; l < WS_LAYERS; ++l) n += (int64_t)kLayers[l].cout * 9 * kLayers[l].cin + kLayers[l].cout;
  return n;
}

int ws_forward_dev(omb_warmstart* W, const void* feat, int B, float** out) {
  WS_TRY(ws_forward(W, static_cast<const bf16*>(feat), B));
  *out = W->out.p;
  return OMB_OK;
}

int ws_guesses(omb_warmstart* W, const std::vector<const Problem*>& probs, const std::vector<double>& omegas,
               DevBuf<double2>& cols, std::vector<size_t>& col_off, std::vector<std::array<double, 4>>& kb) {
  cudaStream_t st = W->ctx->stream;
  const int n = (int)probs.size();
  col_off.assign(n, 0);
  kb.assign(n, {0, 0, 0, 0});
  if (n == 0) return OMB_OK;
  size_t tot = 0, maxN = 0;
  for (int i = 0; i < n; ++i) {
    const Problem& P = *probs[i];
    if (!(P.Nx == P.Ny && (P.Nx == 128 || P.Nx == 256 || P.Nx == 512)))
      return fail(OMB_ERR_UNSUPPORTED, "learned warm start: 128x128, 256x256 or 512x512 grids");
    col_off[i] = tot;
    tot += 4 * 2 * P.N();
    maxN = std::max(maxN, P.N());
  }
  OMB_CU(cols.alloc(tot, st));
  DevBuf<bf16> feat;
  OMB_CU(feat.alloc((size_t)n * WS_IN * WS_IN * WS_CIN, st));
  DevBuf<float> outs;
  OMB_CU(outs.alloc((size_t)n * 4096 * WS_OUT_LD, st));
  for (int i = 0; i < n; ++i) {
    const Problem& P = *probs[i];
    k_features_cell<<<64, 256, 0, st>>>(P.e64.p, P.Nx, P.Ny, omegas[i], feat.p + (size_t)i * WS_IN * WS_IN * WS_CIN);
  }
  OMB_CU(cudaGetLastError());
  for (int i0 = 0; i0 < n; i0 += W->cap) {
    const int B = std::min(W->cap, n - i0);
    int rc = ws_forward(W, feat.p + (size_t)i0 * WS_IN * WS_IN * WS_CIN, B);
    if (rc) return rc;
    OMB_CU(cudaMemcpyAsync(outs.p + (size_t)i0 * 4096 * WS_OUT_LD, W->out.p, (size_t)B * 4096 * WS_OUT_LD * 4,
                           cudaMemcpyDeviceToDevice, st));
  }
  DevBuf<double> dn;
  OMB_CU(dn.alloc((size_t)n * 4, st));
  k_neff_mean<<<dim3(n, 4), 256, 0, st>>>(outs.p, dn.p);
  OMB_CU(cudaGetLastError());
  std::vector<double> hn((size_t)n * 4);
  OMB_CU(cudaMemcpyAsync(hn.data(), dn.p, hn.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  int rc = ws_check_err(W);  // synchronises
  if (rc) return rc;
  DevBuf<double2> planar, scr;
  OMB_CU(planar.alloc(4 * 3 * maxN, st));
  OMB_CU(scr.alloc(4 * 3 * maxN, st));
  DevBuf<double> kd;
  OMB_CU(kd.alloc((size_t)n * 4, st));
  std::vector<double> hk((size_t)n * 4);
  for (int i = 0; i < n; ++i)
    for (int b = 0; b < 4; ++b) {
      // an index outside the physical range falls back to the cell's own k_guess scale
      const double nb = hn[i * 4 + b];
      hk[i * 4 + b] = omegas[i] * ((nb > 1.0 && nb < 4.0 && std::isfinite(nb)) ? nb : std::sqrt(1.0 / probs[i]->min_diag));
      kb[i][b] = hk[i * 4 + b];
    }
  OMB_CU(cudaMemcpyAsync(kd.p, hk.data(), hk.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  DevBuf<OpUnit<double>> du;
  OMB_CU(du.alloc(1, st));
  for (int i = 0; i < n; ++i) {
    const Problem& P = *probs[i];
    const size_t N = P.N();
    k_fields_to_grid<<<blocks_for_n(4 * (long long)N), 256, 0, st>>>(outs.p + (size_t)i * 4096 * WS_OUT_LD, P.Nx,
                                                                     P.Ny, planar.p);
    OMB_CU(cudaGetLastError());
    OpUnit<double> u{};
    u.in = planar.p; u.scr = scr.p; u.k_dev = kd.p + 4 * i;
    u.in_cs = (long long)(3 * N); u.scr_cs = (long long)(3 * N); u.ncol = 4;
    u.Nx = P.Nx; u.Ny = P.Ny; u.inv_dx = 1.0 / P.Dx; u.inv_dy = 1.0 / P.Dy;
    u.part_stride = row_blocks(P.Nx, P.Ny);
    OMB_CU(cudaMemcpyAsync(du.p, &u, sizeof(u), cudaMemcpyHostToDevice, st));
    OMB_CU(launch_op<double>(OP_R2G, du.p, 1, P.Nx, P.Ny, 4, W->ctx->tw, st));
    k_project_guess<<<blocks_for_n(4 * (long long)N), 256, 0, st>>>(scr.p, P.Nx, P.Ny, 1.0 / P.Dx, 1.0 / P.Dy,
                                                                   kd.p + 4 * i, cols.p + col_off[i]);
    OMB_CU(cudaGetLastError());
    // the unit block is re-written for the next instance only after this one's passes ran
    OMB_CU(cudaStreamSynchronize(st));
  }
  return OMB_OK;
}

void ws_release_all(omb_ctx* ctx) {
  for (omb_warmstart* W : ctx->nets) {
    for (WsLayer& L : W->L) L = WsLayer{};
    W->up = DevBuf<bf16>{};
    W->out = DevBuf<float>{};
    W->dout = DevBuf<float>{};
    W->dy = DevBuf<float>{};
    W->dx = DevBuf<float>{};
    W->dym = DevBuf<float>{};
    W->dz = DevBuf<bf16>{};
    W->dzt = DevBuf<bf16>{};
    W->at = DevBuf<bf16>{};
    W->da = DevBuf<float>{};
    W->loss = DevBuf<float>{};
    W->err = DevBuf<int>{};
    W->ctx = nullptr;
  }
  ctx->nets.clear();
  ctx->ws = nullptr;
  cudaStreamSynchronize(ctx->stream);
}

}  // namespace omb

using namespace omb;

extern "C" {

int omb_warmstart_create(omb_ctx* ctx, int32_t batch_cap, uint64_t seed, omb_warmstart** out) {
  if (!ctx || !out) return fail(OMB_ERR_INVALID_ARG, "ctx/out is NULL");
  if (batch_cap < 1 || batch_cap > 256) return fail(OMB_ERR_INVALID_ARG, "batch_cap must be in 1..256");
  OMB_CU(cudaSetDevice(ctx->device));
  auto W = std::make_unique<omb_warmstart>();
  W->ctx = ctx;
  W->device = ctx->device;
  W->cap = batch_cap;
  cudaStream_t st = ctx->stream;
  std::mt19937_64 rng(seed);
  for (int l = 0; l < WS_LAYERS; ++l) {
    WsLayer& L = W->L[l];
    L.s = kLayers[l];
    L.Ho = L.s.H / L.s.stride;
    L.K9 = 9 * L.s.cin;
    L.Kp = rup(L.K9, 64);
    L.cout_p64 = rup(L.s.cout, 64);
    L.cout_rows = rup(L.s.cout, 16);
    OMB_CU(L.w.alloc((size_t)L.s.cout * L.Kp, st));
    OMB_CU(L.b.alloc(L.s.cout, st));
    for (DevBuf<float>* p : {&L.mw, &L.vw, &L.gw}) OMB_CU(p->alloc((size_t)L.s.cout * L.Kp, st));
    for (DevBuf<float>* p : {&L.mb, &L.vb, &L.gb}) OMB_CU(p->alloc(L.s.cout, st));
    for (DevBuf<float>* p : {&L.mw, &L.vw, &L.mb, &L.vb}) OMB_CU(p->zero());
    OMB_CU(L.w16.alloc((size_t)L.cout_rows * L.Kp, st));
    OMB_CU(L.wt16.alloc((size_t)L.Kp * L.cout_p64, st));
    OMB_CU(L.wt16.zero());
    // He initialisation (seeded), zero in the padding columns, zero biases
    std::vector<float> hw((size_t)L.s.cout * L.Kp, 0.f), hb(L.s.cout, 0.f);
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (float)L.K9) * (l == WS_LAYERS - 1 ? 0.5f : 1.f));
    for (int o = 0; o < L.s.cout; ++o)
      for (int k = 0; k < L.K9; ++k) hw[(size_t)o * L.Kp + k] = nd(rng);
    OMB_CU(cudaMemcpyAsync(L.w.p, hw.data(), hw.size() * 4, cudaMemcpyHostToDevice, st));
    OMB_CU(cudaMemcpyAsync(L.b.p, hb.data(), hb.size() * 4, cudaMemcpyHostToDevice, st));
    OMB_CU(cudaStreamSynchronize(st));
    int rc = ws_refresh_bf16(W.get(), l);
    if (rc) return rc;
  }
  int rc = ws_alloc(W.get(), batch_cap);
  if (rc) return rc;
  OMB_CU(cudaStreamSynchronize(st));
  ctx->nets.push_back(W.get());
  *out = W.release();
  return OMB_OK;
}

int omb_ctx_set_warmstart(omb_ctx* ctx, omb_warmstart* W) {
  if (!ctx) return fail(OMB_ERR_INVALID_ARG, "ctx is NULL");
  if (W && W->ctx != ctx) return fail(OMB_ERR_INVALID_ARG, "the network belongs to another context");
  ctx->ws = W;
  return OMB_OK;
}

int omb_warmstart_destroy(omb_warmstart* W) {
  if (!W) return OMB_OK;
  cudaSetDevice(W->device);
  if (omb_ctx* ctx = W->ctx) {
    if (ctx->ws == W) ctx->ws = nullptr;
    auto& v = ctx->nets;
    v.erase(std::remove(v.begin(), v.end(), W), v.end());
    cudaStreamSynchronize(ctx->stream);
  }
  delete W;  // (an orphaned network holds no device memory any more)
  return OMB_OK;
}

int64_t omb_warmstart_num_params(void) { return ws_num_params(); }

// Parameters layer by layer: W as [cout × 9·cin] row-major (k = tap·cin + c), then b[cout].
int omb_warmstart_get_params(omb_warmstart* W, float* host) {
  if (!W || !host) return fail(OMB_ERR_INVALID_ARG, "NULL argument");
  cudaStream_t st = W->ctx->stream;
  size_t off = 0;
  for (int l = 0; l < WS_LAYERS; ++l) {
    WsLayer& L = W->L[l];
    OMB_CU(cudaMemcpy2DAsync(host + off, L.K9 * 4, L.w.p, L.Kp * 4, L.K9 * 4, L.s.cout, cudaMemcpyDeviceToHost, st));
    off += (size_t)L.s.cout * L.K9;
    OMB_CU(cudaMemcpyAsync(host + off, L.b.p, L.s.cout * 4, cudaMemcpyDeviceToHost, st));
    off += L.s.cout;
  }
  OMB_CU(cudaStreamSynchronize(st));
  return OMB_OK;
}

int omb_warmstart_set_params(omb_warmstart* W, const float* host) {
  if (!W || !host) return fail(OMB_ERR_INVALID_ARG, "NULL argument");
  cudaStream_t st = W->ctx->stream;
  size_t off = 0;
  for (int l = 0; l < WS_LAYERS; ++l) {
    WsLayer& L = W->L[l];
    for (int64_t i = 0; i < (int64_t)L.s.cout * L.K9 + L.s.cout; ++i)
      if (!std::isfinite(host[off + i])) return fail(OMB_ERR_NAN, "non-finite network parameter");
    OMB_CU(L.w.zero());
    OMB_CU(cudaMemcpy2DAsync(L.w.p, L.Kp * 4, host + off, L.K9 * 4, L.K9 * 4, L.s.cout, cudaMemcpyHostToDevice, st));
    off += (size_t)L.s.cout * L.K9;
    OMB_CU(cudaMemcpyAsync(L.b.p, host + off, L.s.cout * 4, cudaMemcpyHostToDevice, st));
    off += L.s.cout;
    int rc = ws_refresh_bf16(W, l);
    if (rc) return rc;
  }
  OMB_CU(cudaStreamSynchronize(st));
  return OMB_OK;
}

int omb_warmstart_features(omb_warmstart* W, const double* d_epsinv, int32_t Nx, int32_t Ny, double omega,
                           void* d_feat, void* stream) {
  if (!W || !d_epsinv || !d_feat) return fail(OMB_ERR_INVALID_ARG, "NULL argument");
  if (!(Nx == Ny && (Nx == 128 || Nx == 256 || Nx == 512)))
    return fail(OMB_ERR_UNSUPPORTED, "warm-start network input: 128x128, 256x256 or 512x512 grids");
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : W->ctx->stream;
  k_features<<<64, 256, 0, st>>>(d_epsinv, Nx, Ny, omega, static_cast<bf16*>(d_feat));
  OMB_CU(cudaGetLastError());
  return OMB_OK;
}

int omb_warmstart_forward(omb_warmstart* W, const void* d_feat, int32_t batch, float* d_out) {
  if (!W || !d_feat || !d_out) return fail(OMB_ERR_INVALID_ARG, "NULL argument");
  if (batch < 1 || batch > W->cap) return fail(OMB_ERR_INVALID_ARG, "batch outside 1..batch_cap");
  int rc = ws_forward(W, static_cast<const bf16*>(d_feat), batch);
  if (rc) return rc;
  OMB_CU(cudaMemcpyAsync(d_out, W->out.p, (size_t)batch * 4096 * WS_OUT_LD * 4, cudaMemcpyDeviceToDevice, W->ctx->stream));
  return ws_check_err(W);
}

int omb_warmstart_train_step(omb_warmstart* W, const void* d_feat, const float* d_tfield, const float* d_tneff,
                             int32_t batch, float lr, int32_t update, float* loss, float* grads) {
  if (!W || !d_feat || !d_tfield || !d_tneff) return fail(OMB_ERR_INVALID_ARG, "NULL argument");
  if (batch < 1 || batch > W->cap) return fail(OMB_ERR_INVALID_ARG, "batch outside 1..batch_cap");
  cudaStream_t st = W->ctx->stream;
  int rc = ws_forward(W, static_cast<const bf16*>(d_feat), batch);
  if (rc) return rc;
  OMB_CU(cudaMemsetAsync(W->loss.p, 0, sizeof(float), st));
  OMB_CU(cudaMemsetAsync(W->dout.p, 0, (size_t)batch * 4096 * WS_OUT_LD * 4, st));
  k_loss<<<dim3(batch, 4), 256, 0, st>>>(W->out.p, d_tfield, d_tneff, batch, W->dout.p, W->loss.p);
  OMB_CU(cudaGetLastError());
  rc = ws_backward(W, static_cast<const bf16*>(d_feat), batch);
  if (rc) return rc;
  if (grads) {
    size_t off = 0;
    for (int l = 0; l < WS_LAYERS; ++l) {
      WsLayer& L = W->L[l];
      OMB_CU(cudaMemcpy2DAsync(grads + off, L.K9 * 4, L.gw.p, L.Kp * 4, L.K9 * 4, L.s.cout, cudaMemcpyDeviceToHost, st));
      off += (size_t)L.s.cout * L.K9;
      OMB_CU(cudaMemcpyAsync(grads + off, L.gb.p, L.s.cout * 4, cudaMemcpyDeviceToHost, st));
      off += L.s.cout;
    }
  }
  if (update) {
    W->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)W->step), c2 = 1.f - std::pow(b2, (float)W->step);
    for (int l = 0; l < WS_LAYERS; ++l) {
      WsLayer& L = W->L[l];
      const long long nw = (long long)L.s.cout * L.Kp;
      k_adam<<<blocks_for_n(nw), 256, 0, st>>>(L.w.p, L.mw.p, L.vw.p, L.gw.p, nw, lr, b1, b2, c1, c2, 1e-8f);
      k_adam<<<1, 256, 0, st>>>(L.b.p, L.mb.p, L.vb.p, L.gb.p, L.s.cout, lr, b1, b2, c1, c2, 1e-8f);
      OMB_CU(cudaGetLastError());
      rc = ws_refresh_bf16(W, l);
      if (rc) return rc;
    }
  }
  if (loss) OMB_CU(cudaMemcpyAsync(loss, W->loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
  return ws_check_err(W);
}

}  // extern "C"
