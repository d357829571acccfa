// Operator passes on the two-level register FFT (fft_reg.cuh) for line lengths that split
// into two register DFTs (≤ 256 here); longer lines use the Stockham passes of
// op_kernels.cuh.  Same three passes, modes, layouts and results as those kernels:
//
//   row_in  : G grid rows per CTA; global H → prologue → step 1 (A-point DFTs) → padded
//             block → step 2 (B-point DFTs) → planar scratch, coalesced along x;
//   col     : TX adjacent columns per CTA; scratch → step 1 → block → step 2 → per-pixel
//             ε⁻¹ contraction → reverse step 1 → block → reverse step 2 → scratch;
//   row_out : G rows per CTA; scratch → reverse steps → curl epilogue → H out.
//
// Each transform touches shared memory once (one conflict-free transpose), global loads
// go straight into the registers of the DFT that consumes them, and ε⁻¹ is read at the
// point of use with the three field components of the pixel in registers (FP32), or in
// the thread's own slots of the block (FP64, which keeps the register count below 128).
#pragma once

#include "fft_reg.cuh"
#include "op_kernels.cuh"

namespace omb {

// Elements per 128-byte shared-memory row.
template <typename C> __host__ __device__ constexpr int smem_row_elems() { return 128 / (int)sizeof(C); }

// Per-line stride of a row pass: ≡ B (mod row elements), so that the step-1 column writes of
// consecutive threads (line-major, n2 fastest) fall in consecutive banks.
template <typename C, int L> __host__ __device__ constexpr int l2_row_lstr() {
  constexpr int A = plan2_a(L), B = L / A, E = smem_row_elems<C>();
  constexpr int base = A * (B + 1);
  return base + (((B % E) - (base % E)) % E + E) % E;
}
// Per-line stride of the column pass: ≡ E/TX (mod E) (threads are column-fastest).
template <typename C, int L, int TX> __host__ __device__ constexpr int l2_col_lstr() {
  constexpr int A = plan2_a(L), B = L / A, E = smem_row_elems<C>();
  constexpr int base = A * (B + 1);
  constexpr int want = (E / TX) % E;
  return base + ((want - (base % E)) % E + E) % E;
}
// Rows per CTA of the row passes and threads per CTA.
// (thread counts are rounded up to whole warps; the extra threads idle in the strided loops)
__host__ __device__ constexpr int l2_rows(int NX) {
  return plan2_max(NX) == 0 ? 1 : (128 / plan2_max(NX) > 0 ? 128 / plan2_max(NX) : 1);
}
__host__ __device__ constexpr int l2_row_threads(int NX, int G) { return (G * plan2_max(NX) + 31) / 32 * 32; }
__host__ __device__ constexpr int l2_row_threads(int NX) { return l2_row_threads(NX, l2_rows(NX)); }
template <typename T> __host__ __device__ constexpr int l2_tx(int NY) { return 8; }
__host__ __device__ constexpr int l2_col_threads_tx(int NY, int TX) { return (TX * plan2_max(NY) + 31) / 32 * 32; }
template <typename T> __host__ __device__ constexpr int l2_col_threads(int NY) {
  return l2_col_threads_tx(NY, l2_tx<T>(NY));
}

// Transverse basis for the pass kernels.  FP64 is basis_at itself; FP32 takes 1/|k+G| and
// 1/|G| from the hardware reciprocal square root (≤ 2 ulp), which keeps the prologue and
// epilogue at two MUFU operations per pixel instead of two square roots and two divisions.
template <typename T> __device__ __forceinline__ Basis<T> basis_pass(T k, T gx, T gy) { return basis_at<T>(k, gx, gy); }
template <> __device__ __forceinline__ Basis<float> basis_pass<float>(float k, float gx, float gy) {
  Basis<float> b;
  const float p2 = gx * gx + gy * gy, m2 = p2 + k * k;
  const float im = rsqrtf(m2);
  b.imag = im;
  b.mag = m2 * im;
  if (p2 > 0.f) {
    const float ip = rsqrtf(p2);
    const float kim = k * ip * im;
    b.nx = gy * ip; b.ny = -gx * ip;
    b.mx = -gx * kim; b.my = -gy * kim; b.mz = -p2 * ip * im;
  } else {
    b.nx = 0.f; b.ny = 1.f;
    b.mx = (k >= 0.f) ? 1.f : -1.f; b.my = 0.f; b.mz = 0.f;
  }
  return b;
}

// Field value of the prologue at one pixel (three components).
template <typename T, int MODE>
__device__ __forceinline__ void prologue_at(const OpUnit<T>& U, const cplx<T>* __restrict__ H, size_t p, size_t N,
                                            int ix, int iy, int NX, T k, cplx<T>& d0, cplx<T>& d1, cplx<T>& d2) {
  using C = cplx<T>;
  if constexpr (MODE == RI_LOAD3) {
    d0 = H[p]; d1 = H[N + p]; d2 = H[2 * N + p];
  } else {
    const C h1 = H[2 * p], h2 = H[2 * p + 1];
    const Basis<T> b = basis_pass<T>(k, T(freq_index(ix, NX)) * U.inv_dx, T(freq_index(iy, U.Ny)) * U.inv_dy);
    if constexpr (MODE == RI_KXTC) {
      const T s_ = -b.mag;
      d0 = (h1 * b.nx - h2 * b.mx) * s_;
      d1 = (h1 * b.ny - h2 * b.my) * s_;
      d2 = h2 * (-b.mz * s_);
    } else if constexpr (MODE == RI_KXINV) {
      const T s_ = b.imag;
      d0 = (h1 * b.nx - h2 * b.mx) * s_;
      d1 = (h1 * b.ny - h2 * b.my) * s_;
      d2 = h2 * (-b.mz * s_);
    } else if constexpr (MODE == RI_HCART) {  // Cartesian H = h1 m̂ + h2 n̂
      d0 = h1 * b.mx + h2 * b.nx;
      d1 = h1 * b.my + h2 * b.ny;
      d2 = h1 * b.mz;
    } else {  // RI_ZXTC: ẑ × (h1 m̂ + h2 n̂)
      d0 = (h1 * b.my + h2 * b.ny) * T(-1);
      d1 = h1 * b.mx + h2 * b.nx;
      d2 = mk<C>(0, 0);
      if (U.zx_weight_gz) {  // the period derivative: each plane wave weighted by g_z/Λ
        const T wz = (T)(U.kz_shift * U.inv_dz);
        d0 = d0 * wz;
        d1 = d1 * wz;
      }
    }
  }
}

// ------------------------------------------------------------------------------------
// row_in.  Grid: (ceil(Ny/G), max columns, units); l2_row_threads(NX) threads.
template <typename T, int NX, int MODE, bool INV, int G = l2_rows(NX)>
__global__ void __launch_bounds__(l2_row_threads(NX, G)) k_row_in2(const OpUnit<T>* __restrict__ units,
                                                                  const cplx<T>* __restrict__ tw_g) {
  using C = cplx<T>;
  constexpr int A = plan2_a(NX), B = NX / A, NT = l2_row_threads(NX, G);
  constexpr int LS = l2_row_lstr<C, NX>();
  constexpr bool REG3 = sizeof(T) == 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* blk = reinterpret_cast<C*>(smem_raw);  // [3][G][LS]
  const OpUnit<T>& U = units[blockIdx.z];
  const int col = blockIdx.y;
  if (col >= unit_ncol(U)) return;
  const int Ny = U.Ny;
  const int row0 = blockIdx.x * G;
  if (row0 >= Ny) return;
  const size_t N = U.comp_stride ? (size_t)U.comp_stride : (size_t)NX * Ny;
  const T k = (T)(*U.k_dev - U.kz_shift);
  const C* __restrict__ H = U.in + (size_t)(col + unit_col0(U)) * U.in_cs;
  const C* tw1 = tw_g + NX;
  for (int q = threadIdx.x; q < G * B; q += NT) {
    const int r = q / B, n2 = q - r * B, iy = row0 + r;
    C* l0 = blk + (0 * G + r) * LS;
    C* l1 = blk + (1 * G + r) * LS;
    C* l2 = blk + (2 * G + r) * LS;
    if constexpr (REG3) {
      C v0[A], v1[A], v2[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) {
        const int ix = B * n1 + n2;
        if (iy < Ny) prologue_at<T, MODE>(U, H, ix + (size_t)NX * iy, N, ix, iy, NX, k, v0[n1], v1[n1], v2[n1]);
        else v0[n1] = v1[n1] = v2[n1] = mk<C>(0, 0);
      }
      l2_first<NX, INV>(v0, n2, l0, tw1);
      l2_first<NX, INV>(v1, n2, l1, tw1);
      l2_first<NX, INV>(v2, n2, l2, tw1);
    } else {
      // stage the three components in this thread's own column of the block
#pragma unroll 4
      for (int n1 = 0; n1 < A; ++n1) {
        const int ix = B * n1 + n2;
        C d0 = mk<C>(0, 0), d1 = d0, d2 = d0;
        if (iy < Ny) prologue_at<T, MODE>(U, H, ix + (size_t)NX * iy, N, ix, iy, NX, k, d0, d1, d2);
        l0[n1 * (B + 1) + n2] = d0;
        l1[n1 * (B + 1) + n2] = d1;
        l2[n1 * (B + 1) + n2] = d2;
      }
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C* lc = blk + (c * G + r) * LS;
        C v[A];
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) v[n1] = lc[n1 * (B + 1) + n2];
        l2_first<NX, INV>(v, n2, lc, tw1);
      }
    }
  }
  __syncthreads();
  C* __restrict__ D = U.scr + (size_t)col * U.scr_cs;
  for (int q = threadIdx.x; q < G * A; q += NT) {
    const int r = q / A, k1 = q - r * A, iy = row0 + r;
    if (iy >= Ny) continue;
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      C w[B];
      l2_second<NX, INV>(blk + (c * G + r) * LS, k1, w);
      C* Dc = D + c * N + (size_t)NX * iy + k1;
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) Dc[A * k2] = w[k2];
    }
  }
}

// Per-pixel step of the column pass on the three components.
template <typename T, int PW>
__device__ __forceinline__ void pointwise_at(const OpUnit<T>& U, size_t p, cplx<T>& a0, cplx<T>& a1, cplx<T>& a2) {
  const cplx<T> d0 = a0, d1 = a1, d2 = a2;
  if constexpr (PW == PW_EPS || PW == PW_EPS9) {
    T e[6];
    if constexpr (PW == PW_EPS) {
      load_eps<T>(U, p, e);
    } else {  // the reference's (3, 3, Nx, Ny) column-major layout, 9 entries per pixel
      const T* m = U.e9 + 9 * p;
      e[0] = m[0]; e[1] = m[4]; e[2] = m[8];
      e[3] = T(0.5) * (m[1] + m[3]); e[4] = T(0.5) * (m[2] + m[6]); e[5] = T(0.5) * (m[5] + m[7]);
    }
    a0 = d0 * e[0] + d1 * e[3] + d2 * e[4];
    a1 = d0 * e[3] + d1 * e[1] + d2 * e[5];
    a2 = d0 * e[4] + d1 * e[5] + d2 * e[2];
  } else if constexpr (PW == PW_EAVE) {
    const T w = U.eave[p];
    a0 = d0 * w; a1 = d1 * w; a2 = d2 * w;
  }
}

// ------------------------------------------------------------------------------------
// col.  Grid: (ceil(Nx/TX), max columns, units); l2_col_threads(NY) threads.
// (MINB: CTAs per SM the register budget is set for)
template <typename T, int NY, int S1, int PW, int S2, int TX = l2_tx<T>(NY),
          int MINB = sizeof(T) == 4 ? (384 / l2_col_threads_tx(NY, TX) > 1 ? 384 / l2_col_threads_tx(NY, TX) : 1) : 1>
__global__ void __launch_bounds__(l2_col_threads_tx(NY, TX), MINB)
    k_col2(const OpUnit<T>* __restrict__ units, const cplx<T>* __restrict__ tw_g) {
  using C = cplx<T>;
  constexpr int A = plan2_a(NY), B = NY / A, NT = l2_col_threads_tx(NY, TX);
  constexpr int LS = l2_col_lstr<C, NY, TX>();
  constexpr bool REG3 = sizeof(T) == 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* blk = reinterpret_cast<C*>(smem_raw);  // [3][TX][LS]
  // vectors in the reverse of the row passes' order: the first tiles read are the ones
  // row_in wrote last (still in L2), and row_out then starts on the ones written last here
  const OpUnit<T>& U = units[gridDim.z - 1 - blockIdx.z];
  const int col = gridDim.y - 1 - blockIdx.y;
  if (col >= unit_ncol(U)) return;
  const int Nx = U.Nx;
  const int ix0 = blockIdx.x * TX;
  if (ix0 >= Nx) return;
  const size_t N = U.comp_stride ? (size_t)U.comp_stride : (size_t)Nx * NY;
  const C* tw1 = tw_g + NY;
  const C* tw3 = tw_g + 2 * NY;
  C* __restrict__ D = U.scr + (size_t)col * U.scr_cs;
  if constexpr (S1 != CS_NONE) {
    for (int q = threadIdx.x; q < TX * B; q += NT) {
      const int t = q % TX, n2 = q / TX, ix = ix0 + t;
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C v[A];
        const C* Dc = D + c * N + (size_t)n2 * Nx + ix;
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) v[n1] = (ix < Nx) ? Dc[(size_t)(B * n1) * Nx] : mk<C>(0, 0);
        l2_first<NY, S1 == CS_INV>(v, n2, blk + (c * TX + t) * LS, tw1);
      }
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < TX * A; q += NT) {
    const int t = q % TX, k1 = q / TX, ix = ix0 + t;
    C* l0 = blk + (0 * TX + t) * LS + k1 * (B + 1);
    C* l1 = blk + (1 * TX + t) * LS + k1 * (B + 1);
    C* l2 = blk + (2 * TX + t) * LS + k1 * (B + 1);
    if constexpr (REG3) {
      C V0[B], V1[B], V2[B];
      if constexpr (S1 != CS_NONE) {
        l2_second<NY, S1 == CS_INV>(blk + (0 * TX + t) * LS, k1, V0);
        l2_second<NY, S1 == CS_INV>(blk + (1 * TX + t) * LS, k1, V1);
        l2_second<NY, S1 == CS_INV>(blk + (2 * TX + t) * LS, k1, V2);
      } else {
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) {
          const size_t p = (size_t)(k1 + A * k2) * Nx + ix;
          const bool ok = ix < Nx;
          V0[k2] = ok ? D[p] : mk<C>(0, 0);
          V1[k2] = ok ? D[N + p] : mk<C>(0, 0);
          V2[k2] = ok ? D[2 * N + p] : mk<C>(0, 0);
        }
      }
      if constexpr (PW != PW_NONE) {
        if (ix < Nx) {
#pragma unroll
          for (int k2 = 0; k2 < B; ++k2) pointwise_at<T, PW>(U, (size_t)(k1 + A * k2) * Nx + ix, V0[k2], V1[k2], V2[k2]);
        }
      }
      if constexpr (S2 != CS_NONE) {
        l2_rfirst<NY, S2 == CS_INV>(V0, k1, blk + (0 * TX + t) * LS, tw3);
        l2_rfirst<NY, S2 == CS_INV>(V1, k1, blk + (1 * TX + t) * LS, tw3);
        l2_rfirst<NY, S2 == CS_INV>(V2, k1, blk + (2 * TX + t) * LS, tw3);
      } else if (ix < Nx) {
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) {
          const size_t p = (size_t)(k1 + A * k2) * Nx + ix;
          D[p] = V0[k2]; D[N + p] = V1[k2]; D[2 * N + p] = V2[k2];
        }
      }
    } else {
      // FP64: results of step 2 go back to this thread's own row k1 of each block
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C* lc = c == 0 ? l0 : (c == 1 ? l1 : l2);
        C w[B];
        if constexpr (S1 != CS_NONE) {
          l2_second<NY, S1 == CS_INV>(blk + (c * TX + t) * LS, k1, w);
        } else {
#pragma unroll
          for (int k2 = 0; k2 < B; ++k2)
            w[k2] = (ix < Nx) ? D[c * N + (size_t)(k1 + A * k2) * Nx + ix] : mk<C>(0, 0);
        }
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) lc[k2] = w[k2];
      }
      if constexpr (PW != PW_NONE) {
        if (ix < Nx) {
#pragma unroll 2
          for (int k2 = 0; k2 < B; ++k2) {
            C a0 = l0[k2], a1 = l1[k2], a2 = l2[k2];
            pointwise_at<T, PW>(U, (size_t)(k1 + A * k2) * Nx + ix, a0, a1, a2);
            l0[k2] = a0; l1[k2] = a1; l2[k2] = a2;
          }
        }
      }
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C* lc = c == 0 ? l0 : (c == 1 ? l1 : l2);
        C w[B];
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) w[k2] = lc[k2];
        if constexpr (S2 != CS_NONE) {
          l2_rfirst<NY, S2 == CS_INV>(w, k1, blk + (c * TX + t) * LS, tw3);
        } else if (ix < Nx) {
#pragma unroll
          for (int k2 = 0; k2 < B; ++k2) D[c * N + (size_t)(k1 + A * k2) * Nx + ix] = w[k2];
        }
      }
    }
  }
  if constexpr (S2 != CS_NONE) {
    __syncthreads();
    for (int q = threadIdx.x; q < TX * B; q += NT) {
      const int t = q % TX, m2 = q / TX, ix = ix0 + t;
      if (ix >= Nx) continue;
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C v[A];
        l2_rsecond<NY, S2 == CS_INV>(blk + (c * TX + t) * LS, m2, v);
        C* Dc = D + c * N + (size_t)m2 * Nx + ix;
#pragma unroll
        for (int m1 = 0; m1 < A; ++m1) Dc[(size_t)(B * m1) * Nx] = v[m1];
      }
    }
  }
}

// ------------------------------------------------------------------------------------
// row_out.  Grid: (ceil(Ny/G), max columns, units); l2_row_threads(NX) threads.
template <typename T, int NX, int MODE, bool INV, int G = l2_rows(NX)>
__global__ void __launch_bounds__(l2_row_threads(NX, G)) k_row_out2(const OpUnit<T>* __restrict__ units,
                                                                   const cplx<T>* __restrict__ tw_g) {
  using C = cplx<T>;
  constexpr int A = plan2_a(NX), B = NX / A, NT = l2_row_threads(NX, G);
  constexpr int LS = l2_row_lstr<C, NX>();
  constexpr bool REG3 = sizeof(T) == 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* blk = reinterpret_cast<C*>(smem_raw);  // [3][G][LS]
  __shared__ double red[2][NT / 32 + 1];
  const OpUnit<T>& U = units[blockIdx.z];
  const int col = blockIdx.y;
  if (col >= unit_ncol(U)) return;
  const int Ny = U.Ny;
  const int row0 = blockIdx.x * G;
  if (row0 >= Ny) return;
  const size_t N = U.comp_stride ? (size_t)U.comp_stride : (size_t)NX * Ny;
  const C* tw3 = tw_g + 2 * NX;
  const C* __restrict__ D = U.scr + (size_t)col * U.scr_cs;
  for (int q = threadIdx.x; q < G * A; q += NT) {
    const int r = q / A, k1 = q - r * A, iy = row0 + r;
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      C w[B];
      const C* Dc = D + c * N + (size_t)NX * iy + k1;
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) w[k2] = (iy < Ny) ? Dc[A * k2] : mk<C>(0, 0);
      l2_rfirst<NX, INV>(w, k1, blk + (c * G + r) * LS, tw3);
    }
  }
  __syncthreads();
  const T k = (T)(*U.k_dev - U.kz_shift);
  const T sN = T(1) / T(N);
  const int c0 = unit_col0(U);
  C* __restrict__ O = U.out + (size_t)(col + c0) * U.out_cs;
  const C* __restrict__ Hin = U.in + (size_t)(col + c0) * U.in_cs;
  double accr = 0.0, acci = 0.0;
  auto epilogue = [&](int ix, int iy, const C e0, const C e1, const C e2) {
    const size_t p = ix + (size_t)NX * iy;
    if constexpr (MODE == RO_STORE3) {
      O[p] = e0; O[N + p] = e1; O[2 * N + p] = e2;
    } else {
      const Basis<T> b = basis_pass<T>(k, T(freq_index(ix, NX)) * U.inv_dx, T(freq_index(iy, Ny)) * U.inv_dy);
      const C en = e0 * b.nx + e1 * b.ny;              // e·n̂ (n̂_z = 0)
      const C em = e0 * b.mx + e1 * b.my + e2 * b.mz;  // e·m̂
      C h1, h2;
      if constexpr (MODE == RO_KXINVCT) {
        const T sc = sN * b.imag;
        h1 = en * sc; h2 = em * (-sc);
      } else {
        const T sc = b.mag * sN;
        h1 = en * (-sc); h2 = em * sc;
      }
      if constexpr (MODE == RO_KXCT_DOT) {
        const C g1 = Hin[2 * p], g2 = Hin[2 * p + 1];
        // ⟨H_in, out⟩ = Σ conj(H_in)·out
        accr += (double)g1.x * h1.x + (double)g1.y * h1.y + (double)g2.x * h2.x + (double)g2.y * h2.y;
        acci += (double)g1.x * h1.y - (double)g1.y * h1.x + (double)g2.x * h2.y - (double)g2.y * h2.x;
      } else {
        O[2 * p] = h1; O[2 * p + 1] = h2;
      }
    }
  };
  for (int q = threadIdx.x; q < G * B; q += NT) {
    const int r = q / B, m2 = q - r * B, iy = row0 + r;
    if (iy >= Ny) continue;
    if constexpr (REG3) {
      C y0[A], y1[A], y2[A];
      l2_rsecond<NX, INV>(blk + (0 * G + r) * LS, m2, y0);
      l2_rsecond<NX, INV>(blk + (1 * G + r) * LS, m2, y1);
      l2_rsecond<NX, INV>(blk + (2 * G + r) * LS, m2, y2);
#pragma unroll
      for (int m1 = 0; m1 < A; ++m1) epilogue(m2 + B * m1, iy, y0[m1], y1[m1], y2[m1]);
    } else {
      // FP64: each transformed component goes back to this thread's own column m2
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C* lc = blk + (c * G + r) * LS;
        C v[A];
        l2_rsecond<NX, INV>(lc, m2, v);
#pragma unroll
        for (int m1 = 0; m1 < A; ++m1) lc[m1 * (B + 1) + m2] = v[m1];
      }
      const C* l0 = blk + (0 * G + r) * LS;
      const C* l1 = blk + (1 * G + r) * LS;
      const C* l2 = blk + (2 * G + r) * LS;
#pragma unroll 4
      for (int m1 = 0; m1 < A; ++m1) {
        const int o = m1 * (B + 1) + m2;
        epilogue(m2 + B * m1, iy, l0[o], l1[o], l2[o]);
      }
    }
  }
  if constexpr (MODE == RO_KXCT_DOT) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      accr += __shfl_xor_sync(0xffffffffu, accr, o);
      acci += __shfl_xor_sync(0xffffffffu, acci, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = accr; red[1][w] = acci; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double sr = 0, si = 0;
      for (int i = 0; i < (NT + 31) / 32; ++i) { sr += red[0][i]; si += red[1][i]; }
      double* P = U.partial + 2 * ((size_t)col * U.part_stride + blockIdx.x);
      P[0] = sr; P[1] = si;
    }
  }
}

}  // namespace omb
