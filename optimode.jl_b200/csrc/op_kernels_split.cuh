// Component-parallel operator passes for two-level lines (≤ 256 points): FP32 row and
// column passes (tile variants) and the FP64 row passes.
//
// The same transforms, modes, layouts and results as k_row_in2 / k_col2 / k_row_out2
// (op_kernels_2l.cuh), with one thread per (line slot, field component) instead of one per
// line slot.  A thread then holds the A or B points of ONE component (≈40 live registers
// instead of the 126–168 that three register-resident components need), so three times as
// many warps share an SM's registers and hide the latency of the global loads that the
// one-thread-per-slot passes stall on (long-scoreboard).  The three components of a pixel
// meet in shared memory where they must: the prologue (basis + curl, computed once per pixel
// and written in the step-1 input layout), the per-pixel ε⁻¹ contraction of the column pass
// and the curl epilogue of row_out.  Every transform is done in place in the thread's own
// row or column of the padded A×(B+1) block, so the shared-memory footprint and its
// bank-conflict-free strides are those of the two-level passes.
#pragma once

#include "op_kernels_2l.cuh"

namespace omb {

__host__ __device__ constexpr int sp_row_threads(int NX, int G) { return (3 * G * plan2_max(NX) + 31) / 32 * 32; }
__host__ __device__ constexpr int sp_col_threads(int NY, int TX) { return (3 * TX * plan2_max(NY) + 31) / 32 * 32; }
// CTAs per SM the register budget is set for (the 52 KB FP32 block allows four; an FP64 row
// block is twice as large and its A or B complex doubles need ≈80 registers)
__host__ __device__ constexpr int sp_min_blocks(int nt) { return nt <= 384 ? 3 : (nt <= 512 ? 2 : 1); }
template <typename T> __host__ __device__ constexpr int sp_row_min_blocks(int nt) {
  return sizeof(T) == 4 ? sp_min_blocks(nt) : (nt <= 512 ? 2 : 1);
}

// ------------------------------------------------------------------------------------
// row_in.  Grid: (ceil(Ny/G), max columns, units); sp_row_threads(NX, G) threads.
template <typename T, int NX, int MODE, bool INV, int G>
__global__ void __launch_bounds__(sp_row_threads(NX, G), sp_row_min_blocks<T>(sp_row_threads(NX, G)))
    k_row_in_sp(const OpUnit<T>* __restrict__ units, const cplx<T>* __restrict__ tw_g) {
  using C = cplx<T>;
  constexpr int A = plan2_a(NX), B = NX / A, NT = sp_row_threads(NX, G);
  constexpr int LS = l2_row_lstr<C, NX>();
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
  // prologue, one thread per pixel (x fastest: coalesced loads of H), into the step-1 layout
  // x[B·n1 + n2] → block position n1·(B+1) + n2
  for (int q = threadIdx.x; q < G * NX; q += NT) {
    const int r = q / NX, ix = q - r * NX, iy = row0 + r;
    C d0 = mk<C>(0, 0), d1 = d0, d2 = d0;
    if (iy < Ny) prologue_at<T, MODE>(U, H, ix + (size_t)NX * iy, N, ix, iy, NX, k, d0, d1, d2);
    const int o = (ix / B) * (B + 1) + (ix % B);
    blk[(0 * G + r) * LS + o] = d0;
    blk[(1 * G + r) * LS + o] = d1;
    blk[(2 * G + r) * LS + o] = d2;
  }
  __syncthreads();
  const C* tw1 = tw_g + NX;
  // step 1 in place: thread (c, r, n2) owns column n2 of block (c, r)
  for (int q = threadIdx.x; q < 3 * G * B; q += NT) {
    const int cr = q / B, n2 = q - cr * B;
    C* line = blk + cr * LS;
    C v[A];
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1) v[n1] = line[n1 * (B + 1) + n2];
    l2_first<NX, INV>(v, n2, line, tw1);
  }
  __syncthreads();
  // step 2: thread (c, r, k1) → X[k1 + A·k2] straight to the planar scratch
  C* __restrict__ D = U.scr + (size_t)col * U.scr_cs;
  for (int q = threadIdx.x; q < 3 * G * A; q += NT) {
    const int cr = q / A, k1 = q - cr * A, c = cr / G, r = cr - c * G, iy = row0 + r;
    if (iy >= Ny) continue;
    C w[B];
    l2_second<NX, INV>(blk + cr * LS, k1, w);
    C* Dc = D + c * N + (size_t)NX * iy + k1;
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) Dc[A * k2] = w[k2];
  }
}

// ------------------------------------------------------------------------------------
// col.  Grid: (ceil(Nx/TX), max columns, units); sp_col_threads(NY, TX) threads.
// (MINB: CTAs per SM the register budget is set for; 3 leaves ≈56 registers a thread, 2 ≈85)
template <int NY, int S1, int PW, int S2, int TX, int MINB = sp_min_blocks(sp_col_threads(NY, TX))>
__global__ void __launch_bounds__(sp_col_threads(NY, TX), MINB)
    k_col_sp(const OpUnit<float>* __restrict__ units, const float2* __restrict__ tw_g) {
  using T = float;
  using C = cplx<float>;
  constexpr int A = plan2_a(NY), B = NY / A, NT = sp_col_threads(NY, TX);
  constexpr int LS = l2_col_lstr<C, NY, TX>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* blk = reinterpret_cast<C*>(smem_raw);  // [3][TX][LS]
  // vectors in the reverse of the row passes' order (the tiles row_in wrote last are in L2)
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
  // step 1: thread (c, n2, t), t fastest (coalesced row segments of TX columns)
  if constexpr (S1 != CS_NONE) {
    for (int q = threadIdx.x; q < 3 * TX * B; q += NT) {
      const int c = q / (TX * B), rq = q - c * (TX * B), t = rq % TX, n2 = rq / TX, ix = ix0 + t;
      C v[A];
      const C* Dc = D + c * N + (size_t)n2 * Nx + ix;
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) v[n1] = (ix < Nx) ? Dc[(size_t)(B * n1) * Nx] : mk<C>(0, 0);
      l2_first<NY, S1 == CS_INV>(v, n2, blk + (c * TX + t) * LS, tw1);
    }
    __syncthreads();
  }
  // step 2: thread (c, k1, t); the B outputs go back to row k1 (or on to reverse step 1)
  for (int q = threadIdx.x; q < 3 * TX * A; q += NT) {
    const int c = q / (TX * A), rq = q - c * (TX * A), t = rq % TX, k1 = rq / TX, ix = ix0 + t;
    C* line = blk + (c * TX + t) * LS;
    C w[B];
    if constexpr (S1 != CS_NONE) {
      l2_second<NY, S1 == CS_INV>(line, k1, w);
    } else {
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2)
        w[k2] = (ix < Nx) ? D[c * N + (size_t)(k1 + A * k2) * Nx + ix] : mk<C>(0, 0);
    }
    if constexpr (PW != PW_NONE) {
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) line[k1 * (B + 1) + k2] = w[k2];
    } else if constexpr (S2 != CS_NONE) {
      l2_rfirst<NY, S2 == CS_INV>(w, k1, line, tw3);
    } else if (ix < Nx) {
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) D[c * N + (size_t)(k1 + A * k2) * Nx + ix] = w[k2];
    }
  }
  if constexpr (PW != PW_NONE) {
    __syncthreads();
    // per-pixel step, one thread per pixel (t fastest: coalesced ε⁻¹ loads)
    for (int q = threadIdx.x; q < TX * NY; q += NT) {
      const int t = q % TX, rq = q / TX, k2 = rq % B, k1 = rq / B, ix = ix0 + t;
      if (ix >= Nx) continue;
      const int o = t * LS + k1 * (B + 1) + k2;
      C a0 = blk[o], a1 = blk[TX * LS + o], a2 = blk[2 * TX * LS + o];
      pointwise_at<T, PW>(U, (size_t)(k1 + A * k2) * Nx + ix, a0, a1, a2);
      blk[o] = a0;
      blk[TX * LS + o] = a1;
      blk[2 * TX * LS + o] = a2;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 3 * TX * A; q += NT) {
      const int c = q / (TX * A), rq = q - c * (TX * A), t = rq % TX, k1 = rq / TX, ix = ix0 + t;
      C* line = blk + (c * TX + t) * LS;
      C w[B];
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) w[k2] = line[k1 * (B + 1) + k2];
      if constexpr (S2 != CS_NONE) {
        l2_rfirst<NY, S2 == CS_INV>(w, k1, line, tw3);
      } else if (ix < Nx) {
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) D[c * N + (size_t)(k1 + A * k2) * Nx + ix] = w[k2];
      }
    }
  }
  if constexpr (S2 != CS_NONE) {
    __syncthreads();
    for (int q = threadIdx.x; q < 3 * TX * B; q += NT) {
      const int c = q / (TX * B), rq = q - c * (TX * B), t = rq % TX, m2 = rq / TX, ix = ix0 + t;
      if (ix >= Nx) continue;
      C v[A];
      l2_rsecond<NY, S2 == CS_INV>(blk + (c * TX + t) * LS, m2, v);
      C* Dc = D + c * N + (size_t)m2 * Nx + ix;
#pragma unroll
      for (int m1 = 0; m1 < A; ++m1) Dc[(size_t)(B * m1) * Nx] = v[m1];
    }
  }
}

// ------------------------------------------------------------------------------------
// row_out.  Grid: (ceil(Ny/G), max columns, units); sp_row_threads(NX, G) threads.
template <typename T, int NX, int MODE, bool INV, int G>
__global__ void __launch_bounds__(sp_row_threads(NX, G), sp_row_min_blocks<T>(sp_row_threads(NX, G)))
    k_row_out_sp(const OpUnit<T>* __restrict__ units, const cplx<T>* __restrict__ tw_g) {
  using C = cplx<T>;
  constexpr int A = plan2_a(NX), B = NX / A, NT = sp_row_threads(NX, G);
  constexpr int LS = l2_row_lstr<C, NX>();
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
  // reverse step 1: thread (c, r, k1) reads V[k1 + A·k2] of its component (coalesced in k1)
  for (int q = threadIdx.x; q < 3 * G * A; q += NT) {
    const int cr = q / A, k1 = q - cr * A, c = cr / G, r = cr - c * G, iy = row0 + r;
    C w[B];
    const C* Dc = D + c * N + (size_t)NX * iy + k1;
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) w[k2] = (iy < Ny) ? Dc[A * k2] : mk<C>(0, 0);
    l2_rfirst<NX, INV>(w, k1, blk + cr * LS, tw3);
  }
  __syncthreads();
  // reverse step 2 in place: thread (c, r, m2) owns column m2 of block (c, r)
  for (int q = threadIdx.x; q < 3 * G * B; q += NT) {
    const int cr = q / B, m2 = q - cr * B;
    C* line = blk + cr * LS;
    C v[A];
    l2_rsecond<NX, INV>(line, m2, v);
#pragma unroll
    for (int m1 = 0; m1 < A; ++m1) line[m1 * (B + 1) + m2] = v[m1];
  }
  __syncthreads();
  const T k = (T)(*U.k_dev - U.kz_shift);
  const T sN = T(1) / T(N);
  const int c0 = unit_col0(U);
  C* __restrict__ O = U.out + (size_t)(col + c0) * U.out_cs;
  const C* __restrict__ Hin = U.in + (size_t)(col + c0) * U.in_cs;
  double accr = 0.0, acci = 0.0;
  // epilogue, one thread per pixel (x fastest: coalesced stores)
  for (int q = threadIdx.x; q < G * NX; q += NT) {
    const int r = q / NX, ix = q - r * NX, iy = row0 + r;
    if (iy >= Ny) continue;
    const int o = (ix % B) + (ix / B) * (B + 1);
    const C e0 = blk[(0 * G + r) * LS + o], e1 = blk[(1 * G + r) * LS + o], e2 = blk[(2 * G + r) * LS + o];
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
        accr += (double)g1.x * h1.x + (double)g1.y * h1.y + (double)g2.x * h2.x + (double)g2.y * h2.y;
        acci += (double)g1.x * h1.y - (double)g1.y * h1.x + (double)g2.x * h2.y - (double)g2.y * h2.x;
      } else {
        O[2 * p] = h1; O[2 * p + 1] = h2;
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
      for (int i = 0; i < NT / 32; ++i) { sr += red[0][i]; si += red[1][i]; }
      double* P = U.partial + 2 * ((size_t)col * U.part_stride + blockIdx.x);
      P[0] = sr; P[1] = si;
    }
  }
}

}  // namespace omb
