// Fused plane-wave Helmholtz operator passes (sm_100a).
//
// One operator application M̂(k)H = kx_ct · (1/N)·bfft · ε⁻¹ · fft · kx_tc H
// (reference: _M!, lib/MaxwellEigenmodes/src/maxwell.jl:471-481) runs as three passes:
//
//   row_in  : per grid row, regenerate (mag, m̂, n̂) from (k, gx, gy) in registers, form
//             the 3-component field (kx_tc, kxinv_tc or zx_tc), FFT along x in shared
//             memory, store planar to the scratch field (stays in L2 between passes);
//   col     : per tile of TX adjacent columns, FFT along y, per-pixel 3×3 ε⁻¹ contraction
//             (6 unique entries: float4 + float2 loads) or ε_ave scaling, FFT back along y,
//             in place;
//   row_out : per grid row, FFT back along x, then the curl epilogue (kx_ct or kxinv_ct)
//             that writes the 2-component output, optionally reducing ⟨H_in, out⟩.
//
// The same passes with other prologue/epilogue choices give the MPB-style preconditioner
// (_P!, maxwell.jl:459-469), ⟨H|∂M̂/∂k|H⟩ (HMₖH, maxwell.jl:267-269), E = ε⁻¹·fft(kx_tc H)
// (E⃗, fields.jl:194-210) and the adjoint's _H2d!/_d2ẽ! (fields.jl:81-93).
//
// Layouts: H is the reference's column-major (2, Nx, Ny) complex vector (component
// fastest); scratch fields are planar [c][iy][ix]; ε⁻¹ is stored as 6 unique entries
// (xx, yy, zz, xy) + (xz, yz) per pixel.
#pragma once

#include "fft_smem.cuh"

namespace omb {

template <typename T> struct OpUnit {
  const cplx<T>* in;      // 2-component input block (or planar 3-component for RI_LOAD3)
  cplx<T>* out;           // 2-component output block (or planar 3-component for RO_STORE3)
  cplx<T>* scr;           // planar 3·N scratch per column
  const float4* e32a;     // (xx, yy, zz, xy) FP32
  const float2* e32b;     // (xz, yz)         FP32
  const double2* e64;     // 3 double2 per pixel: (xx,yy), (zz,xy), (xz,yz)
  const T* eave;          // 3/tr(ε⁻¹) per pixel
  const T* e9;            // ε⁻¹ in the reference's (3, 3, Nx, Ny) layout (PW_EPS9 only)
  const double* k_dev;    // wavevector magnitude (device, so the solver can update it)
  double* partial;        // per-(column, row-block) partial sums for RO_KXCT_DOT
  const int* ncol_dev;    // optional device-side column count
  const int* col0_dev;    // optional device-side first column of in/out (scratch is not offset)
  long long in_cs, out_cs, scr_cs;  // column strides in complex elements
  int Nx, Ny, ncol;
  int part_stride;        // partial sums per column (≥ gridDim.x of row_out)
  T inv_dx, inv_dy;
  // z-periodic cells: one unit per z-slab (or per z-line set) of a 3D field
  long long comp_stride;  // component stride of planar 3-component fields (0: Nx·Ny of the pass)
  double kz_shift;        // g_z of the slab: the passes see k − g_z (w = k ẑ − G)
  double inv_dz;          // 1/Λ of a z-periodic cell (0 for a 2D cell)
  int zx_weight_gz;       // RI_ZXTC only: weight ẑ×H by g_z/Λ (⟨H|∂M̂/∂Λ|H⟩, the period derivative)
};

enum RowIn : int { RI_KXTC = 0, RI_KXINV = 1, RI_ZXTC = 2, RI_LOAD3 = 3, RI_HCART = 4 };
enum RowOut : int { RO_KXCT = 0, RO_KXINVCT = 1, RO_STORE3 = 2, RO_KXCT_DOT = 3 };
enum ColStep : int { CS_NONE = 0, CS_FWD = 1, CS_INV = 2 };
enum ColPw : int { PW_NONE = 0, PW_EPS = 1, PW_EAVE = 2, PW_EPS9 = 3 };

template <typename T> __device__ __forceinline__ void load_eps(const OpUnit<T>& U, size_t p, T e[6]);
template <> __device__ __forceinline__ void load_eps<float>(const OpUnit<float>& U, size_t p, float e[6]) {
  float4 a = __ldg(U.e32a + p);
  float2 b = __ldg(U.e32b + p);
  e[0] = a.x; e[1] = a.y; e[2] = a.z; e[3] = a.w; e[4] = b.x; e[5] = b.y;
}
template <> __device__ __forceinline__ void load_eps<double>(const OpUnit<double>& U, size_t p, double e[6]) {
  double2 a = __ldg(U.e64 + 3 * p), b = __ldg(U.e64 + 3 * p + 1), c = __ldg(U.e64 + 3 * p + 2);
  e[0] = a.x; e[1] = a.y; e[2] = b.x; e[3] = b.y; e[4] = c.x; e[5] = c.y;
}

template <typename T> __device__ __forceinline__ int unit_ncol(const OpUnit<T>& U) {
  return U.ncol_dev ? *U.ncol_dev : U.ncol;
}
template <typename T> __device__ __forceinline__ int unit_col0(const OpUnit<T>& U) {
  return U.col0_dev ? *U.col0_dev : 0;
}

template <typename C> __device__ __forceinline__ void load_tw(C* tw, const C* tw_g, int L) {
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = tw_g[i];
}

// ------------------------------------------------------------------------------------
// row_in: prologue + FFT along x.  Grid: (ceil(Ny/ROWS), max columns, units).
template <typename T, int NX, int ROWS, int NT, int MODE, bool INV>
__global__ void __launch_bounds__(NT) k_row_in(const OpUnit<T>* __restrict__ units,
                                               const cplx<T>* __restrict__ tw_g) {
  using C = cplx<T>;
  constexpr int LS = NX + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* s = tw + NX;
  const OpUnit<T>& U = units[blockIdx.z];
  const int col = blockIdx.y;
  if (col >= unit_ncol(U)) return;
  const int Ny = U.Ny;
  const int row0 = blockIdx.x * ROWS;
  if (row0 >= Ny) return;
  const size_t N = U.comp_stride ? (size_t)U.comp_stride : (size_t)NX * Ny;
  load_tw(tw, tw_g, NX);
  const T k = (T)(*U.k_dev - U.kz_shift);
  const C* __restrict__ H = U.in + (size_t)(col + unit_col0(U)) * U.in_cs;
#pragma unroll
  for (int q = threadIdx.x; q < ROWS * NX; q += NT) {
    const int r = q / NX, ix = q - r * NX, iy = row0 + r;
    C d0 = mk<C>(0, 0), d1 = d0, d2 = d0;
    if (iy < Ny) {
      const size_t p = ix + (size_t)NX * iy;
      if constexpr (MODE == RI_LOAD3) {
        d0 = H[p]; d1 = H[N + p]; d2 = H[2 * N + p];
      } else {
        C h1 = H[2 * p], h2 = H[2 * p + 1];
        const Basis<T> b = basis_at<T>(k, T(freq_index(ix, NX)) * U.inv_dx, T(freq_index(iy, Ny)) * U.inv_dy);
        if constexpr (MODE == RI_KXTC) {
          const T s_ = -b.mag;
          d0 = (h1 * b.nx - h2 * b.mx) * s_;
          d1 = (h1 * b.ny - h2 * b.my) * s_;
          d2 = h2 * (-b.mz * s_);
        } else if constexpr (MODE == RI_KXINV) {
          const T s_ = T(1) / b.mag;
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
          if (U.zx_weight_gz) {
            const T wz = (T)(U.kz_shift * U.inv_dz);
            d0 = d0 * wz;
            d1 = d1 * wz;
          }
        }
      }
    }
    s[(0 * ROWS + r) * LS + ix] = d0;
    s[(1 * ROWS + r) * LS + ix] = d1;
    s[(2 * ROWS + r) * LS + ix] = d2;
  }
  __syncthreads();
  fft_lines<C, NX, INV, 3 * ROWS, NT>(s, LS, tw);
  C* __restrict__ D = U.scr + (size_t)col * U.scr_cs;
#pragma unroll
  for (int q = threadIdx.x; q < ROWS * NX; q += NT) {
    const int r = q / NX, ix = q - r * NX, iy = row0 + r;
    if (iy < Ny) {
      const size_t p = ix + (size_t)NX * iy;
#pragma unroll
      for (int c = 0; c < 3; ++c) D[c * N + p] = s[(c * ROWS + r) * LS + ix];
    }
  }
}

// ------------------------------------------------------------------------------------
// col: FFT along y, pointwise, FFT along y (each optional), in place on the scratch.
// Grid: (ceil(Nx/TX), max columns, units).
template <typename T, int NY, int TX, int NT, int S1, int PW, int S2>
__global__ void __launch_bounds__(NT) k_col(const OpUnit<T>* __restrict__ units,
                                            const cplx<T>* __restrict__ tw_g) {
  using C = cplx<T>;
  constexpr int LS = NY + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* s = tw + NY;
  const OpUnit<T>& U = units[blockIdx.z];
  const int col = blockIdx.y;
  if (col >= unit_ncol(U)) return;
  const int Nx = U.Nx;
  const int ix0 = blockIdx.x * TX;
  if (ix0 >= Nx) return;
  const size_t N = U.comp_stride ? (size_t)U.comp_stride : (size_t)Nx * NY;
  load_tw(tw, tw_g, NY);
  C* __restrict__ D = U.scr + (size_t)col * U.scr_cs;
#pragma unroll
  for (int q = threadIdx.x; q < 3 * NY * TX; q += NT) {
    const int t = q % TX, rest = q / TX, iy = rest % NY, c = rest / NY, ix = ix0 + t;
    s[(c * TX + t) * LS + iy] = (ix < Nx) ? D[c * N + (size_t)iy * Nx + ix] : mk<C>(0, 0);
  }
  __syncthreads();
  if constexpr (S1 != CS_NONE) fft_lines<C, NY, S1 == CS_INV, 3 * TX, NT>(s, LS, tw);
  if constexpr (PW != PW_NONE) {
#pragma unroll
    for (int q = threadIdx.x; q < TX * NY; q += NT) {
      const int t = q % TX, iy = q / TX, ix = ix0 + t;
      if (ix < Nx) {
        const size_t p = ix + (size_t)Nx * iy;
        C* a0 = &s[(0 * TX + t) * LS + iy];
        C* a1 = &s[(1 * TX + t) * LS + iy];
        C* a2 = &s[(2 * TX + t) * LS + iy];
        const C d0 = *a0, d1 = *a1, d2 = *a2;
        if constexpr (PW == PW_EPS || PW == PW_EPS9) {
          T e[6];
          if constexpr (PW == PW_EPS) {
            load_eps<T>(U, p, e);
          } else {  // the reference's (3, 3, Nx, Ny) column-major layout, 9 entries per pixel
            const T* m = U.e9 + 9 * p;
            e[0] = m[0]; e[1] = m[4]; e[2] = m[8];
            e[3] = T(0.5) * (m[1] + m[3]); e[4] = T(0.5) * (m[2] + m[6]); e[5] = T(0.5) * (m[5] + m[7]);
          }
          // symmetric ε⁻¹ = [[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]]
          *a0 = d0 * e[0] + d1 * e[3] + d2 * e[4];
          *a1 = d0 * e[3] + d1 * e[1] + d2 * e[5];
          *a2 = d0 * e[4] + d1 * e[5] + d2 * e[2];
        } else {
          const T w = U.eave[p];
          *a0 = d0 * w; *a1 = d1 * w; *a2 = d2 * w;
        }
      }
    }
    __syncthreads();
  }
  if constexpr (S2 != CS_NONE) fft_lines<C, NY, S2 == CS_INV, 3 * TX, NT>(s, LS, tw);
#pragma unroll
  for (int q = threadIdx.x; q < 3 * NY * TX; q += NT) {
    const int t = q % TX, rest = q / TX, iy = rest % NY, c = rest / NY, ix = ix0 + t;
    if (ix < Nx) D[c * N + (size_t)iy * Nx + ix] = s[(c * TX + t) * LS + iy];
  }
}

// ------------------------------------------------------------------------------------
// row_out: FFT along x + epilogue.  Grid: (ceil(Ny/ROWS), max columns, units).
template <typename T, int NX, int ROWS, int NT, int MODE, bool INV>
__global__ void __launch_bounds__(NT) k_row_out(const OpUnit<T>* __restrict__ units,
                                                const cplx<T>* __restrict__ tw_g) {
  using C = cplx<T>;
  constexpr int LS = NX + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* s = tw + NX;
  __shared__ double red[2][NT / 32];
  const OpUnit<T>& U = units[blockIdx.z];
  const int col = blockIdx.y;
  if (col >= unit_ncol(U)) return;
  const int Ny = U.Ny;
  const int row0 = blockIdx.x * ROWS;
  if (row0 >= Ny) return;
  const size_t N = U.comp_stride ? (size_t)U.comp_stride : (size_t)NX * Ny;
  load_tw(tw, tw_g, NX);
  const C* __restrict__ D = U.scr + (size_t)col * U.scr_cs;
#pragma unroll
  for (int q = threadIdx.x; q < ROWS * NX; q += NT) {
    const int r = q / NX, ix = q - r * NX, iy = row0 + r;
    const bool ok = iy < Ny;
    const size_t p = ix + (size_t)NX * iy;
#pragma unroll
    for (int c = 0; c < 3; ++c) s[(c * ROWS + r) * LS + ix] = ok ? D[c * N + p] : mk<C>(0, 0);
  }
  __syncthreads();
  fft_lines<C, NX, INV, 3 * ROWS, NT>(s, LS, tw);
  const T k = (T)(*U.k_dev - U.kz_shift);
  const T sN = T(1) / T(N);
  const int c0 = unit_col0(U);
  C* __restrict__ O = U.out + (size_t)(col + c0) * U.out_cs;
  double accr = 0.0, acci = 0.0;
#pragma unroll
  for (int q = threadIdx.x; q < ROWS * NX; q += NT) {
    const int r = q / NX, ix = q - r * NX, iy = row0 + r;
    if (iy >= Ny) continue;
    const size_t p = ix + (size_t)NX * iy;
    const C e0 = s[(0 * ROWS + r) * LS + ix], e1 = s[(1 * ROWS + r) * LS + ix], e2 = s[(2 * ROWS + r) * LS + ix];
    if constexpr (MODE == RO_STORE3) {
      O[p] = e0; O[N + p] = e1; O[2 * N + p] = e2;
    } else {
      const Basis<T> b = basis_at<T>(k, T(freq_index(ix, NX)) * U.inv_dx, T(freq_index(iy, Ny)) * U.inv_dy);
      const C en = e0 * b.nx + e1 * b.ny;                 // e·n̂ (n̂_z = 0)
      const C em = e0 * b.mx + e1 * b.my + e2 * b.mz;     // e·m̂
      C h1, h2;
      if constexpr (MODE == RO_KXINVCT) {
        const T sc = sN / b.mag;
        h1 = en * sc; h2 = em * (-sc);
      } else {
        const T sc = b.mag * sN;
        h1 = en * (-sc); h2 = em * sc;
      }
      if constexpr (MODE == RO_KXCT_DOT) {
        const C* Hin = U.in + (size_t)(col + c0) * U.in_cs;
        const C g1 = Hin[2 * p], g2 = Hin[2 * p + 1];
        // ⟨H_in, out⟩ = Σ conj(H_in)·out
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
