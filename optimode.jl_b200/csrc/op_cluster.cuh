// M̂(k)H in ONE kernel on thread-block clusters (FP32, 2D cells whose lines split into two
// register DFTs; instantiated for 256 × 256).
//
// The three-pass apply (op_kernels_2l.cuh) moves a 3-component intermediate through global
// memory twice each way, 2.6× the algorithmic bytes.  Here a cluster of 8 CTAs (one per SM,
// 512 threads) holds the whole 3-component field of one (cell, column) unit in its
// distributed shared memory (3 · 256 · 256 · 8 B = 1.5 MiB, ≈205 KB per CTA; or 16 CTAs of 256
// threads, two per SM, ≈102 KB each), so H is read
// once, ε⁻¹ once per pixel and H written once:
//
//   A  CTA r owns grid rows [r·RPC, (r+1)·RPC): H → prologue (basis + kx_tc) → two-level
//      FFT along x, kept in its own shared memory in the "k1-major" order of the register
//      FFT (x = k1 + AX·k2 at slot k1·(BX+1) + k2 of the row's line);
//   B  CTA r owns the x positions with k1 ∈ [r·K1C, (r+1)·K1C) (NX/CTAS columns whose slots
//      in every row line form one contiguous run): it reads its columns out of all the
//      CTAs' shared memory (ld.shared::cluster), FFTs along y, contracts with ε⁻¹ per pixel,
//      FFTs back, and writes the columns back into the owners' row lines
//      (st.shared::cluster);
//   C  CTA r FFTs its rows back along x and applies the kx_ct epilogue, H → global.
//
// Between the phases a cluster barrier (arrive.release / wait.acquire) orders the shared
// memory traffic.  Phase B needs a working block as large as the row lines, so a CTA first
// holds its columns in registers, waits until every CTA has read its lines, and then reuses
// its own lines as the column block; the finished columns are held again until every CTA is
// done with its block.  The same arithmetic as the three passes, in the same order, so the
// results agree with them to FP32 rounding.
//
// A persistent grid: cluster c takes units c, c + nclusters, ...; every CTA of a cluster
// runs the same unit sequence and the same barriers (the column-count test that skips a unit
// reads the same device value in all of them).  No shared memory of another CTA is touched
// before the first cluster barrier or after the last one of a unit.
#pragma once

#include "op_kernels_2l.cuh"

namespace omb {

// Step 1 and reverse step 1 of the two-level transform (fft_reg.cuh) with the twiddles read
// from a shared-memory copy of the table (the carve-out leaves almost no L1 for cached
// global loads in this kernel).
template <int L, bool INV>
__device__ __forceinline__ void cl_first(float2* v, int n2, float2* line, const float2* tw1) {
  constexpr int A = plan2_a(L), B = L / A;
  dft_reg<A, INV>(v);
  line[n2] = v[0];
#pragma unroll
  for (int k1 = 1; k1 < A; ++k1) line[k1 * (B + 1) + n2] = INV ? cmulc(v[k1], tw1[k1 * B + n2]) : cmul(v[k1], tw1[k1 * B + n2]);
}
template <int L, bool INV>
__device__ __forceinline__ void cl_rfirst(float2* w, int k1, float2* line, const float2* tw3) {
  constexpr int A = plan2_a(L), B = L / A;
  dft_reg<B, INV>(w);
  line[k1 * (B + 1)] = w[0];
#pragma unroll
  for (int m2 = 1; m2 < B; ++m2) line[k1 * (B + 1) + m2] = INV ? cmulc(w[m2], tw3[m2 * A + k1]) : cmul(w[m2], tw3[m2 * A + k1]);
}

// Cluster shapes: 8 CTAs of 512 threads (one CTA per SM, the portable cluster size) or 16 CTAs
// of 256 threads (two CTAs per SM, so that two units' phases interleave on an SM).

__device__ __forceinline__ uint32_t cl_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cl_index() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cl_count() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}
// every thread of every CTA of the cluster; orders shared::cluster accesses across it
__device__ __forceinline__ void cl_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// address of the same shared-memory offset in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cl_map(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ float2 cl_load(uint32_t a) {
  float2 v;
  asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ void cl_store(uint32_t a, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}

// Shape of the cluster apply for an NX × NY grid on clusters of CTAS CTAs.
template <int NX, int NY, int CTAS> struct ClShape {
  static constexpr int AX = plan2_a(NX), BX = NX / AX, AY = plan2_a(NY), BY = NY / AY;
  static constexpr int RPC = NY / CTAS;  // grid rows per CTA (phases A and C)
  static constexpr int CPC = NX / CTAS;  // x positions per CTA (phase B)
  static constexpr int K1C = AX / CTAS;  // k1 values per CTA in phase B
  static constexpr int THREADS = RPC * BX;
  static constexpr int LSR = AX * (BX + 1);  // row line stride (k1-major slots)
  static constexpr int LSC = (AY * (BY + 1)) | 1;  // column line stride, odd: conflict-free across columns
  static constexpr size_t SMEM = (size_t)(3 * RPC * LSR > 3 * CPC * LSC ? 3 * RPC * LSR : 3 * CPC * LSC) * sizeof(float2);
  // one work item per thread in every step
  static constexpr bool OK = AX != 0 && AY != 0 && NX % CTAS == 0 && NY % CTAS == 0 && AX % CTAS == 0 &&
                             RPC * AX == THREADS && CPC * BY == THREADS && CPC * AY == THREADS &&
                             RPC % BY == 0 && THREADS <= 1024 && SMEM + 2 * (NX + NY) * sizeof(float2) <= 227 * 1024;
  static constexpr size_t TW_BYTES = (NX == NY ? 2 * NX : 2 * (NX + NY)) * sizeof(float2);  // static twiddles
  static constexpr int MIN_BLOCKS = (2 * (SMEM + TW_BYTES + 1024) <= 228 * 1024) ? 2 : 1;
};

// Launched with a cluster dimension of CTAS (cudaLaunchKernelEx).
template <int NX, int NY, int CTAS>
__global__ void __launch_bounds__(ClShape<NX, NY, CTAS>::THREADS, ClShape<NX, NY, CTAS>::MIN_BLOCKS)
    k_apply_cluster(const OpUnit<float>* __restrict__ units, int nunits, int maxcol,
                    const float2* __restrict__ twx_g, const float2* __restrict__ twy_g) {
  using T = float;
  using C = float2;
  using S = ClShape<NX, NY, CTAS>;
  constexpr int AX = S::AX, BX = S::BX, AY = S::AY, BY = S::BY, RPC = S::RPC, CPC = S::CPC;
  constexpr int LSR = S::LSR, LSC = S::LSC;
  static_assert(S::OK, "cluster apply shape");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* F = reinterpret_cast<C*>(smem_raw);
  const uint32_t F_s = (uint32_t)__cvta_generic_to_shared(F);
  const int tid = threadIdx.x;
  const uint32_t rank = cl_rank();
  // per-level twiddle tables of both axes in shared memory (x and y share them when NX = NY)
  __shared__ C s_tw[NX == NY ? 2 * NX : 2 * (NX + NY)];
  for (int i = tid; i < 2 * NX; i += S::THREADS) s_tw[i] = twx_g[NX + i];
  if constexpr (NX != NY)
    for (int i = tid; i < 2 * NY; i += S::THREADS) s_tw[2 * NX + i] = twy_g[NY + i];
  const C* tw1x = s_tw;
  const C* tw3x = s_tw + NX;
  const C* tw1y = NX == NY ? tw1x : s_tw + 2 * NX;
  const C* tw3y = NX == NY ? tw3x : s_tw + 2 * NX + NY;
  __syncthreads();
  constexpr int N = NX * NY;
  const T sN = T(1) / T(N);
  // phase-B column of this thread: x = k1x + AX·k2x, slot k1x·(BX+1) + k2x of every row line
  const int tB = tid % CPC;
  const int k1x = S::K1C * (int)rank + tB / BX, k2x = tB % BX;
  const int ixB = k1x + AX * k2x;
  const int slotB = k1x * (BX + 1) + k2x;
  // remote lines are addressed by mapa at the point of use (a register array of the CTAs'
  // base addresses would cost CTAS registers for the whole kernel)

  const int total = nunits * maxcol;
  for (int w = (int)cl_index(); w < total; w += (int)cl_count()) {
    const int z = w / maxcol, col = w - z * maxcol;
    const OpUnit<T>& U = units[z];
    if (col >= unit_ncol(U)) continue;  // the same value in every CTA of the cluster
    const int c0 = unit_col0(U);
    const T k = (T)(*U.k_dev - U.kz_shift);
    const C* __restrict__ H = U.in + (size_t)(col + c0) * U.in_cs;
    C* __restrict__ O = U.out + (size_t)(col + c0) * U.out_cs;

    // ---- A: prologue + FFT along x of rows [rank·RPC, +RPC) --------------------------
    // The prologue writes each component straight into the thread's own column n2 of the
    // padded block (x = BX·n1 + n2 at n1·(BX+1) + n2); step 1 then transforms that column
    // in place, one component at a time.
    {
      const int r = tid / BX, n2 = tid % BX, iy = (int)rank * RPC + r;
      C* l0 = F + (0 * RPC + r) * LSR;
      C* l1 = F + (1 * RPC + r) * LSR;
      C* l2 = F + (2 * RPC + r) * LSR;
      float4 h[AX];
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) h[n1] = __ldg(reinterpret_cast<const float4*>(H) + BX * n1 + n2 + (size_t)NX * iy);
      const T gy = T(freq_index(iy, NY)) * U.inv_dy;
      __syncthreads();  // the previous unit's phase C has finished reading F
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) {
        const int ix = BX * n1 + n2;
        const C h1 = mk<C>(h[n1].x, h[n1].y), h2 = mk<C>(h[n1].z, h[n1].w);
        const Basis<T> b = basis_pass<T>(k, T(freq_index(ix, NX)) * U.inv_dx, gy);
        const T s_ = -b.mag;
        l0[n1 * (BX + 1) + n2] = (h1 * b.nx - h2 * b.mx) * s_;
        l1[n1 * (BX + 1) + n2] = (h1 * b.ny - h2 * b.my) * s_;
        l2[n1 * (BX + 1) + n2] = h2 * (-b.mz * s_);
      }
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C* line = F + (c * RPC + r) * LSR;
        C v[AX];
#pragma unroll
        for (int n1 = 0; n1 < AX; ++n1) v[n1] = line[n1 * (BX + 1) + n2];
        cl_first<NX, false>(v, n2, line, tw1x);
      }
    }
    __syncthreads();
    {
      const int r = tid / AX, k1 = tid % AX;
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C* line = F + (c * RPC + r) * LSR;
        C wv[BX];
        l2_second<NX, false>(line, k1, wv);
#pragma unroll
        for (int k2 = 0; k2 < BX; ++k2) line[k1 * (BX + 1) + k2] = wv[k2];
      }
    }
    cl_barrier();  // every row line of the unit is complete

    // ---- B: columns along y (ε⁻¹ between the transforms) ------------------------------
    {
      const int n2 = tid / CPC;
      C v0[AY], v1[AY], v2[AY];
      // y = BY·n1 + n2 lives in CTA (BY·n1)/RPC, line (BY·n1)%RPC + n2 (RPC is a multiple of BY)
      auto col_load = [&](int c, C* v) {
#pragma unroll
        for (int n1 = 0; n1 < AY; ++n1) {
          const int line = c * RPC + (BY * n1) % RPC + n2;
          v[n1] = cl_load(cl_map(F_s + (uint32_t)((line * LSR + slotB) * sizeof(C)), (uint32_t)((BY * n1) / RPC)));
        }
        dft_reg<AY, false>(v);
#pragma unroll
        for (int k1 = 1; k1 < AY; ++k1) v[k1] = cmul(v[k1], tw1y[k1 * BY + n2]);
      };
      col_load(0, v0);
      col_load(1, v1);
      col_load(2, v2);
      cl_barrier();  // every CTA has read its columns: the lines become column blocks
      C* l0 = F + (0 * CPC + tB) * LSC;
      C* l1 = F + (1 * CPC + tB) * LSC;
      C* l2 = F + (2 * CPC + tB) * LSC;
#pragma unroll
      for (int k1 = 0; k1 < AY; ++k1) {
        l0[k1 * (BY + 1) + n2] = v0[k1];
        l1[k1 * (BY + 1) + n2] = v1[k1];
        l2[k1 * (BY + 1) + n2] = v2[k1];
      }
    }
    __syncthreads();
    {
      const int k1 = tid / CPC;
      C* l0 = F + (0 * CPC + tB) * LSC;
      C* l1 = F + (1 * CPC + tB) * LSC;
      C* l2 = F + (2 * CPC + tB) * LSC;
      // components 0 and 1 go back to the thread's own row k1 after their forward DFT;
      // component 2 stays in registers through the ε⁻¹ contraction
      C V[BY];
      C* const r0 = l0 + k1 * (BY + 1);
      C* const r1 = l1 + k1 * (BY + 1);
      // ε⁻¹ of the first half of the thread's pixels is requested before the transforms (its
      // latency hides behind them), the second half after the first half's contraction
      constexpr int EH = BY / 2;
      float4 ea[EH];
      float2 eb[EH];
      auto eps_fetch = [&](int k20) {
#pragma unroll
        for (int j = 0; j < EH; ++j) {
          const size_t p = (size_t)(k1 + AY * (k20 + j)) * NX + ixB;
          ea[j] = __ldg(U.e32a + p);
          eb[j] = __ldg(U.e32b + p);
        }
      };
      auto eps_apply = [&](int k20) {
#pragma unroll
        for (int j = 0; j < EH; ++j) {
          const int k2 = k20 + j;
          const C d0 = r0[k2], d1 = r1[k2], d2 = V[k2];
          const float4 a = ea[j];
          const float2 b = eb[j];
          r0[k2] = d0 * a.x + d1 * a.w + d2 * b.x;
          r1[k2] = d0 * a.w + d1 * a.y + d2 * b.y;
          V[k2] = d0 * b.x + d1 * b.y + d2 * a.z;
        }
      };
      eps_fetch(0);
      l2_second<NY, false>(l0, k1, V);
#pragma unroll
      for (int k2 = 0; k2 < BY; ++k2) r0[k2] = V[k2];
      l2_second<NY, false>(l1, k1, V);
#pragma unroll
      for (int k2 = 0; k2 < BY; ++k2) r1[k2] = V[k2];
      l2_second<NY, false>(l2, k1, V);
      eps_apply(0);
      eps_fetch(EH);
      eps_apply(EH);
      cl_rfirst<NY, true>(V, k1, l2, tw3y);
#pragma unroll
      for (int k2 = 0; k2 < BY; ++k2) V[k2] = r1[k2];
      cl_rfirst<NY, true>(V, k1, l1, tw3y);
#pragma unroll
      for (int k2 = 0; k2 < BY; ++k2) V[k2] = r0[k2];
      cl_rfirst<NY, true>(V, k1, l0, tw3y);
    }
    __syncthreads();
    {
      const int m2 = tid / CPC;
      C v0[AY], v1[AY], v2[AY];
      l2_rsecond<NY, true>(F + (0 * CPC + tB) * LSC, m2, v0);
      l2_rsecond<NY, true>(F + (1 * CPC + tB) * LSC, m2, v1);
      l2_rsecond<NY, true>(F + (2 * CPC + tB) * LSC, m2, v2);
      cl_barrier();  // every CTA is done with its column block: the lines are row lines again
#pragma unroll
      for (int m1 = 0; m1 < AY; ++m1) {
        const int line = (BY * m1) % RPC + m2;  // y = m2 + BY·m1
        const uint32_t a = cl_map(F_s + (uint32_t)((line * LSR + slotB) * sizeof(C)), (uint32_t)((BY * m1) / RPC));
        constexpr uint32_t cstr = (uint32_t)(RPC * LSR * sizeof(C));
        cl_store(a, v0[m1]);
        cl_store(a + cstr, v1[m1]);
        cl_store(a + 2 * cstr, v2[m1]);
      }
    }
    cl_barrier();  // every column is back in its row line

    // ---- C: FFT back along x + kx_ct epilogue ----------------------------------------
    {
      const int r = tid / AX, k1 = tid % AX;
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C* line = F + (c * RPC + r) * LSR;
        C wv[BX];
#pragma unroll
        for (int k2 = 0; k2 < BX; ++k2) wv[k2] = line[k1 * (BX + 1) + k2];
        cl_rfirst<NX, true>(wv, k1, line, tw3x);
      }
    }
    __syncthreads();
    {
      // components 0 and 1 go back to the thread's own column m2 after the transform
      // (x = m2 + BX·m1 at m1·(BX+1) + m2); component 2 stays in registers for the epilogue
      const int r = tid / BX, m2 = tid % BX, iy = (int)rank * RPC + r;
      C y[AX];
#pragma unroll 1
      for (int c = 0; c < 2; ++c) {
        C* line = F + (c * RPC + r) * LSR;
        l2_rsecond<NX, true>(line, m2, y);
#pragma unroll
        for (int m1 = 0; m1 < AX; ++m1) line[m1 * (BX + 1) + m2] = y[m1];
      }
      l2_rsecond<NX, true>(F + (2 * RPC + r) * LSR, m2, y);
      const C* c0l = F + (0 * RPC + r) * LSR + m2;
      const C* c1l = F + (1 * RPC + r) * LSR + m2;
      const T gy = T(freq_index(iy, NY)) * U.inv_dy;
#pragma unroll
      for (int m1 = 0; m1 < AX; ++m1) {
        const int ix = m2 + BX * m1;
        const size_t p = ix + (size_t)NX * iy;
        const Basis<T> b = basis_pass<T>(k, T(freq_index(ix, NX)) * U.inv_dx, gy);
        const C e0 = c0l[m1 * (BX + 1)], e1 = c1l[m1 * (BX + 1)];
        const C en = e0 * b.nx + e1 * b.ny;
        const C em = e0 * b.mx + e1 * b.my + y[m1] * b.mz;
        const T sc = b.mag * sN;
        const C h1 = en * (-sc), h2 = em * sc;
        reinterpret_cast<float4*>(O)[p] = make_float4(h1.x, h1.y, h2.x, h2.y);
      }
    }
  }
}

}  // namespace omb
