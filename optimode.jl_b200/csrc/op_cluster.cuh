// M̂(k)H in ONE kernel on thread-block clusters (FP32, 2D cells whose lines split into two
// register DFTs; instantiated for 256 × 256).
//
// The three-pass apply (op_kernels_2l.cuh) moves a 3-component intermediate through global
// memory twice each way, 2.6× the algorithmic bytes.  Here a cluster of 8 CTAs (one per SM,
// 512 threads) holds the whole 3-component field of one (cell, column) unit in its
// distributed shared memory (3 · 256 · 256 · 8 B = 1.5 MiB, ≈205 KB per CTA), so H is read
// once, ε⁻¹ once per pixel and H written once:
//
//   A  CTA r owns grid rows [r·RPC, (r+1)·RPC): H → prologue (basis + kx_tc) → two-level
//      FFT along x, kept in its own shared memory in the "k1-major" order of the register
//      FFT (x = k1 + AX·k2 at slot k1·(BX+1) + k2 of the row's line);
//   B  CTA r owns the x positions with k1 ∈ [r·AX/8, (r+1)·AX/8) (NX/8 columns whose slots
//      in every row line form one contiguous run): it reads its columns out of all eight
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

constexpr int CL_CTAS = 8;      // CTAs per cluster
constexpr int CL_THREADS = 512;

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

// Shape of the cluster apply for an NX × NY grid.
template <int NX, int NY> struct ClShape {
  static constexpr int AX = plan2_a(NX), BX = NX / AX, AY = plan2_a(NY), BY = NY / AY;
  static constexpr int RPC = NY / CL_CTAS;  // grid rows per CTA (phases A and C)
  static constexpr int CPC = NX / CL_CTAS;  // x positions per CTA (phase B)
  static constexpr int K1C = AX / CL_CTAS;  // k1 values per CTA in phase B
  static constexpr int LSR = AX * (BX + 1);  // row line stride (k1-major slots)
  static constexpr int LSC = (AY * (BY + 1)) | 1;  // column line stride, odd: conflict-free across columns
  static constexpr size_t SMEM = (size_t)(3 * RPC * LSR > 3 * CPC * LSC ? 3 * RPC * LSR : 3 * CPC * LSC) * sizeof(float2);
  // one work item per thread in every step
  static constexpr bool OK = AX != 0 && AY != 0 && NX % CL_CTAS == 0 && NY % CL_CTAS == 0 && AX % CL_CTAS == 0 &&
                             RPC * BX == CL_THREADS && RPC * AX == CL_THREADS && CPC * BY == CL_THREADS &&
                             CPC * AY == CL_THREADS && RPC % BY == 0 && SMEM <= 227 * 1024;
};

template <int NX, int NY>
__global__ void __cluster_dims__(CL_CTAS, 1, 1) __launch_bounds__(CL_THREADS, 1)
    k_apply_cluster(const OpUnit<float>* __restrict__ units, int nunits, int maxcol,
                    const float2* __restrict__ twx_g, const float2* __restrict__ twy_g) {
  using T = float;
  using C = float2;
  using S = ClShape<NX, NY>;
  constexpr int AX = S::AX, BX = S::BX, AY = S::AY, BY = S::BY, RPC = S::RPC, CPC = S::CPC;
  constexpr int LSR = S::LSR, LSC = S::LSC;
  static_assert(S::OK, "cluster apply shape");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* F = reinterpret_cast<C*>(smem_raw);
  const uint32_t F_s = (uint32_t)__cvta_generic_to_shared(F);
  const int tid = threadIdx.x;
  const uint32_t rank = cl_rank();
  const C* tw1x = twx_g + NX;
  const C* tw3x = twx_g + 2 * NX;
  const C* tw1y = twy_g + NY;
  const C* tw3y = twy_g + 2 * NY;
  constexpr int N = NX * NY;
  const T sN = T(1) / T(N);
  // phase-B column of this thread: x = k1x + AX·k2x, slot k1x·(BX+1) + k2x of every row line
  const int tB = tid % CPC;
  const int k1x = S::K1C * (int)rank + tB / BX, k2x = tB % BX;
  const int ixB = k1x + AX * k2x;
  const int slotB = k1x * (BX + 1) + k2x;
  // remote base addresses of the eight CTAs' lines
  uint32_t rbase[CL_CTAS];
#pragma unroll
  for (int r = 0; r < CL_CTAS; ++r) rbase[r] = cl_map(F_s, (uint32_t)r);

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
    {
      const int r = tid / BX, n2 = tid % BX, iy = (int)rank * RPC + r;
      C v0[AX], v1[AX], v2[AX];
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) {
        const int ix = BX * n1 + n2;
        const size_t p = ix + (size_t)NX * iy;
        const float4 h = __ldg(reinterpret_cast<const float4*>(H) + p);
        const C h1 = mk<C>(h.x, h.y), h2 = mk<C>(h.z, h.w);
        const Basis<T> b = basis_pass<T>(k, T(freq_index(ix, NX)) * U.inv_dx, T(freq_index(iy, NY)) * U.inv_dy);
        const T s_ = -b.mag;
        v0[n1] = (h1 * b.nx - h2 * b.mx) * s_;
        v1[n1] = (h1 * b.ny - h2 * b.my) * s_;
        v2[n1] = h2 * (-b.mz * s_);
      }
      __syncthreads();  // the previous unit's phase C has finished reading F
      l2_first<NX, false>(v0, n2, F + (0 * RPC + r) * LSR, tw1x);
      l2_first<NX, false>(v1, n2, F + (1 * RPC + r) * LSR, tw1x);
      l2_first<NX, false>(v2, n2, F + (2 * RPC + r) * LSR, tw1x);
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
#pragma unroll
      for (int n1 = 0; n1 < AY; ++n1) {
        // y = BY·n1 + n2 lives in CTA (BY·n1)/RPC, line (BY·n1)%RPC + n2 (RPC is a multiple of BY)
        const int line = (BY * n1) % RPC + n2;
        const uint32_t a = rbase[(BY * n1) / RPC] + (uint32_t)((line * LSR + slotB) * sizeof(C));
        constexpr uint32_t cstr = (uint32_t)(RPC * LSR * sizeof(C));
        v0[n1] = cl_load(a);
        v1[n1] = cl_load(a + cstr);
        v2[n1] = cl_load(a + 2 * cstr);
      }
      dft_reg<AY, false>(v0);
      dft_reg<AY, false>(v1);
      dft_reg<AY, false>(v2);
#pragma unroll
      for (int k1 = 1; k1 < AY; ++k1) {
        const C t = __ldg(tw1y + k1 * BY + n2);
        v0[k1] = cmul(v0[k1], t);
        v1[k1] = cmul(v1[k1], t);
        v2[k1] = cmul(v2[k1], t);
      }
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
      C V0[BY], V1[BY], V2[BY];
      l2_second<NY, false>(l0, k1, V0);
      l2_second<NY, false>(l1, k1, V1);
      l2_second<NY, false>(l2, k1, V2);
#pragma unroll
      for (int k2 = 0; k2 < BY; ++k2) pointwise_at<T, PW_EPS>(U, (size_t)(k1 + AY * k2) * NX + ixB, V0[k2], V1[k2], V2[k2]);
      l2_rfirst<NY, true>(V0, k1, l0, tw3y);
      l2_rfirst<NY, true>(V1, k1, l1, tw3y);
      l2_rfirst<NY, true>(V2, k1, l2, tw3y);
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
        const uint32_t a = rbase[(BY * m1) / RPC] + (uint32_t)((line * LSR + slotB) * sizeof(C));
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
        l2_rfirst<NX, true>(wv, k1, line, tw3x);
      }
    }
    __syncthreads();
    {
      const int r = tid / BX, m2 = tid % BX, iy = (int)rank * RPC + r;
      C y0[AX], y1[AX], y2[AX];
      l2_rsecond<NX, true>(F + (0 * RPC + r) * LSR, m2, y0);
      l2_rsecond<NX, true>(F + (1 * RPC + r) * LSR, m2, y1);
      l2_rsecond<NX, true>(F + (2 * RPC + r) * LSR, m2, y2);
#pragma unroll
      for (int m1 = 0; m1 < AX; ++m1) {
        const int ix = m2 + BX * m1;
        const size_t p = ix + (size_t)NX * iy;
        const Basis<T> b = basis_pass<T>(k, T(freq_index(ix, NX)) * U.inv_dx, T(freq_index(iy, NY)) * U.inv_dy);
        const C en = y0[m1] * b.nx + y1[m1] * b.ny;
        const C em = y0[m1] * b.mx + y1[m1] * b.my + y2[m1] * b.mz;
        const T sc = b.mag * sN;
        const C h1 = en * (-sc), h2 = em * sc;
        reinterpret_cast<float4*>(O)[p] = make_float4(h1.x, h1.y, h2.x, h2.y);
      }
    }
  }
}

}  // namespace omb
