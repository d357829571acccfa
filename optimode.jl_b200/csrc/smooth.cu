// Kottke sub-pixel smoothing on the device: the geometry pass (`smoothing_plan`) and the
// per-frequency material pass (`smooth_ε(plan, mat_vals)`) of lib/DielectricSmoothing, with
// `sliceinv_3x3` of the ε slice fused into the material pass so the solver's ε⁻¹ input is
// produced in the same sweep over the pixels.
//
// Reference semantics (paths relative to the OptiMode.jl project root):
//   corners          lib/DielectricSmoothing/src/grid.jl:271-312 (myrange, grid.jl:107-110)
//   classification   corner_sinds / proc_sinds, src/smooth.jl:24-72
//   interface pixel  smooth_ε_single! / _interface_geometry, src/smooth.jl:80-121
//   Kottke kernel    normcart, τ_trans, τ⁻¹_trans, avg_param_rot, J2 jet and the lab-frame
//                    εₑ_∂ωεₑ_∂²ωεₑ, src/kottke.jl:13-20, 44-99, 114-137, 218-268
//   plan / apply     SmoothingPlan, smoothing_plan, smooth_ε(plan, mat_vals),
//                    src/smoothing_plan.jl:26-140
//   ε⁻¹              sliceinv_3x3, lib/MaxwellEigenmodes/src/linalg.jl:126-147
// GeometryPrimitives' polygon queries (un-vendored in the reference) are restated for convex
// polygons: inclusive point-in-polygon, the clamped projection onto the nearest edge (first
// edge on ties) with that edge's outward normal, and the voxel fraction on the inner side of
// the tangent line through that point ("plane" fill) or the exact polygon ∩ voxel area
// ("exact" fill).
//
// This file is compiled without floating-point contraction (-fmad=false): every value is a
// chain of individually rounded IEEE operations in a fixed order, so corner classification is
// exact and the results reproduce a CPU restatement that performs the same operations.
//
// Layout in HBM.  Plan: per pixel (x fastest) a uint2 code {kind | m0<<8 | m1<<16 | m2<<24,
// m3} of the pixel kind and four 8-bit material columns, the fill fraction (double) and the
// interface normal (double2) — 32 B per pixel.  Apply: outputs are the reference's column-major
// (3, 3, 3, Nx, Ny) — 27 contiguous doubles per pixel — and (3, 3, Nx, Ny) ε⁻¹, one block of
// each per material set; a CTA stages its 128 pixels' results in shared memory and writes them
// back as one contiguous, coalesced range.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "context.h"

namespace omb {

namespace sm {

constexpr int KIND_UNIFORM = 1;
constexpr int KIND_INTERFACE = 2;
constexpr int KIND_MULTI = 3;
constexpr int MAX_VERTS = 64;          // vertices per polygon
constexpr int MAX_SHAPES = 255;        // shapes per geometry (slot 255 = background at most)
constexpr int MAX_MATS = 256;          // material columns (8-bit indices)
constexpr int CLIP_CAP = MAX_VERTS + 8;
constexpr int PLAN_NT = 128;
constexpr int BULK_NT = 256;
constexpr int SPECIAL_NT = 128;

struct Shapes {
  const double2* verts;  // counter-clockwise vertices of every shape, shape after shape
  const int* voff;       // shape s owns verts[voff[s], voff[s+1])
  const int* minds;      // material column of slot s (nshapes + 1 slots, background last)
  int nshapes;
};

struct Axis {
  double a, step;  // corner i at a + step·i
};

__device__ __forceinline__ double corner(const Axis& ax, int i) { return ax.a + ax.step * (double)i; }

__device__ __forceinline__ double edge_cross(double2 a, double2 b, double px, double py) {
  return (b.x - a.x) * (py - a.y) - (b.y - a.y) * (px - a.x);
}

__device__ int slot_at(const Shapes& sh, double px, double py) {
  for (int s = 0; s < sh.nshapes; ++s) {
    const int v0 = sh.voff[s], v1 = sh.voff[s + 1];
    bool in = true;
    for (int i = v0; i < v1 && in; ++i) {
      const int j = (i + 1 < v1) ? i + 1 : v0;
      in = edge_cross(sh.verts[i], sh.verts[j], px, py) >= 0.0;
    }
    if (in) return s;
  }
  return sh.nshapes;
}

struct Surf {
  double r0x, r0y, nx, ny;
};

__device__ Surf surfpt_nearby(const Shapes& sh, int s, double cx, double cy) {
  const int v0 = sh.voff[s], v1 = sh.voff[s + 1];
  double best = INFINITY;
  Surf out{0.0, 0.0, 1.0, 0.0};
  for (int i = v0; i < v1; ++i) {
    const int j = (i + 1 < v1) ? i + 1 : v0;
    const double2 a = sh.verts[i], b = sh.verts[j];
    const double dx = b.x - a.x, dy = b.y - a.y;
    const double dd = dx * dx + dy * dy;
    double t = ((cx - a.x) * dx + (cy - a.y) * dy) / dd;
    t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
    const double px = a.x + t * dx, py = a.y + t * dy;
    const double ex = cx - px, ey = cy - py;
    const double d2 = ex * ex + ey * ey;
    if (d2 < best) {
      best = d2;
      const double L = sqrt(dd);
      out = Surf{px, py, dy / L, -dx / L};
    }
  }
  return out;
}

// One Sutherland–Hodgman step over `n` vertices (keep f ≥ 0); returns the new count.
template <typename F>
__device__ int clip_step(const double2* in, int n, double2* out, F f) {
  int m = 0;
  for (int j = 0; j < n; ++j) {
    const double2 p = in[j], q = in[(j + 1 < n) ? j + 1 : 0];
    const double sp = f(p), sq = f(q);
    if (sp >= 0.0 && m < CLIP_CAP) out[m++] = p;
    if ((sp >= 0.0) != (sq >= 0.0) && m < CLIP_CAP) {
      const double t = sp / (sp - sq);
      out[m++] = make_double2(p.x + t * (q.x - p.x), p.y + t * (q.y - p.y));
    }
  }
  return m;
}

__device__ double poly_area(const double2* p, int n) {
  if (n < 3) return 0.0;
  double s = 0.0;
  for (int j = 0; j < n; ++j) {
    const double2 a = p[j], b = p[(j + 1 < n) ? j + 1 : 0];
    s += a.x * b.y - b.x * a.y;
  }
  return 0.5 * fabs(s);
}

__device__ double volfrac_plane(double x0, double x1, double y0, double y1, const Surf& sf) {
  double2 box[4] = {make_double2(x0, y0), make_double2(x1, y0), make_double2(x1, y1), make_double2(x0, y1)};
  double2 out[8];
  int m = 0;
  for (int j = 0; j < 4; ++j) {
    const double2 p = box[j], q = box[(j + 1) & 3];
    const double sp = -((p.x - sf.r0x) * sf.nx + (p.y - sf.r0y) * sf.ny);
    const double sq = -((q.x - sf.r0x) * sf.nx + (q.y - sf.r0y) * sf.ny);
    if (sp >= 0.0) out[m++] = p;
    if ((sp >= 0.0) != (sq >= 0.0)) {
      const double t = sp / (sp - sq);
      out[m++] = make_double2(p.x + t * (q.x - p.x), p.y + t * (q.y - p.y));
    }
  }
  return poly_area(out, m) / ((x1 - x0) * (y1 - y0));
}

__device__ double volfrac_exact(const Shapes& sh, int s, double x0, double x1, double y0, double y1) {
  double2 A[CLIP_CAP], B[CLIP_CAP];
  A[0] = make_double2(x0, y0); A[1] = make_double2(x1, y0); A[2] = make_double2(x1, y1); A[3] = make_double2(x0, y1);
  int n = 4;
  double2* cur = A;
  double2* nxt = B;
  const int v0 = sh.voff[s], v1 = sh.voff[s + 1];
  for (int i = v0; i < v1; ++i) {
    const int j = (i + 1 < v1) ? i + 1 : v0;
    const double2 a = sh.verts[i], b = sh.verts[j];
    n = clip_step(cur, n, nxt, [&](double2 p) { return edge_cross(a, b, p.x, p.y); });
    double2* t = cur; cur = nxt; nxt = t;
    if (n == 0) return 0.0;
  }
  return poly_area(cur, n) / ((x1 - x0) * (y1 - y0));
}

// Geometry pass: one thread per pixel.
__global__ void __launch_bounds__(PLAN_NT) k_smooth_plan(Shapes sh, Axis ax, Axis ay, int Nx, int Ny, int fill,
                                                         uint2* __restrict__ code, double* __restrict__ rvol,
                                                         double2* __restrict__ nrm,
                                                         unsigned long long* __restrict__ counts) {
  __shared__ unsigned int cnt[3];
  if (threadIdx.x < 3) cnt[threadIdx.x] = 0;
  __syncthreads();
  const long long N = (long long)Nx * Ny;
  const long long v = (long long)blockIdx.x * PLAN_NT + threadIdx.x;
  if (v < N) {
    const int ix = (int)(v % Nx), iy = (int)(v / Nx);
    const double x0 = corner(ax, ix), x1 = corner(ax, ix + 1);
    const double y0 = corner(ay, iy), y1 = corner(ay, iy + 1);
    // corners (x0,y0), (x0,y1), (x1,y1), (x1,y0)
    const int c0 = slot_at(sh, x0, y0), c1 = slot_at(sh, x0, y1);
    const int c2 = slot_at(sh, x1, y1), c3 = slot_at(sh, x1, y0);
    const int lo = min(min(c0, c1), min(c2, c3)), hi = max(max(c0, c1), max(c2, c3));
    int nd = 1;
    bool mid = false;  // a third distinct slot strictly between lo and hi
    for (int c : {c0, c1, c2, c3}) mid |= (c != lo && c != hi);
    if (hi != lo) nd = mid ? 3 : 2;
    uint2 cd;
    double r = 0.0;
    double2 n = make_double2(0.0, 0.0);
    if (nd == 1) {
      cd = make_uint2(KIND_UNIFORM | ((unsigned)sh.minds[lo] << 8), 0u);
    } else if (nd == 2) {
      const double cx = (((x0 + x0) + x1) + x1) / 4.0;
      const double cy = (((y0 + y1) + y1) + y0) / 4.0;
      const Surf sf = surfpt_nearby(sh, lo, cx, cy);
      r = fill == 0 ? volfrac_plane(x0, x1, y0, y1, sf) : volfrac_exact(sh, lo, x0, x1, y0, y1);
      r = r < 0.0 ? 0.0 : (r > 1.0 ? 1.0 : r);
      n = make_double2(sf.nx, sf.ny);
      cd = make_uint2(KIND_INTERFACE | ((unsigned)sh.minds[lo] << 8) | ((unsigned)sh.minds[hi] << 16), 0u);
    } else {
      cd = make_uint2(KIND_MULTI | ((unsigned)sh.minds[c0] << 8) | ((unsigned)sh.minds[c1] << 16) |
                          ((unsigned)sh.minds[c2] << 24),
                      (unsigned)sh.minds[c3]);
    }
    code[v] = cd;
    rvol[v] = r;
    nrm[v] = n;
    atomicAdd(&cnt[nd - 1], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 3 && cnt[threadIdx.x]) atomicAdd(&counts[threadIdx.x], (unsigned long long)cnt[threadIdx.x]);
}

// ---- the dispersive Kottke kernel: a second-order Taylor jet (f, f′, f″) ----------------
// Written over a scalar type R: double for the material pass, Dual (value and one forward
// derivative with respect to a material entry) for the material-data VJP.

struct Dual {
  double v, d;
  Dual() = default;
  __device__ constexpr Dual(double x) : v(x), d(0.0) {}
  __device__ constexpr Dual(double x, double y) : v(x), d(y) {}
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
__device__ __forceinline__ Dual operator/(double a, Dual b) {
  const double i = a / b.v;
  return Dual(i, -(i * b.d) / b.v);
}

template <typename R> struct J2 {
  R v, d, dd;
};

template <typename R> __device__ __forceinline__ J2<R> jadd(J2<R> a, J2<R> b) {
  return J2<R>{a.v + b.v, a.d + b.d, a.dd + b.dd};
}
template <typename R> __device__ __forceinline__ J2<R> jsub(J2<R> a, J2<R> b) {
  return J2<R>{a.v - b.v, a.d - b.d, a.dd - b.dd};
}
template <typename R> __device__ __forceinline__ J2<R> jneg(J2<R> a) { return J2<R>{-a.v, -a.d, -a.dd}; }
template <typename R> __device__ __forceinline__ J2<R> jmul(J2<R> a, J2<R> b) {
  return J2<R>{a.v * b.v, a.d * b.v + a.v * b.d, (a.dd * b.v + 2.0 * a.d * b.d) + a.v * b.dd};
}
template <typename R> __device__ __forceinline__ J2<R> jinv(J2<R> a) {
  const R i = 1.0 / a.v;
  return J2<R>{i, -a.d * i * i, -a.dd * i * i + 2.0 * a.d * a.d * i * i * i};
}

// τ_trans in place on a row-major jet matrix e[r*3+c]
template <typename R> __device__ __forceinline__ void tau(J2<R>* e) {
  const J2<R> i = jinv(e[0]);
  const J2<R> e01 = e[1], e02 = e[2], e10 = e[3], e20 = e[6];
  e[0] = jneg(i);
  e[1] = jmul(e01, i);
  e[2] = jmul(e02, i);
  e[3] = jmul(e10, i);
  e[4] = jsub(e[4], jmul(jmul(e10, e01), i));
  e[5] = jsub(e[5], jmul(jmul(e10, e02), i));
  e[6] = jmul(e20, i);
  e[7] = jsub(e[7], jmul(jmul(e20, e01), i));
  e[8] = jsub(e[8], jmul(jmul(e20, e02), i));
}

template <typename R> __device__ __forceinline__ void tau_inv(J2<R>* t) {
  const J2<R> i = jinv(t[0]);
  const J2<R> t01 = t[1], t02 = t[2], t10 = t[3], t20 = t[6];
  t[0] = jneg(i);
  t[1] = jmul(jneg(t01), i);
  t[2] = jmul(jneg(t02), i);
  t[3] = jmul(jneg(t10), i);
  t[4] = jsub(t[4], jmul(jmul(t10, t01), i));
  t[5] = jsub(t[5], jmul(jmul(t10, t02), i));
  t[6] = jmul(jneg(t20), i);
  t[7] = jsub(t[7], jmul(jmul(t20, t01), i));
  t[8] = jsub(t[8], jmul(jmul(t20, t02), i));
}

// C = A·B for row-major 3×3 (sum in index order)
template <typename RA, typename RB, typename RC>
__device__ __forceinline__ void mm3(const RA* A, const RB* B, RC* C) {
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) C[r * 3 + c] = (A[r * 3] * B[c] + A[r * 3 + 1] * B[3 + c]) + A[r * 3 + 2] * B[6 + c];
}

// slice s of a 27-entry column (column-major 3×3) → row-major X = Sᵀ (E S)
template <typename R>
__device__ __forceinline__ void rotate_in(const R* col, int s, const double* S, const double* St, R* X) {
  R E[9], T[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) E[r * 3 + c] = col[9 * s + r + 3 * c];
  mm3(E, S, T);
  mm3(St, T, X);
}

template <typename R>
__device__ void kottke_jet(double r1, double nx, double ny, const R* c1, const R* c2, R* out) {
  // S = normcart((nx, ny, 0)), columns n, h, v (row-major S[r*3+c])
  const double hx0 = -ny, hy0 = nx;
  const double L = sqrt(hx0 * hx0 + hy0 * hy0);
  const double h0 = hx0 / L, h1 = hy0 / L, h2 = 0.0 / L;
  const double n0 = nx, n1 = ny, n2 = 0.0;
  const double w0 = n1 * h2 - n2 * h1, w1 = n2 * h0 - n0 * h2, w2 = n0 * h1 - n1 * h0;
  const double S[9] = {n0, h0, w0, n1, h1, w1, n2, h2, w2};
  const double St[9] = {n0, n1, n2, h0, h1, h2, w0, w1, w2};
  J2<R> a[9], b[9];
  {
    R X0[9], X1[9], X2[9];
    rotate_in(c1, 0, S, St, X0);
    rotate_in(c1, 1, S, St, X1);
    rotate_in(c1, 2, S, St, X2);
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = J2<R>{X0[k], X1[k], X2[k]};
    rotate_in(c2, 0, S, St, X0);
    rotate_in(c2, 1, S, St, X1);
    rotate_in(c2, 2, S, St, X2);
#pragma unroll
    for (int k = 0; k < 9; ++k) b[k] = J2<R>{X0[k], X1[k], X2[k]};
  }
  tau(a);
  tau(b);
  const J2<R> ra{R(r1), R(0.0), R(0.0)}, rb{R(1.0 - r1), R(0.0), R(0.0)};
#pragma unroll
  for (int k = 0; k < 9; ++k) a[k] = jadd(jmul(ra, a[k]), jmul(rb, b[k]));
  tau_inv(a);
  // back to the lab frame: S (X Sᵀ), written column-major per slice
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    R X[9], T[9], Y[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) X[k] = s == 0 ? a[k].v : (s == 1 ? a[k].d : a[k].dd);
    mm3(X, St, T);
    mm3(S, T, Y);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) out[9 * s + r + 3 * c] = Y[r * 3 + c];
  }
}

// column-major 3×3 inverse by the adjugate
__device__ __forceinline__ void inv3(const double* m, double* o) {
  const double a = m[0], b = m[3], c = m[6];
  const double d = m[1], e = m[4], f = m[7];
  const double g = m[2], h = m[5], i = m[8];
  const double A = e * i - f * h, B = f * g - d * i, C = d * h - e * g;
  const double det = (a * A + b * B) + c * C;
  const double r = 1.0 / det;
  o[0] = A * r; o[1] = B * r; o[2] = C * r;
  o[3] = (c * h - b * i) * r; o[4] = (a * i - c * g) * r; o[5] = (b * g - a * h) * r;
  o[6] = (b * f - c * e) * r; o[7] = (c * d - a * f) * r; o[8] = (a * e - b * d) * r;
}

// Material pass, part 1 (uniform pixels, all but a thin layer of the cell): grid
// (⌈N/256⌉, nsets), 256 threads, one tile of 256 pixels per CTA.  Shared memory holds the
// set's material columns, their ε⁻¹ and the tile's codes; the CTA then writes the tile's
// 27·256 and 9·256 output doubles as contiguous ranges, consecutive threads on consecutive
// addresses.  Interface and multi-material pixels are left to part 2.
__global__ void __launch_bounds__(BULK_NT) k_smooth_bulk(const uint2* __restrict__ code, long long N,
                                                         const double* __restrict__ mats, int nmat,
                                                         double* __restrict__ eps, double* __restrict__ epsinv) {
  extern __shared__ double smem[];
  double* M = smem;              // 27·nmat
  double* Mi = M + 27 * nmat;    // 9·nmat
  uint2* cds = reinterpret_cast<uint2*>(Mi + 9 * nmat);  // BULK_NT
  const int set = blockIdx.y;
  const double* src = mats + (size_t)set * 27 * nmat;
  for (int k = threadIdx.x; k < 27 * nmat; k += BULK_NT) M[k] = src[k];
  const long long base = (long long)blockIdx.x * BULK_NT;
  const long long rem = N - base;
  const int np = rem < BULK_NT ? (int)rem : BULK_NT;
  if (threadIdx.x < np) cds[threadIdx.x] = code[base + threadIdx.x];
  __syncthreads();
  if (epsinv) {
    for (int m = threadIdx.x; m < nmat; m += BULK_NT) inv3(M + 27 * m, Mi + 9 * m);
    __syncthreads();
  }
  if (eps) {
    double* dst = eps + (size_t)set * 27 * N + (size_t)base * 27;
    for (int e = threadIdx.x; e < 27 * np; e += BULK_NT) {
      const int p = e / 27, k = e - 27 * p;
      const unsigned x = cds[p].x;
      if ((x & 0xff) == KIND_UNIFORM) dst[e] = M[27 * ((x >> 8) & 0xff) + k];
    }
  }
  if (epsinv) {
    double* dst = epsinv + (size_t)set * 9 * N + (size_t)base * 9;
    for (int e = threadIdx.x; e < 9 * np; e += BULK_NT) {
      const int p = e / 9, k = e - 9 * p;
      const unsigned x = cds[p].x;
      if ((x & 0xff) == KIND_UNIFORM) dst[e] = Mi[9 * ((x >> 8) & 0xff) + k];
    }
  }
}

// Material pass, part 2: one thread per (listed interface or multi-material pixel, set).
__global__ void __launch_bounds__(SPECIAL_NT) k_smooth_special(const int* __restrict__ list, int nspecial, int nsets,
                                                               const uint2* __restrict__ code,
                                                               const double* __restrict__ rvol,
                                                               const double2* __restrict__ nrm, long long N,
                                                               const double* __restrict__ mats, int nmat,
                                                               double* __restrict__ eps, double* __restrict__ epsinv) {
  const long long i = (long long)blockIdx.x * SPECIAL_NT + threadIdx.x;
  if (i >= (long long)nspecial * nsets) return;
  const int set = (int)(i / nspecial);
  const long long v = list[i - (long long)set * nspecial];
  const double* M = mats + (size_t)set * 27 * nmat;
  const uint2 cd = code[v];
  double o[27];
  if ((cd.x & 0xff) == KIND_INTERFACE) {
    const double2 n = nrm[v];
    kottke_jet(rvol[v], n.x, n.y, M + 27 * ((cd.x >> 8) & 0xff), M + 27 * ((cd.x >> 16) & 0xff), o);
  } else {
    const double* p0 = M + 27 * ((cd.x >> 8) & 0xff);
    const double* p1 = M + 27 * ((cd.x >> 16) & 0xff);
    const double* p2 = M + 27 * ((cd.x >> 24) & 0xff);
    const double* p3 = M + 27 * (cd.y & 0xff);
#pragma unroll
    for (int k = 0; k < 27; ++k) o[k] = ((((0.0 + p0[k]) + p1[k]) + p2[k]) + p3[k]) / 4.0;
  }
  if (eps) {
    double* dst = eps + (size_t)set * 27 * N + (size_t)v * 27;
#pragma unroll
    for (int k = 0; k < 27; ++k) dst[k] = o[k];
  }
  if (epsinv) {
    double q[9];
    inv3(o, q);
    double* dst = epsinv + (size_t)set * 9 * N + (size_t)v * 9;
#pragma unroll
    for (int k = 0; k < 9; ++k) dst[k] = q[k];
  }
}

// Scalar material property on the plan (`smooth_scalar_single`): uniform pixels take their
// material's value, interface pixels r·v_a + (1 − r)·v_b, multi-material pixels the mean of
// their four corners' values (summed in corner order).
__global__ void k_smooth_scalar(const uint2* __restrict__ code, const double* __restrict__ rvol, long long N,
                                const double* __restrict__ vals, double* __restrict__ out) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const uint2 cd = code[v];
  const int kind = cd.x & 0xff;
  const double a = vals[(cd.x >> 8) & 0xff];
  double o;
  if (kind == KIND_UNIFORM) {
    o = a;
  } else if (kind == KIND_INTERFACE) {
    const double r = rvol[v];
    o = r * a + (1.0 - r) * vals[(cd.x >> 16) & 0xff];
  } else {
    o = (((a + vals[(cd.x >> 16) & 0xff]) + vals[(cd.x >> 24) & 0xff]) + vals[cd.y & 0xff]) / 4.0;
  }
  out[v] = o;
}

// ---- material-data VJP of the material pass (`_plan_vjp`) ------------------------------

// Part 1: per tile of 256 pixels and set, the uniform and multi-material pixels' cotangents
// summed per material entry (one thread per entry, pixels in order), written as the tile's
// partial sums.
__global__ void __launch_bounds__(BULK_NT) k_vjp_tiles(const uint2* __restrict__ code, long long N, int nmat,
                                                       const double* __restrict__ ybar, double* __restrict__ part) {
  __shared__ uint2 cds[BULK_NT];
  const int set = blockIdx.y, tile = blockIdx.x;
  const long long base = (long long)tile * BULK_NT;
  const long long rem = N - base;
  const int np = rem < BULK_NT ? (int)rem : BULK_NT;
  if (threadIdx.x < np) cds[threadIdx.x] = code[base + threadIdx.x];
  __syncthreads();
  const double* y = ybar + (size_t)set * 27 * N + (size_t)base * 27;
  double* out = part + ((size_t)set * gridDim.x + tile) * 27 * nmat;
  for (int e = threadIdx.x; e < 27 * nmat; e += BULK_NT) {
    const unsigned m = (unsigned)(e / 27);
    const int k = e - 27 * (int)m;
    double acc = 0.0;
    for (int p = 0; p < np; ++p) {
      const uint2 x = cds[p];
      const int kind = x.x & 0xff;
      if (kind == KIND_UNIFORM) {
        if (((x.x >> 8) & 0xff) == m) acc = acc + y[27 * p + k];
      } else if (kind == KIND_MULTI) {
        const double q = y[27 * p + k] / 4.0;
        if (((x.x >> 8) & 0xff) == m) acc = acc + q;
        if (((x.x >> 16) & 0xff) == m) acc = acc + q;
        if (((x.x >> 24) & 0xff) == m) acc = acc + q;
        if ((x.y & 0xff) == m) acc = acc + q;
      }
    }
    out[e] = acc;
  }
}

// Part 2: one thread per (listed pixel, set, material entry j ∈ [0, 54)): for an interface
// pixel, ȳ · ∂(Kottke kernel)/∂(entry j of column a, or j − 27 of column b), by a forward
// derivative through the Taylor-jet kernel; 0 for a multi-material pixel.
__global__ void __launch_bounds__(SPECIAL_NT) k_vjp_interface(const int* __restrict__ list, int nspecial, int nsets,
                                                              const uint2* __restrict__ code,
                                                              const double* __restrict__ rvol,
                                                              const double2* __restrict__ nrm, long long N,
                                                              const double* __restrict__ mats, int nmat,
                                                              const double* __restrict__ ybar,
                                                              double* __restrict__ ib) {
  const long long i = (long long)blockIdx.x * SPECIAL_NT + threadIdx.x;
  if (i >= (long long)nspecial * nsets * 54) return;
  const int j = (int)(i % 54);
  const long long rest = i / 54;
  const int sp = (int)(rest % nspecial), set = (int)(rest / nspecial);
  const long long v = list[sp];
  const uint2 cd = code[v];
  if ((cd.x & 0xff) != KIND_INTERFACE) { ib[i] = 0.0; return; }
  const double* M = mats + (size_t)set * 27 * nmat;
  const double* ca = M + 27 * ((cd.x >> 8) & 0xff);
  const double* cb = M + 27 * ((cd.x >> 16) & 0xff);
  Dual c1[27], c2[27], o[27];
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    c1[q] = Dual(ca[q], q == j ? 1.0 : 0.0);
    c2[q] = Dual(cb[q], q + 27 == j ? 1.0 : 0.0);
  }
  const double2 n = nrm[v];
  kottke_jet(rvol[v], n.x, n.y, c1, c2, o);
  const double* y = ybar + (size_t)set * 27 * N + (size_t)v * 27;
  double acc = 0.0;
#pragma unroll
  for (int q = 0; q < 27; ++q) acc = acc + y[q] * o[q].d;
  ib[i] = acc;
}

// Part 3: one thread per (set, material entry): the tiles' partial sums in tile order, then
// the interface contributions in pixel order.
__global__ void k_vjp_reduce(const double* __restrict__ part, int ntiles, const double* __restrict__ ib,
                             const int* __restrict__ list, int nspecial, const uint2* __restrict__ code, int nmat,
                             int nsets, double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nsets * 27 * nmat) return;
  const int set = (int)(i / (27 * nmat));
  const int e = (int)(i - (long long)set * 27 * nmat);
  const unsigned m = (unsigned)(e / 27);
  const int k = e - 27 * (int)m;
  double acc = 0.0;
  for (int t = 0; t < ntiles; ++t) acc = acc + part[((size_t)set * ntiles + t) * 27 * nmat + e];
  for (int sp = 0; sp < nspecial; ++sp) {
    const uint2 cd = code[list[sp]];
    if ((cd.x & 0xff) != KIND_INTERFACE) continue;
    const double* g = ib + ((size_t)set * nspecial + sp) * 54;
    if (((cd.x >> 8) & 0xff) == m) acc = acc + g[k];
    if (((cd.x >> 16) & 0xff) == m) acc = acc + g[27 + k];
  }
  out[i] = acc;
}

// Geometry pass, part 2: the list of interface and multi-material pixels (in any order; the
// host sorts it).
__global__ void k_smooth_list(const uint2* __restrict__ code, long long N, int* __restrict__ list,
                              unsigned int* __restrict__ count) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < N && (code[v].x & 0xff) != KIND_UNIFORM) list[atomicAdd(count, 1u)] = (int)v;
}

}  // namespace sm

}  // namespace omb

struct omb_smoothing_plan {
  omb_ctx* ctx = nullptr;
  int Nx = 0, Ny = 0;
  double Dx = 0, Dy = 0;
  int fill = 0;
  int max_mat = 0;  // largest material column the plan references
  long long counts[3] = {0, 0, 0};
  omb::DevBuf<uint2> code;
  omb::DevBuf<double> rvol;
  omb::DevBuf<double2> nrm;
  omb::DevBuf<int> special;  // interface and multi-material pixels
  int nspecial = 0;
  // part 2 of the material pass runs on `aux`, beside part 1 (they write disjoint pixels)
  cudaStream_t aux = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  ~omb_smoothing_plan() {
    if (join) cudaEventDestroy(join);
    if (fork) cudaEventDestroy(fork);
    if (aux) cudaStreamDestroy(aux);
  }
};


using namespace omb;

namespace {

bool is_finite(double x) { return std::isfinite(x); }

int check_plan(const omb_smoothing_plan* p) {
  if (!p || !p->ctx) return fail(OMB_ERR_INVALID_ARG, "smoothing plan is NULL");
  return OMB_OK;
}

sm::Axis axis(double D, int N) {
  const double d = D / N;
  const double a = -(D + d) / 2;
  const double b = (D - d) / 2;
  return sm::Axis{a, (b - a) / N};
}

int apply_launch(omb_smoothing_plan* p, const double* d_mats, int nmat, int nsets, double* d_eps, double* d_inv,
                 cudaStream_t st) {
  static bool attr_set[64] = {};
  const size_t smem = sizeof(double) * 36 * (size_t)nmat + sizeof(uint2) * sm::BULK_NT;
  const int dev = p->ctx->device;
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    OMB_CU(cudaFuncSetAttribute(sm::k_smooth_bulk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(double) * 36 * sm::MAX_MATS + sizeof(uint2) * sm::BULK_NT)));
    attr_set[dev] = true;
  }
  const long long N = (long long)p->Nx * p->Ny;
  if (p->nspecial > 0) {
    OMB_CU(cudaEventRecord(p->fork, st));
    OMB_CU(cudaStreamWaitEvent(p->aux, p->fork, 0));
    const long long work = (long long)p->nspecial * nsets;
    sm::k_smooth_special<<<(unsigned)((work + sm::SPECIAL_NT - 1) / sm::SPECIAL_NT), sm::SPECIAL_NT, 0, p->aux>>>(
        p->special.p, p->nspecial, nsets, p->code.p, p->rvol.p, p->nrm.p, N, d_mats, nmat, d_eps, d_inv);
    OMB_CU(cudaGetLastError());
    OMB_CU(cudaEventRecord(p->join, p->aux));
  }
  const dim3 grid((unsigned)((N + sm::BULK_NT - 1) / sm::BULK_NT), (unsigned)nsets);
  sm::k_smooth_bulk<<<grid, sm::BULK_NT, smem, st>>>(p->code.p, N, d_mats, nmat, d_eps, d_inv);
  OMB_CU(cudaGetLastError());
  if (p->nspecial > 0) OMB_CU(cudaStreamWaitEvent(st, p->join, 0));
  return OMB_OK;
}

int check_apply_args(const omb_smoothing_plan* p, const double* mat_vals, int nmat, int nsets) {
  int rc = check_plan(p);
  if (rc) return rc;
  if (!mat_vals) return fail(OMB_ERR_INVALID_ARG, "mat_vals is NULL");
  if (nmat < 1 || nmat > sm::MAX_MATS)
    return fail(OMB_ERR_INVALID_ARG, "nmat must be in [1, 256], got " + std::to_string(nmat));
  if (nmat <= p->max_mat)
    return fail(OMB_ERR_INVALID_ARG, "the plan references material column " + std::to_string(p->max_mat) +
                                         " but mat_vals has " + std::to_string(nmat) + " columns");
  if (nsets < 1 || nsets > 65535) return fail(OMB_ERR_INVALID_ARG, "nsets must be in [1, 65535]");
  return OMB_OK;
}

}  // namespace

extern "C" int omb_smoothing_plan_create(omb_ctx* ctx, const omb_grid* grid, int32_t nshapes, const int32_t* nverts,
                                         const double* verts, const int32_t* minds, int32_t fill_rule,
                                         omb_smoothing_plan** out) {
  if (!ctx || !grid || !out) return fail(OMB_ERR_INVALID_ARG, "NULL context, grid or output handle");
  *out = nullptr;
  if (grid->Nx < 1 || grid->Ny < 1 || !(grid->Dx > 0) || !(grid->Dy > 0) || !is_finite(grid->Dx) || !is_finite(grid->Dy))
    return fail(OMB_ERR_INVALID_ARG, "grid needs Nx, Ny ≥ 1 and finite Dx, Dy > 0");
  if ((long long)grid->Nx * grid->Ny > (1LL << 31))
    return fail(OMB_ERR_INVALID_ARG, "grid has more than 2^31 pixels");
  if (nshapes < 0 || nshapes > sm::MAX_SHAPES)
    return fail(OMB_ERR_INVALID_ARG, "nshapes must be in [0, 255], got " + std::to_string(nshapes));
  if (fill_rule != OMB_FILL_PLANE && fill_rule != OMB_FILL_EXACT)
    return fail(OMB_ERR_INVALID_ARG, "fill_rule must be OMB_FILL_PLANE or OMB_FILL_EXACT");
  if (!minds || (nshapes > 0 && (!nverts || !verts))) return fail(OMB_ERR_INVALID_ARG, "NULL shape arrays");
  // counter-clockwise convex polygons
  std::vector<int> voff(nshapes + 1, 0);
  std::vector<double2> hv;
  size_t pos = 0;
  for (int s = 0; s < nshapes; ++s) {
    const int nv = nverts[s];
    if (nv < 3 || nv > sm::MAX_VERTS)
      return fail(OMB_ERR_INVALID_ARG, "shape " + std::to_string(s) + " needs 3 to 64 vertices");
    std::vector<double2> v(nv);
    for (int i = 0; i < nv; ++i) {
      v[i] = make_double2(verts[2 * (pos + i)], verts[2 * (pos + i) + 1]);
      if (!is_finite(v[i].x) || !is_finite(v[i].y))
        return fail(OMB_ERR_INVALID_ARG, "shape " + std::to_string(s) + " has a non-finite vertex");
    }
    pos += nv;
    double area2 = 0.0;
    for (int i = 0; i < nv; ++i) {
      const int j = (i + 1) % nv;
      area2 += v[i].x * v[j].y - v[j].x * v[i].y;
    }
    if (area2 < 0) std::reverse(v.begin(), v.end());
    if (area2 == 0) return fail(OMB_ERR_INVALID_ARG, "shape " + std::to_string(s) + " has zero area");
    for (int i = 0; i < nv; ++i) {
      const double2 a = v[i], b = v[(i + 1) % nv], c = v[(i + 2) % nv];
      const double turn = (b.x - a.x) * (c.y - b.y) - (b.y - a.y) * (c.x - b.x);
      if (turn < 0) return fail(OMB_ERR_INVALID_ARG, "shape " + std::to_string(s) + " is not convex");
    }
    voff[s + 1] = voff[s] + nv;
    hv.insert(hv.end(), v.begin(), v.end());
  }
  int max_mat = 0;
  for (int s = 0; s <= nshapes; ++s) {
    if (minds[s] < 0 || minds[s] >= sm::MAX_MATS)
      return fail(OMB_ERR_INVALID_ARG, "minds entries must be material columns in [0, 255]");
    max_mat = std::max(max_mat, (int)minds[s]);
  }
  auto* p = new omb_smoothing_plan();
  p->ctx = ctx;
  p->Nx = grid->Nx; p->Ny = grid->Ny; p->Dx = grid->Dx; p->Dy = grid->Dy;
  p->fill = fill_rule;
  p->max_mat = max_mat;
  cudaStream_t st = ctx->stream;
  const size_t N = (size_t)p->Nx * p->Ny;
  auto bail = [&](int rc) { delete p; return rc; };
  DevBuf<double2> dv;
  DevBuf<int> doff, dm;
  DevBuf<unsigned long long> dcnt;
  if (cudaError_t e = cudaSetDevice(ctx->device); e != cudaSuccess) return bail(cuda_fail(e, "cudaSetDevice"));
#define PLAN_CU(x)                                          \
  do {                                                      \
    cudaError_t e__ = (x);                                  \
    if (e__ != cudaSuccess) return bail(cuda_fail(e__, #x)); \
  } while (0)
  PLAN_CU(cudaStreamCreateWithFlags(&p->aux, cudaStreamNonBlocking));
  PLAN_CU(cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming));
  PLAN_CU(cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming));
  PLAN_CU(p->code.alloc(N, st));
  PLAN_CU(p->rvol.alloc(N, st));
  PLAN_CU(p->nrm.alloc(N, st));
  PLAN_CU(dv.alloc(std::max<size_t>(hv.size(), 1), st));
  PLAN_CU(doff.alloc(nshapes + 1, st));
  PLAN_CU(dm.alloc(nshapes + 1, st));
  PLAN_CU(dcnt.alloc(3, st));
  if (!hv.empty()) PLAN_CU(cudaMemcpyAsync(dv.p, hv.data(), hv.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
  PLAN_CU(cudaMemcpyAsync(doff.p, voff.data(), voff.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  std::vector<int> hm(minds, minds + nshapes + 1);
  PLAN_CU(cudaMemcpyAsync(dm.p, hm.data(), hm.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  PLAN_CU(dcnt.zero());
  sm::Shapes sh{dv.p, doff.p, dm.p, nshapes};
  const unsigned blocks = (unsigned)((N + sm::PLAN_NT - 1) / sm::PLAN_NT);
  sm::k_smooth_plan<<<blocks, sm::PLAN_NT, 0, st>>>(sh, axis(p->Dx, p->Nx), axis(p->Dy, p->Ny), p->Nx, p->Ny,
                                                    fill_rule, p->code.p, p->rvol.p, p->nrm.p, dcnt.p);
  PLAN_CU(cudaGetLastError());
  unsigned long long hc[3];
  PLAN_CU(cudaMemcpyAsync(hc, dcnt.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
  PLAN_CU(cudaStreamSynchronize(st));
  for (int k = 0; k < 3; ++k) p->counts[k] = (long long)hc[k];
  p->nspecial = (int)(hc[1] + hc[2]);
  if (p->nspecial > 0) {
    DevBuf<unsigned int> dn;
    PLAN_CU(p->special.alloc(p->nspecial, st));
    PLAN_CU(dn.alloc(1, st));
    PLAN_CU(dn.zero());
    sm::k_smooth_list<<<blocks, sm::PLAN_NT, 0, st>>>(p->code.p, (long long)N, p->special.p, dn.p);
    PLAN_CU(cudaGetLastError());
    unsigned int hn = 0;
    PLAN_CU(cudaMemcpyAsync(&hn, dn.p, sizeof(hn), cudaMemcpyDeviceToHost, st));
    PLAN_CU(cudaStreamSynchronize(st));
    if ((int)hn != p->nspecial) return bail(fail(OMB_ERR_CUDA, "smoothing plan: inconsistent pixel list"));
    std::vector<int> hl(p->nspecial);
    PLAN_CU(cudaMemcpy(hl.data(), p->special.p, hl.size() * sizeof(int), cudaMemcpyDeviceToHost));
    std::sort(hl.begin(), hl.end());  // pixel order: deterministic sums in the VJP
    PLAN_CU(cudaMemcpyAsync(p->special.p, hl.data(), hl.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    PLAN_CU(cudaStreamSynchronize(st));
  }
#undef PLAN_CU
  *out = p;
  return OMB_OK;
}

extern "C" int omb_smoothing_plan_query(const omb_smoothing_plan* p, int64_t* counts, uint8_t* kind, int32_t* mats,
                                        double* rvol, double* normal) {
  int rc = check_plan(p);
  if (rc) return rc;
  if (counts)
    for (int k = 0; k < 3; ++k) counts[k] = p->counts[k];
  const size_t N = (size_t)p->Nx * p->Ny;
  cudaStream_t st = p->ctx->stream;
  OMB_CU(cudaSetDevice(p->ctx->device));
  if (kind || mats) {
    std::vector<uint2> c(N);
    OMB_CU(cudaMemcpyAsync(c.data(), p->code.p, N * sizeof(uint2), cudaMemcpyDeviceToHost, st));
    OMB_CU(cudaStreamSynchronize(st));
    for (size_t v = 0; v < N; ++v) {
      const int kd = c[v].x & 0xff;
      if (kind) kind[v] = (uint8_t)kd;
      if (mats) {
        int32_t* m = mats + 4 * v;
        m[0] = (int32_t)((c[v].x >> 8) & 0xff);
        m[1] = kd >= sm::KIND_INTERFACE ? (int32_t)((c[v].x >> 16) & 0xff) : -1;
        m[2] = kd == sm::KIND_MULTI ? (int32_t)((c[v].x >> 24) & 0xff) : -1;
        m[3] = kd == sm::KIND_MULTI ? (int32_t)(c[v].y & 0xff) : -1;
      }
    }
  }
  if (rvol) OMB_CU(cudaMemcpyAsync(rvol, p->rvol.p, N * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (normal) OMB_CU(cudaMemcpyAsync(normal, p->nrm.p, N * sizeof(double2), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaStreamSynchronize(st));
  return OMB_OK;
}

extern "C" int omb_smooth_eps(omb_smoothing_plan* p, const double* mat_vals, int32_t nmat, int32_t nsets,
                              double* eps, double* epsinv) {
  int rc = check_apply_args(p, mat_vals, nmat, nsets);
  if (rc) return rc;
  if (!eps && !epsinv) return fail(OMB_ERR_INVALID_ARG, "both outputs are NULL");
  cudaStream_t st = p->ctx->stream;
  OMB_CU(cudaSetDevice(p->ctx->device));
  const size_t N = (size_t)p->Nx * p->Ny, nm = 27 * (size_t)nmat * nsets;
  DevBuf<double> dmat, de, di;
  OMB_CU(dmat.alloc(nm, st));
  OMB_CU(cudaMemcpyAsync(dmat.p, mat_vals, nm * sizeof(double), cudaMemcpyHostToDevice, st));
  if (eps) OMB_CU(de.alloc(27 * N * nsets, st));
  if (epsinv) OMB_CU(di.alloc(9 * N * nsets, st));
  rc = apply_launch(p, dmat.p, nmat, nsets, de.p, di.p, st);
  if (rc) return rc;
  if (eps) OMB_CU(cudaMemcpyAsync(eps, de.p, 27 * N * nsets * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (epsinv) OMB_CU(cudaMemcpyAsync(epsinv, di.p, 9 * N * nsets * sizeof(double), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaStreamSynchronize(st));
  return OMB_OK;
}

extern "C" int omb_smooth_eps_device(omb_smoothing_plan* p, const double* mat_vals, int32_t nmat, int32_t nsets,
                                     double* d_eps, double* d_epsinv, void* stream) {
  int rc = check_apply_args(p, mat_vals, nmat, nsets);
  if (rc) return rc;
  if (!d_eps && !d_epsinv) return fail(OMB_ERR_INVALID_ARG, "both outputs are NULL");
  cudaStream_t st = stream ? (cudaStream_t)stream : p->ctx->stream;
  OMB_CU(cudaSetDevice(p->ctx->device));
  const size_t nm = 27 * (size_t)nmat * nsets;
  DevBuf<double> dmat;
  OMB_CU(dmat.alloc(nm, st));
  OMB_CU(cudaMemcpyAsync(dmat.p, mat_vals, nm * sizeof(double), cudaMemcpyHostToDevice, st));
  return apply_launch(p, dmat.p, nmat, nsets, d_eps, d_epsinv, st);
}

extern "C" int omb_smooth_eps_vjp(omb_smoothing_plan* p, const double* mat_vals, int32_t nmat, int32_t nsets,
                                  const double* eps_bar, double* mat_vals_bar) {
  int rc = check_apply_args(p, mat_vals, nmat, nsets);
  if (rc) return rc;
  if (!eps_bar || !mat_vals_bar) return fail(OMB_ERR_INVALID_ARG, "eps_bar and mat_vals_bar must be non-NULL");
  cudaStream_t st = p->ctx->stream;
  OMB_CU(cudaSetDevice(p->ctx->device));
  const long long N = (long long)p->Nx * p->Ny;
  const size_t nm = 27 * (size_t)nmat * nsets, ny = 27 * (size_t)N * nsets;
  const int ntiles = (int)((N + sm::BULK_NT - 1) / sm::BULK_NT);
  DevBuf<double> dmat, dy, dpart, dib, dout;
  OMB_CU(dmat.alloc(nm, st));
  OMB_CU(dy.alloc(ny, st));
  OMB_CU(dpart.alloc((size_t)ntiles * 27 * nmat * nsets, st));
  OMB_CU(dib.alloc(std::max<size_t>((size_t)p->nspecial * nsets * 54, 1), st));
  OMB_CU(dout.alloc(nm, st));
  OMB_CU(cudaMemcpyAsync(dmat.p, mat_vals, nm * sizeof(double), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaMemcpyAsync(dy.p, eps_bar, ny * sizeof(double), cudaMemcpyHostToDevice, st));
  sm::k_vjp_tiles<<<dim3((unsigned)ntiles, (unsigned)nsets), sm::BULK_NT, 0, st>>>(p->code.p, N, nmat, dy.p, dpart.p);
  OMB_CU(cudaGetLastError());
  if (p->nspecial > 0) {
    const long long work = (long long)p->nspecial * nsets * 54;
    sm::k_vjp_interface<<<(unsigned)((work + sm::SPECIAL_NT - 1) / sm::SPECIAL_NT), sm::SPECIAL_NT, 0, st>>>(
        p->special.p, p->nspecial, nsets, p->code.p, p->rvol.p, p->nrm.p, N, dmat.p, nmat, dy.p, dib.p);
    OMB_CU(cudaGetLastError());
  }
  sm::k_vjp_reduce<<<(unsigned)((nm + 127) / 128), 128, 0, st>>>(dpart.p, ntiles, dib.p, p->special.p, p->nspecial,
                                                                p->code.p, nmat, nsets, dout.p);
  OMB_CU(cudaGetLastError());
  OMB_CU(cudaMemcpyAsync(mat_vals_bar, dout.p, nm * sizeof(double), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaStreamSynchronize(st));
  return OMB_OK;
}

extern "C" int omb_smooth_scalar(omb_smoothing_plan* p, const double* vals, int32_t nmat, double* out) {
  int rc = check_apply_args(p, vals, nmat, 1);
  if (rc) return rc;
  if (!out) return fail(OMB_ERR_INVALID_ARG, "out is NULL");
  cudaStream_t st = p->ctx->stream;
  OMB_CU(cudaSetDevice(p->ctx->device));
  const long long N = (long long)p->Nx * p->Ny;
  DevBuf<double> dv, dout;
  OMB_CU(dv.alloc(nmat, st));
  OMB_CU(dout.alloc(N, st));
  OMB_CU(cudaMemcpyAsync(dv.p, vals, nmat * sizeof(double), cudaMemcpyHostToDevice, st));
  sm::k_smooth_scalar<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(p->code.p, p->rvol.p, N, dv.p, dout.p);
  OMB_CU(cudaGetLastError());
  OMB_CU(cudaMemcpyAsync(out, dout.p, N * sizeof(double), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaStreamSynchronize(st));
  return OMB_OK;
}

extern "C" int omb_smoothing_plan_destroy(omb_smoothing_plan* p) {
  if (!p) return OMB_OK;
  if (p->ctx) {
    cudaSetDevice(p->ctx->device);
    cudaDeviceSynchronize();  // applies on caller streams may still read the plan
  }
  delete p;
  return OMB_OK;
}
