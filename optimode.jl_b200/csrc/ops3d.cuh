// Operator pipelines on z-periodic (3D) cells, built from the 2D passes of ops_impl.cuh.
//
// A 3D field (component, x, y, z) is transformed as Nz slabs along x and y, and as Nx·Ny
// lines along z:
//   * slab units: one per (unit, z-slab); the row pass (x) and the column pass (y) of the
//     2D operator act on the slab, with the slab's g_z subtracted from k in the basis
//     (w = k ẑ − G) and the planar components Nx·Ny·Nz apart;
//   * line units: one per unit; the 2D column kernel run with "columns" = the Nx·Ny pixels
//     of a slab and "rows" = the Nz slabs (stride Nx·Ny), where the per-pixel step (ε⁻¹, ε_ave)
//     sits between the forward and inverse z-transforms.
// M̂ = row_out(x) · col(y⁻¹) · [z · ε⁻¹ · z⁻¹] · col(y) · row_in(x), and the same pattern for
// P̂, HMₖH, E, H2D and D2E.  The expanded units are written on the device from the caller's
// units by one small kernel (so a captured graph replays them with the caller's current k
// and column counts).
#pragma once

#include "ops_impl.cuh"

namespace omb {

// How the slab offset applies to a unit's input / output: 2-component interleaved fields
// (offset 2·Nx·Ny per slab) or planar 3-component fields (offset Nx·Ny).
enum SlabLayout : int { SL_IN_H = 1, SL_IN_PLANAR = 2, SL_OUT_H = 4, SL_OUT_PLANAR = 8 };

template <typename T>
__global__ void k_expand_units3d(const OpUnit<T>* __restrict__ base, int nunits, int Nx, int Ny, int Nz, int layout,
                                 int rb, OpUnit<T>* __restrict__ slab, OpUnit<T>* __restrict__ line) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const long long S = (long long)Nx * Ny, N3 = S * Nz;
  if (i < nunits * Nz) {
    const int u = i / Nz, s = i - u * Nz;
    OpUnit<T> v = base[u];
    const long long in_off = (layout & SL_IN_H) ? 2 * S * s : S * s;
    const long long out_off = (layout & SL_OUT_H) ? 2 * S * s : S * s;
    if (v.in) v.in += in_off;
    if (v.out) v.out += out_off;
    if (v.scr) v.scr += S * s;
    if (v.partial) v.partial += 2 * (long long)rb * s;
    v.Nx = Nx;
    v.Ny = Ny;
    v.comp_stride = N3;
    v.kz_shift = freq_index(s, Nz) * v.inv_dz;
    slab[i] = v;
  }
  if (i < nunits) {
    OpUnit<T> v = base[i];
    v.Nx = Nx * Ny;  // the column kernel's "x" runs over the pixels of a slab
    v.Ny = Nz;
    v.comp_stride = N3;
    v.kz_shift = 0;
    line[i] = v;
  }
}

template <typename T>
cudaError_t launch_op3d(OpKind op, const OpUnit<T>* u, int nunits, int Nx, int Ny, int Nz, int maxcol,
                        const TwTables& t, OpUnit<T>* expand, cudaStream_t st) {
  if (nunits <= 0 || maxcol <= 0) return cudaSuccess;
  OpUnit<T>* slab = expand;
  OpUnit<T>* line = expand + (size_t)nunits * Nz;
  int layout = SL_IN_H | SL_OUT_H;
  if (op == OP_EFIELD || op == OP_H2D) layout = SL_IN_H | SL_OUT_PLANAR;
  if (op == OP_D2E) layout = SL_IN_PLANAR | SL_OUT_PLANAR;
  const int rb = row_blocks(Nx, Ny);
  const int n = nunits * Nz;
  k_expand_units3d<T><<<(n + 127) / 128, 128, 0, st>>>(u, nunits, Nx, Ny, Nz, layout, rb, slab, line);
  OMB_TRY(cudaGetLastError());
  const int NxNy = Nx * Ny;
  switch (op) {
    case OP_M:
    case OP_MDOT:
      OMB_TRY(row_in<T>(RI_KXTC, slab, n, Nx, Ny, maxcol, t, st));
      OMB_TRY(col<T>(CM_FWD, slab, n, Nx, Ny, maxcol, t, st));
      OMB_TRY(col<T>(CM_M, line, nunits, NxNy, Nz, maxcol, t, st));
      OMB_TRY(col<T>(CM_BWD, slab, n, Nx, Ny, maxcol, t, st));
      return row_out<T>(op == OP_M ? RO_KXCT : RO_KXCT_DOT, slab, n, Nx, Ny, maxcol, t, st);
    case OP_HMKH:
      OMB_TRY(row_in<T>(RI_ZXTC, slab, n, Nx, Ny, maxcol, t, st));
      OMB_TRY(col<T>(CM_FWD, slab, n, Nx, Ny, maxcol, t, st));
      OMB_TRY(col<T>(CM_M, line, nunits, NxNy, Nz, maxcol, t, st));
      OMB_TRY(col<T>(CM_BWD, slab, n, Nx, Ny, maxcol, t, st));
      return row_out<T>(RO_KXCT_DOT, slab, n, Nx, Ny, maxcol, t, st);
    case OP_P:
      OMB_TRY(row_in<T>(RI_KXINV, slab, n, Nx, Ny, maxcol, t, st));
      OMB_TRY(col<T>(CM_BWD, slab, n, Nx, Ny, maxcol, t, st));
      OMB_TRY(col<T>(CM_P, line, nunits, NxNy, Nz, maxcol, t, st));
      OMB_TRY(col<T>(CM_FWD, slab, n, Nx, Ny, maxcol, t, st));
      return row_out<T>(RO_KXINVCT, slab, n, Nx, Ny, maxcol, t, st);
    case OP_EFIELD:
      OMB_TRY(row_in<T>(RI_KXTC, slab, n, Nx, Ny, maxcol, t, st));
      OMB_TRY(col<T>(CM_FWD, slab, n, Nx, Ny, maxcol, t, st));
      return col<T>(CM_E, line, nunits, NxNy, Nz, maxcol, t, st);
    case OP_H2D:
      OMB_TRY(row_in<T>(RI_KXTC, slab, n, Nx, Ny, maxcol, t, st));
      OMB_TRY(col<T>(CM_FWD, slab, n, Nx, Ny, maxcol, t, st));
      return col<T>(CM_FWD, line, nunits, NxNy, Nz, maxcol, t, st);
    case OP_D2E:
      OMB_TRY(col<T>(CM_EPSINV, line, nunits, NxNy, Nz, maxcol, t, st));
      OMB_TRY(col<T>(CM_BWD, slab, n, Nx, Ny, maxcol, t, st));
      return row_out<T>(RO_STORE3, slab, n, Nx, Ny, maxcol, t, st);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace omb
