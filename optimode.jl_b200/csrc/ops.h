// Host-side launchers for the fused operator passes.
#pragma once

#include "op_kernels.cuh"

namespace omb {

// Operator pipelines built from the row_in / col / row_out passes.
enum OpKind : int {
  OP_M = 0,       // Hout = M̂(k) Hin                       (_M!)
  OP_P = 1,       // Hout = P̂(k) Hin, MPB-style              (_P!)
  OP_HMKH = 2,    // partial sums of ⟨Hin, kx_ct bfft ε⁻¹ fft zx_tc Hin⟩/N  (HMₖH)
  OP_EFIELD = 3,  // scratch ← ε⁻¹·fft2(kx_tc Hin)            (E⃗, un-normalised)
  OP_H2D = 4,     // scratch ← fft2(kx_tc Hin)                (_H2d!)
  OP_D2E = 5,     // out (planar 3N) ← bfft2(ε⁻¹·scratch)     (_d2ẽ!)
  OP_MDOT = 6,    // like OP_M but reduces ⟨Hin, M̂ Hin⟩ partials instead of storing
  OP_HFIELD = 7,  // scratch ← fft2(h1 m̂ + h2 n̂): the Cartesian H field in real space
  OP_R2G = 8,     // scratch ← bfft2(planar 3-component in): real space back to plane waves
};

// Twiddle tables exp(-2πi m/L) for every supported length, per precision.
struct TwTables {
  const float2* f32[1025];
  const double2* f64[1025];
};

bool fft_size_supported(int L);

// Tile variants of the FP32 M̂ passes (0, 1, 2: half, default, double the rows per CTA of the
// row passes / columns per CTA of the column pass; row 3: row_in with one thread per line
// slot and field component, row 4: both row passes so; column 3 and 4: the column pass so,
// with a register budget for three or two CTAs per SM; column 5: the default tile with a
// budget for four; rows 5 and 6: the whole M̂ application in one kernel on thread-block
// clusters of 8 or 16 CTAs (op_cluster.cuh) where the grid has that kernel, the column and
// wave choices then unused) and the wave size (0: every column in one
// launch of each pass; w > 0: the units are cut into waves of about wave_columns(w) columns,
// each wave running its three passes while its intermediate stays in L2), chosen per grid by
// the autotuner (tune.cu); grids never tuned use the defaults.
struct TileChoice {
  int row = 1, col = 1, wave = 0;
};
constexpr int ROW_VARIANTS = 7;
constexpr int ROW_CLUSTER = 5, ROW_CLUSTER16 = 6;
constexpr int COL_VARIANTS = 6;
constexpr int WAVE_VARIANTS = 4;
__host__ __device__ constexpr int wave_columns(int w) { return w == 1 ? 32 : w == 2 ? 64 : w == 3 ? 128 : 0; }
TileChoice tiles_for(int Nx, int Ny);  // for the calling thread's current device
// Raise a kernel's dynamic shared-memory limit once per (kernel, device), and with
// `max_shared` ask for the whole L1/shared carve-out; later calls for the same or a smaller
// size return without touching the driver (so they are safe inside a stream capture after a
// warm-up launch).
cudaError_t ensure_smem(const void* func, size_t bytes, bool max_shared = false);
// Clusters of `cluster_ctas` CTAs of `threads` threads and `smem` dynamic shared bytes that can
// be resident at once on the current device (cudaOccupancyMaxActiveClusters, cached per kernel
// and device; at least 1).
int cluster_slots(const void* func, int cluster_ctas, int threads, size_t smem);
// Whether the one-kernel cluster apply exists for this grid (FP32 M̂).
bool cluster_apply_available(int Nx, int Ny);
// Number of row blocks row_out uses for a grid with Ny rows (partial sums per column).
int row_blocks(int Nx, int Ny);

template <typename T>
cudaError_t launch_op(OpKind op, const OpUnit<T>* d_units, int nunits, int Nx, int Ny, int maxcol,
                      const TwTables& tw, cudaStream_t st);
// The same pipelines on z-periodic cells (Nz slabs; ops3d.cuh); `expand` is device memory for
// (Nz + 1)·nunits units.
template <typename T>
cudaError_t launch_op3d(OpKind op, const OpUnit<T>* d_units, int nunits, int Nx, int Ny, int Nz, int maxcol,
                        const TwTables& tw, OpUnit<T>* expand, cudaStream_t st);

}  // namespace omb
