// Learned warm-start network (warmstart.cu): internal interface for the solver.
#pragma once

#include <stdint.h>

#include <array>
#include <vector>

#include "context.h"

namespace omb {

constexpr int WS_LAYERS = 6;
int64_t ws_num_params();
// Forward pass on `B` device feature images (128×128×8 BF16 each); *out receives the
// network's output buffer, [B·64·64 × 16] FP32 (channels 0..11 valid).
int ws_forward_dev(omb_warmstart* W, const void* feat, int B, float** out);
// Learned starting blocks for uploaded cells (128² or 256²) at frequencies `omegas`: four FP64
// device columns (2N each, the (h1, h2) plane-wave coefficients of bands 0..3) per cell at
// cols + col_off[i], and per band the Newton start kb = n_eff·ω from the network (the cell's
// k_guess when the network's n_eff leaves (1, 4)); the columns are projected at kb.
int ws_guesses(omb_warmstart* W, const std::vector<const Problem*>& probs, const std::vector<double>& omegas,
               DevBuf<double2>& cols, std::vector<size_t>& col_off, std::vector<std::array<double, 4>>& kb);

}  // namespace omb
