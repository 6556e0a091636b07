// Kernel instantiations, part A: D3Q27, MRT collision (FP64 / FP32 storage, pull and AA); the
// one-cell, batched and sparse sweeps, the boundary pre-pass and the setter.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_REDUCED_A(q27_mrt, 27, MK_MRT)
}  // namespace lbm
