// Kernel instantiations, part A: D3Q27, central-moment collision (FP64 / FP32 storage, pull and
// AA); the one-cell, batched and sparse sweeps, the boundary pre-pass and the setter.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_REDUCED_A(q27_cm, 27, MK_CM)
}  // namespace lbm
