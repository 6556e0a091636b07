// Kernel instantiations, part A: D3Q27, cumulant collision with every order >= 3 relaxed by 1,
// every storage type and pattern; the one-cell, batched and sparse sweeps, the boundary pre-pass
// and the setter.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_A(q27_cum1, 27, MK_CUM1)
}  // namespace lbm
