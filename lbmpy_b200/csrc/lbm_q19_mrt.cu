// Kernel instantiations, part A: D3Q19, MRT collision, every storage type and pattern; the
// one-cell, batched and sparse sweeps, the boundary pre-pass and the setter.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_A(q19_mrt, 19, MK_MRT)
}  // namespace lbm
