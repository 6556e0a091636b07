// Kernel instantiations, part A: D3Q27, SRT/TRT collision, every storage type and pattern; the
// one-cell, batched and sparse sweeps, the boundary pre-pass and the setter.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_A(q27_pop, 27, MK_POP)
}  // namespace lbm
