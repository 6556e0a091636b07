// Kernel instantiations, part B: D3Q27, SRT/TRT collision; the pair, quad and staged sweeps.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_B(q27_pop, 27, MK_POP)
}  // namespace lbm
