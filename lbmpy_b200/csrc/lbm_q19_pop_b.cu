// Kernel instantiations, part B: D3Q19, SRT/TRT collision; the pair, quad and staged sweeps.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_B(q19_pop, 19, MK_POP)
}  // namespace lbm
