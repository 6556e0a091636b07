// Kernel instantiations: D3Q19, POP collision, every storage type and pattern.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY(q19_pop, 19, MK_POP)
}  // namespace lbm
