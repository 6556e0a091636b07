// Kernel instantiations: D3Q27, POP collision, every storage type and pattern.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY(q27_pop, 27, MK_POP)
}  // namespace lbm
