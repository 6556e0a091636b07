// Kernel instantiations: D3Q27 cumulant with every order >= 3 relaxed by 1, every storage type and pattern.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY(q27_cum1, 27, MK_CUM1)
}  // namespace lbm
