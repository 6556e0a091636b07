// Kernel instantiations: D3Q27, CUM collision, every storage type and pattern.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY(q27_cum, 27, MK_CUM)
}  // namespace lbm
