// Kernel instantiations: D3Q19, MRT collision, every storage type and pattern.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY(q19_mrt, 19, MK_MRT)
}  // namespace lbm
