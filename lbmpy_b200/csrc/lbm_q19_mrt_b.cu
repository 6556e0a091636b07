// Kernel instantiations, part B: D3Q19, MRT collision; the pair, quad and staged sweeps.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_B(q19_mrt, 19, MK_MRT)
}  // namespace lbm
