// Kernel instantiations, part B: D3Q27, cumulant collision with every order >= 3 relaxed by 1; the
// pair, quad and staged sweeps.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_B(q27_cum1, 27, MK_CUM1)
}  // namespace lbm
