// Kernel instantiations, part B: D3Q27, cumulant collision with general rates; the pair, quad and
// staged sweeps.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_B(q27_cum, 27, MK_CUM)
}  // namespace lbm
