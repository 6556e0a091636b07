// Kernel instantiations, part B: D3Q27, central-moment collision (FP64 / FP32 storage, pull and
// AA); the pair and staged sweeps.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_REDUCED_B(q27_cm, 27, MK_CM)
}  // namespace lbm
