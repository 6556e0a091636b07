// Kernel instantiations, part B: D3Q27, cumulant collision with every order >= 3 relaxed by 1; the
// pair, quad and staged sweeps, and the pipelined z-column sweep.
#include "lbm_dispatch.h"

namespace lbm {
LBM_DEFINE_FAMILY_B(q27_cum1, 27, MK_CUM1)

SweepLauncher sweep_zpipe_q27_cum1(int store, int pat) {
    if (store != ST_F32) return nullptr;
    switch (pat) {
        case PAT_PULL: return &launch_sweep_zpipe<float, float, 27, MK_CUM1, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_sweep_zpipe<float, float, 27, MK_CUM1, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_sweep_zpipe<float, float, 27, MK_CUM1, PAT_AA_ODD>;
    }
    return nullptr;
}
}  // namespace lbm
