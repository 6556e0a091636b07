// D3Q27 cumulant sweep (orders >= 3 relaxed by 1) with the learned eddy-viscosity closure folded
// into the shear rate.  This translation unit owns the constant-memory copy of the closure
// parameters that its kernels read (c_closure); closure_upload writes it.
#include "lbm_closure.cuh"
#include "lbm_dispatch.h"

namespace lbm {

static __constant__ float c_closure[MLP_PARAMS];

// Reads the parameters by name, so that the unrolled network addresses constant memory directly.
struct ConstClosureWeights {
    __device__ __forceinline__ float operator[](int i) const { return c_closure[i]; }
};

// FP64: the exact network (parity with the CPU oracle); FP32: the hardware-tanh SiLU.
template <class R> struct ClosureNu {
    __device__ __forceinline__ R operator()(R pxx, R pyy, R pzz, R pxy, R pxz, R pyz, R rho, R ux, R uy,
                                            R uz) const {
        R x[MLP_IN];
        closure_features<R>(pxx, pyy, pzz, pxy, pxz, pyz, rho, ux, uy, uz, x);
        return closure_nu_t<R, ConstClosureWeights, true, std::is_same<R, float>::value>(x, ConstClosureWeights{});
    }
};

template <class S, class R>
static SweepLauncher closure_sweep_pat(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_sweep<S, R, 27, MK_CUM1_MLP, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_sweep<S, R, 27, MK_CUM1_MLP, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_sweep<S, R, 27, MK_CUM1_MLP, PAT_AA_ODD>;
    }
    return nullptr;
}

SweepLauncher sweep_q27_closure(int store, int pat) {
    if (store == ST_F64) return closure_sweep_pat<double, double>(pat);
    if (store == ST_F32) return closure_sweep_pat<float, float>(pat);
    return nullptr;
}

cudaError_t closure_upload(const float* host_params, cudaStream_t stream) {
    return cudaMemcpyToSymbolAsync(c_closure, host_params, sizeof(float) * MLP_PARAMS, 0, cudaMemcpyHostToDevice,
                                   stream);
}

}  // namespace lbm
