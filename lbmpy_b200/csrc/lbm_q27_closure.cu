// D3Q27 cumulant sweep (orders >= 3 relaxed by 1) with the learned eddy-viscosity closure folded
// into the shear rate.  This translation unit owns the constant-memory copy of the closure
// parameters that its kernels read (c_closure); closure_upload writes it.
#include "lbm_closure.cuh"
#include "lbm_dispatch.h"

namespace lbm {

static __constant__ float c_closure[MLP_PARAMS];
// The parameters as the FP32 sweep's tensor-core network reads them (stage_mlp_params), built
// once per upload; each sweep block copies it into shared memory with 16-byte loads.
static __device__ MlpShared g_closure_image;

// Reads the parameters by name, so that the unrolled network addresses constant memory directly.
struct ConstClosureWeights {
    __device__ __forceinline__ float operator[](int i) const { return c_closure[i]; }
};

// The exact network from constant memory (the FP64 sweep: parity with the CPU oracle).
template <class R> struct ClosureNu {
    __device__ __forceinline__ R operator()(R pxx, R pyy, R pzz, R pxy, R pxz, R pyz, R rho, R ux, R uy,
                                            R uz) const {
        R x[MLP_IN];
        closure_features<R>(pxx, pyy, pzz, pxy, pxz, pyz, rho, ux, uy, uz, x);
        return closure_nu_t<R, ConstClosureWeights, true, false>(x, ConstClosureWeights{});
    }
};

// FP32: the network of the warp's 32 cells on the tensor cores (warp_mlp_nu).
struct WarpClosureNu {
    const MlpShared* s;
    uint32_t* X;
    __device__ __forceinline__ float operator()(float pxx, float pyy, float pzz, float pxy, float pxz, float pyz,
                                                float rho, float ux, float uy, float uz) const {
        float x[MLP_IN];
        closure_features<float, true>(pxx, pyy, pzz, pxy, pxz, pyz, rho, ux, uy, uz, x);
        return warp_mlp_nu(x, *s, X);
    }
};

// FP32 closure sweep.  The network works on whole warps, so no lane leaves early: lanes past the
// row end work on a clamped copy of the last cell and boundary cells collide their own (unused)
// values; only fluid cells inside the domain store.  Each thread sweeps a.zc consecutive planes
// (amortising the parameter staging) and prefetches the next plane to L2.  Otherwise as k_sweep.
template <int PAT>
__global__ void __launch_bounds__(256, 3) k_sweep_closure_tc(const SweepArgs a) {
    using A = Access<PAT>;
    __shared__ MlpShared sp;
    __shared__ __align__(16) uint32_t tiles[8][32 * MLP_XLD];
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    static_assert(sizeof(MlpShared) % 16 == 0, "the image is copied in 16-byte pieces");
    for (int i = tid; i < int(sizeof(MlpShared) / 16); i += blockDim.x * blockDim.y)
        reinterpret_cast<uint4*>(&sp)[i] = reinterpret_cast<const uint4*>(&g_closure_image)[i];
    __syncthreads();
    const WarpClosureNu nu{&sp, tiles[tid >> 5]};
    const Grid& g = a.g;
    const int xr = blockIdx.x * blockDim.x + threadIdx.x;
    const int yr = blockIdx.y * blockDim.y + threadIdx.y;
    const bool inside = xr < g.nx && yr < g.ny;
    const int x = min(xr, g.nx - 1), y = min(yr, g.ny - 1);
    const int z0 = blockIdx.z * a.zc;
    const int z1 = min(z0 + a.zc, g.nz);
    const float* src = static_cast<const float*>(a.src);
    float* dst = static_cast<float*>(a.dst);
#pragma unroll 1
    for (int z = z0; z < z1; ++z) {
        if (z + 1 < z1) prefetch_cell<float, 27, PAT>(a, x, y, z + 1);
        const int fl = (g.flags != nullptr && row_flagged(g, y, z)) ? g.flags[(x + 1) + (y + 1) * g.fsy + (z + 1) * g.fsz] : 0;
        NbrOffsets nb;
        nb.init(g, x, y, z);
        const int cell = (x + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
        float f[27];
#pragma unroll
        for (int i = 0; i < 27; ++i) {
            const int off = nb.off(A::template roff<27>(i, 0), A::template roff<27>(i, 1), A::template roff<27>(i, 2));
            f[i] = src[eidx(A::template rslot<27>(i) * g.sq, cell + off)];
        }
        const bool fluid = inside && !(fl & FLAG_TYPE_MASK);
        if (fluid && (fl & FLAG_NEAR_WALL)) bounce_back<float, float, 27, PAT>(f, a, nb, cell, x, y, z);
        __syncwarp();
        const float om = collide_cum_ho1<float, true>(f, a.p, nu);
        if (fluid) {
#pragma unroll
            for (int i = 0; i < 27; ++i) {
                const int off = nb.off(A::template woff<27>(i, 0), A::template woff<27>(i, 1), A::template woff<27>(i, 2));
                dst[eidx(A::template wslot<27>(i) * g.sq, cell + off)] = f[i];
            }
            if (a.omega_out != nullptr) a.omega_out[x + g.nx * (y + (long long)g.ny * z)] = om;
        }
    }
}

template <int PAT>
cudaError_t launch_closure_tc(const SweepArgs& a, dim3 grid, dim3 block, cudaStream_t s) {
    if (block.x * block.y != 256) return cudaErrorInvalidConfiguration;
    k_sweep_closure_tc<PAT><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

SweepLauncher sweep_q27_closure(int store, int pat) {
    if (store == ST_F64) {
        switch (pat) {
            case PAT_PULL: return &launch_sweep<double, double, 27, MK_CUM1_MLP, PAT_PULL>;
            case PAT_AA_EVEN: return &launch_sweep<double, double, 27, MK_CUM1_MLP, PAT_AA_EVEN>;
            case PAT_AA_ODD: return &launch_sweep<double, double, 27, MK_CUM1_MLP, PAT_AA_ODD>;
        }
    }
    if (store == ST_F32) {
        switch (pat) {
            case PAT_PULL: return &launch_closure_tc<PAT_PULL>;
            case PAT_AA_EVEN: return &launch_closure_tc<PAT_AA_EVEN>;
            case PAT_AA_ODD: return &launch_closure_tc<PAT_AA_ODD>;
        }
    }
    return nullptr;
}

__global__ void __launch_bounds__(256) k_closure_image() {
    stage_mlp_params(ConstClosureWeights{}, g_closure_image, threadIdx.x, blockDim.x);
}

cudaError_t closure_upload(const float* host_params, cudaStream_t stream) {
    cudaError_t e = cudaMemcpyToSymbolAsync(c_closure, host_params, sizeof(float) * MLP_PARAMS, 0,
                                            cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    k_closure_image<<<1, 256, 0, stream>>>();
    return cudaGetLastError();
}

}  // namespace lbm
