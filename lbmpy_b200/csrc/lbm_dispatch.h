// Launcher tables: one instantiated kernel per (stencil, method, storage type, pattern).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <type_traits>

#include "lbm_quad.cuh"
#include "lbm_staged.cuh"

namespace lbm {

using SweepLauncher = cudaError_t (*)(const SweepArgs&, dim3, dim3, cudaStream_t);
using MacroLauncher = cudaError_t (*)(const MacroArgs&, dim3, dim3, cudaStream_t);

template <class S, class R, int Q, int MK, int PAT>
cudaError_t launch_sweep(const SweepArgs& a, dim3 grid, dim3 block, cudaStream_t s) {
    k_sweep<S, R, Q, MK, PAT><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

template <class S, class R, int Q, int MK, int PAT>
cudaError_t launch_set_eq(const MacroArgs& a, dim3 grid, dim3 block, cudaStream_t s) {
    k_set_equilibrium<S, R, Q, MK, PAT><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

template <class S, int Q, int MK, int PAT>
cudaError_t launch_sweep_pair(const SweepArgs& a, dim3 grid, dim3 block, cudaStream_t s) {
    k_sweep_pair<S, Q, MK, PAT><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

template <class S, int Q, int MK>
SweepLauncher pick_pair_pattern(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_sweep_pair<S, Q, MK, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_sweep_pair<S, Q, MK, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_sweep_pair<S, Q, MK, PAT_AA_ODD>;
    }
    return nullptr;
}

template <class S, int Q, int MK, int PAT>
cudaError_t launch_sweep_quad(const SweepArgs& a, dim3 grid, dim3 block, cudaStream_t s) {
    k_sweep_quad<S, Q, MK, PAT><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

template <class S, int Q, int MK>
SweepLauncher pick_quad_pattern(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_sweep_quad<S, Q, MK, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_sweep_quad<S, Q, MK, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_sweep_quad<S, Q, MK, PAT_AA_ODD>;
    }
    return nullptr;
}

// Staged sweep: the launcher sizes the persistent grid itself (resident CTAs per SM x SMs, at
// most one CTA per tile).  W = cells per tile = threads per CTA.
using StagedLauncher = cudaError_t (*)(const SweepArgs&, int ns, int sms, cudaStream_t);

template <class S> struct StagedWidth { static constexpr int value = 128; };
template <> struct StagedWidth<double> { static constexpr int value = 128; };

template <class S, class R, int Q, int MK, int PAT>
cudaError_t launch_sweep_staged(const SweepArgs& a, int ns, int sms, cudaStream_t s) {
    constexpr int W = StagedWidth<S>::value;
    using Lay = StagedLayout<S, Q, W>;
    if (ns < 2 || ns > STAGED_MAX_NS) return cudaErrorInvalidValue;
    auto kern = &k_sweep_staged<S, R, Q, MK, PAT, W>;
    const size_t smem = Lay::smem_bytes(ns);
    // resident CTAs per SM for the last stage count asked for, packed as ns << 8 | blocks
    static std::atomic<int> cached{0};
    const int c = cached.load(std::memory_order_relaxed);
    int per_sm = c & 255;
    if ((c >> 8) != ns) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, W, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        per_sm = per_sm > 255 ? 255 : per_sm;
        cached.store((ns << 8) | per_sm, std::memory_order_relaxed);
    }
    const long long tiles = (long long)((a.g.nx + W - 1) / W) * a.g.ny * a.g.nz;
    const long long slots = (long long)per_sm * sms;
    const unsigned grid = (unsigned)(tiles < slots ? tiles : slots);
    kern<<<grid, W, smem, s>>>(a, ns);
    return cudaGetLastError();
}

template <class S, class R, int Q, int MK>
StagedLauncher pick_staged_pattern(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_sweep_staged<S, R, Q, MK, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_sweep_staged<S, R, Q, MK, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_sweep_staged<S, R, Q, MK, PAT_AA_ODD>;
    }
    return nullptr;
}

using SparseLauncher = cudaError_t (*)(const SparseArgs&, cudaStream_t);
using SparseSetLauncher = cudaError_t (*)(const SparseArgs&, const double*, const double*, cudaStream_t);

template <class S, class R, int Q, int MK>
cudaError_t launch_sparse(const SparseArgs& a, cudaStream_t s) {
    const long long blocks = (a.n_fluid + 255) / 256;
    k_sweep_sparse<S, R, Q, MK><<<(unsigned)blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <class S, class R, int Q, int MK>
cudaError_t launch_sparse_set(const SparseArgs& a, const double* rho, const double* u, cudaStream_t s) {
    const long long blocks = (a.n_fluid + 255) / 256;
    k_sparse_set_equilibrium<S, R, Q, MK><<<(unsigned)blocks, 256, 0, s>>>(a, rho, u);
    return cudaGetLastError();
}

template <class S, class R, int Q, int MK, int PAT>
cudaError_t launch_sweep_zpipe(const SweepArgs& a, dim3 grid, dim3 block, cudaStream_t s) {
    k_sweep_zpipe<S, R, Q, MK, PAT><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

using BatchLauncher = cudaError_t (*)(const BatchArgs&, dim3, dim3, cudaStream_t);

template <class S, class R, int Q, int MK, int PAT>
cudaError_t launch_batched(const BatchArgs& b, dim3 grid, dim3 block, cudaStream_t s) {
    k_sweep_batched<S, R, Q, MK, PAT><<<grid, block, 0, s>>>(b);
    return cudaGetLastError();
}

template <class S, class R, int Q, int MK>
BatchLauncher pick_batched_pattern(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_batched<S, R, Q, MK, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_batched<S, R, Q, MK, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_batched<S, R, Q, MK, PAT_AA_ODD>;
    }
    return nullptr;
}

template <class S, class R, int Q, int MK>
SweepLauncher pick_sweep_pattern(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_sweep<S, R, Q, MK, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_sweep<S, R, Q, MK, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_sweep<S, R, Q, MK, PAT_AA_ODD>;
    }
    if constexpr (std::is_same<S, e3m12>::value) {
        return nullptr;   // e3m12: pull and AA
    } else {
        switch (pat) {
            case PAT_ESO_EVEN: return &launch_sweep<S, R, Q, MK, PAT_ESO_EVEN>;
            case PAT_ESO_ODD: return &launch_sweep<S, R, Q, MK, PAT_ESO_ODD>;
        }
        if constexpr (sizeof(S) >= 4) {
            switch (pat) {
                case PAT_PUSH: return &launch_sweep<S, R, Q, MK, PAT_PUSH>;
                case PAT_EPULL_EVEN: return &launch_sweep<S, R, Q, MK, PAT_EPULL_EVEN>;
                case PAT_EPULL_ODD: return &launch_sweep<S, R, Q, MK, PAT_EPULL_ODD>;
                case PAT_EPUSH_EVEN: return &launch_sweep<S, R, Q, MK, PAT_EPUSH_EVEN>;
                case PAT_EPUSH_ODD: return &launch_sweep<S, R, Q, MK, PAT_EPUSH_ODD>;
            }
        }
        return nullptr;
    }
}

template <class S, class R, int Q, int MK, int PAT>
cudaError_t launch_prepass(const SweepArgs& a, dim3 grid, dim3 block, cudaStream_t s) {
    k_boundary_prepass<S, R, Q, MK, PAT><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

template <class S, class R, int Q, int MK>
SweepLauncher pick_prepass_pattern(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_prepass<S, R, Q, MK, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_prepass<S, R, Q, MK, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_prepass<S, R, Q, MK, PAT_AA_ODD>;
    }
    if constexpr (std::is_same<S, e3m12>::value) {
        return nullptr;   // e3m12: pull and AA
    } else {
        switch (pat) {
            case PAT_ESO_EVEN: return &launch_prepass<S, R, Q, MK, PAT_ESO_EVEN>;
            case PAT_ESO_ODD: return &launch_prepass<S, R, Q, MK, PAT_ESO_ODD>;
        }
        if constexpr (sizeof(S) >= 4) {
            switch (pat) {
                case PAT_PUSH: return &launch_prepass<S, R, Q, MK, PAT_PUSH>;
                case PAT_EPULL_EVEN: return &launch_prepass<S, R, Q, MK, PAT_EPULL_EVEN>;
                case PAT_EPULL_ODD: return &launch_prepass<S, R, Q, MK, PAT_EPULL_ODD>;
                case PAT_EPUSH_EVEN: return &launch_prepass<S, R, Q, MK, PAT_EPUSH_EVEN>;
                case PAT_EPUSH_ODD: return &launch_prepass<S, R, Q, MK, PAT_EPUSH_ODD>;
            }
        }
        return nullptr;
    }
}

template <class S, class R, int Q, int MK>
MacroLauncher pick_set_eq_pattern(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_set_eq<S, R, Q, MK, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_set_eq<S, R, Q, MK, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_set_eq<S, R, Q, MK, PAT_AA_ODD>;
    }
    if constexpr (std::is_same<S, e3m12>::value) {
        return nullptr;   // e3m12: pull and AA
    } else {
        switch (pat) {
            case PAT_ESO_EVEN: return &launch_set_eq<S, R, Q, MK, PAT_ESO_EVEN>;
            case PAT_ESO_ODD: return &launch_set_eq<S, R, Q, MK, PAT_ESO_ODD>;
        }
        if constexpr (sizeof(S) >= 4) {
            switch (pat) {
                case PAT_PUSH: return &launch_set_eq<S, R, Q, MK, PAT_PUSH>;
                case PAT_EPULL_EVEN: return &launch_set_eq<S, R, Q, MK, PAT_EPULL_EVEN>;
                case PAT_EPULL_ODD: return &launch_set_eq<S, R, Q, MK, PAT_EPULL_ODD>;
                case PAT_EPUSH_EVEN: return &launch_set_eq<S, R, Q, MK, PAT_EPUSH_EVEN>;
                case PAT_EPUSH_ODD: return &launch_set_eq<S, R, Q, MK, PAT_EPUSH_ODD>;
            }
        }
        return nullptr;
    }
}

// Instantiates the sweep and setter families of one (Q, method) pair in one translation unit.
// The setter always evaluates the equilibrium in FP64 from FP64 density / velocity fields, so
// that the density deviation rho - 1 keeps its digits before the PDFs are rounded to storage.
// The families are instantiated in two translation units each (part A: the one-cell sweep, the
// batched sweep, the boundary pre-pass, the sparse sweeps and the setter; part B: the pair, quad
// and staged sweeps), so that the build compiles them in parallel.
#define LBM_DEFINE_FAMILY_A(NAME, Q, MK)                                                          \
    SweepLauncher sweep_##NAME(int store, int pat) {                                            \
        switch (store) {                                                                        \
            case ST_F64: return pick_sweep_pattern<double, double, Q, MK>(pat);                  \
            case ST_F32: return pick_sweep_pattern<float, float, Q, MK>(pat);                    \
            case ST_F16: return pick_sweep_pattern<__half, float, Q, MK>(pat);                   \
            case ST_BF16: return pick_sweep_pattern<__nv_bfloat16, float, Q, MK>(pat);          \
            case ST_E3M12: return pick_sweep_pattern<e3m12, float, Q, MK>(pat);                 \
        }                                                                                       \
        return nullptr;                                                                         \
    }                                                                                           \
    BatchLauncher batched_##NAME(int store, int pat) {                                          \
        if (store == ST_F64) return pick_batched_pattern<double, double, Q, MK>(pat);           \
        if (store == ST_F32) return pick_batched_pattern<float, float, Q, MK>(pat);             \
        return nullptr;                                                                         \
    }                                                                                           \
    SweepLauncher prepass_##NAME(int store, int pat) {                                    \
        switch (store) {                                                                        \
            case ST_F64: return pick_prepass_pattern<double, double, Q, MK>(pat);          \
            case ST_F32: return pick_prepass_pattern<float, float, Q, MK>(pat);            \
            case ST_F16: return pick_prepass_pattern<__half, float, Q, MK>(pat);           \
            case ST_BF16: return pick_prepass_pattern<__nv_bfloat16, float, Q, MK>(pat);  \
            case ST_E3M12: return pick_prepass_pattern<e3m12, float, Q, MK>(pat);         \
        }                                                                                       \
        return nullptr;                                                                         \
    }                                                                                           \
    SparseLauncher sparse_##NAME(int store) {                                                   \
        if (store == ST_F64) return &launch_sparse<double, double, Q, MK>;                      \
        if (store == ST_F32) return &launch_sparse<float, float, Q, MK>;                        \
        return nullptr;                                                                         \
    }                                                                                           \
    SparseSetLauncher sparse_set_##NAME(int store) {                                            \
        if (store == ST_F64) return &launch_sparse_set<double, double, Q, MK>;                  \
        if (store == ST_F32) return &launch_sparse_set<float, double, Q, MK>;                   \
        return nullptr;                                                                         \
    }                                                                                           \
    MacroLauncher set_eq_##NAME(int store, int pat) {                                           \
        switch (store) {                                                                        \
            case ST_F64: return pick_set_eq_pattern<double, double, Q, MK>(pat);                 \
            case ST_F32: return pick_set_eq_pattern<float, double, Q, MK>(pat);                   \
            case ST_F16: return pick_set_eq_pattern<__half, double, Q, MK>(pat);                  \
            case ST_BF16: return pick_set_eq_pattern<__nv_bfloat16, double, Q, MK>(pat);         \
            case ST_E3M12: return pick_set_eq_pattern<e3m12, double, Q, MK>(pat);                \
        }                                                                                       \
        return nullptr;                                                                         \
    }

#define LBM_DEFINE_FAMILY_B(NAME, Q, MK)                                                          \
    SweepLauncher sweep_quad_##NAME(int store, int pat) {                                       \
        switch (store) {                                                                        \
            case ST_F16: return pick_quad_pattern<__half, Q, MK>(pat);                           \
            case ST_BF16: return pick_quad_pattern<__nv_bfloat16, Q, MK>(pat);                  \
            case ST_E3M12: return pick_quad_pattern<e3m12, Q, MK>(pat);                         \
        }                                                                                       \
        return nullptr;                                                                         \
    }                                                                                           \
    StagedLauncher sweep_staged_##NAME(int store, int pat) {                                    \
        switch (store) {                                                                        \
            case ST_F64: return pick_staged_pattern<double, double, Q, MK>(pat);                 \
            case ST_F32: return pick_staged_pattern<float, float, Q, MK>(pat);                   \
            case ST_F16: return pick_staged_pattern<__half, float, Q, MK>(pat);                  \
            case ST_BF16: return pick_staged_pattern<__nv_bfloat16, float, Q, MK>(pat);         \
        }                                                                                       \
        return nullptr;                                                                         \
    }                                                                                           \
    SweepLauncher sweep_pair_##NAME(int store, int pat) {                                       \
        switch (store) {                                                                        \
            case ST_F32: return pick_pair_pattern<float, Q, MK>(pat);                            \
            case ST_F16: return pick_pair_pattern<__half, Q, MK>(pat);                           \
            case ST_BF16: return pick_pair_pattern<__nv_bfloat16, Q, MK>(pat);                  \
            case ST_E3M12: return pick_pair_pattern<e3m12, Q, MK>(pat);                         \
        }                                                                                       \
        return nullptr;                                                                         \
    }

// Reduced family (FP64 / FP32 storage, pull and AA): for bases whose fully unrolled 27x27
// transforms make every extra instantiation expensive to compile.
#define LBM_DEFINE_FAMILY_REDUCED_A(NAME, Q, MK)                                              \
    template <class S, class R>                                                                 \
    static SweepLauncher NAME##_sweep_pat(int pat) {                                            \
        switch (pat) {                                                                          \
            case PAT_PULL: return &launch_sweep<S, R, Q, MK, PAT_PULL>;                         \
            case PAT_AA_EVEN: return &launch_sweep<S, R, Q, MK, PAT_AA_EVEN>;                   \
            case PAT_AA_ODD: return &launch_sweep<S, R, Q, MK, PAT_AA_ODD>;                     \
        }                                                                                       \
        return nullptr;                                                                         \
    }                                                                                           \
    template <class S, class R>                                                                 \
    static MacroLauncher NAME##_set_pat(int pat) {                                              \
        switch (pat) {                                                                          \
            case PAT_PULL: return &launch_set_eq<S, R, Q, MK, PAT_PULL>;                        \
            case PAT_AA_EVEN: return &launch_set_eq<S, R, Q, MK, PAT_AA_EVEN>;                  \
            case PAT_AA_ODD: return &launch_set_eq<S, R, Q, MK, PAT_AA_ODD>;                    \
        }                                                                                       \
        return nullptr;                                                                         \
    }                                                                                           \
    BatchLauncher batched_##NAME(int store, int pat) {                                          \
        if (store == ST_F32) return pick_batched_pattern<float, float, Q, MK>(pat);             \
        return nullptr;                                                                         \
    }                                                                                           \
    SweepLauncher sweep_quad_##NAME(int, int) { return nullptr; }                               \
    SweepLauncher prepass_##NAME(int store, int pat) {                                    \
        if (pat != PAT_PULL && pat != PAT_AA_EVEN && pat != PAT_AA_ODD) return nullptr;          \
        if (store == ST_F64) return pick_prepass_pattern<double, double, Q, MK>(pat);     \
        if (store == ST_F32) return pick_prepass_pattern<float, float, Q, MK>(pat);       \
        return nullptr;                                                                         \
    }                                                                                           \
    SweepLauncher sweep_##NAME(int store, int pat) {                                            \
        if (store == ST_F64) return NAME##_sweep_pat<double, double>(pat);                      \
        if (store == ST_F32) return NAME##_sweep_pat<float, float>(pat);                        \
        return nullptr;                                                                         \
    }                                                                                           \
    SparseLauncher sparse_##NAME(int store) {                                                   \
        if (store == ST_F64) return &launch_sparse<double, double, Q, MK>;                      \
        if (store == ST_F32) return &launch_sparse<float, float, Q, MK>;                        \
        return nullptr;                                                                         \
    }                                                                                           \
    SparseSetLauncher sparse_set_##NAME(int store) {                                            \
        if (store == ST_F64) return &launch_sparse_set<double, double, Q, MK>;                  \
        if (store == ST_F32) return &launch_sparse_set<float, double, Q, MK>;                   \
        return nullptr;                                                                         \
    }                                                                                           \
    MacroLauncher set_eq_##NAME(int store, int pat) {                                           \
        if (store == ST_F64) return NAME##_set_pat<double, double>(pat);                        \
        if (store == ST_F32) return NAME##_set_pat<float, double>(pat);                          \
        return nullptr;                                                                         \
    }

#define LBM_DEFINE_FAMILY_REDUCED_B(NAME, Q, MK)                                              \
    StagedLauncher sweep_staged_##NAME(int store, int pat) {                                    \
        if (store == ST_F64) return pick_staged_pattern<double, double, Q, MK>(pat);            \
        if (store == ST_F32) return pick_staged_pattern<float, float, Q, MK>(pat);              \
        return nullptr;                                                                         \
    }                                                                                           \
    SweepLauncher sweep_pair_##NAME(int store, int pat) {                                       \
        if (store == ST_F32) return pick_pair_pattern<float, Q, MK>(pat);                       \
        return nullptr;                                                                         \
    }

#define LBM_DECLARE_FAMILY(NAME)                        \
    SparseLauncher sparse_##NAME(int store);             \
    SparseSetLauncher sparse_set_##NAME(int store);      \
    BatchLauncher batched_##NAME(int store, int pat);    \
    SweepLauncher sweep_##NAME(int store, int pat);      \
    SweepLauncher sweep_pair_##NAME(int store, int pat); \
    SweepLauncher sweep_quad_##NAME(int store, int pat); \
    StagedLauncher sweep_staged_##NAME(int store, int pat); \
    SweepLauncher prepass_##NAME(int store, int pat); \
    MacroLauncher set_eq_##NAME(int store, int pat);

LBM_DECLARE_FAMILY(q19_pop)
LBM_DECLARE_FAMILY(q19_mrt)
LBM_DECLARE_FAMILY(q27_pop)
LBM_DECLARE_FAMILY(q27_mrt)
LBM_DECLARE_FAMILY(q27_cum)
LBM_DECLARE_FAMILY(q27_cum1)
LBM_DECLARE_FAMILY(q27_cm)

// Pipelined z-column sweep of the D3Q27 cumulant (orders >= 3 relaxed by 1), FP32, pull and AA.
SweepLauncher sweep_zpipe_q27_cum1(int store, int pat);

// error reporting shared by the entry points of every translation unit (lbm_abi.cu)
int abi_fail(int code, const char* fmt, ...);

// learned closure (lbm_q27_closure.cu)
SweepLauncher sweep_q27_closure(int store, int pat);
cudaError_t closure_upload(const float* host_params, cudaStream_t stream);

}  // namespace lbm
