// C ABI of liblbmb200.so (declared in include/lbm_b200.h): plan validation, launch
// configuration and the macroscopic / reduction / flag kernels that do not depend on the method.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lbm_b200.h"
#include "lbm_closure.cuh"
#include "lbm_dispatch.h"

using namespace lbm;

struct LbmPlan {
    LbmPlanDesc desc;
    int device;
    int q, mk, store;
    int use_pair;          // -1 default policy, 0 never, 1 whenever applicable (environment LBM_B200_PAIR)
    int zc;                // z-planes per thread of the FP32 closure sweep (environment LBM_B200_ZC, else 8)
    int use_quad;          // -1 default policy, 0 never, 1 whenever applicable (environment LBM_B200_QUAD)
    int use_staged;        // -1 default policy, 0 never, 1 whenever applicable (environment LBM_B200_STAGED)
    int ns;                // shared-memory stages of the staged sweep (environment LBM_B200_NS, else 2)
    int zpipe;             // cells per thread of the pipelined z-column sweep, 0 off (environment LBM_B200_ZPIPE)
    int block_x;           // x extent of the one-cell sweep's 256-thread blocks, 0 automatic (LBM_B200_BX)
    int sms;               // multiprocessors of the plan's device
    unsigned* status;      // device status word (lbm_plan_status), inside the reduction scratch
    uint32_t* rowmask;     // row summary of the flag field last finalized with this plan
    mutable const uint8_t* rowmask_flags;  // that flag field (sweeps given it use the summary)
    void* ubb_rho;         // compressible + moving UBB walls: density gathered before the sweep
    const int* ubb_block;  // per-link boundary tables (lbm_plan_set_links), caller-owned
    const double* ubb_link_vel;
    const int* link_code;
    double* link_value;
    uint32_t ubb_link_mask;
    unsigned long long stage_wait_ns;   // bound of the staged sweep's barrier waits (0: default)
    int stage_probe;                    // staged sweep: wait on a barrier nothing arrives at (test)
    Physics phys;
    double* partial;       // reduction scratch: RED_BLOCKS * 5 doubles
    double* red_out;       // 5 doubles on the device
    int red_blocks;
};

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(LBM_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int check_device(const LbmPlan* p) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev != p->device)
        return fail(LBM_E_DEVICE, "plan was created on device %d but device %d is current", p->device, dev);
    return LBM_OK;
}

int check_device_ptr(const LbmPlan* p, const void* ptr, const char* name, bool nullable) {
    if (ptr == nullptr) {
        if (nullable) return LBM_OK;
        return fail(LBM_E_INVALID, "%s is NULL", name);
    }
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(LBM_E_INVALID, "%s is not a CUDA pointer", name);
    }
    if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
        return fail(LBM_E_INVALID, "%s must point to device memory", name);
    if (at.device != p->device)
        return fail(LBM_E_DEVICE, "%s lives on device %d, the plan on device %d", name, at.device, p->device);
    return LBM_OK;
}

int check_strides(const LbmPlan* p, const int64_t s[4]) {
    if (s == nullptr) return fail(LBM_E_INVALID, "strides is NULL");
    const int64_t ex = p->desc.dims[0] + 2, ey = p->desc.dims[1] + 2, ez = p->desc.dims[2] + 2;
    if (s[0] != 1) return fail(LBM_E_INVALID, "x stride must be 1 (fzyx layout), got %lld", (long long)s[0]);
    if (s[1] < ex || s[2] < s[1] * ey || s[3] < s[2] * ez)
        return fail(LBM_E_INVALID,
                    "strides {%lld, %lld, %lld, %lld} overlap for a ghost-layered %lldx%lldx%lld field "
                    "(need x fastest, then y, z, q)",
                    (long long)s[0], (long long)s[1], (long long)s[2], (long long)s[3], (long long)ex,
                    (long long)ey, (long long)ez);
    if ((ex - 1) + (ey - 1) * s[1] + (ez - 1) * s[2] >= (int64_t(1) << 31))
        return fail(LBM_E_INVALID, "one PDF slot plane must hold fewer than 2^31 elements");
    if (s[3] * (int64_t)p->q >= (int64_t(1) << 32))
        return fail(LBM_E_INVALID, "the PDF field must span fewer than 2^32 elements (32-bit indexing)");
    return LBM_OK;
}

Grid make_grid(const LbmPlan* p, const int64_t s[4], const uint8_t* flags) {
    Grid g;
    g.nx = p->desc.dims[0];
    g.ny = p->desc.dims[1];
    g.nz = p->desc.dims[2];
    g.sy = (int)s[1];
    g.sz = (int)s[2];
    g.sq = (unsigned)s[3];
    g.periodic = (p->desc.periodic[0] ? 1 : 0) | (p->desc.periodic[1] ? 2 : 0) | (p->desc.periodic[2] ? 4 : 0);
    g.flags = flags;
    g.fsy = g.nx + 2;
    g.fsz = (g.nx + 2) * (g.ny + 2);
    g.rowmask = nullptr;
    return g;
}

// 256-thread blocks shaped along x: the widest of 128 / 64 / 32 threads whose last block in a
// row idles at most 1/8 of the row (else 32).
void launch_shape(const Grid& g, int zc, dim3& grid, dim3& block) {
    int bx = 32;
    for (int c : {128, 64}) {
        const int waste = (g.nx + c - 1) / c * c - g.nx;
        if (c <= 2 * g.nx && 8 * waste <= g.nx) { bx = c; break; }
    }
    const int by = 256 / bx;
    block = dim3(bx, by, 1);
    grid = dim3((g.nx + bx - 1) / bx, (g.ny + by - 1) / by, (g.nz + zc - 1) / zc);
}

// In-place patterns update one field (src == dst); pull and push use two.
bool pattern_inplace(int pattern) {
    return pattern == LBM_PATTERN_AA || pattern == LBM_PATTERN_ESOTWIST || pattern == LBM_PATTERN_ESOPULL ||
           pattern == LBM_PATTERN_ESOPUSH;
}

int pattern_kind(const LbmPlan* p, int parity) {
    switch (p->desc.pattern) {
        case LBM_PATTERN_PULL: return PAT_PULL;
        case LBM_PATTERN_AA: return parity ? PAT_AA_ODD : PAT_AA_EVEN;
        case LBM_PATTERN_ESOTWIST: return parity ? PAT_ESO_ODD : PAT_ESO_EVEN;
        case LBM_PATTERN_PUSH: return PAT_PUSH;
        case LBM_PATTERN_ESOPULL: return parity ? PAT_EPULL_ODD : PAT_EPULL_EVEN;
        case LBM_PATTERN_ESOPUSH: return parity ? PAT_EPUSH_ODD : PAT_EPUSH_EVEN;
    }
    return -1;
}

SweepLauncher sweep_launcher(const LbmPlan* p, int pat) {
    if (p->q == 19 && p->mk == MK_POP) return sweep_q19_pop(p->store, pat);
    if (p->q == 19 && p->mk == MK_MRT) return sweep_q19_mrt(p->store, pat);
    if (p->q == 27 && p->mk == MK_POP) return sweep_q27_pop(p->store, pat);
    if (p->q == 27 && p->mk == MK_MRT) return sweep_q27_mrt(p->store, pat);
    if (p->q == 27 && p->mk == MK_CUM) return sweep_q27_cum(p->store, pat);
    if (p->q == 27 && p->mk == MK_CUM1) return sweep_q27_cum1(p->store, pat);
    if (p->q == 27 && p->mk == MK_CUM1_MLP) return sweep_q27_closure(p->store, pat);
    if (p->q == 27 && p->mk == MK_CM) return sweep_q27_cm(p->store, pat);
    return nullptr;
}

SweepLauncher pair_launcher(const LbmPlan* p, int pat) {
    if (p->q == 19 && p->mk == MK_POP) return sweep_pair_q19_pop(p->store, pat);
    if (p->q == 19 && p->mk == MK_MRT) return sweep_pair_q19_mrt(p->store, pat);
    if (p->q == 27 && p->mk == MK_POP) return sweep_pair_q27_pop(p->store, pat);
    if (p->q == 27 && p->mk == MK_MRT) return sweep_pair_q27_mrt(p->store, pat);
    if (p->q == 27 && p->mk == MK_CUM) return sweep_pair_q27_cum(p->store, pat);
    if (p->q == 27 && p->mk == MK_CUM1) return sweep_pair_q27_cum1(p->store, pat);
    return nullptr;
}

size_t store_size(int store) { return store == ST_F64 ? 8 : (store == ST_F32 ? 4 : 2); }

size_t rowmask_bytes(const LbmPlan* p) {
    return sizeof(uint32_t) * ((size_t(p->desc.dims[1]) * p->desc.dims[2] + 31) / 32);
}

SweepLauncher quad_launcher(const LbmPlan* p, int pat) {
    if (p->q == 19 && p->mk == MK_POP) return sweep_quad_q19_pop(p->store, pat);
    if (p->q == 19 && p->mk == MK_MRT) return sweep_quad_q19_mrt(p->store, pat);
    if (p->q == 27 && p->mk == MK_POP) return sweep_quad_q27_pop(p->store, pat);
    if (p->q == 27 && p->mk == MK_CUM) return sweep_quad_q27_cum(p->store, pat);
    if (p->q == 27 && p->mk == MK_CUM1) return sweep_quad_q27_cum1(p->store, pat);
    return nullptr;
}

// The quad sweep (16-bit storage): four x-adjacent cells per thread, 8-byte accesses.  Needs
// nx a multiple of 4 and interior cell x = 0 of every row and slot on an 8-byte boundary.
// Default policy, from B200 measurements: SRT/TRT (D3Q19 TRT FP16 pull 61.3 -> 68.2 GLUPS at
// 256^3, 62.8 -> 70.0 at 512^3); not the moment-space methods, whose larger collision state
// spills (MRT) or loses occupancy (cumulant AA: 29.0 -> 25.9).
bool quad_applicable(const LbmPlan* p, const void* src, const void* dst, const int64_t s[4], int pat,
                     const float* omega_out) {
    if (p->use_quad == 0 || (p->use_quad < 0 && p->mk != MK_POP)) return false;
    if (p->store != ST_F16 && p->store != ST_BF16 && p->store != ST_E3M12) return false;
    if (omega_out != nullptr || (pat != PAT_PULL && pat != PAT_AA_EVEN && pat != PAT_AA_ODD)) return false;
    if (p->desc.dims[0] % 4 != 0) return false;
    const size_t es = store_size(p->store);
    if ((reinterpret_cast<uintptr_t>(src) + es) % (4 * es) != 0) return false;
    if ((reinterpret_cast<uintptr_t>(dst) + es) % (4 * es) != 0) return false;
    if (s[1] % 4 != 0 || s[2] % 4 != 0 || s[3] % 4 != 0) return false;
    return quad_launcher(p, pat) != nullptr;
}

// The pair sweep needs an even row length, no omega output, and every row's interior cell x = 0
// (ghost-inclusive x = 1) on a 2-element boundary so that paired loads / stores are aligned.
// Default policy, from B200 measurements: the pair sweep wins where the one-cell sweep is limited by
// instruction issue (16-bit storage, the cumulant with pull streaming); for FP32 storage the
// one-cell sweep already streams at HBM speed and keeps twice the occupancy.
bool pair_preferred(const LbmPlan* p, int pat) {
    if (p->use_pair >= 0) return p->use_pair == 1;
    if (p->store == ST_F16 || p->store == ST_BF16 || p->store == ST_E3M12) return true;
    return (p->mk == MK_CUM || p->mk == MK_CUM1) && pat == PAT_PULL;
}

bool pair_applicable(const LbmPlan* p, const void* src, const void* dst, const int64_t s[4], int pat,
                     const float* omega_out) {
    if (!pair_preferred(p, pat) || p->store == ST_F64 || omega_out != nullptr) return false;
    if (pat != PAT_PULL && pat != PAT_AA_EVEN && pat != PAT_AA_ODD) return false;
    if (p->desc.dims[0] % 2 != 0) return false;
    const size_t es = store_size(p->store);
    if ((reinterpret_cast<uintptr_t>(src) + es) % (2 * es) != 0) return false;
    if ((reinterpret_cast<uintptr_t>(dst) + es) % (2 * es) != 0) return false;
    if (s[1] % 2 != 0 || s[2] % 2 != 0 || s[3] % 2 != 0) return false;
    return pair_launcher(p, pat) != nullptr;
}

SweepLauncher prepass_launcher(const LbmPlan* p, int pat) {
    if (p->q == 19 && p->mk == MK_POP) return prepass_q19_pop(p->store, pat);
    if (p->q == 19 && p->mk == MK_MRT) return prepass_q19_mrt(p->store, pat);
    if (p->q == 27 && p->mk == MK_POP) return prepass_q27_pop(p->store, pat);
    if (p->q == 27 && p->mk == MK_MRT) return prepass_q27_mrt(p->store, pat);
    if (p->q == 27 && p->mk == MK_CUM) return prepass_q27_cum(p->store, pat);
    if (p->q == 27 && (p->mk == MK_CUM1 || p->mk == MK_CUM1_MLP)) return prepass_q27_cum1(p->store, pat);
    if (p->q == 27 && p->mk == MK_CM) return prepass_q27_cm(p->store, pat);
    return nullptr;
}

StagedLauncher staged_launcher(const LbmPlan* p, int pat) {
    if (p->q == 19 && p->mk == MK_POP) return sweep_staged_q19_pop(p->store, pat);
    if (p->q == 19 && p->mk == MK_MRT) return sweep_staged_q19_mrt(p->store, pat);
    if (p->q == 27 && p->mk == MK_POP) return sweep_staged_q27_pop(p->store, pat);
    if (p->q == 27 && p->mk == MK_MRT) return sweep_staged_q27_mrt(p->store, pat);
    if (p->q == 27 && p->mk == MK_CUM) return sweep_staged_q27_cum(p->store, pat);
    if (p->q == 27 && p->mk == MK_CUM1) return sweep_staged_q27_cum1(p->store, pat);
    return nullptr;
}

// The staged sweep copies row segments in 16-byte chunks: the source rows of every slot must
// start (interior cell x = 0) on a 16-byte boundary, the y / z / slot strides and the row length
// must be whole 16-byte units.  The tile count must fit an int.
bool staged_applicable(const LbmPlan* p, const void* src, const int64_t s[4], int pat) {
    if (p->use_staged <= 0) return false;
    if (pat != PAT_PULL && pat != PAT_AA_EVEN && pat != PAT_AA_ODD) return false;
    const size_t es = store_size(p->store);
    if (size_t(p->desc.dims[0]) * es % 16 != 0) return false;
    if ((reinterpret_cast<uintptr_t>(src) + es * size_t(1 + s[1] + s[2])) % 16 != 0) return false;
    if (size_t(s[1]) * es % 16 != 0 || size_t(s[2]) * es % 16 != 0 || size_t(s[3]) * es % 16 != 0) return false;
    // 16-bit storage copies the halo element after a row's ghost cell as a 4-byte word with its
    // successor, which must lie in the row's padding
    if (es == 2 && s[1] < int64_t(p->desc.dims[0]) + 3) return false;
    const long long tiles = (long long)((p->desc.dims[0] + 31) / 32) * p->desc.dims[1] * p->desc.dims[2];
    if (tiles > 0x7fffffffLL) return false;
    return staged_launcher(p, pat) != nullptr;
}

MacroLauncher set_eq_launcher(const LbmPlan* p, int pat) {
    if (p->q == 19 && p->mk == MK_POP) return set_eq_q19_pop(p->store, pat);
    if (p->q == 19 && p->mk == MK_MRT) return set_eq_q19_mrt(p->store, pat);
    if (p->q == 27 && p->mk == MK_POP) return set_eq_q27_pop(p->store, pat);
    if (p->q == 27 && p->mk == MK_MRT) return set_eq_q27_mrt(p->store, pat);
    if (p->q == 27 && (p->mk == MK_CUM || p->mk == MK_CUM1 || p->mk == MK_CUM1_MLP))
        return set_eq_q27_cum(p->store, pat);
    if (p->q == 27 && p->mk == MK_CM) return set_eq_q27_cm(p->store, pat);
    return nullptr;
}

// ---- method-independent kernels, instantiated here
template <class S, class R, int Q, int PAT>
cudaError_t launch_get(const MacroArgs& a, dim3 grid, dim3 block, cudaStream_t s) {
    k_get_macroscopic<S, R, Q, PAT><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

template <class S, class R, int Q>
MacroLauncher pick_get(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_get<S, R, Q, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_get<S, R, Q, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_get<S, R, Q, PAT_AA_ODD>;
        case PAT_ESO_EVEN: return &launch_get<S, R, Q, PAT_ESO_EVEN>;
        case PAT_ESO_ODD: return &launch_get<S, R, Q, PAT_ESO_ODD>;
    }
    if constexpr (sizeof(S) >= 4) {
        switch (pat) {
            case PAT_PUSH: return &launch_get<S, R, Q, PAT_PUSH>;
            case PAT_EPULL_EVEN: return &launch_get<S, R, Q, PAT_EPULL_EVEN>;
            case PAT_EPULL_ODD: return &launch_get<S, R, Q, PAT_EPULL_ODD>;
            case PAT_EPUSH_EVEN: return &launch_get<S, R, Q, PAT_EPUSH_EVEN>;
            case PAT_EPUSH_ODD: return &launch_get<S, R, Q, PAT_EPUSH_ODD>;
        }
    }
    return nullptr;
}

template <int Q>
MacroLauncher get_launcher_q(int store, int pat) {
    switch (store) {
        case ST_F64: return pick_get<double, double, Q>(pat);
        case ST_F32: return pick_get<float, float, Q>(pat);
        case ST_F16: return pick_get<__half, float, Q>(pat);
        case ST_BF16: return pick_get<__nv_bfloat16, float, Q>(pat);
        case ST_E3M12: return pick_get<e3m12, float, Q>(pat);
    }
    return nullptr;
}

using ReduceLauncher = cudaError_t (*)(const MacroArgs&, int, double*, cudaStream_t);

template <class S, int Q, int PAT>
cudaError_t launch_reduce(const MacroArgs& a, int blocks, double* partial, cudaStream_t s) {
    k_reduce_partial<S, Q, PAT><<<blocks, RED_THREADS, 0, s>>>(a, partial);
    return cudaGetLastError();
}

template <class S, int Q>
ReduceLauncher pick_reduce(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_reduce<S, Q, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_reduce<S, Q, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_reduce<S, Q, PAT_AA_ODD>;
        case PAT_ESO_EVEN: return &launch_reduce<S, Q, PAT_ESO_EVEN>;
        case PAT_ESO_ODD: return &launch_reduce<S, Q, PAT_ESO_ODD>;
    }
    if constexpr (sizeof(S) >= 4) {
        switch (pat) {
            case PAT_PUSH: return &launch_reduce<S, Q, PAT_PUSH>;
            case PAT_EPULL_EVEN: return &launch_reduce<S, Q, PAT_EPULL_EVEN>;
            case PAT_EPULL_ODD: return &launch_reduce<S, Q, PAT_EPULL_ODD>;
            case PAT_EPUSH_EVEN: return &launch_reduce<S, Q, PAT_EPUSH_EVEN>;
            case PAT_EPUSH_ODD: return &launch_reduce<S, Q, PAT_EPUSH_ODD>;
        }
    }
    return nullptr;
}

template <int Q>
ReduceLauncher reduce_launcher_q(int store, int pat) {
    switch (store) {
        case ST_F64: return pick_reduce<double, Q>(pat);
        case ST_F32: return pick_reduce<float, Q>(pat);
        case ST_F16: return pick_reduce<__half, Q>(pat);
        case ST_BF16: return pick_reduce<__nv_bfloat16, Q>(pat);
        case ST_E3M12: return pick_reduce<e3m12, Q>(pat);
    }
    return nullptr;
}

// ---- previous-step density next to moving walls (k_ubb_density)
using UbbLauncher = cudaError_t (*)(const SweepArgs&, void*, dim3, dim3, cudaStream_t);

template <class S, class R, int Q, int PAT>
cudaError_t launch_ubb(const SweepArgs& a, void* out, dim3 grid, dim3 block, cudaStream_t s) {
    k_ubb_density<S, R, Q, PAT><<<grid, block, 0, s>>>(a, static_cast<R*>(out));
    return cudaGetLastError();
}

template <class S, class R, int Q>
UbbLauncher pick_ubb(int pat) {
    switch (pat) {
        case PAT_PULL: return &launch_ubb<S, R, Q, PAT_PULL>;
        case PAT_AA_EVEN: return &launch_ubb<S, R, Q, PAT_AA_EVEN>;
        case PAT_AA_ODD: return &launch_ubb<S, R, Q, PAT_AA_ODD>;
        case PAT_ESO_EVEN: return &launch_ubb<S, R, Q, PAT_ESO_EVEN>;
        case PAT_ESO_ODD: return &launch_ubb<S, R, Q, PAT_ESO_ODD>;
    }
    if constexpr (sizeof(S) >= 4) {
        switch (pat) {
            case PAT_PUSH: return &launch_ubb<S, R, Q, PAT_PUSH>;
            case PAT_EPULL_EVEN: return &launch_ubb<S, R, Q, PAT_EPULL_EVEN>;
            case PAT_EPULL_ODD: return &launch_ubb<S, R, Q, PAT_EPULL_ODD>;
            case PAT_EPUSH_EVEN: return &launch_ubb<S, R, Q, PAT_EPUSH_EVEN>;
            case PAT_EPUSH_ODD: return &launch_ubb<S, R, Q, PAT_EPUSH_ODD>;
        }
    }
    return nullptr;
}

template <int Q>
UbbLauncher ubb_launcher_q(int store, int pat) {
    switch (store) {
        case ST_F64: return pick_ubb<double, double, Q>(pat);
        case ST_F32: return pick_ubb<float, float, Q>(pat);
        case ST_F16: return pick_ubb<__half, float, Q>(pat);
        case ST_BF16: return pick_ubb<__nv_bfloat16, float, Q>(pat);
        case ST_E3M12: return pick_ubb<e3m12, float, Q>(pat);
    }
    return nullptr;
}

// The compressible UBB of a moving wall needs the cell's previous-step density (unless the wall
// density is prescribed): a non-zero constant velocity, per-link velocities, or a wall velocity
// shifted by the force.
bool needs_ubb_density(const LbmPlanDesc* d, uint32_t link_mask) {
    if (!d->compressible) return false;
    const bool force = d->force[0] != 0.0 || d->force[1] != 0.0 || d->force[2] != 0.0;
    for (int u = 0; u < 4; ++u) {
        if (d->ubb_density[u] > 0.0) continue;
        if ((link_mask >> u) & 1u) return true;
        if (force && ((d->ubb_adapt_mask >> u) & 1u)) return true;
        for (int k = 0; k < 3; ++k)
            if (d->ubb_velocity[u][k] != 0.0) return true;
    }
    return false;
}

int ensure_ubb_buffer(LbmPlan* p) {
    if (!needs_ubb_density(&p->desc, p->ubb_link_mask) || p->ubb_rho != nullptr) return LBM_OK;
    const size_t n = size_t(p->desc.dims[0]) * p->desc.dims[1] * p->desc.dims[2];
    cudaError_t e = cudaMalloc(&p->ubb_rho, n * (p->store == ST_F64 ? 8 : 4));
    if (e != cudaSuccess) {
        p->ubb_rho = nullptr;
        return cuda_fail(e, "cudaMalloc(wall density)");
    }
    return LBM_OK;
}

// Row summary of a finalized flag field: bit y + ny*z for every interior row with a non-zero flag.
__global__ void k_row_mask(Grid g, uint32_t* mask) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.ny * g.nz) return;
    const int y = r % g.ny, z = r / g.ny;
    const uint8_t* row = g.flags + 1 + (y + 1) * g.fsy + (z + 1) * g.fsz;
    for (int x = 0; x < g.nx; ++x)
        if (row[x] != 0) {
            atomicOr(mask + (r >> 5), 1u << (r & 31));
            break;
        }
}

// Marks fluid cells that have a boundary neighbour along the stencil.
template <int Q>
__global__ void k_flags_finalize(Grid g) {
    using L = Lat<Q>;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    uint8_t* fl = const_cast<uint8_t*>(g.flags);
    const int fc = (x + 1) + (y + 1) * g.fsy + (z + 1) * g.fsz;
    int v = fl[fc] & ~FLAG_NEAR_WALL;
    if ((v & FLAG_TYPE_MASK) == 0) {
        Grid gf = g;
        gf.sy = g.fsy;
        gf.sz = g.fsz;
        NbrOffsets nb;
        nb.init(gf, x, y, z);
        bool near = false;
#pragma unroll
        for (int i = 1; i < Q; ++i)
            if (fl[fc + nb.off(L::cx(i), L::cy(i), L::cz(i))] & FLAG_TYPE_MASK) near = true;
        if (near) v |= FLAG_NEAR_WALL;
    }
    fl[fc] = (uint8_t)v;
}

// Optimal third-order rates w3..w5 (before the per-cell limiters) and the parameters a, b of the
// fourth-order correction for shear rate w1 and bulk rate w2 (Geier et al. 2017, eq. 111-116;
// methods/cumulantbased/fourth_order_correction.py:79-97, :149-170).  False if a denominator vanishes.
bool fourth_order_params(double w1, double w2, double w[3], double ab[2]) {
    const double w11 = w1 * w1, w12 = w1 * w2, w22 = w2 * w2;
    const double d3 = 8.0 * (5.0 - 2.0 * w1) * w1 + w2 * (8.0 + w1 * (9.0 * w1 - 26.0));
    const double d4 = w2 * (56.0 - 42.0 * w1 + 9.0 * w11) - 8.0 * w1;
    const double d5 = 16.0 * w11 * (w1 - 6.0) - 2.0 * w12 * (216.0 + 5.0 * w1 * (9.0 * w1 - 46.0)) +
                      w22 * (w1 * (3.0 * w1 - 10.0) * (15.0 * w1 - 28.0) - 48.0);
    const double dab = (w1 - w2) * (w2 * (2.0 + 3.0 * w1) - 8.0 * w1);
    if (d3 == 0.0 || d4 == 0.0 || d5 == 0.0 || dab == 0.0) return false;
    w[0] = 8.0 * (w1 - 2.0) * (w2 * (3.0 * w1 - 1.0) - 5.0 * w1) / d3;
    w[1] = 8.0 * (w1 - 2.0) * (w1 + w2 * (3.0 * w1 - 7.0)) / d4;
    w[2] = 24.0 * (w1 - 2.0) * (4.0 * w11 + w12 * (18.0 - 13.0 * w1) + w22 * (2.0 + w1 * (6.0 * w1 - 11.0))) / d5;
    ab[0] = (4.0 * w11 + 2.0 * w12 * (w1 - 6.0) + w22 * (w1 * (10.0 - 3.0 * w1) - 4.0)) / dab;
    ab[1] = (4.0 * w12 * (9.0 * w1 - 16.0) - 4.0 * w11 - 2.0 * w22 * (2.0 + 9.0 * w1 * (w1 - 2.0))) / (3.0 * dab);
    return std::isfinite(w[0]) && std::isfinite(w[1]) && std::isfinite(w[2]) && std::isfinite(ab[0]) &&
           std::isfinite(ab[1]);
}

int fill_physics(LbmPlan* p, const LbmPlanDesc* d) {
    Physics& ph = p->phys;
    memset(&ph, 0, sizeof(ph));
    for (int k = 0; k < 27; ++k) ph.rates[k] = d->rates[k];
    for (int k = 0; k < 3; ++k) ph.force[k] = d->force[k];
    ph.force_model = d->force_model;
    ph.compressible = d->compressible ? 1 : 0;
    ph.continuous_eq = d->continuous_equilibrium ? 1 : 0;
    ph.sgs = d->sgs;
    ph.sgs_c18 = 18.0 * d->sgs_constant * d->sgs_constant;
    ph.tau0 = d->shear_rate != 0.0 ? 1.0 / d->shear_rate : 0.0;
    ph.sgs_mask = d->sgs_mask;
    ph.galilean = d->galilean_correction ? 1 : 0;
    for (int u = 0; u < MAX_UBB; ++u)
        for (int k = 0; k < 3; ++k) ph.ubb[u][k] = d->ubb_velocity[u][k];
    if (d->method == LBM_METHOD_SRT) ph.rates[1] = ph.rates[0];
    ph.fixed_density = d->fixed_density;
    ph.fixed_density1 = d->fixed_density1;
    for (int u = 0; u < MAX_UBB; ++u) ph.ubb_density[u] = d->ubb_density[u];
    ph.ubb_adapt_mask = d->ubb_adapt_mask & 0xfu;
    ph.ubb_link_mask = p->ubb_link_mask;
    if (d->method == LBM_METHOD_CUMULANT && d->fourth_order_limiter > 0.0) {
        double w[3], ab[2];
        fourth_order_params(d->rates[4], d->rates[9], w, ab);
        for (int k = 10; k < 13; ++k) ph.rates[k] = w[0];
        for (int k = 13; k < 16; ++k) ph.rates[k] = w[1];
        ph.rates[16] = w[2];
        for (int k = 17; k < 27; ++k) ph.rates[k] = 1.0;
        ph.foc_limiter = d->fourth_order_limiter;
        ph.foc_a = ab[0];
        ph.foc_b = ab[1];
    }
    return LBM_OK;
}

// Every cumulant group of order >= 3 (canonical indices 10..26) has rate 1 and no SGS adaptation:
// the specialised cumulant sweep applies.
bool cumulant_high_orders_relax_to_equilibrium(const LbmPlanDesc* d) {
    for (int k = 10; k < 27; ++k) {
        if (d->rates[k] != 1.0) return false;
        if (d->sgs != LBM_SGS_NONE && ((d->sgs_mask >> k) & 1u)) return false;
    }
    return true;
}

int method_kind(const LbmPlanDesc* d) {
    if (d->method == LBM_METHOD_MRT) return MK_MRT;
    if (d->method == LBM_METHOD_CENTRAL_MOMENT) return MK_CM;
    if (d->method != LBM_METHOD_CUMULANT) return MK_POP;
    if (d->fourth_order_limiter > 0.0 || !cumulant_high_orders_relax_to_equilibrium(d)) return MK_CUM;
    return d->sgs == LBM_SGS_MLP ? MK_CUM1_MLP : MK_CUM1;
}

int validate_desc(const LbmPlanDesc* d) {
    if (d->stencil != 19 && d->stencil != 27) return fail(LBM_E_UNSUPPORTED, "stencil must be D3Q19 or D3Q27");
    if (d->method < 0 || d->method > 4) return fail(LBM_E_INVALID, "unknown method %d", d->method);
    if (d->method == LBM_METHOD_CENTRAL_MOMENT) {
        if (d->stencil != 27) return fail(LBM_E_UNSUPPORTED, "the central-moment sweep is built for D3Q27 only");
        if (!d->compressible)
            return fail(LBM_E_UNSUPPORTED, "the central-moment sweep is built for compressible methods");
        if (d->sgs != LBM_SGS_NONE)
            return fail(LBM_E_UNSUPPORTED, "subgrid-scale models are not built for the central-moment sweep");
        if (d->store_dtype != LBM_DTYPE_F64 && d->store_dtype != LBM_DTYPE_F32)
            return fail(LBM_E_UNSUPPORTED, "the central-moment sweep is built for FP64 and FP32 storage");
        if (d->pattern != LBM_PATTERN_PULL && d->pattern != LBM_PATTERN_AA)
            return fail(LBM_E_UNSUPPORTED, "the central-moment sweep is built for the pull and AA patterns");
    }
    if (d->method == LBM_METHOD_CUMULANT && d->stencil != 27)
        return fail(LBM_E_UNSUPPORTED, "the cumulant sweep is built for D3Q27 only");
    if (!(d->fourth_order_limiter >= 0.0))
        return fail(LBM_E_INVALID, "fourth_order_limiter must be >= 0 (0: no fourth-order correction)");
    if (d->fourth_order_limiter > 0.0) {
        if (d->method != LBM_METHOD_CUMULANT)
            return fail(LBM_E_INVALID, "Fourth-order correction can only be applied to D3Q27 cumulant methods.");
        if (d->sgs != LBM_SGS_NONE)
            return fail(LBM_E_UNSUPPORTED, "the fourth-order correction is not built with subgrid-scale models");
        double w[3], ab[2];
        if (!fourth_order_params(d->rates[4], d->rates[9], w, ab))
            return fail(LBM_E_INVALID, "the fourth-order correction is undefined for shear rate %g and bulk rate %g",
                        d->rates[4], d->rates[9]);
    }
    if (d->method == LBM_METHOD_CUMULANT && !d->compressible)
        return fail(LBM_E_INVALID, "Incompressible cumulant-based methods are not supported (yet).");
    if (d->store_dtype < 0 || d->store_dtype > 4) return fail(LBM_E_INVALID, "unknown dtype %d", d->store_dtype);
    if (d->pattern < 0 || d->pattern > 5) return fail(LBM_E_INVALID, "unknown streaming pattern %d", d->pattern);
    if (d->force_model < 0 || d->force_model > 4) return fail(LBM_E_INVALID, "unknown force model");
    if (d->method == LBM_METHOD_CUMULANT && d->force_model != LBM_FORCE_NONE &&
        d->force_model != LBM_FORCE_CENTRAL_MOMENT)
        return fail(LBM_E_UNSUPPORTED, "the cumulant sweep supports the CentralMoment force model only");
    if (d->method != LBM_METHOD_CUMULANT && d->force_model == LBM_FORCE_CENTRAL_MOMENT)
        return fail(LBM_E_INVALID, "This force model can only be combined with the Cumulant collision model");
    if (d->galilean_correction && d->method != LBM_METHOD_CUMULANT)
        return fail(LBM_E_INVALID, "Galilean correction is only defined for D3Q27 cumulant methods.");
    if (d->sgs != LBM_SGS_NONE && d->sgs != LBM_SGS_SMAGORINSKY && d->sgs != LBM_SGS_MLP)
        return fail(LBM_E_INVALID, "unknown SGS model");
    if (d->sgs != LBM_SGS_NONE && !(d->shear_rate > 0.0))
        return fail(LBM_E_INVALID, "a subgrid-scale model needs a positive shear relaxation rate");
    if (d->sgs == LBM_SGS_MLP &&
        (d->method != LBM_METHOD_CUMULANT || d->stencil != 27 || !cumulant_high_orders_relax_to_equilibrium(d)))
        return fail(LBM_E_UNSUPPORTED,
                    "the learned closure is built for the D3Q27 cumulant method with orders >= 3 relaxed by 1");
    if (d->sgs == LBM_SGS_MLP && d->store_dtype != LBM_DTYPE_F32 && d->store_dtype != LBM_DTYPE_F64)
        return fail(LBM_E_UNSUPPORTED, "the learned closure is built for FP32 and FP64 storage");
    if (d->sgs == LBM_SGS_MLP && d->pattern != LBM_PATTERN_PULL && d->pattern != LBM_PATTERN_AA)
        return fail(LBM_E_UNSUPPORTED, "the learned closure is built for the pull and AA patterns");
    if (!(d->fixed_density >= 0.0) || !(d->fixed_density1 >= 0.0))
        return fail(LBM_E_INVALID, "fixed_density must be >= 0 (0: no FixedDensity cells)");
    if (d->fixed_density1 > 0.0 && d->force_model != LBM_FORCE_NONE)
        return fail(LBM_E_UNSUPPORTED, "FixedDensity boundaries are built for force-free methods");
    for (int u = 0; u < 4; ++u)
        if (!(d->ubb_density[u] >= 0.0))
            return fail(LBM_E_INVALID, "ubb_density must be >= 0 (0: the density of the fluid cell)");
    if (d->ubb_adapt_mask & ~0xfu) return fail(LBM_E_INVALID, "ubb_adapt_mask has bits beyond UBB number 3");
    if (d->fixed_density > 0.0 && d->force_model != LBM_FORCE_NONE)
        return fail(LBM_E_UNSUPPORTED, "FixedDensity boundaries are built for force-free methods");
    for (int k = 0; k < 3; ++k)
        if (d->dims[k] < 1) return fail(LBM_E_INVALID, "dims must be positive, got %d in axis %d", d->dims[k], k);
    if (d->dims[1] > 65535 * 8 || d->dims[2] > 65535)
        return fail(LBM_E_INVALID, "domain too large for the launch grid");
    return LBM_OK;
}

}  // namespace

int lbm::abi_fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

extern "C" {

int lbm_version(void) { return 1; }

int lbm_last_error(char* buf, size_t n) {
    if (buf == nullptr || n == 0) return LBM_E_INVALID;
    snprintf(buf, n, "%s", g_err.c_str());
    return LBM_OK;
}

int lbm_plan_create(const LbmPlanDesc* desc, LbmPlan** out) {
    if (desc == nullptr || out == nullptr) return fail(LBM_E_INVALID, "desc and out must not be NULL");
    *out = nullptr;
    int rc = validate_desc(desc);
    if (rc) return rc;
    LbmPlan* p = new LbmPlan();
    p->desc = *desc;
    cudaError_t e = cudaGetDevice(&p->device);
    if (e != cudaSuccess) { delete p; return cuda_fail(e, "cudaGetDevice"); }
    p->q = desc->stencil;
    p->mk = method_kind(desc);
    p->store = desc->store_dtype;
    {
        const char* env = getenv("LBM_B200_PAIR");
        p->use_pair = env == nullptr ? -1 : (env[0] == '0' ? 0 : 1);
        const char* qenv = getenv("LBM_B200_QUAD");
        p->use_quad = qenv == nullptr ? -1 : (qenv[0] == '0' ? 0 : 1);
        const char* zenv = getenv("LBM_B200_ZC");
        p->zc = zenv != nullptr ? atoi(zenv) : 8;
        if (p->zc < 1) p->zc = 1;
        const char* senv = getenv("LBM_B200_STAGED");
        p->use_staged = senv == nullptr ? -1 : (senv[0] == '0' ? 0 : 1);
        const char* benv = getenv("LBM_B200_BX");
        p->block_x = benv != nullptr ? atoi(benv) : 0;
        if (p->block_x != 32 && p->block_x != 64 && p->block_x != 128 && p->block_x != 256) p->block_x = 0;
        const char* penv = getenv("LBM_B200_ZPIPE");
        p->zpipe = penv != nullptr ? atoi(penv) : 0;
        if (p->zpipe < 2) p->zpipe = 0;
        if (p->zpipe > 64) p->zpipe = 64;
        const char* nenv = getenv("LBM_B200_NS");
        p->ns = nenv != nullptr ? atoi(nenv) : 2;
        if (p->ns < 2) p->ns = 2;
        if (p->ns > STAGED_MAX_NS) p->ns = STAGED_MAX_NS;
    }
    p->ubb_block = nullptr;
    p->ubb_link_vel = nullptr;
    p->link_code = nullptr;
    p->link_value = nullptr;
    p->ubb_link_mask = 0;
    p->stage_wait_ns = 0;
    p->stage_probe = 0;
    fill_physics(p, desc);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
    p->sms = sms;
    p->red_blocks = sms * 4;
    e = cudaMalloc(&p->partial, sizeof(double) * (5 * (p->red_blocks + 1) + 1));
    if (e != cudaSuccess) { delete p; return cuda_fail(e, "cudaMalloc(reduction scratch)"); }
    p->red_out = p->partial + 5 * p->red_blocks;
    p->status = reinterpret_cast<unsigned*>(p->partial + 5 * (p->red_blocks + 1));
    e = cudaMemset(p->status, 0, sizeof(double));
    if (e != cudaSuccess) { cudaFree(p->partial); delete p; return cuda_fail(e, "cudaMemset(status)"); }
    p->ubb_rho = nullptr;
    p->rowmask = nullptr;
    p->rowmask_flags = nullptr;
    if (sweep_launcher(p, PAT_PULL) == nullptr) {
        cudaFree(p->partial);
        delete p;
        return fail(LBM_E_UNSUPPORTED, "no kernel built for this stencil/method/dtype");
    }
    if (int rc2 = ensure_ubb_buffer(p)) {
        cudaFree(p->partial);
        delete p;
        return rc2;
    }
    e = cudaMalloc(&p->rowmask, rowmask_bytes(p));
    if (e != cudaSuccess) {
        cudaFree(p->partial);
        if (p->ubb_rho) cudaFree(p->ubb_rho);
        delete p;
        return cuda_fail(e, "cudaMalloc(row summary)");
    }
    *out = p;
    return LBM_OK;
}

int lbm_plan_update(LbmPlan* p, const LbmPlanDesc* desc) {
    if (p == nullptr || desc == nullptr) return fail(LBM_E_INVALID, "plan and desc must not be NULL");
    if (desc->stencil != p->desc.stencil || desc->method != p->desc.method ||
        desc->store_dtype != p->desc.store_dtype || desc->pattern != p->desc.pattern ||
        memcmp(desc->dims, p->desc.dims, sizeof(desc->dims)) != 0)
        return fail(LBM_E_INVALID, "lbm_plan_update may only change physical parameters");
    int rc = validate_desc(desc);
    if (rc) return rc;
    p->desc = *desc;
    p->mk = method_kind(desc);
    fill_physics(p, desc);
    return ensure_ubb_buffer(p);
}

int lbm_plan_destroy(LbmPlan* p) {
    if (p == nullptr) return LBM_OK;
    if (p->partial) cudaFree(p->partial);
    if (p->ubb_rho) cudaFree(p->ubb_rho);
    if (p->rowmask) cudaFree(p->rowmask);
    delete p;
    return LBM_OK;
}

static int validate_sweep(const LbmPlan* p, const void* src, const void* dst, const int64_t strides[4],
                          const uint8_t* flags, const float* omega_out) {
    if (p == nullptr) return fail(LBM_E_INVALID, "plan is NULL");
    int rc;
    if ((rc = check_device(p))) return rc;
    if ((rc = check_strides(p, strides))) return rc;
    if ((rc = check_device_ptr(p, src, "src", false))) return rc;
    if ((rc = check_device_ptr(p, dst, "dst", false))) return rc;
    if ((rc = check_device_ptr(p, flags, "flags", true))) return rc;
    if ((rc = check_device_ptr(p, omega_out, "omega_out", true))) return rc;
    const bool inplace = pattern_inplace(p->desc.pattern);
    if (inplace && src != dst) return fail(LBM_E_INVALID, "in-place streaming patterns need src == dst");
    if (!inplace && src == dst) return fail(LBM_E_INVALID, "the pull and push patterns need two distinct fields");
    return LBM_OK;
}

// Which sweep kernel a launch with these arguments uses (LBM_VARIANT_*), in order of preference.
static bool zpipe_applicable(const LbmPlan* p, int pat, const float* omega_out) {
    return p->zpipe >= 2 && p->mk == MK_CUM1 && p->store == ST_F32 && omega_out == nullptr &&
           (pat == PAT_PULL || pat == PAT_AA_EVEN || pat == PAT_AA_ODD);
}

static int sweep_variant(const LbmPlan* p, const void* src, const void* dst, const int64_t strides[4], int pat,
                         const float* omega_out) {
    if (zpipe_applicable(p, pat, omega_out)) return LBM_VARIANT_ZPIPE;
    if (staged_applicable(p, src, strides, pat)) return LBM_VARIANT_STAGED;
    if (quad_applicable(p, src, dst, strides, pat, omega_out)) return LBM_VARIANT_QUAD;
    if (pair_applicable(p, src, dst, strides, pat, omega_out)) return LBM_VARIANT_PAIR;
    return LBM_VARIANT_CELL;
}

// Launch without re-validating (arguments checked by the caller).
static int launch_sweep_checked(const LbmPlan* p, const void* src, void* dst, const int64_t strides[4],
                                const uint8_t* flags, int parity, float* omega_out, cudaStream_t stream) {
    const int pat = pattern_kind(p, parity);
    SweepArgs a;
    a.g = make_grid(p, strides, flags);
    a.p = p->phys;
    a.src = src;
    a.dst = dst;
    a.omega_out = omega_out;
    a.zc = (p->mk == MK_CUM1_MLP && p->store == ST_F32) ? p->zc : 1;
    a.stage_probe = p->stage_probe;
    a.stage_wait_ns = p->stage_wait_ns;
    a.ubb_rho = nullptr;
    a.status = p->status;
    a.ubb_block = p->ubb_block;
    a.ubb_link_vel = p->ubb_link_vel;
    a.link_code = p->link_code;
    a.link_value = p->link_value;
    if (flags != nullptr && flags == p->rowmask_flags) a.g.rowmask = p->rowmask;
    if (flags != nullptr && p->ubb_rho != nullptr && needs_ubb_density(&p->desc, p->ubb_link_mask)) {
        UbbLauncher U = p->q == 19 ? ubb_launcher_q<19>(p->store, pat) : ubb_launcher_q<27>(p->store, pat);
        if (U == nullptr) return fail(LBM_E_UNSUPPORTED, "no wall-density kernel for this storage type / pattern");
        dim3 ug, ub;
        launch_shape(a.g, 1, ug, ub);
        cudaError_t e = U(a, p->ubb_rho, ug, ub, stream);
        if (e != cudaSuccess) return cuda_fail(e, "wall-density launch");
        a.ubb_rho = p->ubb_rho;
    }
    if (flags != nullptr && (p->desc.fixed_density > 0 || p->desc.fixed_density1 > 0 || p->link_code != nullptr ||
                             p->link_value != nullptr)) {
        SweepLauncher F = prepass_launcher(p, pat);
        if (F == nullptr) return fail(LBM_E_UNSUPPORTED, "no boundary pre-pass kernel for this storage type / pattern");
        dim3 fg, fb;
        launch_shape(a.g, 1, fg, fb);
        cudaError_t e = F(a, fg, fb, stream);
        if (e != cudaSuccess) return cuda_fail(e, "boundary pre-pass launch");
    }
    const int variant = sweep_variant(p, src, dst, strides, pat, omega_out);
    if (variant == LBM_VARIANT_STAGED) {
        StagedLauncher SL = staged_launcher(p, pat);
        cudaError_t e = SL(a, p->ns, p->sms, stream);
        if (e != cudaSuccess) return cuda_fail(e, "staged sweep launch");
        return LBM_OK;
    }
    dim3 grid, block;
    SweepLauncher L;
    if (variant == LBM_VARIANT_QUAD) {
        L = quad_launcher(p, pat);
        block = dim3(32, QUAD_ROWS, 1);
        grid = dim3((a.g.nx + 127) / 128, (a.g.ny + QUAD_ROWS - 1) / QUAD_ROWS, a.g.nz);
    } else if (variant == LBM_VARIANT_ZPIPE) {
        L = sweep_zpipe_q27_cum1(p->store, pat);
        a.zc = p->zpipe;
        launch_shape(a.g, a.zc, grid, block);
    } else if (variant == LBM_VARIANT_PAIR) {
        L = pair_launcher(p, pat);
        block = dim3(32, PAIR_ROWS, 1);
        grid = dim3((a.g.nx + 63) / 64, (a.g.ny + PAIR_ROWS - 1) / PAIR_ROWS, a.g.nz);
    } else {
        L = sweep_launcher(p, pat);
        launch_shape(a.g, a.zc, grid, block);
        if (p->block_x > 0 && a.zc == 1) {
            block = dim3(p->block_x, 256 / p->block_x, 1);
            grid = dim3((a.g.nx + block.x - 1) / block.x, (a.g.ny + block.y - 1) / block.y, a.g.nz);
        }
    }
    if (L == nullptr) return fail(LBM_E_UNSUPPORTED, "no kernel for this storage type / pattern");
    cudaError_t e = L(a, grid, block, stream);
    if (e != cudaSuccess) return cuda_fail(e, "sweep launch");
    return LBM_OK;
}

int lbm_sweep(const LbmPlan* p, const void* src, void* dst, const int64_t strides[4], const uint8_t* flags,
              int parity, float* omega_out, void* stream) {
    int rc = validate_sweep(p, src, dst, strides, flags, omega_out);
    if (rc) return rc;
    if (parity != 0 && parity != 1) return fail(LBM_E_INVALID, "parity must be 0 (EVEN) or 1 (ODD)");
    return launch_sweep_checked(p, src, dst, strides, flags, parity, omega_out, static_cast<cudaStream_t>(stream));
}

int lbm_sweep_variant(const LbmPlan* p, const void* src, const void* dst, const int64_t strides[4], int parity,
                      const float* omega_out, int* variant) {
    if (variant == nullptr) return fail(LBM_E_INVALID, "variant must not be NULL");
    int rc = validate_sweep(p, src, dst, strides, nullptr, omega_out);
    if (rc) return rc;
    if (parity != 0 && parity != 1) return fail(LBM_E_INVALID, "parity must be 0 (EVEN) or 1 (ODD)");
    *variant = sweep_variant(p, src, dst, strides, pattern_kind(p, parity), omega_out);
    return LBM_OK;
}

int lbm_plan_status(LbmPlan* p, uint32_t* status, int clear) {
    if (p == nullptr || status == nullptr) return fail(LBM_E_INVALID, "plan and status must not be NULL");
    int rc = check_device(p);
    if (rc) return rc;
    unsigned v = 0;
    cudaError_t e = cudaMemcpy(&v, p->status, sizeof(v), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "reading the plan status");
    if (clear) {
        e = cudaMemset(p->status, 0, sizeof(unsigned));
        if (e != cudaSuccess) return cuda_fail(e, "clearing the plan status");
    }
    *status = v;
    return LBM_OK;
}

int lbm_run(const LbmPlan* p, void* a, void* b, const int64_t strides[4], const uint8_t* flags, int first_parity,
            int steps, int* result_in_b, void* stream) {
    if (p == nullptr) return fail(LBM_E_INVALID, "plan is NULL");
    if (steps < 0) return fail(LBM_E_INVALID, "steps must be >= 0");
    if (first_parity != 0 && first_parity != 1) return fail(LBM_E_INVALID, "parity must be 0 (EVEN) or 1 (ODD)");
    const bool inplace = pattern_inplace(p->desc.pattern);
    int rc = validate_sweep(p, a, inplace ? a : b, strides, flags, nullptr);
    if (rc) return rc;
    void* src = a;
    void* dst = inplace ? a : b;
    int parity = first_parity;
    int in_b = 0;
    for (int t = 0; t < steps; ++t) {
        rc = launch_sweep_checked(p, src, dst, strides, flags, parity, nullptr, static_cast<cudaStream_t>(stream));
        if (rc) return rc;
        if (inplace) parity ^= 1;
        else { void* tmp = src; src = dst; dst = tmp; in_b ^= 1; }
    }
    if (result_in_b) *result_in_b = in_b;
    return LBM_OK;
}

static int macro_common(const LbmPlan* p, const void* pdfs, const int64_t strides[4], const void* rho,
                        const int64_t rs[3], const void* u, const int64_t us[4], MacroArgs& a) {
    int rc;
    if ((rc = check_device(p))) return rc;
    if ((rc = check_strides(p, strides))) return rc;
    if ((rc = check_device_ptr(p, pdfs, "pdfs", false))) return rc;
    if ((rc = check_device_ptr(p, rho, "rho", true))) return rc;
    if ((rc = check_device_ptr(p, u, "u", true))) return rc;
    if (rho && rs == nullptr) return fail(LBM_E_INVALID, "rho_strides is NULL");
    if (u && us == nullptr) return fail(LBM_E_INVALID, "u_strides is NULL");
    a.g = make_grid(p, strides, nullptr);
    a.p = p->phys;
    a.pdfs = const_cast<void*>(pdfs);
    a.rho = const_cast<void*>(rho);
    a.u = const_cast<void*>(u);
    for (int k = 0; k < 3; ++k) a.rs[k] = rho ? rs[k] : 0;
    for (int k = 0; k < 4; ++k) a.us[k] = u ? us[k] : 0;
    return LBM_OK;
}

int lbm_set_equilibrium(const LbmPlan* p, void* pdfs, const int64_t strides[4], const void* rho,
                        const int64_t rho_strides[3], const void* u, const int64_t u_strides[4], int prev_parity,
                        void* stream) {
    if (p == nullptr) return fail(LBM_E_INVALID, "plan is NULL");
    if (rho == nullptr || u == nullptr) return fail(LBM_E_INVALID, "rho and u are required");
    MacroArgs a;
    int rc = macro_common(p, pdfs, strides, rho, rho_strides, u, u_strides, a);
    if (rc) return rc;
    MacroLauncher L = set_eq_launcher(p, pattern_kind(p, prev_parity ? 1 : 0));
    if (L == nullptr) return fail(LBM_E_UNSUPPORTED, "no setter kernel");
    dim3 grid, block;
    launch_shape(a.g, 1, grid, block);
    cudaError_t e = L(a, grid, block, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? LBM_OK : cuda_fail(e, "setter launch");
}

int lbm_get_macroscopic(const LbmPlan* p, const void* pdfs, const int64_t strides[4], void* rho,
                        const int64_t rho_strides[3], void* u, const int64_t u_strides[4], int prev_parity,
                        void* stream) {
    if (p == nullptr) return fail(LBM_E_INVALID, "plan is NULL");
    MacroArgs a;
    int rc = macro_common(p, pdfs, strides, rho, rho_strides, u, u_strides, a);
    if (rc) return rc;
    const int pat = pattern_kind(p, prev_parity ? 1 : 0);
    MacroLauncher L = p->q == 19 ? get_launcher_q<19>(p->store, pat) : get_launcher_q<27>(p->store, pat);
    if (L == nullptr) return fail(LBM_E_UNSUPPORTED, "no getter kernel");
    dim3 grid, block;
    launch_shape(a.g, 1, grid, block);
    cudaError_t e = L(a, grid, block, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? LBM_OK : cuda_fail(e, "getter launch");
}

int lbm_reduce_conserved(const LbmPlan* p, const void* pdfs, const int64_t strides[4], const uint8_t* flags,
                         int prev_parity, double out[5], void* stream) {
    if (p == nullptr || out == nullptr) return fail(LBM_E_INVALID, "plan and out must not be NULL");
    MacroArgs a;
    int rc = macro_common(p, pdfs, strides, nullptr, nullptr, nullptr, nullptr, a);
    if (rc) return rc;
    if ((rc = check_device_ptr(p, flags, "flags", true))) return rc;
    a.g.flags = flags;
    const int pat = pattern_kind(p, prev_parity ? 1 : 0);
    ReduceLauncher L = p->q == 19 ? reduce_launcher_q<19>(p->store, pat) : reduce_launcher_q<27>(p->store, pat);
    if (L == nullptr) return fail(LBM_E_UNSUPPORTED, "no reduction kernel for this storage type / pattern");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = L(a, p->red_blocks, p->partial, s);
    if (e != cudaSuccess) return cuda_fail(e, "reduction launch");
    k_reduce_finish<<<1, 32, 0, s>>>(p->partial, p->red_blocks, p->red_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "reduction finish launch");
    e = cudaMemcpyAsync(out, p->red_out, 5 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(e, "reduction copy");
    e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? LBM_OK : cuda_fail(e, "reduction sync");
}

int lbm_closure_set_weights(const float* params, int n, void* stream) {
    if (params == nullptr) return fail(LBM_E_INVALID, "params is NULL");
    if (n != MLP_PARAMS) return fail(LBM_E_INVALID, "the closure takes %d parameters, got %d", MLP_PARAMS, n);
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, params) == cudaSuccess && at.type == cudaMemoryTypeDevice)
        return fail(LBM_E_INVALID, "params must be host memory");
    cudaGetLastError();
    cudaError_t e = closure_upload(params, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "closure upload");
    return LBM_OK;
}

int lbm_flags_finalize(const LbmPlan* p, uint8_t* flags, void* stream) {
    if (p == nullptr) return fail(LBM_E_INVALID, "plan is NULL");
    int rc;
    if ((rc = check_device(p))) return rc;
    if ((rc = check_device_ptr(p, flags, "flags", false))) return rc;
    int64_t s[4] = {1, p->desc.dims[0] + 2, (int64_t)(p->desc.dims[0] + 2) * (p->desc.dims[1] + 2), 0};
    Grid g = make_grid(p, s, flags);
    dim3 grid, block;
    launch_shape(g, 1, grid, block);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (p->q == 19) k_flags_finalize<19><<<grid, block, 0, st>>>(g);
    else k_flags_finalize<27><<<grid, block, 0, st>>>(g);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "flag finalize launch");
    // the row summary the sweeps of this plan use with this flag field
    p->rowmask_flags = nullptr;
    e = cudaMemsetAsync(p->rowmask, 0, rowmask_bytes(p), st);
    if (e != cudaSuccess) return cuda_fail(e, "clearing the row summary");
    const int rows = g.ny * g.nz;
    k_row_mask<<<(rows + 255) / 256, 256, 0, st>>>(g, p->rowmask);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "row summary launch");
    p->rowmask_flags = flags;
    return LBM_OK;
}

int lbm_plan_set_stage_wait(LbmPlan* p, uint64_t wait_ns, int probe) {
    if (p == nullptr) return fail(LBM_E_INVALID, "plan is NULL");
    if (wait_ns > 60ull * 1000000000ull) return fail(LBM_E_INVALID, "wait_ns above 60 s");
    p->stage_wait_ns = wait_ns;
    p->stage_probe = probe ? 1 : 0;
    return LBM_OK;
}

int lbm_plan_set_links(LbmPlan* p, const LbmLinkTables* t) {
    if (p == nullptr) return fail(LBM_E_INVALID, "plan is NULL");
    int rc;
    if ((rc = check_device(p))) return rc;
    if (t == nullptr) {                          // detach
        p->ubb_block = nullptr;
        p->ubb_link_vel = nullptr;
        p->link_code = nullptr;
        p->link_value = nullptr;
        p->ubb_link_mask = 0;
        p->phys.ubb_link_mask = 0;
        return LBM_OK;
    }
    if (t->ubb_mask & ~0xfu) return fail(LBM_E_INVALID, "ubb_mask has bits beyond UBB number 3");
    if ((rc = check_device_ptr(p, t->cell_block, "cell_block", false))) return rc;
    if (t->n_blocks < 1) return fail(LBM_E_INVALID, "n_blocks must be positive");
    if ((rc = check_device_ptr(p, t->ubb_velocity, "ubb_velocity", t->ubb_mask == 0))) return rc;
    if ((rc = check_device_ptr(p, t->link_code, "link_code", true))) return rc;
    if ((rc = check_device_ptr(p, t->link_value, "link_value", true))) return rc;
    p->ubb_block = reinterpret_cast<const int*>(t->cell_block);
    p->ubb_link_vel = t->ubb_mask ? t->ubb_velocity : nullptr;
    p->link_code = reinterpret_cast<const int*>(t->link_code);
    p->link_value = t->link_value;
    p->ubb_link_mask = t->ubb_mask;
    p->phys.ubb_link_mask = t->ubb_mask;
    return ensure_ubb_buffer(p);
}

}  // extern "C"

// ------------------------------------------------------------------ sparse (list-based) domains
namespace {

SparseLauncher sparse_launcher(const LbmPlan* p) {
    if (p->q == 19 && p->mk == MK_POP) return sparse_q19_pop(p->store);
    if (p->q == 19 && p->mk == MK_MRT) return sparse_q19_mrt(p->store);
    if (p->q == 27 && p->mk == MK_POP) return sparse_q27_pop(p->store);
    if (p->q == 27 && p->mk == MK_MRT) return sparse_q27_mrt(p->store);
    if (p->q == 27 && p->mk == MK_CUM) return sparse_q27_cum(p->store);
    if (p->q == 27 && p->mk == MK_CUM1) return sparse_q27_cum1(p->store);
    if (p->q == 27 && p->mk == MK_CM) return sparse_q27_cm(p->store);
    return nullptr;
}

SparseSetLauncher sparse_set_launcher(const LbmPlan* p) {
    if (p->q == 19 && p->mk == MK_POP) return sparse_set_q19_pop(p->store);
    if (p->q == 19 && p->mk == MK_MRT) return sparse_set_q19_mrt(p->store);
    if (p->q == 27 && p->mk == MK_POP) return sparse_set_q27_pop(p->store);
    if (p->q == 27 && p->mk == MK_MRT) return sparse_set_q27_mrt(p->store);
    if (p->q == 27 && (p->mk == MK_CUM || p->mk == MK_CUM1)) return sparse_set_q27_cum(p->store);
    if (p->q == 27 && p->mk == MK_CM) return sparse_set_q27_cm(p->store);
    return nullptr;
}

template <class S, class R, int Q>
cudaError_t launch_sparse_get(const SparseArgs& a, double* rho, double* u, cudaStream_t s) {
    k_sparse_get_macroscopic<S, R, Q><<<(unsigned)((a.n_fluid + 255) / 256), 256, 0, s>>>(a, rho, u);
    return cudaGetLastError();
}

template <class S, class R, int Q>
cudaError_t launch_sparse_ubb(const SparseArgs& a, const uint32_t* links, int64_t n, const double* u,
                              cudaStream_t s) {
    k_sparse_ubb<S, R, Q><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, links, n, u[0], u[1], u[2]);
    return cudaGetLastError();
}

int sparse_common(const LbmPlan* p, const void* src, const void* dst, int64_t n_fluid, int64_t n_cells,
                  SparseArgs& a) {
    if (p == nullptr) return fail(LBM_E_INVALID, "plan is NULL");
    int rc;
    if ((rc = check_device(p))) return rc;
    if (p->store != ST_F64 && p->store != ST_F32)
        return fail(LBM_E_UNSUPPORTED, "sparse domains are built for FP64 and FP32 storage");
    if (p->desc.pattern != LBM_PATTERN_PULL)
        return fail(LBM_E_UNSUPPORTED, "sparse domains stream by the pull pattern (the index list encodes it)");
    if (p->desc.sgs == LBM_SGS_MLP)
        return fail(LBM_E_UNSUPPORTED, "the learned closure is not built for sparse domains");
    if (n_fluid < 0 || n_cells < n_fluid)
        return fail(LBM_E_INVALID, "need 0 <= n_fluid <= n_cells (got %lld, %lld)", (long long)n_fluid,
                    (long long)n_cells);
    if (n_cells * (int64_t)p->q > (int64_t)UINT32_MAX)
        return fail(LBM_E_INVALID, "n_cells * Q must fit the 32-bit index list");
    if (n_fluid / 256 >= (int64_t)INT32_MAX) return fail(LBM_E_INVALID, "too many fluid cells for one launch");
    if ((rc = check_device_ptr(p, src, "src", false))) return rc;
    if ((rc = check_device_ptr(p, dst, "dst", false))) return rc;
    memset(&a, 0, sizeof(a));
    a.p = p->phys;
    a.src = src;
    a.dst = const_cast<void*>(dst);
    a.n_fluid = n_fluid;
    a.n_cells = n_cells;
    return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_sparse_sweep(const LbmPlan* p, const void* src, void* dst, const uint32_t* index, int64_t n_fluid,
                     int64_t n_cells, void* stream) {
    SparseArgs a;
    int rc = sparse_common(p, src, dst, n_fluid, n_cells, a);
    if (rc) return rc;
    if (src == dst) return fail(LBM_E_INVALID, "the sparse sweep needs two distinct PDF lists");
    if ((rc = check_device_ptr(p, index, "index", false))) return rc;
    a.index = index;
    SparseLauncher L = sparse_launcher(p);
    if (L == nullptr) return fail(LBM_E_UNSUPPORTED, "no sparse kernel built for this stencil/method/dtype");
    if (n_fluid == 0) return LBM_OK;
    cudaError_t e = L(a, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? LBM_OK : cuda_fail(e, "sparse sweep launch");
}

int lbm_sparse_set_equilibrium(const LbmPlan* p, void* pdfs, const double* rho, const double* u, int64_t n_fluid,
                               int64_t n_cells, void* stream) {
    SparseArgs a;
    int rc = sparse_common(p, pdfs, pdfs, n_fluid, n_cells, a);
    if (rc) return rc;
    if ((rc = check_device_ptr(p, rho, "rho", false))) return rc;
    if ((rc = check_device_ptr(p, u, "u", false))) return rc;
    SparseSetLauncher L = sparse_set_launcher(p);
    if (L == nullptr) return fail(LBM_E_UNSUPPORTED, "no sparse setter kernel");
    if (n_fluid == 0) return LBM_OK;
    cudaError_t e = L(a, rho, u, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? LBM_OK : cuda_fail(e, "sparse setter launch");
}

int lbm_sparse_get_macroscopic(const LbmPlan* p, const void* pdfs, double* rho, double* u, int64_t n_fluid,
                               int64_t n_cells, void* stream) {
    SparseArgs a;
    int rc = sparse_common(p, pdfs, pdfs, n_fluid, n_cells, a);
    if (rc) return rc;
    if ((rc = check_device_ptr(p, rho, "rho", true))) return rc;
    if ((rc = check_device_ptr(p, u, "u", true))) return rc;
    if (n_fluid == 0) return LBM_OK;
    cudaError_t e;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (p->q == 19)
        e = p->store == ST_F64 ? launch_sparse_get<double, double, 19>(a, rho, u, s)
                               : launch_sparse_get<float, float, 19>(a, rho, u, s);
    else
        e = p->store == ST_F64 ? launch_sparse_get<double, double, 27>(a, rho, u, s)
                               : launch_sparse_get<float, float, 27>(a, rho, u, s);
    return e == cudaSuccess ? LBM_OK : cuda_fail(e, "sparse getter launch");
}

int lbm_sparse_ubb(const LbmPlan* p, void* pdfs, const uint32_t* links, int64_t n_links, int64_t n_cells,
                   const double velocity[3], void* stream) {
    SparseArgs a;
    int rc = sparse_common(p, pdfs, pdfs, 0, n_cells, a);
    if (rc) return rc;
    if (velocity == nullptr) return fail(LBM_E_INVALID, "velocity must not be NULL");
    if (n_links < 0 || n_links / 256 >= (int64_t)INT32_MAX) return fail(LBM_E_INVALID, "bad number of links");
    if (n_links == 0) return LBM_OK;
    if ((rc = check_device_ptr(p, links, "links", false))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (p->q == 19)
        e = p->store == ST_F64 ? launch_sparse_ubb<double, double, 19>(a, links, n_links, velocity, s)
                               : launch_sparse_ubb<float, float, 19>(a, links, n_links, velocity, s);
    else
        e = p->store == ST_F64 ? launch_sparse_ubb<double, double, 27>(a, links, n_links, velocity, s)
                               : launch_sparse_ubb<float, float, 27>(a, links, n_links, velocity, s);
    return e == cudaSuccess ? LBM_OK : cuda_fail(e, "sparse UBB launch");
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Batched domains: one persistent launch per step over a tile table spanning every domain.

struct LbmBatch {
    int device;
    int q, mk, store, pattern;
    int n_domains;
    LbmBatchTiling tiling;
    int64_t n_tiles, grid_blocks, cells;
    SweepArgs* d_domains;      // [2][n_domains]: parity 0 and parity 1 source/destination
    BatchTile* d_tiles;
};

namespace {

BatchLauncher batched_launcher(int q, int mk, int store, int pat) {
    if (q == 19 && mk == MK_POP) return batched_q19_pop(store, pat);
    if (q == 19 && mk == MK_MRT) return batched_q19_mrt(store, pat);
    if (q == 27 && mk == MK_POP) return batched_q27_pop(store, pat);
    if (q == 27 && mk == MK_MRT) return batched_q27_mrt(store, pat);
    if (q == 27 && mk == MK_CUM) return batched_q27_cum(store, pat);
    if (q == 27 && mk == MK_CUM1) return batched_q27_cum1(store, pat);
    if (q == 27 && mk == MK_CM) return batched_q27_cm(store, pat);
    return nullptr;
}

// The plan-shaped view of one domain, for the shared validation and physics helpers.
void domain_plan(const LbmPlanDesc* common, const LbmDomainDesc& d, int device, LbmPlan& p) {
    p.desc = *common;
    memcpy(p.desc.dims, d.dims, sizeof(d.dims));
    memcpy(p.desc.periodic, d.periodic, sizeof(d.periodic));
    memcpy(p.desc.rates, d.rates, sizeof(d.rates));
    memcpy(p.desc.ubb_velocity, d.ubb_velocity, sizeof(d.ubb_velocity));
    p.device = device;
    p.q = common->stencil;
    p.store = common->store_dtype;
    p.partial = nullptr;
    p.red_out = nullptr;
    p.ubb_block = nullptr;
    p.ubb_link_vel = nullptr;
    p.ubb_link_mask = 0;
    fill_physics(&p, &p.desc);
}

int64_t field_extent(const LbmDomainDesc& d, int q) {
    const int64_t ex = d.dims[0] + 2, ey = d.dims[1] + 2, ez = d.dims[2] + 2;
    return (q - 1) * d.strides[3] + (ez - 1) * d.strides[2] + (ey - 1) * d.strides[1] + ex;
}

int64_t flags_extent(const LbmDomainDesc& d) {
    return int64_t(d.dims[0] + 2) * (d.dims[1] + 2) * (d.dims[2] + 2);
}

// Intervals [begin, end) must not overlap.
bool disjoint(std::vector<std::pair<int64_t, int64_t>>& iv) {
    std::sort(iv.begin(), iv.end());
    for (size_t k = 1; k < iv.size(); ++k)
        if (iv[k].first < iv[k - 1].second) return false;
    return true;
}

}  // namespace

extern "C" {

int lbm_batch_create(const LbmPlanDesc* common, const LbmDomainDesc* domains, int n_domains, void* buffer_a,
                     void* buffer_b, int64_t buffer_elems, uint8_t* flags, int64_t flags_bytes,
                     const LbmBatchTiling* tiling, LbmBatch** out) {
    if (common == nullptr || domains == nullptr || tiling == nullptr || out == nullptr)
        return fail(LBM_E_INVALID, "common, domains, tiling and out must not be NULL");
    *out = nullptr;
    if (n_domains < 1) return fail(LBM_E_INVALID, "a batch needs at least one domain");
    const LbmBatchTiling t = *tiling;
    if (t.tile_x < 1 || t.tile_y < 1 || t.tile_x * t.tile_y > 256 || t.cells_z < 1 || t.blocks_per_sm < 0)
        return fail(LBM_E_INVALID, "tiling %dx%dx%d (%d blocks/SM): need tile_x*tile_y in [1, 256], cells_z >= 1",
                    t.tile_x, t.tile_y, t.cells_z, t.blocks_per_sm);
    if (common->pattern != LBM_PATTERN_PULL && common->pattern != LBM_PATTERN_AA)
        return fail(LBM_E_UNSUPPORTED, "batched sweeps are built for the pull and AA patterns");
    if (common->fixed_density != 0.0 || common->fixed_density1 != 0.0)
        return fail(LBM_E_UNSUPPORTED, "batched sweeps are built without FixedDensity boundaries");
    if (common->fourth_order_limiter != 0.0)
        return fail(LBM_E_UNSUPPORTED, "batched sweeps are built without the fourth-order correction");
    const bool inplace = common->pattern != LBM_PATTERN_PULL;
    if (inplace && buffer_b == nullptr) buffer_b = buffer_a;
    if (inplace && buffer_b != buffer_a) return fail(LBM_E_INVALID, "in-place patterns use buffer_a only");
    if (!inplace && buffer_a == buffer_b) return fail(LBM_E_INVALID, "the pull pattern needs two distinct buffers");

    int device = -1;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    LbmPlan p0{};
    domain_plan(common, domains[0], device, p0);
    int rc;
    if ((rc = check_device_ptr(&p0, buffer_a, "buffer_a", false))) return rc;
    if ((rc = check_device_ptr(&p0, buffer_b, "buffer_b", false))) return rc;
    if ((rc = check_device_ptr(&p0, flags, "flags", true))) return rc;

    // Every domain on its own, then the batch as a whole.
    bool all_cum1 = true;
    std::vector<std::pair<int64_t, int64_t>> fields, flag_ranges;
    int64_t cells = 0;
    for (int k = 0; k < n_domains; ++k) {
        const LbmDomainDesc& d = domains[k];
        LbmPlan pk{};
        domain_plan(common, d, device, pk);
        if ((rc = validate_desc(&pk.desc))) return fail(rc, "domain %d: %s", k, g_err.c_str());
        if ((rc = check_strides(&pk, d.strides))) return fail(rc, "domain %d: %s", k, g_err.c_str());
        if (d.offset < 0 || d.offset + field_extent(d, pk.q) > buffer_elems)
            return fail(LBM_E_INVALID, "domain %d: field at offset %lld runs past the %lld-element buffers", k,
                        (long long)d.offset, (long long)buffer_elems);
        fields.emplace_back(d.offset, d.offset + field_extent(d, pk.q));
        if (d.flags_offset >= 0) {
            if (flags == nullptr) return fail(LBM_E_INVALID, "domain %d has flags but the flag buffer is NULL", k);
            if (d.flags_offset + flags_extent(d) > flags_bytes)
                return fail(LBM_E_INVALID, "domain %d: flags at byte %lld run past the %lld-byte flag buffer", k,
                            (long long)d.flags_offset, (long long)flags_bytes);
            flag_ranges.emplace_back(d.flags_offset, d.flags_offset + flags_extent(d));
        } else if (d.flags_offset != -1) {
            return fail(LBM_E_INVALID, "domain %d: flags_offset must be >= 0 or -1", k);
        }
        if (!cumulant_high_orders_relax_to_equilibrium(&pk.desc)) all_cum1 = false;
        if (needs_ubb_density(&pk.desc, 0) && d.flags_offset >= 0)
            return fail(LBM_E_UNSUPPORTED, "domain %d: moving UBB walls of a compressible method are not built "
                        "for batches", k);
        cells += int64_t(d.dims[0]) * d.dims[1] * d.dims[2];
    }
    if (!disjoint(fields)) return fail(LBM_E_INVALID, "two domains' fields overlap");
    if (!disjoint(flag_ranges)) return fail(LBM_E_INVALID, "two domains' flags overlap");

    const int q = common->stencil;
    if (common->sgs == LBM_SGS_MLP) return fail(LBM_E_UNSUPPORTED, "batched sweeps do not take the learned closure");
    int mk = common->method == LBM_METHOD_MRT ? MK_MRT
             : common->method == LBM_METHOD_CUMULANT ? MK_CUM
             : common->method == LBM_METHOD_CENTRAL_MOMENT ? MK_CM : MK_POP;
    if (mk == MK_CUM && all_cum1) mk = MK_CUM1;
    const int store = common->store_dtype;
    if (batched_launcher(q, mk, store, PAT_PULL) == nullptr)
        return fail(LBM_E_UNSUPPORTED, "no batched kernel for this stencil/method/dtype");

    // Per-domain arguments for both parities, and the tile table (domain-major, then z, y, x).
    const size_t es = store_size(store);
    char* A = static_cast<char*>(buffer_a);
    char* B = static_cast<char*>(buffer_b);
    std::vector<SweepArgs> args(2 * size_t(n_domains));
    std::vector<BatchTile> tiles;
    for (int k = 0; k < n_domains; ++k) {
        const LbmDomainDesc& d = domains[k];
        LbmPlan pk{};
        domain_plan(common, d, device, pk);
        SweepArgs a;
        memset(&a, 0, sizeof(a));
        a.g = make_grid(&pk, d.strides, d.flags_offset >= 0 ? flags + d.flags_offset : nullptr);
        a.p = pk.phys;
        a.omega_out = nullptr;
        a.src = A + d.offset * es;
        a.dst = B + d.offset * es;
        args[k] = a;
        a.src = B + d.offset * es;
        a.dst = A + d.offset * es;
        args[n_domains + k] = a;
        for (int z = 0; z < d.dims[2]; z += t.cells_z)
            for (int y = 0; y < d.dims[1]; y += t.tile_y)
                for (int x = 0; x < d.dims[0]; x += t.tile_x) tiles.push_back(BatchTile{k, x, y, z});
    }
    if (tiles.size() >= (size_t(1) << 31)) return fail(LBM_E_INVALID, "too many tiles for one launch");

    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    LbmBatch* b = new LbmBatch();
    b->device = device;
    b->q = q;
    b->mk = mk;
    b->store = store;
    b->pattern = common->pattern;
    b->n_domains = n_domains;
    b->tiling = t;
    b->n_tiles = (int64_t)tiles.size();
    b->grid_blocks = t.blocks_per_sm == 0 ? b->n_tiles : std::min<int64_t>(b->n_tiles, int64_t(sms) * t.blocks_per_sm);
    b->cells = cells;
    b->d_domains = nullptr;
    b->d_tiles = nullptr;
    e = cudaMalloc(&b->d_domains, sizeof(SweepArgs) * args.size());
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tiles, sizeof(BatchTile) * tiles.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_domains, args.data(), sizeof(SweepArgs) * args.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_tiles, tiles.data(), sizeof(BatchTile) * tiles.size(), cudaMemcpyHostToDevice);
    // Near-wall marks, per domain with flags (as lbm_flags_finalize does for one field).
    for (int k = 0; k < n_domains && e == cudaSuccess; ++k) {
        if (domains[k].flags_offset < 0) continue;
        const Grid& g = args[k].g;
        const dim3 block(32, 8, 1), grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz);
        if (q == 19) k_flags_finalize<19><<<grid, block>>>(g);
        else k_flags_finalize<27><<<grid, block>>>(g);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(b->d_domains);
        cudaFree(b->d_tiles);
        delete b;
        return cuda_fail(e, "lbm_batch_create");
    }
    *out = b;
    return LBM_OK;
}

int lbm_batch_sweep(const LbmBatch* b, int parity, void* stream) {
    if (b == nullptr) return fail(LBM_E_INVALID, "batch is NULL");
    if (parity != 0 && parity != 1) return fail(LBM_E_INVALID, "parity must be 0 (EVEN) or 1 (ODD)");
    const bool inplace = b->pattern != LBM_PATTERN_PULL;
    const int pat = inplace ? (parity ? PAT_AA_ODD : PAT_AA_EVEN) : PAT_PULL;
    BatchLauncher L = batched_launcher(b->q, b->mk, b->store, pat);
    if (L == nullptr) return fail(LBM_E_UNSUPPORTED, "no batched kernel for this pattern");
    BatchArgs a;
    a.domains = b->d_domains;
    a.tiles = b->d_tiles;
    a.n_domains = b->n_domains;
    a.n_tiles = (int)b->n_tiles;
    a.cells_z = b->tiling.cells_z;
    a.parity = inplace ? 0 : parity;
    cudaError_t e = L(a, dim3((unsigned)b->grid_blocks), dim3(b->tiling.tile_x, b->tiling.tile_y, 1),
                      static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "batched sweep launch");
    return LBM_OK;
}

int lbm_batch_info(const LbmBatch* b, int64_t info[4]) {
    if (b == nullptr || info == nullptr) return fail(LBM_E_INVALID, "batch and info must not be NULL");
    info[0] = b->n_tiles;
    info[1] = b->grid_blocks;
    info[2] = b->cells;
    info[3] = b->n_tiles * b->tiling.tile_x * b->tiling.tile_y * b->tiling.cells_z;
    return LBM_OK;
}

int lbm_batch_destroy(LbmBatch* b) {
    if (b == nullptr) return LBM_OK;
    cudaFree(b->d_domains);
    cudaFree(b->d_tiles);
    delete b;
    return LBM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Allocation-free variant of lbm_reduce_conserved.
//
// Some callers cannot call cudaMalloc at all: code running where device allocation is forbidden
// or must stay predictable (inside a fixed memory budget, an allocator-less embedding, or a
// process whose memory is all pre-reserved by another framework).  For them this entry point
// takes the plan description instead of a plan (lbm_plan_create allocates the reduction
// scratch) and keeps its block partial sums in a file-scope device array instead.
//
// Capacity: LBM_NOALLOC_MAX_BLOCKS partial sums of 5 doubles (80 KiB).  The launch uses at most
// 4 blocks per SM; a call that would need more partials than the array holds is rejected.  The
// array exists once per GPU that loads the library, for the life of the process.  Every call
// overwrites the partials it reads, so no state carries over between calls, but calls that
// overlap on the GPU (different streams, or concurrent host threads) share the array and race.
// The first call on a device resolves the array's device address (cudaGetSymbolAddress); with
// lazy module loading that first call may also load the library's module on the device, which
// reserves the array itself and the code.  Make that first call at start-up, before the caller's
// memory budget is fixed.  The call waits for its result (cudaStreamSynchronize), so it cannot
// be recorded into a CUDA graph.
static constexpr int LBM_NOALLOC_MAX_BLOCKS = 2048;
static __device__ __align__(256) double g_noalloc_scratch[LBM_NOALLOC_MAX_BLOCKS * 5 + 5];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kMaxDevices] = {};

int noalloc_scratch(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return fail(LBM_E_DEVICE, "device index %d out of range", device);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_ptr[device] == nullptr) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);   // the current device's copy
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(reduction scratch)");
        g_noalloc_ptr[device] = static_cast<double*>(ptr);
    }
    *out = g_noalloc_ptr[device];
    return LBM_OK;
}
}  // namespace

extern "C" int lbm_reduce_conserved_noalloc(const LbmPlanDesc* desc, const void* pdfs, const int64_t strides[4],
                                            const uint8_t* flags, int prev_parity, double out[5], void* stream) {
    if (desc == nullptr || out == nullptr) return fail(LBM_E_INVALID, "desc and out must not be NULL");
    int rc = validate_desc(desc);
    if (rc) return rc;
    LbmPlan p;                                   // on the stack: nothing is allocated
    memset(&p, 0, sizeof(p));
    p.desc = *desc;
    cudaError_t e = cudaGetDevice(&p.device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    p.q = desc->stencil;
    p.mk = method_kind(desc);
    p.store = desc->store_dtype;
    fill_physics(&p, desc);
    MacroArgs a;
    if ((rc = macro_common(&p, pdfs, strides, nullptr, nullptr, nullptr, nullptr, a))) return rc;
    if ((rc = check_device_ptr(&p, flags, "flags", true))) return rc;
    a.g.flags = flags;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    const long long cells = (long long)desc->dims[0] * desc->dims[1] * desc->dims[2];
    const long long wanted = (cells + RED_THREADS - 1) / RED_THREADS;
    const int blocks = (int)(wanted < (long long)sms * 4 ? wanted : (long long)sms * 4);
    if (blocks > LBM_NOALLOC_MAX_BLOCKS)
        return fail(LBM_E_INVALID,
                    "lbm_reduce_conserved_noalloc needs %d partial sums but its static scratch holds %d "
                    "(at most 4 blocks per SM on up to %d SMs)", blocks, LBM_NOALLOC_MAX_BLOCKS,
                    LBM_NOALLOC_MAX_BLOCKS / 4);
    double* scratch = nullptr;
    if ((rc = noalloc_scratch(p.device, &scratch))) return rc;
    double* partial = scratch;
    double* result = scratch + 5 * LBM_NOALLOC_MAX_BLOCKS;
    const int pat = pattern_kind(&p, prev_parity ? 1 : 0);
    ReduceLauncher L = p.q == 19 ? reduce_launcher_q<19>(p.store, pat) : reduce_launcher_q<27>(p.store, pat);
    if (L == nullptr) return fail(LBM_E_UNSUPPORTED, "no reduction kernel for this storage type / pattern");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    e = L(a, blocks, partial, s);
    if (e != cudaSuccess) return cuda_fail(e, "reduction launch");
    k_reduce_finish<<<1, 32, 0, s>>>(partial, blocks, result);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "reduction finish launch");
    e = cudaMemcpyAsync(out, result, 5 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(e, "reduction copy");
    e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? LBM_OK : cuda_fail(e, "reduction sync");
}
