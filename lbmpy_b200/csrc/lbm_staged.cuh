// Row-staged sweep.  Persistent CTAs walk row segments ("tiles") of W cells of one (y, z) row.
// The Q population rows a tile reads are copied into a ring of NS shared-memory stages NS-1
// tiles ahead by the CTA's own threads with asynchronous 16-byte copies (cp.async; each warp
// owns whole population rows), completion counted on one mbarrier per stage
// (cp.async.mbarrier.arrive).  DRAM requests therefore stay in flight while the CTA collides,
// however many registers the collision holds, which is what limits the one-cell sweep: it issues
// its Q loads, then collides with nothing in flight.  (One 1D bulk copy per population row was
// tried first: at 0.5-1 KB per copy the copies, not DRAM, set the pace.)
//
// Stage layout, per population i: a 16-byte pad, the W staged cells, a 16-byte pad.  The value a
// tile's edge cell pulls from outside the segment (x = xs - 1 or xs + w, with the periodic wrap)
// is copied into the pad next to the segment by the same asynchronous copies (4 / 8 bytes; for
// 16-bit storage the aligned 4-byte word holding it, whose other half lies in the row or in its
// padding).  Each cell's flag is loaded one tile ahead.  Writes go straight to global memory.
//
// Every wait on a barrier is bounded (SweepArgs::stage_wait_ns, default STAGED_WAIT_NS); a CTA
// whose stage does not complete sets
// the plan's device status word, waits for its own copies in flight and returns.
//
// Opt-in (LBM_B200_STAGED=1).  Measured on B200 it matches but does not beat the other sweeps
// where they are latency-bound (D3Q27 cumulant AA channel 22.2 against 23.1 GLUPS; D3Q27 TRT AA
// channel 22.2 against 21.6), and loses where they stream at HBM speed: the per-tile CTA barrier
// makes each CTA's warps wait and issue in phase, and the shared-memory round trip adds Q loads
// per cell.
#pragma once
#include <type_traits>

#include "lbm_kernels.cuh"

namespace lbm {

constexpr int STAGED_MAX_NS = 8;
constexpr int STAGED_BAR_BYTES = 256;                     // barriers, tile headers, iterator
constexpr unsigned long long STAGED_WAIT_NS = 1000000000ull;
constexpr unsigned STAGED_WAIT_ITERS = 1u << 26;
constexpr unsigned STATUS_STAGE_TIMEOUT = 1u;

template <class S, int Q, int W>
struct StagedLayout {
    static constexpr int PADE = 16 / int(sizeof(S));      // elements in a 16-byte pad
    static constexpr int PS = W + 2 * PADE;               // elements per population row
    static constexpr int STAGE_BYTES = ((Q * PS * int(sizeof(S))) + 127) / 128 * 128;
    static constexpr size_t smem_bytes(int ns) { return STAGED_BAR_BYTES + size_t(ns) * STAGE_BYTES; }
};

namespace staged {
__device__ __forceinline__ unsigned saddr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void bar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_bar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// The suspend-time hint lets the hardware park a waiting warp (no issue slots spent polling)
// until the phase completes or about STAGED_SUSPEND_NS pass.
constexpr unsigned STAGED_SUSPEND_NS = 100000u;
__device__ __forceinline__ bool try_wait(unsigned bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity), "r"(STAGED_SUSPEND_NS)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Phase `parity` of the barrier completed; false once STAGED_WAIT_ITERS polls or `limit_ns`
// have passed without it.
__device__ __forceinline__ bool wait(unsigned bar, unsigned parity, unsigned long long limit_ns) {
    if (try_wait(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    for (unsigned it = 1; it < STAGED_WAIT_ITERS; ++it) {
        if (try_wait(bar, parity)) return true;
        if ((it & 15u) == 0 && now_ns() - t0 > limit_ns) return false;
    }
    return false;
}
// Asynchronous global -> shared copies of this thread (16 bytes bypassing L1; 4 / 8 bytes).
__device__ __forceinline__ void copy16(unsigned dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
template <int N>
__device__ __forceinline__ void copy_small(unsigned dst, const void* src) {
    static_assert(N == 4 || N == 8, "cp.async of 4 or 8 bytes");
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(dst), "l"(src), "n"(N) : "memory");
}
// The barrier's current phase also waits for every copy this thread has issued so far.
__device__ __forceinline__ void copies_arrive(unsigned bar) {
    asm volatile("cp.async.mbarrier.arrive.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void copies_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
}  // namespace staged

// A tile: row segment [xs, xs + w) of row (y, z).  Thread 0 keeps the CTA's tile headers in
// shared memory, so no other thread decodes a tile index.
struct StagedTile {
    int xs, w, y, z;
};

// Calls f(integral_constant<WP>) for the warp's index (a compare chain over the NW warps), so that
// f unrolls over the populations of its warp with compile-time indices.
template <int WP, int NW, class F>
__device__ __forceinline__ void staged_warp_dispatch(int warp, F&& f) {
    if constexpr (WP < NW) {
        if (warp == WP) f(std::integral_constant<int, WP>{});
        else staged_warp_dispatch<WP + 1, NW>(warp, f);
    }
}

// Requirements (checked by the host): pattern pull or AA; the address of interior cell x = 0 of
// every row and slot 16-byte aligned; row / plane / slot strides multiples of 16 bytes; nx a
// multiple of 16 / sizeof(S); for 16-bit storage a row stride of at least nx + 3 elements (the
// element after a row's ghost cell lies in the row's padding); 2 <= ns <= STAGED_MAX_NS.
//
// Shared memory: mbarriers (64 B), the tile header of each stage (8 x 16 B), the headers of the
// next two tiles to issue (2 x 16 B), thread 0's tile iterator (24 B), the probe barrier (8 B at
// byte 248), then the stages.
template <class S, class R, int Q, int MK, int PAT, int W>
__global__ void __launch_bounds__(W) k_sweep_staged(const SweepArgs a, const int ns) {
    static_assert(PAT == PAT_PULL || PAT == PAT_AA_EVEN || PAT == PAT_AA_ODD, "staged sweep: pull and AA");
    static_assert(W % 32 == 0 && W >= 32 && W <= 1024, "staged sweep: whole warps");
    using A = Access<PAT>;
    using Lay = StagedLayout<S, Q, W>;
    constexpr int NW = W / 32;
    constexpr int STAGE_ELEMS = Lay::STAGE_BYTES / int(sizeof(S));
    constexpr int COPIES = (W * int(sizeof(S)) / 16 + 31) / 32;   // 16-byte chunks per lane per row
    const Grid& g = a.g;
    extern __shared__ __align__(128) unsigned char smem[];
    const unsigned bar0 = staged::saddr(smem);
    StagedTile* const hdr = reinterpret_cast<StagedTile*>(smem + 64);
    StagedTile* const nexthdr = hdr + STAGED_MAX_NS;
    int* const iter = reinterpret_cast<int*>(nexthdr + 2);       // seg, y, z of the tile after nexthdr's; step
    S* const stage0 = reinterpret_cast<S*>(smem + STAGED_BAR_BYTES);
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int nseg = (g.nx + W - 1) / W;
    const int ntiles = nseg * g.ny * g.nz;
    const int G = gridDim.x;
    const int mine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / G + 1 : 0;
    const S* src = static_cast<const S*>(a.src);
    S* dst = static_cast<S*>(a.dst);

    const unsigned long long wait_ns = a.stage_wait_ns != 0 ? a.stage_wait_ns : STAGED_WAIT_NS;
    const unsigned probe_bar = bar0 + 248;
    if (tid == 0) {
        for (int s = 0; s < ns; ++s) staged::bar_init(bar0 + 8 * s, W);
        if (a.stage_probe) staged::bar_init(probe_bar, 1);
        staged::fence_bar_init();
        // CTA b sweeps tiles b, b + G, b + 2G, ... (walls spread over all CTAs); the step G is
        // added to (segment, y, z) with carries
        const int b = blockIdx.x;
        int seg = b % nseg, r = b / nseg;
        int y = r % g.ny, z = r / g.ny;
        const int gs = G % nseg, gr = G / nseg;
        iter[3] = gs; iter[4] = gr % g.ny; iter[5] = gr / g.ny;
        for (int k = 0; k <= ns; ++k) {
            const int xs = seg * W;
            const StagedTile t{xs, min(W, g.nx - xs), y, z};
            if (k < ns) hdr[k] = t;
            else nexthdr[0] = t;
            seg += iter[3]; y += iter[4]; z += iter[5];
            if (seg >= nseg) { seg -= nseg; ++y; }
            if (y >= g.ny) { y -= g.ny; ++z; }
        }
        iter[0] = seg; iter[1] = y; iter[2] = z;
    }
    __syncthreads();

    // Issues tile t into stage s: each warp copies its population rows (16-byte chunks over its
    // lanes) and, from lane 0, each row's halo value; then every thread arrives.
    auto issue = [&](const StagedTile t, int s) {
        S* st = stage0 + s * STAGE_ELEMS;
        const unsigned bar = bar0 + 8 * s;
        NbrOffsets nb;
        nb.init(g, t.xs, t.y, t.z);
        const int cell = (t.xs + 1) + (t.y + 1) * g.sy + (t.z + 1) * g.sz;
        const int chunks = t.w * int(sizeof(S)) / 16;
        // element offsets, from the segment's first cell, of the cells left of it and right of it
        const int hl = (t.xs == 0 && (g.periodic & 1)) ? g.nx - 1 : -1;
        const int hr = (t.xs + t.w == g.nx && (g.periodic & 1)) ? -t.xs : t.w;
        staged_warp_dispatch<0, NW>(warp, [&](auto wp) {
            constexpr int WP = decltype(wp)::value;
#pragma unroll
            for (int i = WP; i < Q; i += NW) {
                const S* row = src + eidx(A::template rslot<Q>(i) * g.sq,
                                          cell + nb.off(0, A::template roff<Q>(i, 1), A::template roff<Q>(i, 2)));
                const char* rowb = reinterpret_cast<const char*>(row);
                S* sr = st + i * Lay::PS + Lay::PADE;
                const unsigned sdst = staged::saddr(sr);
#pragma unroll
                for (int c = 0; c < COPIES; ++c) {
                    const int o = lane + 32 * c;
                    if (o < chunks) staged::copy16(sdst + 16u * o, rowb + 16 * o);
                }
                const int rx = A::template roff<Q>(i, 0);
                if (rx != 0 && lane == 0) {
                    const S* hp = row + (rx < 0 ? hl : hr);
                    S* hd = sr + (rx < 0 ? -1 : t.w);
                    if constexpr (sizeof(S) >= 4) {
                        staged::copy_small<int(sizeof(S))>(staged::saddr(hd), hp);
                    } else if (rx < 0) {    // word [x - 1, x]: x lands in the pad's last element
                        staged::copy_small<4>(staged::saddr(hd - 1), hp - 1);
                    } else {                // word [x, x + 1]: x lands in the pad's first element
                        staged::copy_small<4>(staged::saddr(hd), hp);
                    }
                }
            }
        });
        staged::copies_arrive(bar);
        staged::arrive(bar);
    };
    auto flag_of = [&](const StagedTile& t) -> int {
        if (g.flags == nullptr || tid >= t.w || !row_flagged(g, t.y, t.z)) return 0;
        return g.flags[(t.xs + tid + 1) + (t.y + 1) * g.fsy + (t.z + 1) * g.fsz];
    };

    const int npro = min(ns, mine);
    for (int k = 0; k < npro; ++k) issue(hdr[k], k);
    int fl = mine > 0 ? flag_of(hdr[0]) : 0;

    for (int k = 0; k < mine; ++k) {
        const int s = k % ns;
        bool ok = staged::wait(bar0 + 8 * s, unsigned(k / ns) & 1u, wait_ns);
        // probe: the last tile's data have landed and no copy is in flight; a wait on a barrier
        // that no thread arrives at runs out after wait_ns
        if (a.stage_probe && k == mine - 1) ok = ok && staged::wait(probe_bar, 0u, wait_ns);
        const S* st = stage0 + s * STAGE_ELEMS;
        const StagedTile t = hdr[s];
        R f[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i] = Conv<S, R>::ld(st + i * Lay::PS + Lay::PADE + tid + A::template roff<Q>(i, 0));
        if (!__syncthreads_and(ok)) {
            // a stage never completed: report, let this thread's copies in flight land, leave
            if (tid == 0 && a.status != nullptr) atomicOr(a.status, STATUS_STAGE_TIMEOUT);
            staged::copies_wait_all();
            return;
        }
        if (k + ns < mine) {
            const StagedTile tn = nexthdr[k & 1];
            issue(tn, s);
            if (tid == 0) {
                hdr[s] = tn;
                if (k + ns + 1 < mine) {
                    int seg = iter[0], y = iter[1], z = iter[2];
                    nexthdr[(k + 1) & 1] = StagedTile{seg * W, min(W, g.nx - seg * W), y, z};
                    seg += iter[3]; y += iter[4]; z += iter[5];
                    if (seg >= nseg) { seg -= nseg; ++y; }
                    if (y >= g.ny) { y -= g.ny; ++z; }
                    iter[0] = seg; iter[1] = y; iter[2] = z;
                }
            }
        }
        const int fl_next = k + 1 < mine ? flag_of(hdr[(k + 1) % ns]) : 0;

        if (tid < t.w && !(fl & FLAG_TYPE_MASK)) {
            const int x = t.xs + tid;
            NbrOffsets nb;
            nb.init(g, x, t.y, t.z);
            const int cell = (x + 1) + (t.y + 1) * g.sy + (t.z + 1) * g.sz;
            if (fl & FLAG_NEAR_WALL) bounce_back<S, R, Q, PAT>(f, a, nb, cell, x, t.y, t.z);
            const R om = collide<R, Q, MK>(f, a.p);
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const int off = nb.off(A::template woff<Q>(i, 0), A::template woff<Q>(i, 1), A::template woff<Q>(i, 2));
                Conv<S, R>::st(dst + eidx(A::template wslot<Q>(i) * g.sq, cell + off), f[i]);
            }
            if (a.omega_out != nullptr) a.omega_out[x + g.nx * (t.y + (long long)g.ny * t.z)] = (float)om;
        }
        fl = fl_next;
    }
}

}  // namespace lbm
