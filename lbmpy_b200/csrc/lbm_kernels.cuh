// Kernels of the B200 lattice Boltzmann sweep.
//
// k_sweep: one fused stream-collide update of every fluid cell, one thread per cell, SoA
// (fzyx) PDF layout, x fastest.  The PDF accessors follow lbmpy's fieldaccess.py:66-181:
//   pull      read src[x - c_i](i)            write dst[x](i)
//   AA even   read f[x](i)                    write f[x](inv i)
//   AA odd    read f[x - c_i](inv i)          write f[x + c_i](i)
//   EsoTwist  even/odd with offsets max(-c,0) / max(c,0) (fieldaccess.py:160-181)
//   push      read src[x](i)                  write dst[x + c_i](i)   (fieldaccess.py:78-87)
//   EsoPull / EsoPush  in place, by the direction's parity in the 'lehmann' ordering
//                                                                     (fieldaccess.py:184-318)
// Periodicity is an index wrap instead of ghost-layer copies, and NoSlip / UBB bounce-back
// (boundaries/boundaryconditions.py:128-139, 794-841) is fused into the read: where lbmpy's
// boundary kernel would have written the wall slot, the sweep reads the value that kernel
// would have copied (the f_out location of advanced_streaming/indexing.py:12-183).
#pragma once
#include "lbm_collide.cuh"

namespace lbm {

template <int PAT> struct Access {
    template <int Q>
    LBM_HD static constexpr bool leven(int i) { return lehmann_even(Lat<Q>::cx(i), Lat<Q>::cy(i), Lat<Q>::cz(i)); }
    // read location of direction i: offset (ox, oy, oz) and slot
    template <int Q>
    LBM_HD static constexpr int rslot(int i) {
        return (PAT == PAT_AA_ODD || PAT == PAT_ESO_ODD || PAT == PAT_EPULL_ODD || PAT == PAT_EPUSH_EVEN)
                   ? Lat<Q>::inv(i) : i;
    }
    template <int Q>
    LBM_HD static constexpr int roff(int i, int d) {
        const int c = d == 0 ? Lat<Q>::cx(i) : (d == 1 ? Lat<Q>::cy(i) : Lat<Q>::cz(i));
        return PAT == PAT_PULL ? -c
             : PAT == PAT_PUSH ? 0
             : PAT == PAT_AA_EVEN ? 0
             : PAT == PAT_AA_ODD ? -c
             : (PAT == PAT_EPULL_EVEN || PAT == PAT_EPULL_ODD) ? (leven<Q>(i) ? -c : 0)
             : (PAT == PAT_EPUSH_EVEN || PAT == PAT_EPUSH_ODD) ? (leven<Q>(i) ? 0 : -c)
             : (c < 0 ? -c : 0);   // EsoTwist: max(-c, 0)
    }
    template <int Q>
    LBM_HD static constexpr int wslot(int i) {
        return (PAT == PAT_AA_EVEN || PAT == PAT_ESO_EVEN || PAT == PAT_EPULL_EVEN || PAT == PAT_EPUSH_ODD)
                   ? Lat<Q>::inv(i) : i;
    }
    template <int Q>
    LBM_HD static constexpr int woff(int i, int d) {
        const int c = d == 0 ? Lat<Q>::cx(i) : (d == 1 ? Lat<Q>::cy(i) : Lat<Q>::cz(i));
        return PAT == PAT_PULL ? 0
             : PAT == PAT_PUSH ? c
             : PAT == PAT_AA_EVEN ? 0
             : PAT == PAT_AA_ODD ? c
             : (PAT == PAT_EPULL_EVEN || PAT == PAT_EPULL_ODD) ? (leven<Q>(i) ? 0 : c)
             : (PAT == PAT_EPUSH_EVEN || PAT == PAT_EPUSH_ODD) ? (leven<Q>(i) ? c : 0)
             : (c > 0 ? c : 0);    // EsoTwist: max(c, 0)
    }
};

// Write pattern of the previous step (where f_out lives) for the current pattern.
template <int PAT> struct PrevPattern {
    static constexpr int value = PAT == PAT_AA_EVEN ? PAT_AA_ODD
                               : PAT == PAT_AA_ODD ? PAT_AA_EVEN
                               : PAT == PAT_ESO_EVEN ? PAT_ESO_ODD
                               : PAT == PAT_ESO_ODD ? PAT_ESO_EVEN
                               : PAT == PAT_EPULL_EVEN ? PAT_EPULL_ODD
                               : PAT == PAT_EPULL_ODD ? PAT_EPULL_EVEN
                               : PAT == PAT_EPUSH_EVEN ? PAT_EPUSH_ODD
                               : PAT == PAT_EPUSH_ODD ? PAT_EPUSH_EVEN
                               : PAT;
};

// Eddy viscosity of the learned closure for the sweep with MK_CUM1_MLP; defined (with the
// constant-memory parameters it reads) only in the translation unit that instantiates that
// sweep, lbm_q27_closure.cu.
template <class R> struct ClosureNu;

template <class R, int Q, int MK>
__device__ __forceinline__ R collide(R (&f)[Q], const Physics& p) {
    if constexpr (MK == MK_POP) return collide_pop<Q, R>(f, p);
    else if constexpr (MK == MK_MRT) return collide_mrt<Q, R>(f, p);
    else if constexpr (MK == MK_CUM1) return collide_cum_ho1<R>(f, p);
    else if constexpr (MK == MK_CUM1_MLP) return collide_cum_ho1<R, true>(f, p, ClosureNu<R>{});
    else if constexpr (MK == MK_CM) return collide_cm<R>(f, p);
    else return collide_cum<R>(f, p);
}

// Element index of (slot, cell + offset) relative to the field base; 32-bit (host-checked).
__device__ __forceinline__ unsigned eidx(unsigned slot_off, int cell_off) { return slot_off + (unsigned)cell_off; }

// Element offset of cell (x, y, z) (interior coordinates), periodic axes wrapped; false when the
// cell lies beyond the ghost layer of a non-periodic axis.  Used by the boundary conditions that
// read a cell other than the fluid cell itself (FreeSlip, outflows, Bouzidi), where the offset from
// the fluid cell can reach 2.
__device__ __forceinline__ bool cell_offset(const Grid& g, int x, int y, int z, int& out) {
    const int n[3] = {g.nx, g.ny, g.nz};
    int c[3] = {x, y, z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if ((g.periodic >> a) & 1) c[a] = ((c[a] % n[a]) + n[a]) % n[a];
        else if (c[a] < -1 || c[a] > n[a]) return false;
    }
    out = (c[0] + 1) + (c[1] + 1) * g.sy + (c[2] + 1) * g.sz;
    return true;
}

// Where the previous step wrote the outgoing population d of the cell at (x, y, z) + off: the
// value, or `fallback` when that cell lies beyond the ghost layer.
template <class S, class R, int Q, int PAT>
__device__ __forceinline__ R load_f_out(const SweepArgs& a, int x, int y, int z, int ox, int oy, int oz, int d,
                                        R fallback) {
    using PA = Access<PrevPattern<PAT>::value>;
    int off;
    if (!cell_offset(a.g, x + ox + PA::template woff<Q>(d, 0), y + oy + PA::template woff<Q>(d, 1),
                     z + oz + PA::template woff<Q>(d, 2), off))
        return fallback;
    return Conv<S, R>::ld(static_cast<const S*>(a.src) + eidx(PA::template wslot<Q>(d) * a.g.sq, off));
}

// Fused boundary handling for a fluid cell next to a boundary: replaces the pulled value of every
// direction i whose source cell x - c_i is a NoSlip or UBB cell by the value lbmpy's boundary kernel
// would have written there (boundaries/boundaryconditions.py), from the populations the previous
// step wrote.  f_out(x, j) below is where the previous step wrote direction j of cell x.
//   NoSlip (:104-139)   f_out(x, inv i)
//   UBB (:724-841)      f_out(x, inv i) + 6 w_i rho c_i.u_w   (u_w per UBB number or per link)
// Links into FixedDensity, FreeSlip, outflow and Bouzidi cells read values of other cells; inside an
// in-place sweep those cells update concurrently, so k_boundary_prepass stores those links' values
// where the sweep reads them before the sweep runs, as lbmpy's boundary kernel does.
template <class S, class R, int Q, int PAT>
__device__ __forceinline__ void bounce_back(R (&f)[Q], const SweepArgs& a, const NbrOffsets& nb, int cell,
                                         int x, int y, int z) {
    using L = Lat<Q>;
    using PA = Access<PrevPattern<PAT>::value>;
    const Grid& g = a.g;
    const S* src = static_cast<const S*>(a.src);
    NbrOffsets fo;
    {
        Grid gf = g;
        gf.sy = g.fsy; gf.sz = g.fsz;
        fo.init(gf, x, y, z);
    }
    const int fcell = (x + 1) + (y + 1) * g.fsy + (z + 1) * g.fsz;
    // Interior cell indices fit 32 bits (the host bounds the field below 2^32 elements).
    const int icell = x + g.nx * (y + g.ny * z);
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        const int bt = g.flags[fcell + fo.off(-L::cx(i), -L::cy(i), -L::cz(i))] & FLAG_TYPE_MASK;
        if (bt == 0) continue;
        // FixedDensity and per-link types: written by k_boundary_prepass (per-link types bounce back
        // as NoSlip when the plan holds no link tables, so the pre-pass does not run)
        if (bt >= FLAG_FIXED_DENSITY && !(bt >= FLAG_FREE_SLIP && a.link_code == nullptr && a.link_value == nullptr))
            continue;
        // f_out(x, inv i): where the previous step wrote direction inv(i) of this cell
        const int j = L::inv(i);
        const int off = nb.off(PA::template woff<Q>(j, 0), PA::template woff<Q>(j, 1), PA::template woff<Q>(j, 2));
        R v = Conv<S, R>::ld(src + eidx(PA::template wslot<Q>(j) * g.sq, cell + off));
        if (flag_is_ubb(bt)) {
            const int u = bt - FLAG_UBB0;
            const double* uw = a.p.ubb[u];
            if ((a.p.ubb_link_mask >> u) & 1u)   // per-link velocity of the link x -> x - c_i (dir inv i)
                uw = a.ubb_link_vel + (size_t(a.ubb_block[icell]) * Q + size_t(j)) * 3;
            // compressible: the prescribed wall density, else the cell's density at the previous
            // step, gathered before the sweep (k_ubb_density; in-place sweeps overwrite the
            // values it is summed from)
            const R rho = !a.p.compressible ? R(1)
                          : a.p.ubb_density[u] > 0.0 ? R(a.p.ubb_density[u])
                          : a.ubb_rho != nullptr ? static_cast<const R*>(a.ubb_rho)[icell] : R(1);
            R ux = R(uw[0]), uy = R(uw[1]), uz = R(uw[2]);
            if ((a.p.ubb_adapt_mask >> u) & 1u) {   // the equilibrium velocity of the wall
                const R h = R(0.5) / rho;
                ux -= h * R(a.p.force[0]); uy -= h * R(a.p.force[1]); uz -= h * R(a.p.force[2]);
            }
            const R cu = R(L::cx(i)) * ux + R(L::cy(i)) * uy + R(L::cz(i)) * uz;
            v += R(6) * R(L::w(i)) * cu * rho;
        }
        f[i] = v;
    }
}

// The whole update of one cell: pull through the accessor, fused bounce-back, collision, push
// through the accessor.  Shared by the single-domain and the batched sweeps.
template <class S, class R, int Q, int MK, int PAT>
__device__ __forceinline__ void sweep_cell(const SweepArgs& a, int x, int y, int z) {
    using A = Access<PAT>;
    const Grid& g = a.g;
    // Flag first or together with the populations.  Every address below lies inside the
    // ghost-inclusive field whatever the cell type, so the populations can be loaded before the
    // flag is known: a boundary cell wastes a few loads, and no cell waits for a flag round trip
    // before its loads issue.  The specialised cumulant sweep keeps the flag first: its register
    // budget (64 per thread for AA) does not hold the flag alongside 27 loads in flight.
    constexpr bool flag_first = MK == MK_CUM1 || MK == MK_CUM1_MLP;
    const int fl = (g.flags != nullptr && row_flagged(g, y, z)) ? g.flags[(x + 1) + (y + 1) * g.fsy + (z + 1) * g.fsz] : 0;
    if (flag_first && (fl & FLAG_TYPE_MASK)) return;
    NbrOffsets nb;
    nb.init(g, x, y, z);
    const int cell = (x + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
    const S* src = static_cast<const S*>(a.src);
    S* dst = static_cast<S*>(a.dst);
    R f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int off = nb.off(A::template roff<Q>(i, 0), A::template roff<Q>(i, 1), A::template roff<Q>(i, 2));
        f[i] = Conv<S, R>::ld(src + eidx(A::template rslot<Q>(i) * g.sq, cell + off));
    }
    if (!flag_first && (fl & FLAG_TYPE_MASK)) return;
    if (fl & FLAG_NEAR_WALL) bounce_back<S, R, Q, PAT>(f, a, nb, cell, x, y, z);
    const R om = collide<R, Q, MK>(f, a.p);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int off = nb.off(A::template woff<Q>(i, 0), A::template woff<Q>(i, 1), A::template woff<Q>(i, 2));
        Conv<S, R>::st(dst + eidx(A::template wslot<Q>(i) * g.sq, cell + off), f[i]);
    }
    if (a.omega_out != nullptr) a.omega_out[x + g.nx * (y + (long long)g.ny * z)] = (float)om;
}

// Resident 256-thread blocks per SM that the one-cell sweep is compiled for.  The register
// allocator otherwise trades occupancy for registers in ways that move with unrelated code (the
// near-wall path): the D3Q27 cumulant AA odd sweep went from 80 to 92 registers (3 to 2 blocks)
// when the per-link boundary data arrived, and the D3Q19 TRT AA odd sweep took 88 (2 blocks, 0.72
// of the copy bandwidth; 0.92 at 64).  These hot variants are held to register counts checked
// for spills with -Xptxas -v: 80 (3 blocks), 64 (4) and 48 (5).
template <class S, int Q, int MK, int PAT> struct SweepMinBlocks { static constexpr int value = 1; };
template <> struct SweepMinBlocks<float, 27, MK_CUM1, PAT_AA_ODD> { static constexpr int value = 3; };
template <> struct SweepMinBlocks<float, 27, MK_CUM1, PAT_AA_EVEN> { static constexpr int value = 4; };
template <> struct SweepMinBlocks<float, 19, MK_POP, PAT_PULL> { static constexpr int value = 5; };
template <> struct SweepMinBlocks<float, 19, MK_POP, PAT_AA_ODD> { static constexpr int value = 4; };
template <> struct SweepMinBlocks<float, 19, MK_POP, PAT_AA_EVEN> { static constexpr int value = 4; };
template <> struct SweepMinBlocks<float, 27, MK_POP, PAT_AA_ODD> { static constexpr int value = 3; };
template <> struct SweepMinBlocks<float, 27, MK_POP, PAT_AA_EVEN> { static constexpr int value = 4; };
template <> struct SweepMinBlocks<float, 19, MK_MRT, PAT_PULL> { static constexpr int value = 4; };
template <> struct SweepMinBlocks<float, 27, MK_MRT, PAT_PULL> { static constexpr int value = 3; };

template <class S, class R, int Q, int MK, int PAT>
__global__ void __launch_bounds__(256, SweepMinBlocks<S, Q, MK, PAT>::value) k_sweep(const SweepArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= a.g.nx || y >= a.g.ny) return;
    sweep_cell<S, R, Q, MK, PAT>(a, x, y, z);
}

// Pipelined z-columns: each thread sweeps a.zc consecutive cells along z and issues the loads of
// the next cell before it collides the current one, so every warp keeps Q loads in flight through
// its collision (the one-cell sweep has none in flight while it computes).  The second set of Q
// values costs registers: two 256-thread blocks per SM.  Safe in place for AA: the locations a
// cell reads and the locations it writes are the same set, disjoint from every other cell's.
template <class S, class R, int Q, int MK, int PAT>
__global__ void __launch_bounds__(256, 2) k_sweep_zpipe(const SweepArgs a) {
    static_assert(PAT == PAT_PULL || PAT == PAT_AA_EVEN || PAT == PAT_AA_ODD, "pipelined sweep: pull and AA");
    using A = Access<PAT>;
    const Grid& g = a.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z0 = blockIdx.z * a.zc;
    if (x >= g.nx || y >= g.ny || z0 >= g.nz) return;
    const int z1 = min(z0 + a.zc, g.nz);
    const S* src = static_cast<const S*>(a.src);
    S* dst = static_cast<S*>(a.dst);
    auto load = [&](int z, R (&h)[Q], int& hf) {
        hf = (g.flags != nullptr && row_flagged(g, y, z)) ? g.flags[(x + 1) + (y + 1) * g.fsy + (z + 1) * g.fsz] : 0;
        NbrOffsets nb;
        nb.init(g, x, y, z);
        const int cell = (x + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int off = nb.off(A::template roff<Q>(i, 0), A::template roff<Q>(i, 1), A::template roff<Q>(i, 2));
            h[i] = Conv<S, R>::ld(src + eidx(A::template rslot<Q>(i) * g.sq, cell + off));
        }
    };
    R nxt[Q];
    int nfl;
    load(z0, nxt, nfl);
#pragma unroll 1
    for (int z = z0; z < z1; ++z) {
        R f[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i] = nxt[i];
        const int fl = nfl;
        if (z + 1 < z1) load(z + 1, nxt, nfl);
        if (fl & FLAG_TYPE_MASK) continue;
        NbrOffsets nb;
        nb.init(g, x, y, z);
        const int cell = (x + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
        if (fl & FLAG_NEAR_WALL) bounce_back<S, R, Q, PAT>(f, a, nb, cell, x, y, z);
        collide<R, Q, MK>(f, a.p);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int off = nb.off(A::template woff<Q>(i, 0), A::template woff<Q>(i, 1), A::template woff<Q>(i, 2));
            Conv<S, R>::st(dst + eidx(A::template wslot<Q>(i) * g.sq, cell + off), f[i]);
        }
    }
}

// Asks L2 for the lines one cell will pull (prefetch.global.L2 is a hint: no data returns, no
// registers are held, and every address is one the sweep itself reads).
template <class S, int Q, int PAT>
__device__ __forceinline__ void prefetch_cell(const SweepArgs& a, int x, int y, int z) {
    using A = Access<PAT>;
    const Grid& g = a.g;
    NbrOffsets nb;
    nb.init(g, x, y, z);
    const int cell = (x + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
    const S* src = static_cast<const S*>(a.src);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int off = nb.off(A::template roff<Q>(i, 0), A::template roff<Q>(i, 1), A::template roff<Q>(i, 2));
        const S* q = src + eidx(A::template rslot<Q>(i) * g.sq, cell + off);
        asm volatile("prefetch.global.L2 [%0];" ::"l"(q));
    }
}

// Density, at the previous step, of every fluid cell with a moving-wall (UBB) link, for the
// compressible UBB: lbmpy takes it from the cell's own post-collision values in a boundary pass
// before the sweep (boundaries/boundaryconditions.py:794-841).  Inside an in-place sweep the
// neighbours overwrite those locations, and summing them inside any sweep costs every cell
// registers, so they are summed here first, for every pattern.
template <class S, class R, int Q, int PAT>
__global__ void __launch_bounds__(256) k_ubb_density(const SweepArgs a, R* rho_out) {
    using L = Lat<Q>;
    using PA = Access<PrevPattern<PAT>::value>;
    const Grid& g = a.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    const int fcell = (x + 1) + (y + 1) * g.fsy + (z + 1) * g.fsz;
    const int fl = g.flags[fcell];
    if ((fl & FLAG_TYPE_MASK) || !(fl & FLAG_NEAR_WALL)) return;
    NbrOffsets fo;
    {
        Grid gf = g;
        gf.sy = g.fsy;
        gf.sz = g.fsz;
        fo.init(gf, x, y, z);
    }
    bool moving = false;
#pragma unroll
    for (int i = 1; i < Q; ++i)
        if (flag_is_ubb(g.flags[fcell + fo.off(-L::cx(i), -L::cy(i), -L::cz(i))] & FLAG_TYPE_MASK)) moving = true;
    if (!moving) return;
    NbrOffsets nb;
    nb.init(g, x, y, z);
    const int cell = (x + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
    const S* src = static_cast<const S*>(a.src);
    R s = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const int ok = nb.off(PA::template woff<Q>(k, 0), PA::template woff<Q>(k, 1), PA::template woff<Q>(k, 2));
        s += Conv<S, R>::ld(src + eidx(PA::template wslot<Q>(k) * g.sq, cell + ok));
    }
    rho_out[x + g.nx * (y + g.ny * z)] = R(1) + s;
}

// ------------------------------------------------------------------ batched domains
// Many independent domains (each with its own ghost layers, strides, flags and rates) updated by
// one persistent launch: the blocks walk a table of tiles, each tile_x x tile_y cells of
// `cells_z` consecutive x-y planes of one domain (a thread updates up to cells_z cells along z).
// Each domain carries a full SweepArgs whose pointers already point into the shared source and
// destination buffers of the batch, one set per step parity.  A block stages the arguments of
// its current domain in shared memory, so the collision reads its rates from there.
struct BatchTile {
    int domain, x0, y0, z0;
};

struct BatchArgs {
    const SweepArgs* domains;     // device array, [parity][n_domains]
    const BatchTile* tiles;       // device array
    int n_domains, n_tiles;
    int cells_z;
    int parity;                   // selects which half of `domains` (src/dst swapped) to use
};

template <class S, class R, int Q, int MK, int PAT>
__global__ void __launch_bounds__(256, 3) k_sweep_batched(const BatchArgs b) {
    __shared__ __align__(16) SweepArgs sa;
    constexpr int WORDS = sizeof(SweepArgs) / 4;
    static_assert(sizeof(SweepArgs) % 4 == 0, "SweepArgs is copied as 32-bit words");
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthreads = blockDim.x * blockDim.y;
    int staged = -1;
#pragma unroll 1
    for (int t = blockIdx.x; t < b.n_tiles; t += gridDim.x) {
        const BatchTile tile = b.tiles[t];
        if (tile.domain != staged) {
            __syncthreads();                         // every thread is done with the previous domain
            const unsigned* from = reinterpret_cast<const unsigned*>(b.domains + b.parity * b.n_domains + tile.domain);
            unsigned* to = reinterpret_cast<unsigned*>(&sa);
            for (int w = tid; w < WORDS; w += nthreads) to[w] = from[w];
            __syncthreads();
            staged = tile.domain;
        }
        const int x = tile.x0 + threadIdx.x;
        const int y = tile.y0 + threadIdx.y;
        if (x < sa.g.nx && y < sa.g.ny) {
            const int z1 = min(tile.z0 + b.cells_z, sa.g.nz);
#pragma unroll 1
            for (int z = tile.z0; z < z1; ++z) sweep_cell<S, R, Q, MK, PAT>(sa, x, y, z);
        }
    }
}

// ------------------------------------------------------------------ sparse (list-based) domains
// lbmpy's sparse LBM (sparse/mapping.py:13-156, sparse/update_rule_sparse.py:22-52): the cells are a
// list (fluid cells first, then boundary cells), PDF i of list cell c at element c + i * n_cells, and
// an index list gives, per fluid cell and direction i >= 1, the element a pull sweep reads
// (a neighbour's slot, the cell's own inverse slot for NoSlip, or the periodic image).  Index
// layout here: [Q-1][n_fluid] (direction-major, so a warp's reads of one direction are coalesced).
struct SparseArgs {
    Physics p;
    const void* src;
    void* dst;
    const unsigned* index;
    long long n_fluid;
    long long n_cells;
};

template <class S, class R, int Q, int MK>
__global__ void __launch_bounds__(256) k_sweep_sparse(const SparseArgs a) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= a.n_fluid) return;
    const S* src = static_cast<const S*>(a.src);
    S* dst = static_cast<S*>(a.dst);
    R f[Q];
    f[0] = Conv<S, R>::ld(src + c);
#pragma unroll
    for (int i = 1; i < Q; ++i) f[i] = Conv<S, R>::ld(src + a.index[(long long)(i - 1) * a.n_fluid + c]);
    collide<R, Q, MK>(f, a.p);
#pragma unroll
    for (int i = 0; i < Q; ++i) Conv<S, R>::st(dst + c + (long long)i * a.n_cells, f[i]);
}

// Equilibrium of list cells c < n_fluid from rho[c] and u[k * n_fluid + c] (FP64).  The velocity
// enters unshifted, as lbmpy's sparse setter builds it (force_substitution=False,
// sparse/update_rule_sparse.py:70-85).
template <class S, class R, int Q, int MK>
__global__ void __launch_bounds__(256) k_sparse_set_equilibrium(const SparseArgs a, const double* rho,
                                                               const double* u) {
    constexpr int EQ = (MK == MK_CUM1 || MK == MK_CUM1_MLP) ? MK_CUM : MK;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= a.n_fluid) return;
    const R r = R(rho[c]);
    const R ux = R(u[c]), uy = R(u[a.n_fluid + c]), uz = R(u[2 * a.n_fluid + c]);
    R f[Q];
    equilibrium<Q, R, EQ>(f, r, ux, uy, uz, a.p);
    S* dst = static_cast<S*>(a.dst);
#pragma unroll
    for (int i = 0; i < Q; ++i) Conv<S, R>::st(dst + c + (long long)i * a.n_cells, f[i]);
}

// Velocity bounce-back on a sparse list (lbmpy's SparseLbBoundaryMapper with UBB,
// sparse/mapping.py:157-247 and boundaries/boundaryconditions.py UBB): link k runs from fluid cell
// links[n_links + k] in direction links[k] into boundary cell links[2 * n_links + k]; the boundary
// cell's slot inv(d), which the fluid cell pulls next, receives f_out(c, d) - 6 w_d rho (c_d . u_w)
// (rho the cell's density when compressible, else 1).  Runs on the source list before the sweep;
// each link writes its own slot, and only boundary cells are written.
template <class S, class R, int Q>
__global__ void __launch_bounds__(256) k_sparse_ubb(const SparseArgs a, const unsigned* links, long long n_links,
                                                    double ux, double uy, double uz) {
    using L = Lat<Q>;
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= n_links) return;
    const int d = int(links[k]);
    if (d < 1 || d >= Q) return;
    const long long c = links[n_links + k], b = links[2 * n_links + k];
    S* pdf = static_cast<S*>(a.dst);
    R rho = R(1);
    if (a.p.compressible) {
        R s = R(0);
#pragma unroll
        for (int i = 0; i < Q; ++i) s += Conv<S, R>::ld(pdf + c + (long long)i * a.n_cells);
        rho += s;
    }
    const R cu = R(L::cx(d)) * R(ux) + R(L::cy(d)) * R(uy) + R(L::cz(d)) * R(uz);
    const R v = Conv<S, R>::ld(pdf + c + (long long)d * a.n_cells) - R(6) * R(L::w(d)) * cu * rho;
    Conv<S, R>::st(pdf + b + (long long)L::inv(d) * a.n_cells, v);
}

// Density and velocity (FP64) of list cells c < n_fluid (sparse/update_rule_sparse.py:55-67).
template <class S, class R, int Q>
__global__ void __launch_bounds__(256) k_sparse_get_macroscopic(const SparseArgs a, double* rho, double* u) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= a.n_fluid) return;
    const S* src = static_cast<const S*>(a.src);
    R f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = Conv<S, R>::ld(src + c + (long long)i * a.n_cells);
    Macro<Q, R> m = conserved<Q, R>(f, a.p, false);
    if (a.p.force_model != FM_NONE) {
        const R h = R(0.5) / m.rho_ref;
        m.ux += h * R(a.p.force[0]); m.uy += h * R(a.p.force[1]); m.uz += h * R(a.p.force[2]);
    }
    if (rho) rho[c] = m.rho;
    if (u) {
        u[c] = m.ux;
        u[a.n_fluid + c] = m.uy;
        u[2 * a.n_fluid + c] = m.uz;
    }
}

// ------------------------------------------------------------------ setter / getter
struct MacroArgs {
    Grid g;
    Physics p;
    void* pdfs;
    void* rho;              // R*, element strides rs[3]
    void* u;                // R*, element strides us[4] (x, y, z, component)
    long long rs[3];
    long long us[4];
};

// Equilibrium initialisation through the write accessor of the previous step
// (macroscopic_value_kernels.py:29-45); the velocity is shifted by -F/(2 rho_ref) when a force
// model is present (forcemodels.py:592-593).
template <class S, class R, int Q, int MK, int PAT>
__global__ void __launch_bounds__(256) k_set_equilibrium(const MacroArgs a) {
    using A = Access<PAT>;
    const Grid& g = a.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    const R* rp = static_cast<const R*>(a.rho);
    const R* up = static_cast<const R*>(a.u);
    const R rho = rp[x * a.rs[0] + y * a.rs[1] + z * a.rs[2]];
    const long long ub = x * a.us[0] + y * a.us[1] + z * a.us[2];
    R ux = up[ub], uy = up[ub + a.us[3]], uz = up[ub + 2 * a.us[3]];
    if (a.p.force_model != FM_NONE) {
        const R h = R(0.5) / (a.p.compressible ? rho : R(1));
        ux -= h * R(a.p.force[0]); uy -= h * R(a.p.force[1]); uz -= h * R(a.p.force[2]);
    }
    R f[Q];
    equilibrium<Q, R, MK>(f, rho, ux, uy, uz, a.p);
    NbrOffsets nb;
    nb.init(g, x, y, z);
    const int cell = (x + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
    S* dst = static_cast<S*>(a.pdfs);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int off = nb.off(A::template woff<Q>(i, 0), A::template woff<Q>(i, 1), A::template woff<Q>(i, 2));
        Conv<S, R>::st(dst + eidx(A::template wslot<Q>(i) * g.sq, cell + off), f[i]);
    }
}

// Boundary pre-pass, before the sweep as lbmpy's boundary kernel runs before its sweep: for every
// fluid cell x next to a cell of a type whose incoming value depends on other cells' populations,
// compute that value per link and store it where the sweep reads direction i of x (a slot that only
// the boundary cell's own update would write, so no fluid cell's outgoing value is overwritten, in
// place or not).  f_out(y, d) is where the previous step wrote direction d of cell y; the link from
// x towards the boundary cell x - c_i has direction j = inv(i).
//   FixedDensity (:1044-1099)            2 feq_even_i(rho_w, u) - f_out(x, j),  feq_even_i =
//                                        (feq_i + feq_j) / 2, u from x's outgoing populations at
//                                        density rho_w (j / rho_w compressible, j otherwise);
//                                        force-free methods (host-checked)
//   FreeSlip (:360-455), SimpleExtrapolationOutflow (:844-889)
//                                        f_out(x + off, d)          (off, d from the link code)
//   ExtrapolationOutflow (:894-1041)     c p + (1 - c) p_nd, c = sqrt(1/3); then
//                                        p <- f_out(x + off, d), p_nd <- the result
//   NoSlipLinearBouzidi (:142-212)       q >= 1/2: (f_out(x, j) + (2q - 1) f_out(x, i)) / (2q)
//                                        0 < q < 1/2: 2q f_out(x, j) + (1 - 2q) f_out(x + c_i, j)
//                                        else f_out(x, j)
// A link whose table is missing, or whose other cell lies beyond the ghost layer, gets NoSlip.
template <class S, class R, int Q, int MK, int PAT>
__global__ void __launch_bounds__(256) k_boundary_prepass(const SweepArgs a) {
    using L = Lat<Q>;
    using A = Access<PAT>;
    using PA = Access<PrevPattern<PAT>::value>;
    constexpr int EQ = (MK == MK_CUM1 || MK == MK_CUM1_MLP) ? MK_CUM : MK;
    const Grid& g = a.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny || !row_flagged(g, y, z)) return;
    const int fcell = (x + 1) + (y + 1) * g.fsy + (z + 1) * g.fsz;
    const int fl = g.flags[fcell];
    if ((fl & FLAG_TYPE_MASK) || !(fl & FLAG_NEAR_WALL)) return;
    NbrOffsets fo;
    {
        Grid gf = g;
        gf.sy = g.fsy;
        gf.sz = g.fsz;
        fo.init(gf, x, y, z);
    }
    unsigned types = 0;   // bit t: a link to a cell of type t
#pragma unroll
    for (int i = 1; i < Q; ++i)
        types |= 1u << (g.flags[fcell + fo.off(-L::cx(i), -L::cy(i), -L::cz(i))] & FLAG_TYPE_MASK);
    constexpr unsigned HANDLED = (1u << FLAG_FIXED_DENSITY) | (1u << FLAG_FIXED_DENSITY1) | (1u << FLAG_FREE_SLIP) |
                                 (1u << FLAG_SIMPLE_OUTFLOW) | (1u << FLAG_OUTFLOW) | (1u << FLAG_BOUZIDI);
    if (!(types & HANDLED)) return;
    NbrOffsets nb;
    nb.init(g, x, y, z);
    const int cell = (x + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
    S* f = const_cast<S*>(static_cast<const S*>(a.src));
    R out[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const int off = nb.off(PA::template woff<Q>(k, 0), PA::template woff<Q>(k, 1), PA::template woff<Q>(k, 2));
        out[k] = Conv<S, R>::ld(f + eidx(PA::template wslot<Q>(k) * g.sq, cell + off));
    }
    // where the sweep reads direction i of this cell
    auto store = [&](int i, R v) {
        const int off = nb.off(A::template roff<Q>(i, 0), A::template roff<Q>(i, 1), A::template roff<Q>(i, 2));
        Conv<S, R>::st(f + eidx(A::template rslot<Q>(i) * g.sq, cell + off), v);
    };
    if (types & ((1u << FLAG_FIXED_DENSITY) | (1u << FLAG_FIXED_DENSITY1))) {
        R jx = 0, jy = 0, jz = 0;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            jx += R(L::cx(k)) * out[k];
            jy += R(L::cy(k)) * out[k];
            jz += R(L::cz(k)) * out[k];
        }
#pragma unroll 1
        for (int t = 0; t < 2; ++t) {
            if (!((types >> (FLAG_FIXED_DENSITY + t)) & 1u)) continue;
            const R rw = R(t == 0 ? a.p.fixed_density : a.p.fixed_density1);
            const R s = a.p.compressible ? R(1) / rw : R(1);
            R feq[Q];
            equilibrium<Q, R, EQ>(feq, rw, jx * s, jy * s, jz * s, a.p);
#pragma unroll
            for (int i = 1; i < Q; ++i) {
                if ((g.flags[fcell + fo.off(-L::cx(i), -L::cy(i), -L::cz(i))] & FLAG_TYPE_MASK) != FLAG_FIXED_DENSITY + t)
                    continue;
                const int q = L::inv(i);
                store(i, feq[q] + feq[i] - out[q]);
            }
        }
    }
    if (!(types & ((1u << FLAG_FREE_SLIP) | (1u << FLAG_SIMPLE_OUTFLOW) | (1u << FLAG_OUTFLOW) | (1u << FLAG_BOUZIDI))))
        return;
    const int icell = x + g.nx * (y + g.ny * z);
    const int blk = a.ubb_block != nullptr ? a.ubb_block[icell] : -1;
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        const int bt = g.flags[fcell + fo.off(-L::cx(i), -L::cy(i), -L::cz(i))] & FLAG_TYPE_MASK;
        if (bt < FLAG_FREE_SLIP || bt > FLAG_BOUZIDI) continue;
        const int j = L::inv(i);
        R v = out[j];                                  // NoSlip fallback
        if (blk >= 0 && bt <= FLAG_OUTFLOW && a.link_code != nullptr) {
            const size_t li = size_t(blk) * Q + size_t(j);
            const int code = a.link_code[li];
            const R w = load_f_out<S, R, Q, PAT>(a, x, y, z, link_off(code, 0), link_off(code, 1), link_off(code, 2),
                                                 link_dir(code), v);
            if (bt == FLAG_OUTFLOW && a.link_value != nullptr) {
                double* st = a.link_value + li * 2;
                const R c = R(0.57735026918962576451);   // sqrt(1/3) dt/dx
                const R fin = c * R(st[0]) + (R(1) - c) * R(st[1]);
                st[0] = double(w);
                st[1] = double(fin);
                v = fin;
            } else {
                v = w;
            }
        } else if (blk >= 0 && bt == FLAG_BOUZIDI && a.link_value != nullptr) {
            const R q = R(a.link_value[(size_t(blk) * Q + size_t(j)) * 2]);
            if (q >= R(0.5)) {
                v = (R(0.5) * (out[j] + out[i] * (R(2) * q - R(1)))) / q;
            } else if (q > R(0)) {
                const R d2 = load_f_out<S, R, Q, PAT>(a, x, y, z, L::cx(i), L::cy(i), L::cz(i), j, out[j]);
                v = R(2) * q * out[j] + (R(1) - R(2) * q) * d2;
            }
        }
        store(i, v);
    }
}

// Density and velocity of the values the previous step wrote (macroscopic_value_kernels.py:48-61,
// conservedquantitycomputation.py:274-374).
template <class S, class R, int Q, int PAT>
__global__ void __launch_bounds__(256) k_get_macroscopic(const MacroArgs a) {
    using A = Access<PAT>;
    const Grid& g = a.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    NbrOffsets nb;
    nb.init(g, x, y, z);
    const int cell = (x + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
    const S* src = static_cast<const S*>(a.pdfs);
    R f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int off = nb.off(A::template woff<Q>(i, 0), A::template woff<Q>(i, 1), A::template woff<Q>(i, 2));
        f[i] = Conv<S, R>::ld(src + eidx(A::template wslot<Q>(i) * g.sq, cell + off));
    }
    Macro<Q, R> m = conserved<Q, R>(f, a.p, false);
    if (a.p.force_model != FM_NONE) {
        const R h = R(0.5) / m.rho_ref;
        m.ux += h * R(a.p.force[0]); m.uy += h * R(a.p.force[1]); m.uz += h * R(a.p.force[2]);
    }
    R* rp = static_cast<R*>(a.rho);
    R* up = static_cast<R*>(a.u);
    if (rp) rp[x * a.rs[0] + y * a.rs[1] + z * a.rs[2]] = m.rho;
    if (up) {
        const long long ub = x * a.us[0] + y * a.us[1] + z * a.us[2];
        up[ub] = m.ux; up[ub + a.us[3]] = m.uy; up[ub + 2 * a.us[3]] = m.uz;
    }
}

// ------------------------------------------------------------------ FP64 conserved sums
// Per-block partial sums of mass, momentum (rho_ref * u, force-shifted) and kinetic energy over
// fluid cells; k_reduce_finish adds the partials in a fixed order (deterministic).
constexpr int RED_THREADS = 256;

template <class S, int Q, int PAT>
__global__ void __launch_bounds__(RED_THREADS) k_reduce_partial(const MacroArgs a, double* partial) {
    using A = Access<PAT>;
    const Grid& g = a.g;
    double acc[5] = {0, 0, 0, 0, 0};
    const long long ncell = (long long)g.nx * g.ny * g.nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(c % g.nx);
        const int y = (int)((c / g.nx) % g.ny);
        const int z = (int)(c / ((long long)g.nx * g.ny));
        if (g.flags != nullptr && (g.flags[(x + 1) + (y + 1) * g.fsy + (z + 1) * g.fsz] & FLAG_TYPE_MASK)) continue;
        NbrOffsets nb;
        nb.init(g, x, y, z);
        const int cell = (x + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
        const S* src = static_cast<const S*>(a.pdfs);
        double f[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int off = nb.off(A::template woff<Q>(i, 0), A::template woff<Q>(i, 1), A::template woff<Q>(i, 2));
            f[i] = Conv<S, double>::ld(src + eidx(A::template wslot<Q>(i) * g.sq, cell + off));
        }
        Macro<Q, double> m = conserved<Q, double>(f, a.p, false);
        if (a.p.force_model != FM_NONE) {
            const double h = 0.5 / m.rho_ref;
            m.ux += h * a.p.force[0]; m.uy += h * a.p.force[1]; m.uz += h * a.p.force[2];
        }
        acc[0] += m.rho;
        acc[1] += m.rho_ref * m.ux;
        acc[2] += m.rho_ref * m.uy;
        acc[3] += m.rho_ref * m.uz;
        acc[4] += 0.5 * m.rho * (m.ux * m.ux + m.uy * m.uy + m.uz * m.uz);
    }
    __shared__ double sh[5][RED_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0;
        for (int w = 0; w < RED_THREADS / 32; ++w) v += sh[threadIdx.x][w];
        partial[blockIdx.x * 5 + threadIdx.x] = v;
    }
}

static __global__ void k_reduce_finish(const double* partial, int nblocks, double* out) {
    const int k = threadIdx.x;
    if (k < 5) {
        double v = 0;
        for (int b = 0; b < nblocks; ++b) v += partial[b * 5 + k];
        out[k] = v;
    }
}

}  // namespace lbm
