// Two cells per thread: the sweep for x-adjacent cell pairs with packed FP32x2 arithmetic.
//
// sm_100 executes FP32 add / multiply / fused multiply-add on register pairs (FADD2 / FMUL2 /
// FFMA2; CUDA exposes them as __fadd2_rn / __fmul2_rn / __ffma2_rn).  F2 is a float2 value whose
// operators map onto those instructions; products are kept lazy so that a*b + c issues one FFMA2.
// The collision templates of lbm_collide.cuh are instantiated on F2 unchanged, so one thread
// collides cells (x0, x0+1) at once: lane .x is the even cell, lane .y the odd one.
#pragma once
#include "lbm_kernels.cuh"

namespace lbm {

struct F2 {
    float2 v;
    __device__ __forceinline__ F2() {}
    __device__ __forceinline__ F2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ F2(double s) : v(make_float2((float)s, (float)s)) {}
    __device__ __forceinline__ F2(int s) : v(make_float2((float)s, (float)s)) {}
    __device__ __forceinline__ explicit F2(float2 x) : v(x) {}
    __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
};

struct F2Prod {   // a * b, materialised only when used as a value
    F2 a, b;
    __device__ __forceinline__ operator F2() const { return F2(__fmul2_rn(a.v, b.v)); }
};

__device__ __forceinline__ float2 neg2(float2 x) { return make_float2(-x.x, -x.y); }

__device__ __forceinline__ F2Prod operator*(F2 a, F2 b) { return F2Prod{a, b}; }
__device__ __forceinline__ F2Prod operator*(F2Prod a, F2 b) { return F2Prod{F2(a), b}; }
__device__ __forceinline__ F2Prod operator*(F2 a, F2Prod b) { return F2Prod{a, F2(b)}; }
__device__ __forceinline__ F2Prod operator*(F2Prod a, F2Prod b) { return F2Prod{F2(a), F2(b)}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(__fadd2_rn(a.v, neg2(b.v))); }
__device__ __forceinline__ F2 operator-(F2 a) { return F2(neg2(a.v)); }
__device__ __forceinline__ F2 operator+(F2Prod p, F2 c) { return F2(__ffma2_rn(p.a.v, p.b.v, c.v)); }
__device__ __forceinline__ F2 operator+(F2 c, F2Prod p) { return F2(__ffma2_rn(p.a.v, p.b.v, c.v)); }
__device__ __forceinline__ F2 operator-(F2Prod p, F2 c) { return F2(__ffma2_rn(p.a.v, p.b.v, neg2(c.v))); }
__device__ __forceinline__ F2 operator-(F2 c, F2Prod p) { return F2(__ffma2_rn(neg2(p.a.v), p.b.v, c.v)); }
__device__ __forceinline__ F2 operator+(F2Prod p, F2Prod q) { return F2(__ffma2_rn(p.a.v, p.b.v, F2(q).v)); }
__device__ __forceinline__ F2 operator-(F2Prod p, F2Prod q) { return F2(__ffma2_rn(p.a.v, p.b.v, neg2(F2(q).v))); }
__device__ __forceinline__ F2 operator-(F2Prod p) { return F2(neg2(F2(p).v)); }
__device__ __forceinline__ F2& operator+=(F2& a, F2 b) { a = a + b; return a; }
__device__ __forceinline__ F2& operator+=(F2& a, F2Prod b) { a = a + b; return a; }
__device__ __forceinline__ F2& operator-=(F2& a, F2 b) { a = a - b; return a; }
__device__ __forceinline__ F2& operator-=(F2& a, F2Prod b) { a = a - b; return a; }
__device__ __forceinline__ F2& operator*=(F2& a, F2 b) { a = F2(__fmul2_rn(a.v, b.v)); return a; }
__device__ __forceinline__ F2 operator/(F2 a, F2 b) { return F2(a.v.x / b.v.x, a.v.y / b.v.y); }
__device__ __forceinline__ F2 sqrt(F2 a) { return F2(sqrtf(a.v.x), sqrtf(a.v.y)); }
__device__ __forceinline__ F2 fabs(F2 a) { return F2(fabsf(a.v.x), fabsf(a.v.y)); }

// ------------------------------------------------------------------ paired storage access
template <class S> struct Pair;
template <> struct Pair<float> {
    using V = float2;
    __device__ __forceinline__ static V ld(const float* p) { return *reinterpret_cast<const float2*>(p); }
    __device__ __forceinline__ static void st(float* p, V v) { *reinterpret_cast<float2*>(p) = v; }
    __device__ __forceinline__ static float2 to_f2(V v) { return v; }
    __device__ __forceinline__ static V from_f2(float2 v) { return v; }
};
template <> struct Pair<__half> {
    using V = __half2;
    __device__ __forceinline__ static V ld(const __half* p) { return *reinterpret_cast<const __half2*>(p); }
    __device__ __forceinline__ static void st(__half* p, V v) { *reinterpret_cast<__half2*>(p) = v; }
    __device__ __forceinline__ static float2 to_f2(V v) { return __half22float2(v); }
    __device__ __forceinline__ static V from_f2(float2 v) { return __float22half2_rn(v); }
};
template <> struct Pair<__nv_bfloat16> {
    using V = __nv_bfloat162;
    __device__ __forceinline__ static V ld(const __nv_bfloat16* p) {
        return *reinterpret_cast<const __nv_bfloat162*>(p);
    }
    __device__ __forceinline__ static void st(__nv_bfloat16* p, V v) { *reinterpret_cast<__nv_bfloat162*>(p) = v; }
    __device__ __forceinline__ static float2 to_f2(V v) { return __bfloat1622float2(v); }
    __device__ __forceinline__ static V from_f2(float2 v) { return __float22bfloat162_rn(v); }
};

template <class R, int Q, int MK>
__device__ __forceinline__ F2 collide2(F2 (&f)[Q], const Physics& p) {
    if constexpr (MK == MK_POP) return collide_pop<Q, F2>(f, p);
    else if constexpr (MK == MK_MRT) return collide_mrt<Q, F2>(f, p);
    else if constexpr (MK == MK_CUM1) return collide_cum_ho1<F2>(f, p);
    else return collide_cum<F2>(f, p);
}

// One warp covers 32 pairs = 64 cells of one x row; block = 32 x PAIR_ROWS threads.
constexpr int PAIR_ROWS = 4;

// Requirements (checked by the host): nx even, the address of interior cell x = 0 of every row
// and every slot 8-byte aligned for the paired type (x = 0 lands at an even element offset).
// Resident blocks of 128 threads per SM the register allocation must allow.  16-bit storage:
// the sweep is limited by latency rather than bandwidth at the occupancy its registers allow; a
// cap of 80 registers (6 blocks) trades a few spilled words for a third more resident warps.
// FP32: 5 blocks (at most 102 registers); without a stated minimum the allocator may take far more.
template <> struct Pair<e3m12> {
    using V = unsigned;
    __device__ __forceinline__ static V ld(const e3m12* p) { return *reinterpret_cast<const unsigned*>(p); }
    __device__ __forceinline__ static void st(e3m12* p, V v) { *reinterpret_cast<unsigned*>(p) = v; }
    __device__ __forceinline__ static float2 to_f2(V v) { return make_float2(e3m12_decode(v & 0xffffu), e3m12_decode(v >> 16)); }
    __device__ __forceinline__ static V from_f2(float2 v) { return e3m12_encode(v.x) | (e3m12_encode(v.y) << 16); }
};

template <class S> struct PairMinBlocks { static constexpr int value = 5; };
template <> struct PairMinBlocks<__half> { static constexpr int value = 6; };
template <> struct PairMinBlocks<__nv_bfloat16> { static constexpr int value = 6; };
template <> struct PairMinBlocks<e3m12> { static constexpr int value = 6; };

template <class S, int Q, int MK, int PAT>
__global__ void __launch_bounds__(32 * PAIR_ROWS, PairMinBlocks<S>::value) k_sweep_pair(const SweepArgs a) {
    static_assert(PAT == PAT_PULL || PAT == PAT_AA_EVEN || PAT == PAT_AA_ODD, "pair sweep: pull and AA");
    using L = Lat<Q>;
    using A = Access<PAT>;
    using PS = Pair<S>;
    const Grid& g = a.g;
    const int lane = threadIdx.x;
    const int pairs_per_row = g.nx >> 1;
    const int pidx = blockIdx.x * 32 + lane;
    const int y = blockIdx.y * PAIR_ROWS + threadIdx.y;
    const int z = blockIdx.z;
    if (y >= g.ny) return;                        // whole warp (same y) leaves together
    const bool active = pidx < pairs_per_row;
    const int x0 = active ? 2 * pidx : g.nx - 2;   // inactive lanes shadow the last pair
    const int last_lane = min(31, pairs_per_row - 1 - blockIdx.x * 32);   // last active lane of this warp

    // neighbour offsets: y/z shared by both cells; x per cell (A = x0, B = x0 + 1)
    NbrOffsets nbA, nbB;
    nbA.init(g, x0, y, z);
    nbB.init(g, x0 + 1, y, z);
    const int cellA = (x0 + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
    const S* src = static_cast<const S*>(a.src);
    S* dst = static_cast<S*>(a.dst);

    int flA = 0, flB = 0;
    if (g.flags != nullptr && row_flagged(g, y, z)) {
        const int fc = (x0 + 1) + (y + 1) * g.fsy + (z + 1) * g.fsz;
        flA = g.flags[fc];
        flB = g.flags[fc + 1];
    }

    F2 f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = A::template roff<Q>(i, 0);
        const int yz = nbA.off(0, A::template roff<Q>(i, 1), A::template roff<Q>(i, 2));
        const unsigned slot = A::template rslot<Q>(i) * g.sq;
        // aligned pair of the source row at (x0, x0 + 1)
        const float2 P = PS::to_f2(PS::ld(src + eidx(slot, cellA + yz)));
        float va, vb;
        if (cx == 0) {
            va = P.x; vb = P.y;
        } else if (cx == -1) {                     // cells read x - 1: (x0 - 1, x0)
            float up = __shfl_up_sync(0xffffffffu, P.y, 1);
            if (lane == 0) up = Conv<S, float>::ld(src + eidx(slot, cellA + yz + nbA.dx[0]));
            va = up; vb = P.x;
        } else {                                   // cells read x + 1: (x0 + 1, x0 + 2)
            float dn = __shfl_down_sync(0xffffffffu, P.x, 1);
            if (lane == last_lane) dn = Conv<S, float>::ld(src + eidx(slot, cellA + 1 + yz + nbB.dx[2]));
            va = P.y; vb = dn;
        }
        f[i] = F2(va, vb);
    }
    // cells next to a boundary: per-cell fused bounce-back on the scalar path
    if ((flA | flB) & FLAG_NEAR_WALL) {
        float ta[Q], tb[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) { ta[i] = f[i].v.x; tb[i] = f[i].v.y; }
        if (flA & FLAG_NEAR_WALL) bounce_back<S, float, Q, PAT>(ta, a, nbA, cellA, x0, y, z);
        if (flB & FLAG_NEAR_WALL) bounce_back<S, float, Q, PAT>(tb, a, nbB, cellA + 1, x0 + 1, y, z);
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i] = F2(ta[i], tb[i]);
    }
    collide2<float, Q, MK>(f, a.p);
    // Non-fluid cells must leave their own slots as they are in AA even steps, where neighbours
    // read them (fused bounce-back): slot inv(i) is rewritten with its current value.  Pull and
    // AA odd never read what a non-fluid cell writes.
    if (PAT == PAT_AA_EVEN && ((flA | flB) & FLAG_TYPE_MASK)) {
        const bool keepA = (flA & FLAG_TYPE_MASK) != 0, keepB = (flB & FLAG_TYPE_MASK) != 0;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const S* q = src + eidx(L::inv(i) * g.sq, cellA);
            f[i] = F2(keepA ? Conv<S, float>::ld(q) : f[i].v.x, keepB ? Conv<S, float>::ld(q + 1) : f[i].v.y);
        }
    }

#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = A::template woff<Q>(i, 0);
        const int yz = nbA.off(0, A::template woff<Q>(i, 1), A::template woff<Q>(i, 2));
        const unsigned slot = A::template wslot<Q>(i) * g.sq;
        const float va = f[i].v.x, vb = f[i].v.y;
        if (cx == 0) {
            if (active) PS::st(dst + eidx(slot, cellA + yz), PS::from_f2(make_float2(va, vb)));
        } else if (cx == 1) {                      // A -> x0 + 1, B -> x0 + 2
            const float prevB = __shfl_up_sync(0xffffffffu, vb, 1);
            if (active) {
                if (lane == 0) Conv<S, float>::st(dst + eidx(slot, cellA + 1 + yz), va);
                else PS::st(dst + eidx(slot, cellA + yz), PS::from_f2(make_float2(prevB, va)));
                if (lane == last_lane) Conv<S, float>::st(dst + eidx(slot, cellA + 1 + yz + nbB.dx[2]), vb);
            }
        } else {                                   // A -> x0 - 1, B -> x0
            const float nextA = __shfl_down_sync(0xffffffffu, va, 1);
            if (active) {
                if (lane == last_lane) Conv<S, float>::st(dst + eidx(slot, cellA + yz), vb);
                else PS::st(dst + eidx(slot, cellA + yz), PS::from_f2(make_float2(vb, nextA)));
                if (lane == 0) Conv<S, float>::st(dst + eidx(slot, cellA + yz + nbA.dx[0]), va);
            }
        }
    }
}

}  // namespace lbm
