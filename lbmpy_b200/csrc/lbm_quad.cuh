// Four cells per thread for 16-bit storage: the pair sweep (lbm_pair.cuh) widened to x-adjacent
// quads.  Every population of a quad is one aligned 8-byte access (four halves), so loads, stores,
// address arithmetic, warp shuffles and edge fix-ups per cell are half the pair sweep's; the
// collision runs as two packed FP32x2 pairs (cells x0, x0+1 and x0+2, x0+3).
#pragma once
#include "lbm_pair.cuh"

namespace lbm {

template <class S> struct Quad;
template <> struct Quad<__half> {
    using H2 = __half2;
    __device__ __forceinline__ static float2 to_f2(unsigned w) {
        return __half22float2(*reinterpret_cast<const __half2*>(&w));
    }
    __device__ __forceinline__ static unsigned from_f2(float2 v) {
        const __half2 h = __float22half2_rn(v);
        return *reinterpret_cast<const unsigned*>(&h);
    }
};
template <> struct Quad<__nv_bfloat16> {
    __device__ __forceinline__ static float2 to_f2(unsigned w) {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w));
    }
    __device__ __forceinline__ static unsigned from_f2(float2 v) {
        const __nv_bfloat162 h = __float22bfloat162_rn(v);
        return *reinterpret_cast<const unsigned*>(&h);
    }
};

template <> struct Quad<e3m12> {
    __device__ __forceinline__ static float2 to_f2(unsigned w) {
        return make_float2(e3m12_decode(w & 0xffffu), e3m12_decode(w >> 16));
    }
    __device__ __forceinline__ static unsigned from_f2(float2 v) {
        return e3m12_encode(v.x) | (e3m12_encode(v.y) << 16);
    }
};

template <class S>
__device__ __forceinline__ void quad_ld(const S* p, float (&v)[4]) {
    const uint2 w = *reinterpret_cast<const uint2*>(p);
    const float2 a = Quad<S>::to_f2(w.x), b = Quad<S>::to_f2(w.y);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

template <class S>
__device__ __forceinline__ void quad_st(S* p, float v0, float v1, float v2, float v3) {
    *reinterpret_cast<uint2*>(p) = make_uint2(Quad<S>::from_f2(make_float2(v0, v1)), Quad<S>::from_f2(make_float2(v2, v3)));
}

constexpr int QUAD_ROWS = 4;

// Requirements (checked by the host): nx a multiple of 4, the address of interior cell x = 0 of
// every row and every slot 8-byte aligned, row / plane / slot strides multiples of 4 elements.
template <class S, int Q, int MK, int PAT>
__global__ void __launch_bounds__(32 * QUAD_ROWS, 4) k_sweep_quad(const SweepArgs a) {
    static_assert(PAT == PAT_PULL || PAT == PAT_AA_EVEN || PAT == PAT_AA_ODD, "quad sweep: pull and AA");
    using L = Lat<Q>;
    using A = Access<PAT>;
    const Grid& g = a.g;
    const int lane = threadIdx.x;
    const int quads_per_row = g.nx >> 2;
    const int qidx = blockIdx.x * 32 + lane;
    const int y = blockIdx.y * QUAD_ROWS + threadIdx.y;
    const int z = blockIdx.z;
    if (y >= g.ny) return;                        // whole warp (same y) leaves together
    const bool active = qidx < quads_per_row;
    const int x0 = active ? 4 * qidx : g.nx - 4;   // inactive lanes shadow the last quad
    const int last_lane = min(31, quads_per_row - 1 - blockIdx.x * 32);

    // y/z offsets shared by the quad; x wrap of the first (A) and last (D) cell
    NbrOffsets nbA, nbD;
    nbA.init(g, x0, y, z);
    nbD.init(g, x0 + 3, y, z);
    const int cellA = (x0 + 1) + (y + 1) * g.sy + (z + 1) * g.sz;
    const S* src = static_cast<const S*>(a.src);
    S* dst = static_cast<S*>(a.dst);

    int fl[4] = {0, 0, 0, 0};
    if (g.flags != nullptr && row_flagged(g, y, z)) {
        const int fc = (x0 + 1) + (y + 1) * g.fsy + (z + 1) * g.fsz;
#pragma unroll
        for (int k = 0; k < 4; ++k) fl[k] = g.flags[fc + k];
    }

    F2 f0[Q], f1[Q];     // cells (x0, x0+1) and (x0+2, x0+3)
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = A::template roff<Q>(i, 0);
        const int yz = nbA.off(0, A::template roff<Q>(i, 1), A::template roff<Q>(i, 2));
        const unsigned slot = A::template rslot<Q>(i) * g.sq;
        float P[4];
        quad_ld<S>(src + eidx(slot, cellA + yz), P);
        float v[4];
        if (cx == 0) {
            v[0] = P[0]; v[1] = P[1]; v[2] = P[2]; v[3] = P[3];
        } else if (cx == -1) {                     // cells read x - 1: (x0 - 1 .. x0 + 2)
            float up = __shfl_up_sync(0xffffffffu, P[3], 1);
            if (lane == 0) up = Conv<S, float>::ld(src + eidx(slot, cellA + yz + nbA.dx[0]));
            v[0] = up; v[1] = P[0]; v[2] = P[1]; v[3] = P[2];
        } else {                                   // cells read x + 1: (x0 + 1 .. x0 + 4)
            float dn = __shfl_down_sync(0xffffffffu, P[0], 1);
            if (lane == last_lane) dn = Conv<S, float>::ld(src + eidx(slot, cellA + 3 + yz + nbD.dx[2]));
            v[0] = P[1]; v[1] = P[2]; v[2] = P[3]; v[3] = dn;
        }
        f0[i] = F2(v[0], v[1]);
        f1[i] = F2(v[2], v[3]);
    }
    // cells next to a boundary: per-cell fused bounce-back on the scalar path
    if ((fl[0] | fl[1] | fl[2] | fl[3]) & FLAG_NEAR_WALL) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (!(fl[k] & FLAG_NEAR_WALL)) continue;
            float t[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const F2& h = k < 2 ? f0[i] : f1[i];
                t[i] = (k & 1) ? h.v.y : h.v.x;
            }
            NbrOffsets nb;
            nb.init(g, x0 + k, y, z);
            bounce_back<S, float, Q, PAT>(t, a, nb, cellA + k, x0 + k, y, z);
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                F2& h = k < 2 ? f0[i] : f1[i];
                if (k & 1) h.v.y = t[i]; else h.v.x = t[i];
            }
        }
    }
    collide2<float, Q, MK>(f0, a.p);
    collide2<float, Q, MK>(f1, a.p);
    // Non-fluid cells leave their own slots as they are in AA even steps (neighbours read them in
    // the fused bounce-back): slot inv(i) is rewritten with its current value.
    if (PAT == PAT_AA_EVEN && ((fl[0] | fl[1] | fl[2] | fl[3]) & FLAG_TYPE_MASK)) {
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const S* q = src + eidx(L::inv(i) * g.sq, cellA);
            if (fl[0] & FLAG_TYPE_MASK) f0[i].v.x = Conv<S, float>::ld(q);
            if (fl[1] & FLAG_TYPE_MASK) f0[i].v.y = Conv<S, float>::ld(q + 1);
            if (fl[2] & FLAG_TYPE_MASK) f1[i].v.x = Conv<S, float>::ld(q + 2);
            if (fl[3] & FLAG_TYPE_MASK) f1[i].v.y = Conv<S, float>::ld(q + 3);
        }
    }

#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = A::template woff<Q>(i, 0);
        const int yz = nbA.off(0, A::template woff<Q>(i, 1), A::template woff<Q>(i, 2));
        const unsigned slot = A::template wslot<Q>(i) * g.sq;
        const float va = f0[i].v.x, vb = f0[i].v.y, vc = f1[i].v.x, vd = f1[i].v.y;
        if (cx == 0) {
            if (active) quad_st<S>(dst + eidx(slot, cellA + yz), va, vb, vc, vd);
        } else if (cx == 1) {                      // A..D -> x0+1 .. x0+4
            const float prevD = __shfl_up_sync(0xffffffffu, vd, 1);
            if (active) {
                if (lane == 0) {                   // x0 belongs to the previous warp's last lane
                    S* p = dst + eidx(slot, cellA + yz);
                    Conv<S, float>::st(p + 1, va);
                    Conv<S, float>::st(p + 2, vb);
                    Conv<S, float>::st(p + 3, vc);
                } else {
                    quad_st<S>(dst + eidx(slot, cellA + yz), prevD, va, vb, vc);
                }
                if (lane == last_lane) Conv<S, float>::st(dst + eidx(slot, cellA + 3 + yz + nbD.dx[2]), vd);
            }
        } else {                                   // A..D -> x0-1 .. x0+2
            const float nextA = __shfl_down_sync(0xffffffffu, va, 1);
            if (active) {
                if (lane == last_lane) {           // x0+3 belongs to the next warp's lane 0
                    S* p = dst + eidx(slot, cellA + yz);
                    Conv<S, float>::st(p, vb);
                    Conv<S, float>::st(p + 1, vc);
                    Conv<S, float>::st(p + 2, vd);
                } else {
                    quad_st<S>(dst + eidx(slot, cellA + yz), vb, vc, vd, nextA);
                }
                if (lane == 0) Conv<S, float>::st(dst + eidx(slot, cellA + yz + nbA.dx[0]), va);
            }
        }
    }
}

}  // namespace lbm
