// Learned eddy-viscosity closure: a 10 -> 32 -> 32 -> 1 perceptron (SiLU hidden layers, softplus
// output) that maps local non-equilibrium quantities of a cell to an eddy viscosity nu_t, folded
// into the shear relaxation rate as omega = 1 / (tau0 + 3 nu_t).  This is where lbmpy's
// Smagorinsky model puts its eddy viscosity (turbulence_models.py:25-84, omega = 2 / (tau0 +
// sqrt(18 C^2 Pi + tau0^2)) with Pi = sqrt(2 Pi_neq:Pi_neq) / rho); the network replaces the
// closed form.
//
// Shared by the in-sweep inference (the cumulant sweep with sgs = MLP), the training kernels and
// the host build of the tests, so that features and network are the same function everywhere.
#pragma once

#ifndef LBM_HD
#ifdef __CUDACC__
#define LBM_HD __host__ __device__ __forceinline__
#else
#define LBM_HD inline
#endif
#endif

#include <cmath>
#include <cstdint>
#include <type_traits>

namespace lbm {

constexpr int MLP_IN = 10;
constexpr int MLP_H = 32;
// parameter block (FP32): W1[in][h], b1[h], W2[h][h] (W2[j][k]: from unit j to unit k), b2[h],
// W3[h], b3, output scale s (nu_t = s * softplus(y)); s is fixed, not trained
constexpr int MLP_W1 = 0;
constexpr int MLP_B1 = MLP_W1 + MLP_IN * MLP_H;
constexpr int MLP_W2 = MLP_B1 + MLP_H;
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;
constexpr int MLP_W3 = MLP_B2 + MLP_H;
constexpr int MLP_B3 = MLP_W3 + MLP_H;
constexpr int MLP_SCALE = MLP_B3 + 1;
constexpr int MLP_TRAINED = MLP_SCALE;          // parameters 0 .. MLP_TRAINED-1 are trained
constexpr int MLP_PARAMS = MLP_SCALE + 1;

template <class R> LBM_HD R mlp_exp(R x) {
#ifdef __CUDA_ARCH__
    if constexpr (std::is_same<R, float>::value) return __expf(x);
#endif
    using std::exp;
    return exp(x);
}
template <class R> LBM_HD R mlp_log1p(R x) { using std::log1p; return log1p(x); }
template <class R> LBM_HD R mlp_sqrt(R x) { using std::sqrt; return sqrt(x); }
template <class R> LBM_HD R mlp_log(R x) { using std::log; return log(x); }
template <class R> LBM_HD R mlp_abs(R x) { return x < R(0) ? -x : x; }

// Division for the activations: on the device in FP32 the fast reciprocal-based quotient (a few
// ulp), everywhere else the IEEE one.
template <class R> LBM_HD R mlp_div(R a, R b) {
#ifdef __CUDA_ARCH__
    if constexpr (std::is_same<R, float>::value) return __fdividef(a, b);
#endif
    return a / b;
}

// SiLU z * sigmoid(z) and its derivative sigmoid(z) * (1 + z * (1 - sigmoid(z))).
template <class R> LBM_HD R mlp_sigmoid(R z) { return mlp_div<R>(R(1), R(1) + mlp_exp<R>(-z)); }
template <class R> LBM_HD R mlp_silu(R z) { return mlp_div<R>(z, R(1) + mlp_exp<R>(-z)); }
template <class R> LBM_HD R mlp_softplus(R y) { return y > R(20) ? y : mlp_log1p<R>(mlp_exp<R>(y)); }

// SiLU for the in-sweep FP32 inference: (z/2)(1 + tanh(z/2)) with the hardware tanh
// approximation (tanh.approx.f32, relative error about 2^-11): three instructions instead of an
// exponential and a division.  Training and the FP64 paths use the exact form.
template <class R> LBM_HD R mlp_silu_sweep(R z) {
#ifdef __CUDA_ARCH__
    if constexpr (std::is_same<R, float>::value) {
        const float h = 0.5f * z;
        float t;
        asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
        return fmaf(h, t, h);
    }
#endif
    return mlp_silu<R>(z);
}

// Features of one cell from the pre-collision non-equilibrium second moments Pi (6 components),
// the density and the velocity.  Scale-free shape features plus log and linear magnitudes:
//  0 log(Pi_m + 1e-9), Pi_m = sqrt(2 Pi:Pi) / rho  (the Smagorinsky invariant)
//  1 100 Pi_m
//  2 tr(Pi) / |Pi|                       (bulk fraction)
//  3 sqrt(6) tr(A^3), A = dev(Pi)/|dev(Pi)| (strain shape: -1 axisymmetric contraction .. +1 expansion)
//  4 30 |u|
//  5 1000 (rho - 1)
//  6 u.A.u / |u|^2                        (alignment of the flow with the principal strain)
//  7 (Pi_xy^2 + Pi_xz^2 + Pi_yz^2) / |Pi|^2 (off-diagonal fraction, lattice-frame)
//  8 max_i |dev(Pi)_ii| / |dev(Pi)|
//  9 1000 |u|^2
//
// FAST (the FP32 sweep, whose network rounds the features to FP16 anyway): square roots, quotients
// and the logarithm with the hardware approximations (relative error about 2^-21).
template <class R, bool FAST = false>
LBM_HD void closure_features(R pxx, R pyy, R pzz, R pxy, R pxz, R pyz, R rho, R ux, R uy, R uz,
                             R (&x)[MLP_IN]) {
    auto sq = [](R v) -> R {
#ifdef __CUDA_ARCH__
        if constexpr (FAST && std::is_same<R, float>::value) {
            float r;
            asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(v));
            return r;
        }
#endif
        return mlp_sqrt<R>(v);
    };
    auto dv = [](R a, R b) -> R {
#ifdef __CUDA_ARCH__
        if constexpr (FAST && std::is_same<R, float>::value) return __fdividef(a, b);
#endif
        return a / b;
    };
    auto lg = [](R v) -> R {
#ifdef __CUDA_ARCH__
        if constexpr (FAST && std::is_same<R, float>::value) return __logf(v);
#endif
        return mlp_log<R>(v);
    };
    const R off2 = pxy * pxy + pxz * pxz + pyz * pyz;
    const R s2 = pxx * pxx + pyy * pyy + pzz * pzz + R(2) * off2;
    const R pim = dv(sq(R(2) * s2), rho);
    const R tr = pxx + pyy + pzz;
    const R t3 = tr * R(1.0 / 3.0);
    const R dxx = pxx - t3, dyy = pyy - t3, dzz = pzz - t3;
    const R d2 = dxx * dxx + dyy * dyy + dzz * dzz + R(2) * off2;
    const R dn = sq(d2);
    const R tr3 = dxx * dxx * dxx + dyy * dyy * dyy + dzz * dzz * dzz +
                  R(3) * (dxx * (pxy * pxy + pxz * pxz) + dyy * (pxy * pxy + pyz * pyz) +
                          dzz * (pxz * pxz + pyz * pyz)) +
                  R(6) * pxy * pxz * pyz;
    const R u2 = ux * ux + uy * uy + uz * uz;
    const R uau = ux * (dxx * ux + pxy * uy + pxz * uz) + uy * (pxy * ux + dyy * uy + pyz * uz) +
                  uz * (pxz * ux + pyz * uy + dzz * uz);
    R mx = mlp_abs<R>(dxx);
    if (mlp_abs<R>(dyy) > mx) mx = mlp_abs<R>(dyy);
    if (mlp_abs<R>(dzz) > mx) mx = mlp_abs<R>(dzz);
    x[0] = lg(pim + R(1e-9));
    x[1] = R(100) * pim;
    x[2] = dv(tr, sq(s2) + R(1e-12));
    x[3] = dv(R(2.449489742783178) * tr3, d2 * dn + R(1e-30));
    x[4] = R(30) * sq(u2);
    x[5] = R(1000) * (rho - R(1));
    x[6] = dv(uau, (u2 + R(1e-12)) * dn + R(1e-30));
    x[7] = dv(off2, s2 + R(1e-30));
    x[8] = dv(mx, dn + R(1e-30));
    x[9] = R(1000) * u2;
}

// Network output y (before the softplus).  `w` is anything indexable that yields the FP32
// parameters: a pointer, or an accessor that reads a __constant__ array by name (then, fully
// unrolled, every parameter becomes an instruction operand).  FULL unrolls both layers;
// otherwise the second layer loops over its units (parameters in shared or global memory are
// loaded as needed instead of all at once).
template <class R, class WA, bool FULL = true, bool SWEEP = false>
LBM_HD R mlp_output(const R (&x)[MLP_IN], const WA& w) {
    auto act = [](R z) { return SWEEP ? mlp_silu_sweep<R>(z) : mlp_silu<R>(z); };
    R h1[MLP_H];
#pragma unroll
    for (int k = 0; k < MLP_H; ++k) {
        R z = R(w[MLP_B1 + k]);
#pragma unroll
        for (int i = 0; i < MLP_IN; ++i) z += x[i] * R(w[MLP_W1 + i * MLP_H + k]);
        h1[k] = act(z);
    }
    R y = R(w[MLP_B3]);
    auto unit = [&](int k) {
        R z = R(w[MLP_B2 + k]);
#pragma unroll
        for (int j = 0; j < MLP_H; ++j) z += h1[j] * R(w[MLP_W2 + j * MLP_H + k]);
        y += act(z) * R(w[MLP_W3 + k]);
    };
    if constexpr (FULL) {
#pragma unroll
        for (int k = 0; k < MLP_H; ++k) unit(k);
    } else {
#pragma unroll 1
        for (int k = 0; k < MLP_H; ++k) unit(k);
    }
    return y;
}

template <class R, class WA, bool FULL = true, bool SWEEP = false>
LBM_HD R closure_nu_t(const R (&x)[MLP_IN], const WA& w) {
    return R(w[MLP_SCALE]) * mlp_softplus<R>(mlp_output<R, WA, FULL, SWEEP>(x, w));
}

#ifdef __CUDACC__
// ------------------------------------------------------------------ tensor-core inference (FP32)
// The network for the 32 cells of a warp at once, as three chained m16n8k16 FP16 products
// (mma.sync; rows are the warp's cells, taken 16 at a time): [16 x 16] features (zero-padded
// from 10) x [16 x 32], [16 x 32] x [32 x 32], [16 x 32] x [32 x 8] (the output unit in column
// 0), accumulating in FP32 from the biases.  The accumulator fragment of a hidden layer has the
// layout of the A fragment of the next product (two adjacent 8-column tiles form one 16-wide
// k-step), so the hidden activations never leave registers: the SiLU and the FP16 packing are
// applied to them in place.  Only the features pass through shared memory once, to be
// transposed into A fragments.  FP16 operands (11-bit significand, as TF32) give nu_t to about
// 1e-3 relative; training and the FP64 sweep use the exact network.

constexpr int MLP_FRAGS = 4 + 8 + 2;             // B fragments: layer 1 (4 n-tiles), 2 (2 k x 4 n), 3 (2 k)
constexpr int MLP_XLD = 12;                      // row stride (32-bit words) of a warp's feature tile

// Shared-memory image of the parameters: per B fragment and lane the two 32-bit registers of
// mma.m16n8k16's B operand (f16 pairs along k), the halved biases of both hidden layers as
// accumulator start values, b3 and the output scale.  Copied in 16-byte pieces.
struct __align__(16) MlpShared {
    uint2 frag[MLP_FRAGS][32];
    float4 hb1[4][4], hb2[4][4];   // [n-tile][t]: halved biases of columns 8 nt + 2t, + 1, twice
    float b3, scale;
    float pad_[2];
};

// Softplus for the in-sweep FP32 inference, with the fast exponential and logarithm (absolute
// error of log(1 + e^y) about 1e-7).
__device__ __forceinline__ float mlp_softplus_sweep(float y) {
    return y > 20.f ? y : __logf(1.f + __expf(y));
}

__device__ __forceinline__ uint32_t pack_half2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// SiLU of two pre-activations given as h = z / 2: h (1 + tanh h) in packed FP16, with the
// hardware tanh (tanh.approx.f16x2).  The result is one A-fragment register of the next product.
__device__ __forceinline__ uint32_t silu_half2(float h_lo, float h_hi) {
    uint32_t r;
    asm("{\n\t.reg .b32 h, t;\n\t"
        "cvt.rn.f16x2.f32 h, %2, %1;\n\t"
        "tanh.approx.f16x2 t, h;\n\t"
        "fma.rn.f16x2 %0, h, t, h;\n\t}"
        : "=r"(r) : "f"(h_lo), "f"(h_hi));
    return r;
}

__device__ __forceinline__ void mma_f16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                        uint2 b) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b.x), "r"(b.y));
}

// Fills `s` from the FP32 parameter block; all threads of the block take part.  Fragment f, lane
// (g = lane / 4, t = lane % 4) holds rows k0 = 16 ks + 2t, k0 + 1 (first register) and k0 + 8,
// k0 + 9 (second) of column n = 8 nt + g of the layer's K x N weight matrix.  The hidden layers'
// weights and biases are stored halved (exact in FP16), so that their products give h = z / 2,
// the argument of the SiLU's tanh, directly.
template <class WA>
__device__ __forceinline__ void stage_mlp_params(const WA& w, MlpShared& s, int tid, int nthreads) {
    for (int i = tid; i < MLP_FRAGS * 32; i += nthreads) {
        const int f = i >> 5, lane = i & 31, g = lane >> 2, t = lane & 3;
        float v[4];
        if (f < 4) {                                   // layer 1: W1[k][n], k < MLP_IN
            const int n = 8 * f + g;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int k = 2 * t + (j & 1) + 8 * (j >> 1);
                v[j] = k < MLP_IN ? 0.5f * w[MLP_W1 + k * MLP_H + n] : 0.f;
            }
        } else if (f < 12) {                           // layer 2: W2[k][n]
            const int ks = (f - 4) >> 2, n = 8 * ((f - 4) & 3) + g;
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = 0.5f * w[MLP_W2 + (16 * ks + 2 * t + (j & 1) + 8 * (j >> 1)) * MLP_H + n];
        } else {                                       // output unit in column 0
            const int ks = f - 12;
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = g == 0 ? w[MLP_W3 + 16 * ks + 2 * t + (j & 1) + 8 * (j >> 1)] : 0.f;
        }
        s.frag[f][lane] = make_uint2(pack_half2(v[0], v[1]), pack_half2(v[2], v[3]));
    }
    for (int i = tid; i < 16; i += nthreads) {
        const int col = 8 * (i >> 2) + 2 * (i & 3);
        const float a0 = 0.5f * w[MLP_B1 + col], a1 = 0.5f * w[MLP_B1 + col + 1];
        const float c0 = 0.5f * w[MLP_B2 + col], c1 = 0.5f * w[MLP_B2 + col + 1];
        s.hb1[i >> 2][i & 3] = make_float4(a0, a1, a0, a1);
        s.hb2[i >> 2][i & 3] = make_float4(c0, c1, c0, c1);
    }
    if (tid == 0) {
        s.b3 = w[MLP_B3];
        s.scale = w[MLP_SCALE];
    }
}

// SiLU of two adjacent 8-column accumulator tiles (h = z / 2 of columns 16 ks .. 16 ks + 15 of a
// hidden layer) into the four A-fragment registers of the next product's k-step ks.
__device__ __forceinline__ void hidden_to_a(const float (&lo)[4], const float (&hi)[4], uint32_t (&a)[4]) {
    a[0] = silu_half2(lo[0], lo[1]);
    a[1] = silu_half2(lo[2], lo[3]);
    a[2] = silu_half2(hi[0], hi[1]);
    a[3] = silu_half2(hi[2], hi[3]);
}

// nu_t of this lane's cell; every lane of the warp must call it together.  X: this warp's feature
// tile, 32 rows of MLP_XLD words.
__device__ __forceinline__ float warp_mlp_nu(const float (&x)[MLP_IN], const MlpShared& s, uint32_t* X) {
    const int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
    const int g = lane >> 2, t = lane & 3;
    {
        uint4* row = reinterpret_cast<uint4*>(X + lane * MLP_XLD);
        row[0] = make_uint4(pack_half2(x[0], x[1]), pack_half2(x[2], x[3]), pack_half2(x[4], x[5]),
                            pack_half2(x[6], x[7]));
        row[1] = make_uint4(pack_half2(x[8], x[9]), 0u, 0u, 0u);
    }
    __syncwarp();
    float y = 0.f;
#pragma unroll 1
    for (int mt = 0; mt < 2; ++mt) {
        const uint32_t* r0 = X + (16 * mt + g) * MLP_XLD + t;
        const uint32_t* r1 = r0 + 8 * MLP_XLD;
        const uint32_t a0 = r0[0], a1 = r1[0], a2 = r0[4], a3 = r1[4];
        // accumulators start at the halved biases (one 16-byte shared load per tile)
        float h1[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const float4 b = s.hb1[nt][t];
            h1[nt][0] = b.x; h1[nt][1] = b.y; h1[nt][2] = b.z; h1[nt][3] = b.w;
            mma_f16(h1[nt], a0, a1, a2, a3, s.frag[nt][lane]);
        }
        uint32_t a[2][4];
        hidden_to_a(h1[0], h1[1], a[0]);
        hidden_to_a(h1[2], h1[3], a[1]);
        float h2[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const float4 b = s.hb2[nt][t];
            h2[nt][0] = b.x; h2[nt][1] = b.y; h2[nt][2] = b.z; h2[nt][3] = b.w;
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) mma_f16(h2[nt], a[ks][0], a[ks][1], a[ks][2], a[ks][3], s.frag[4 + 4 * ks + nt][lane]);
        }
        hidden_to_a(h2[0], h2[1], a[0]);
        hidden_to_a(h2[2], h2[3], a[1]);
        float o[4] = {s.b3, 0.f, s.b3, 0.f};
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) mma_f16(o, a[ks][0], a[ks][1], a[ks][2], a[ks][3], s.frag[12 + ks][lane]);
        // column 0: lane 4r holds the outputs of rows r (o[0]) and r + 8 (o[2]) of this tile
        const int src = 4 * (lane & 7);
        const float lo = __shfl_sync(0xffffffffu, o[0], src), hi = __shfl_sync(0xffffffffu, o[2], src);
        if ((lane >> 4) == mt) y = (lane & 8) ? hi : lo;
    }
    __syncwarp();
    return s.scale * mlp_softplus_sweep(y);
}
#endif

}  // namespace lbm
