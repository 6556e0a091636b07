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
template <class R>
LBM_HD void closure_features(R pxx, R pyy, R pzz, R pxy, R pxz, R pyz, R rho, R ux, R uy, R uz,
                             R (&x)[MLP_IN]) {
    const R off2 = pxy * pxy + pxz * pxz + pyz * pyz;
    const R s2 = pxx * pxx + pyy * pyy + pzz * pzz + R(2) * off2;
    const R pim = mlp_sqrt<R>(R(2) * s2) / rho;
    const R tr = pxx + pyy + pzz;
    const R t3 = tr * R(1.0 / 3.0);
    const R dxx = pxx - t3, dyy = pyy - t3, dzz = pzz - t3;
    const R d2 = dxx * dxx + dyy * dyy + dzz * dzz + R(2) * off2;
    const R dn = mlp_sqrt<R>(d2);
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
    x[0] = mlp_log<R>(pim + R(1e-9));
    x[1] = R(100) * pim;
    x[2] = tr / (mlp_sqrt<R>(s2) + R(1e-12));
    x[3] = R(2.449489742783178) * tr3 / (d2 * dn + R(1e-30));
    x[4] = R(30) * mlp_sqrt<R>(u2);
    x[5] = R(1000) * (rho - R(1));
    x[6] = uau / ((u2 + R(1e-12)) * dn + R(1e-30));
    x[7] = off2 / (s2 + R(1e-30));
    x[8] = mx / (dn + R(1e-30));
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
// The network for the 32 cells of a warp at once: each layer is a 32 x K by K x 32 product done
// as m16n8k8 TF32 tiles (mma.sync; rows are the warp's cells), the hidden activations pass
// through a per-warp shared-memory tile of 32 rows.  TF32 operands (10-bit mantissa) give nu_t to
// about 1e-3 relative; training and the FP64 sweep use the exact network.

constexpr int MLP_TLD = 33;                       // row stride of the per-warp activation tile

__device__ __forceinline__ uint32_t to_tf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return r;
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Parameter block as the tensor-core network reads it from shared memory: the entries of W1 and
// W2 as TF32 bit patterns, everything else as FP32 bit patterns.
template <class WA>
__device__ __forceinline__ void stage_mlp_params(const WA& w, uint32_t* sw, int tid, int nthreads) {
    for (int i = tid; i < MLP_PARAMS; i += nthreads) {
        const float v = w[i];
        const bool matrix = i < MLP_B1 || (i >= MLP_W2 && i < MLP_B2);
        sw[i] = matrix ? to_tf32(v) : __float_as_uint(v);
    }
}

// nu_t of this lane's cell; every lane of the warp must call it together.  T: this warp's
// 32 x MLP_TLD float tile.
__device__ __forceinline__ float warp_mlp_nu(const float (&x)[MLP_IN], const uint32_t* sw, float* T) {
    const int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
    const int gid = lane >> 2, t4 = lane & 3;
    auto F = [&](int i) { return __uint_as_float(sw[i]); };
#pragma unroll
    for (int k = 0; k < 16; ++k) T[lane * MLP_TLD + k] = k < MLP_IN ? x[k] : 0.f;
    __syncwarp();
    float acc[2][4][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[mt][nt][c] = 0.f;
    // layer 1: [32 x 16] (features, zero-padded) x [16 x 32]
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            const int r0 = (mt * 16 + gid) * MLP_TLD, r1 = r0 + 8 * MLP_TLD, c0 = ks * 8 + t4;
            const uint32_t a0 = to_tf32(T[r0 + c0]), a1 = to_tf32(T[r1 + c0]);
            const uint32_t a2 = to_tf32(T[r0 + c0 + 4]), a3 = to_tf32(T[r1 + c0 + 4]);
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int n = nt * 8 + gid;
                const uint32_t b0 = c0 < MLP_IN ? sw[MLP_W1 + c0 * MLP_H + n] : 0u;
                const uint32_t b1 = c0 + 4 < MLP_IN ? sw[MLP_W1 + (c0 + 4) * MLP_H + n] : 0u;
                mma_tf32(acc[mt][nt], a0, a1, a2, a3, b0, b1);
            }
        }
    __syncwarp();
    // bias + SiLU, back into the tile as rows of 32 hidden units
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int col = nt * 8 + 2 * t4, r0 = (mt * 16 + gid) * MLP_TLD, r1 = r0 + 8 * MLP_TLD;
            const float blo = F(MLP_B1 + col), bhi = F(MLP_B1 + col + 1);
            T[r0 + col] = mlp_silu_sweep<float>(acc[mt][nt][0] + blo);
            T[r0 + col + 1] = mlp_silu_sweep<float>(acc[mt][nt][1] + bhi);
            T[r1 + col] = mlp_silu_sweep<float>(acc[mt][nt][2] + blo);
            T[r1 + col + 1] = mlp_silu_sweep<float>(acc[mt][nt][3] + bhi);
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[mt][nt][c] = 0.f;
        }
    __syncwarp();
    // layer 2: [32 x 32] x [32 x 32]
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const int r0 = (mt * 16 + gid) * MLP_TLD, r1 = r0 + 8 * MLP_TLD, c0 = ks * 8 + t4;
            const uint32_t a0 = to_tf32(T[r0 + c0]), a1 = to_tf32(T[r1 + c0]);
            const uint32_t a2 = to_tf32(T[r0 + c0 + 4]), a3 = to_tf32(T[r1 + c0 + 4]);
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int n = nt * 8 + gid;
                mma_tf32(acc[mt][nt], a0, a1, a2, a3, sw[MLP_W2 + c0 * MLP_H + n], sw[MLP_W2 + (c0 + 4) * MLP_H + n]);
            }
        }
    // output unit: per-lane partial sums over its columns, then over the 4 lanes of a row group
    float y[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int col = nt * 8 + 2 * t4;
            const float blo = F(MLP_B2 + col), bhi = F(MLP_B2 + col + 1);
            const float wlo = F(MLP_W3 + col), whi = F(MLP_W3 + col + 1);
            y[mt][0] += mlp_silu_sweep<float>(acc[mt][nt][0] + blo) * wlo +
                        mlp_silu_sweep<float>(acc[mt][nt][1] + bhi) * whi;
            y[mt][1] += mlp_silu_sweep<float>(acc[mt][nt][2] + blo) * wlo +
                        mlp_silu_sweep<float>(acc[mt][nt][3] + bhi) * whi;
        }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            y[mt][h] += __shfl_xor_sync(0xffffffffu, y[mt][h], 1);
            y[mt][h] += __shfl_xor_sync(0xffffffffu, y[mt][h], 2);
        }
    // row `lane` sits in tile lane >> 4, half (lane >> 3) & 1, row group lane & 7
    const int src = 4 * (lane & 7);
    const float v00 = __shfl_sync(0xffffffffu, y[0][0], src), v01 = __shfl_sync(0xffffffffu, y[0][1], src);
    const float v10 = __shfl_sync(0xffffffffu, y[1][0], src), v11 = __shfl_sync(0xffffffffu, y[1][1], src);
    const int mt = lane >> 4, half = (lane >> 3) & 1;
    const float yv = (mt ? (half ? v11 : v10) : (half ? v01 : v00)) + F(MLP_B3);
    __syncwarp();
    return F(MLP_SCALE) * mlp_softplus<float>(yv);
}
#endif

}  // namespace lbm
