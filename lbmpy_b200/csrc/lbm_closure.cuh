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

}  // namespace lbm
