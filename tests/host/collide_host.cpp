// Host build of the sweep's per-cell collision operators (lbmpy_b200/csrc/lbm_collide.cuh) so that
// their arithmetic can be checked against the oracle on the CPU.  Test infrastructure only.
#define __device__
#define __host__
#define __forceinline__ inline
#include <cmath>
using std::sqrt;
#include "../../lbmpy_b200/csrc/lbm_collide.cuh"
#include "../../lbmpy_b200/csrc/lbm_closure.cuh"

using namespace lbm;

template <int Q, int MK>
static double run(double* f, const Physics* p) {
    double g[Q];
    for (int i = 0; i < Q; ++i) g[i] = f[i];
    double om;
    if constexpr (MK == MK_POP) om = collide_pop<Q, double>(g, *p);
    else if constexpr (MK == MK_MRT) om = collide_mrt<Q, double>(g, *p);
    else if constexpr (MK == MK_CUM1) om = collide_cum_ho1<double>(g, *p);
    else om = collide_cum<double>(g, *p);
    for (int i = 0; i < Q; ++i) f[i] = g[i];
    return om;
}

template <int Q, int MK>
static double runf(double* f, const Physics* p) {
    float g[Q];
    for (int i = 0; i < Q; ++i) g[i] = (float)f[i];
    float om;
    if constexpr (MK == MK_POP) om = collide_pop<Q, float>(g, *p);
    else if constexpr (MK == MK_MRT) om = collide_mrt<Q, float>(g, *p);
    else if constexpr (MK == MK_CUM1) om = collide_cum_ho1<float>(g, *p);
    else om = collide_cum<float>(g, *p);
    for (int i = 0; i < Q; ++i) f[i] = g[i];
    return om;
}

template <class R> struct HostClosureNu {
    const float* w;
    R operator()(R pxx, R pyy, R pzz, R pxy, R pxz, R pyz, R rho, R ux, R uy, R uz) const {
        R x[MLP_IN];
        closure_features<R>(pxx, pyy, pzz, pxy, pxz, pyz, rho, ux, uy, uz, x);
        return closure_nu_t<R>(x, w);
    }
};
extern "C" {
int host_sizeof_physics() { return (int)sizeof(Physics); }
double host_collide(int q, int mk, int fp32, double* f, const Physics* p) {
    if (q == 19 && mk == MK_POP) return fp32 ? runf<19, MK_POP>(f, p) : run<19, MK_POP>(f, p);
    if (q == 19 && mk == MK_MRT) return fp32 ? runf<19, MK_MRT>(f, p) : run<19, MK_MRT>(f, p);
    if (q == 27 && mk == MK_POP) return fp32 ? runf<27, MK_POP>(f, p) : run<27, MK_POP>(f, p);
    if (q == 27 && mk == MK_MRT) return fp32 ? runf<27, MK_MRT>(f, p) : run<27, MK_MRT>(f, p);
    if (q == 27 && mk == MK_CUM) return fp32 ? runf<27, MK_CUM>(f, p) : run<27, MK_CUM>(f, p);
    if (q == 27 && mk == MK_CUM1) return fp32 ? runf<27, MK_CUM1>(f, p) : run<27, MK_CUM1>(f, p);
    return -1.0;
}
// learned closure: features, network, and the cumulant collision with the closure folded in
void host_closure_features(const double* s10, double* x) {
    double xx[MLP_IN];
    closure_features<double>(s10[0], s10[1], s10[2], s10[3], s10[4], s10[5], s10[6], s10[7], s10[8], s10[9], xx);
    for (int i = 0; i < MLP_IN; ++i) x[i] = xx[i];
}
double host_closure_nu_t(const double* x, const float* w) {
    double xx[MLP_IN];
    for (int i = 0; i < MLP_IN; ++i) xx[i] = x[i];
    return closure_nu_t<double>(xx, w);
}
double host_collide_closure(int fp32, double* f, const Physics* p, const float* w) {
    if (fp32) {
        float g[27];
        for (int i = 0; i < 27; ++i) g[i] = (float)f[i];
        const float om = collide_cum_ho1<float, true>(g, *p, HostClosureNu<float>{w});
        for (int i = 0; i < 27; ++i) f[i] = g[i];
        return om;
    }
    double g[27];
    for (int i = 0; i < 27; ++i) g[i] = f[i];
    const double om = collide_cum_ho1<double, true>(g, *p, HostClosureNu<double>{w});
    for (int i = 0; i < 27; ++i) f[i] = g[i];
    return om;
}
void host_equilibrium(int q, int mk, double* f, double rho, double ux, double uy, double uz, const Physics* p) {
    if (q == 19 && mk == MK_POP) { double g[19]; equilibrium<19, double, MK_POP>(g, rho, ux, uy, uz, *p); for (int i = 0; i < 19; ++i) f[i] = g[i]; }
    if (q == 19 && mk == MK_MRT) { double g[19]; equilibrium<19, double, MK_MRT>(g, rho, ux, uy, uz, *p); for (int i = 0; i < 19; ++i) f[i] = g[i]; }
    if (q == 27 && mk == MK_POP) { double g[27]; equilibrium<27, double, MK_POP>(g, rho, ux, uy, uz, *p); for (int i = 0; i < 27; ++i) f[i] = g[i]; }
    if (q == 27 && mk == MK_CUM) { double g[27]; equilibrium<27, double, MK_CUM>(g, rho, ux, uy, uz, *p); for (int i = 0; i < 27; ++i) f[i] = g[i]; }
}
}
