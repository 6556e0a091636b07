// Per-cell collision operators of lbmpy's methods, written for registers.
//
// All operators work on zero-centred PDFs f~ = f - w (lbmpy's default storage,
// creationfunctions.py:140) and return post-collision PDFs in place.
//   collide_pop  -- SRT/TRT in population space, delta equilibrium
//                   (methods/momentbased/momentbasedmethod.py:389-398)
//   collide_mrt  -- raw-moment MRT with the weighted-orthogonal basis
//                   (methods/momentbased/momentbasedmethod.py:359-387)
//   collide_cum  -- D3Q27 polynomial cumulants (Geier et al. 2015) with optional Galilean
//                   correction and CentralMoment forcing
//                   (methods/cumulantbased/cumulantbasedmethod.py:296-402,
//                    methods/cumulantbased/galilean_correction.py:56-91, forcemodels.py:213-233)
// Smagorinsky (turbulence_models.py:25-84) is shared by all three.
#pragma once
#include "lbm_common.cuh"

namespace lbm {

// acc + c*x for a compile-time table coefficient c: zeros and unit factors fold away
// (IEEE arithmetic forbids the compiler from dropping 0*x on its own).
template <class R, class A>
__device__ __forceinline__ R cmad(A acc_in, double c, R x) {
    const R acc = acc_in;
    return c == 0.0 ? acc : (c == 1.0 ? acc + x : (c == -1.0 ? acc - x : acc + R(c) * x));
}

// Conserved quantities of zero-centred PDFs (methods/conservedquantitycomputation.py:218-249).
template <int Q, class R> struct Macro {
    R drho, rho, rho_ref, ux, uy, uz;
};

template <int Q, class R>
__device__ __forceinline__ Macro<Q, R> conserved(const R (&f)[Q], const Physics& p, bool eq_shift) {
    using L = Lat<Q>;
    R d = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        d += f[i];
        if (L::cx(i) == 1) jx += f[i]; else if (L::cx(i) == -1) jx -= f[i];
        if (L::cy(i) == 1) jy += f[i]; else if (L::cy(i) == -1) jy -= f[i];
        if (L::cz(i) == 1) jz += f[i]; else if (L::cz(i) == -1) jz -= f[i];
    }
    Macro<Q, R> m;
    m.drho = d;
    m.rho = R(1) + d;
    m.rho_ref = p.compressible ? m.rho : R(1);
    const R inv = R(1) / m.rho_ref;
    m.ux = jx * inv; m.uy = jy * inv; m.uz = jz * inv;
    if (eq_shift) {
        const R h = R(0.5) * inv;
        m.ux += h * R(p.force[0]); m.uy += h * R(p.force[1]); m.uz += h * R(p.force[2]);
    }
    return m;
}

// Smagorinsky rate from the non-equilibrium stress.  f_eq's second raw moments are
// rho_f*u_a*u_b + delta_ab*drho/3 for every method here (they are matched moments).
template <int Q, class R>
__device__ __forceinline__ R smagorinsky_rate(const R (&f)[Q], const Macro<Q, R>& m, const Physics& p) {
    using L = Lat<Q>;
    R sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        if (L::cx(i) != 0) sxx += f[i];
        if (L::cy(i) != 0) syy += f[i];
        if (L::cz(i) != 0) szz += f[i];
        if (L::cx(i) * L::cy(i) == 1) sxy += f[i]; else if (L::cx(i) * L::cy(i) == -1) sxy -= f[i];
        if (L::cx(i) * L::cz(i) == 1) sxz += f[i]; else if (L::cx(i) * L::cz(i) == -1) sxz -= f[i];
        if (L::cy(i) * L::cz(i) == 1) syz += f[i]; else if (L::cy(i) * L::cz(i) == -1) syz -= f[i];
    }
    const R rf = p.compressible ? m.rho : R(1);
    const R third = m.drho * R(1.0 / 3.0);
    const R pxx = sxx - rf * m.ux * m.ux - third;
    const R pyy = syy - rf * m.uy * m.uy - third;
    const R pzz = szz - rf * m.uz * m.uz - third;
    const R pxy = sxy - rf * m.ux * m.uy;
    const R pxz = sxz - rf * m.ux * m.uz;
    const R pyz = syz - rf * m.uy * m.uz;
    const R s2 = pxx * pxx + pyy * pyy + pzz * pzz + R(2) * (pxy * pxy + pxz * pxz + pyz * pyz);
    const R pi = sqrt(R(2) * s2) / m.rho_ref;
    const R tau0 = R(p.tau0);
    return R(2) / (tau0 + sqrt(R(p.sgs_c18) * pi + tau0 * tau0));
}

// ------------------------------------------------------------------ SRT / TRT
template <int Q, class R>
__device__ __forceinline__ R collide_pop(R (&f)[Q], const Physics& p) {
    using L = Lat<Q>;
    const bool shift = p.force_model == FM_GUO || p.force_model == FM_CENTRAL;
    const Macro<Q, R> m = conserved<Q, R>(f, p, shift);
    R wp = R(p.rates[0]), wm = R(p.rates[1]);
    if (p.sgs == 1) {
        const R om = smagorinsky_rate<Q, R>(f, m, p);
        if (p.sgs_mask & 1u) wp = om;
        if (p.sgs_mask & 2u) wm = om;
    }
    const R rf = p.compressible ? m.rho : R(1);
    const R uxx = m.ux * m.ux, uyy = m.uy * m.uy, uzz = m.uz * m.uz;
    const R uxy = m.ux * m.uy, uxz = m.ux * m.uz, uyz = m.uy * m.uz;
    const bool cont = p.continuous_eq != 0;
    const bool has_force = p.force_model == FM_GUO || p.force_model == FM_SIMPLE || p.force_model == FM_LUO;
    const R Fx = R(p.force[0]), Fy = R(p.force[1]), Fz = R(p.force[2]);
    const R uF = m.ux * Fx + m.uy * Fy + m.uz * Fz;
    R fe_scale = R(1), fo_scale = R(1), fe_on = R(1);
    if (p.force_model == FM_GUO) { fe_scale = R(1) - R(0.5) * wp; fo_scale = R(1) - R(0.5) * wm; }
    if (p.force_model == FM_SIMPLE) fe_on = R(0);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int j = L::inv(i);
        if (j < i) continue;   // handle each (i, inverse) pair once
        const R w = R(L::w(i));
        R quad = 0;
        if (cont) {
            quad = cmad(quad, L::eqquad(true, i, 0), uxx); quad = cmad(quad, L::eqquad(true, i, 1), uyy);
            quad = cmad(quad, L::eqquad(true, i, 2), uzz); quad = cmad(quad, L::eqquad(true, i, 3), uxy);
            quad = cmad(quad, L::eqquad(true, i, 4), uxz); quad = cmad(quad, L::eqquad(true, i, 5), uyz);
        } else {
            quad = cmad(quad, L::eqquad(false, i, 0), uxx); quad = cmad(quad, L::eqquad(false, i, 1), uyy);
            quad = cmad(quad, L::eqquad(false, i, 2), uzz); quad = cmad(quad, L::eqquad(false, i, 3), uxy);
            quad = cmad(quad, L::eqquad(false, i, 4), uxz); quad = cmad(quad, L::eqquad(false, i, 5), uyz);
        }
        const R feq_e = m.drho * w + rf * quad;
        R force_e = 0, force_o = 0;
        if (has_force) {
            const R cF = R(L::cx(i)) * Fx + R(L::cy(i)) * Fy + R(L::cz(i)) * Fz;
            const R cu = R(L::cx(i)) * m.ux + R(L::cy(i)) * m.uy + R(L::cz(i)) * m.uz;
            force_e = fe_on * fe_scale * w * (R(9) * cF * cu - R(3) * uF);
            force_o = fo_scale * w * R(3) * cF;
        }
        if (j == i) {   // rest direction: even only
            f[i] = f[i] + wp * (feq_e - f[i]) + force_e;
        } else {
            R lin = 0;
            lin = cmad(lin, L::eqlin(true, i, 0), m.ux);
            lin = cmad(lin, L::eqlin(true, i, 1), m.uy);
            lin = cmad(lin, L::eqlin(true, i, 2), m.uz);
            const R feq_o = rf * lin;
            const R fi = f[i], fj = f[j];
            const R fe = R(0.5) * (fi + fj), fo = R(0.5) * (fi - fj);
            const R de = wp * (feq_e - fe) + force_e;
            const R dod = wm * (feq_o - fo) + force_o;
            f[i] = fi + de + dod;
            f[j] = fj + de - dod;
        }
    }
    return wp;
}

// ------------------------------------------------------------------ MRT (raw moment space)
template <int Q, class R>
__device__ __forceinline__ R collide_mrt(R (&f)[Q], const Physics& p) {
    using L = Lat<Q>;
    const bool shift = p.force_model == FM_GUO || p.force_model == FM_CENTRAL;
    const Macro<Q, R> m = conserved<Q, R>(f, p, shift);
    R om_sgs = R(0);
    if (p.sgs == 1) om_sgs = smagorinsky_rate<Q, R>(f, m, p);
    const R rf = p.compressible ? m.rho : R(1);
    const R uu[6] = {m.ux * m.ux, m.uy * m.uy, m.uz * m.uz, m.ux * m.uy, m.ux * m.uz, m.uy * m.uz};
    const bool has_force = p.force_model == FM_GUO || p.force_model == FM_SIMPLE || p.force_model == FM_LUO;
    // Moments of the force populations (Luo and Guo: w_i (9 (c.F)(c.u) + 3 c.F - 3 u.F); Simple:
    // 3 w_i c.F) in closed form: the even rows see 9 sum_ab T_ab F_a u_b - 3 (u.F) S, the odd rows
    // 3 sum_a B_a F_a (tables generated from the basis).
    const R Fx = R(p.force[0]), Fy = R(p.force[1]), Fz = R(p.force[2]);
    const bool simple = p.force_model == FM_SIMPLE;
    const R FU[6] = {Fx * m.ux, Fy * m.uy, Fz * m.uz, Fx * m.uy + Fy * m.ux, Fx * m.uz + Fz * m.ux,
                     Fy * m.uz + Fz * m.uy};
    const R uF = m.ux * Fx + m.uy * Fy + m.uz * Fz;
    // Every row of the weighted-orthogonal basis is even or odd under c -> -c, so the transforms
    // run on the sums and differences of opposite populations, f_i +- f_inv(i): half the terms of
    // the dense Q x Q products.  The moment changes are folded into the even and odd parts of the
    // result as soon as they are known, so no array of them stays live.
    constexpr int NP = (Q - 1) / 2;
    R fs[NP], fd[NP], ev[NP], od[NP];
    const R f0 = f[0];
#pragma unroll
    for (int q2 = 0; q2 < NP; ++q2) {
        const int i = L::pair(q2), j = L::inv(L::pair(q2));
        fs[q2] = f[i] + f[j];
        fd[q2] = f[i] - f[j];
        ev[q2] = R(0);
        od[q2] = R(0);
    }
    R e0 = R(0);
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const bool even = L::Meven(k);
        R mk = 0;
        if (even) {
            mk = cmad(mk, L::M(k, 0), f0);
#pragma unroll
            for (int q2 = 0; q2 < NP; ++q2) mk = cmad(mk, L::M(k, L::pair(q2)), fs[q2]);
        } else {
#pragma unroll
            for (int q2 = 0; q2 < NP; ++q2) mk = cmad(mk, L::M(k, L::pair(q2)), fd[q2]);
        }
        R lin = 0, quad = 0;
        lin = cmad(lin, L::mlin(k, 0), m.ux);
        lin = cmad(lin, L::mlin(k, 1), m.uy);
        lin = cmad(lin, L::mlin(k, 2), m.uz);
#pragma unroll
        for (int a = 0; a < 6; ++a) quad = cmad(quad, L::mquad(k, a), uu[a]);
        const R meq = cmad(rf * (lin + quad), L::p0(k), m.drho);
        R r = R(p.rates[k]);
        if (p.sgs == 1 && ((p.sgs_mask >> k) & 1u)) r = om_sgs;
        R d = r * (meq - mk);
        if (has_force) {
            R fk = 0;
            if (even) {
                if (!simple) {
#pragma unroll
                    for (int a = 0; a < 6; ++a) fk = cmad(fk, 9.0 * L::fT(k, a), FU[a]);
                    fk = cmad(fk, -3.0 * L::fS(k), uF);
                }
            } else {
                fk = cmad(fk, 3.0 * L::fB(k, 0), Fx);
                fk = cmad(fk, 3.0 * L::fB(k, 1), Fy);
                fk = cmad(fk, 3.0 * L::fB(k, 2), Fz);
            }
            if (p.force_model == FM_GUO) fk *= (R(1) - R(0.5) * r);
            d += fk;
        }
        // back: column k of M^-1 is even or odd with row k of M, so f_i and f_inv(i) receive the
        // even part plus or minus the odd part
        if (even) {
            e0 = cmad(e0, L::Minv(0, k), d);
#pragma unroll
            for (int q2 = 0; q2 < NP; ++q2) ev[q2] = cmad(ev[q2], L::Minv(L::pair(q2), k), d);
        } else {
#pragma unroll
            for (int q2 = 0; q2 < NP; ++q2) od[q2] = cmad(od[q2], L::Minv(L::pair(q2), k), d);
        }
    }
    f[0] = f0 + e0;
#pragma unroll
    for (int q2 = 0; q2 < NP; ++q2) {
        const int i = L::pair(q2), j = L::inv(L::pair(q2));
        f[i] += ev[q2] + od[q2];
        f[j] += ev[q2] - od[q2];
    }
    return p.sgs == 1 ? om_sgs : R(0);
}

// ------------------------------------------------------------------ D3Q27 cumulant
// Index of direction i in the 3x3x3 velocity cube, (cx+1)*9 + (cy+1)*3 + (cz+1).
template <int Q> LBM_HD constexpr int cube(int i) {
    return (Lat<Q>::cx(i) + 1) * 9 + (Lat<Q>::cy(i) + 1) * 3 + (Lat<Q>::cz(i) + 1);
}

// Forward: populations on the velocity cube -> central moments about u, axis by axis.
template <class R>
__device__ __forceinline__ void chimera_forward(R (&g)[27], R u, int stride, int s1, int s2) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const int base = a * s1 + b * s2;
            const R fm = g[base], f0 = g[base + stride], fp = g[base + 2 * stride];
            const R k0 = fm + f0 + fp;
            const R dm = fp - fm;
            const R k1 = dm - u * k0;
            const R k2 = (fp + fm) - R(2) * u * dm + u * u * k0;
            g[base] = k0; g[base + stride] = k1; g[base + 2 * stride] = k2;
        }
    }
}

// Backward: central moments about u -> populations, axis by axis.
template <class R>
__device__ __forceinline__ void chimera_backward(R (&g)[27], R u, int stride, int s1, int s2) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const int base = a * s1 + b * s2;
            const R k0 = g[base], k1 = g[base + stride], k2 = g[base + 2 * stride];
            const R m1 = k1 + u * k0;
            const R m2 = k2 + R(2) * u * k1 + u * u * k0;
            g[base] = R(0.5) * (m2 - m1);
            g[base + stride] = k0 - m2;
            g[base + 2 * stride] = R(0.5) * (m2 + m1);
        }
    }
}

template <class R>
__device__ __forceinline__ R collide_cum(R (&f)[27], const Physics& p) {
    using L = Lat<27>;
    const bool cm_force = p.force_model == FM_CENTRAL;
    const Macro<27, R> m = conserved<27, R>(f, p, cm_force);
    const R rho = m.rho, irho = R(1) / rho;
    const R ux = m.ux, uy = m.uy, uz = m.uz;
    R om_sgs = R(0);
    if (p.sgs == 1) om_sgs = smagorinsky_rate<27, R>(f, m, p);

    R k[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) k[cube<27>(i)] = f[i];
    chimera_forward(k, uz, 1, 9, 3);   // z moments
    chimera_forward(k, uy, 3, 9, 1);   // y moments
    chimera_forward(k, ux, 9, 3, 1);   // x moments
    // background (lattice weights) central moments are separable: B0 = 1, B1 = -u, B2 = 1/3 + u^2
    const R bx[3] = {R(1), -ux, R(1.0 / 3.0) + ux * ux};
    const R by[3] = {R(1), -uy, R(1.0 / 3.0) + uy * uy};
    const R bz[3] = {R(1), -uz, R(1.0 / 3.0) + uz * uz};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) k[a * 9 + b * 3 + c] += bx[a] * by[b] * bz[c];
    // conserved central moments after the symmetric forcing step are exact: rho and 0
#define K(a, b, c) k[(a) * 9 + (b) * 3 + (c)]
    K(0, 0, 0) = rho; K(1, 0, 0) = 0; K(0, 1, 0) = 0; K(0, 0, 1) = 0;

    // ---- monomial cumulants (rho-scaled), zero first-order central moments
    const R k200 = K(2, 0, 0), k020 = K(0, 2, 0), k002 = K(0, 0, 2);
    const R k110 = K(1, 1, 0), k101 = K(1, 0, 1), k011 = K(0, 1, 1);
    const R k111 = K(1, 1, 1), k210 = K(2, 1, 0), k201 = K(2, 0, 1), k120 = K(1, 2, 0);
    const R k021 = K(0, 2, 1), k102 = K(1, 0, 2), k012 = K(0, 1, 2);
    const R C220 = K(2, 2, 0) - (k200 * k020 + R(2) * k110 * k110) * irho;
    const R C202 = K(2, 0, 2) - (k200 * k002 + R(2) * k101 * k101) * irho;
    const R C022 = K(0, 2, 2) - (k020 * k002 + R(2) * k011 * k011) * irho;
    const R C211 = K(2, 1, 1) - (k200 * k011 + R(2) * k110 * k101) * irho;
    const R C121 = K(1, 2, 1) - (k020 * k101 + R(2) * k110 * k011) * irho;
    const R C112 = K(1, 1, 2) - (k002 * k110 + R(2) * k101 * k011) * irho;
    const R C122 = K(1, 2, 2) - (k020 * k102 + k002 * k120 + R(2) * k110 * k012 + R(2) * k101 * k021 +
                                 R(4) * k011 * k111) * irho;
    const R C212 = K(2, 1, 2) - (k200 * k012 + k002 * k210 + R(2) * k110 * k102 + R(4) * k101 * k111 +
                                 R(2) * k011 * k201) * irho;
    const R C221 = K(2, 2, 1) - (k200 * k021 + k020 * k201 + R(4) * k110 * k111 + R(2) * k101 * k120 +
                                 R(2) * k011 * k210) * irho;
    const R C222 = K(2, 2, 2) -
                   (k200 * K(0, 2, 2) + k020 * K(2, 0, 2) + k002 * K(2, 2, 0) +
                    R(4) * (k110 * K(1, 1, 2) + k101 * K(1, 2, 1) + k011 * K(2, 1, 1))) * irho -
                   (R(2) * (k210 * k012 + k201 * k021 + k120 * k102) + R(4) * k111 * k111) * irho +
                   R(2) * (k200 * k020 * k002 + R(2) * (k200 * k011 * k011 + k020 * k101 * k101 +
                                                        k002 * k110 * k110) + R(8) * k110 * k101 * k011) *
                       irho * irho;

    // ---- relaxation of the polynomial cumulants (group rates from the plan)
    auto rate = [&](int idx) -> R {
        R r = R(p.rates[idx]);
        if (p.sgs == 1 && ((p.sgs_mask >> idx) & 1u)) r = om_sgs;
        return r;
    };
    // canonical order (methods.cumulant_groups): 0 rho | 1-3 momentum | 4 xy 5 xz 6 yz 7 x2-y2 8 x2-z2 |
    // 9 bulk | 10-12 (xy2+xz2, x2y+yz2, x2z+y2z) | 13-15 differences | 16 xyz | 17-18 | 19 | 20-22 | 23-25 | 26
    const R w_xy = rate(4), w_xz = rate(5), w_yz = rate(6), w_d1 = rate(7), w_d2 = rate(8), w_b = rate(9);
    const R P_d1 = k200 - k020, P_d2 = k200 - k002, P_b = k200 + k020 + k002;
    R Ps_d1 = P_d1 - w_d1 * P_d1;
    R Ps_d2 = P_d2 - w_d2 * P_d2;
    R Ps_b = P_b + w_b * (rho - P_b);
    const R c110 = k110 - w_xy * k110, c101 = k101 - w_xz * k101, c011 = k011 - w_yz * k011;
    if (p.galilean) {
        const R o1 = R(p.rates[7]), o2 = R(p.rates[9]);   // base rates, not the SGS-adapted ones
        const R h = R(0.5) * irho;
        const R Dx = -o1 * h * (R(2) * k200 - k020 - k002) - o2 * h * (k200 + k020 + k002 - rho);
        const R Dy = Dx + R(3) * o1 * h * (k200 - k020);
        const R Dz = Dx + R(3) * o1 * h * (k200 - k002);
        const R a1 = R(-3) * rho * (R(1) - R(0.5) * o1);
        const R a2 = R(-3) * rho * (R(1) - R(0.5) * o2);
        Ps_d1 += a1 * (ux * ux * Dx - uy * uy * Dy);
        Ps_d2 += a1 * (ux * ux * Dx - uz * uz * Dz);
        Ps_b += a2 * (ux * ux * Dx + uy * uy * Dy + uz * uz * Dz);
    }
    const R c200 = (Ps_b + Ps_d1 + Ps_d2) * R(1.0 / 3.0);
    const R c020 = c200 - Ps_d1;
    const R c002 = c200 - Ps_d2;
    // third order: sums and differences relax separately, xyz alone
    R w_s[3] = {rate(10), rate(11), rate(12)}, w_d[3] = {rate(13), rate(14), rate(15)}, w_xyz = rate(16);
    if (p.foc_limiter > 0.0) {
        // fourth-order correction: the optimal third-order rates of the plan, limited per cell by
        // the magnitude of the x-variant cumulant of each group (fourth_order_correction.py:199-211)
        const R lim = R(p.foc_limiter) * rho;
        const R a3 = fabs(k120 + k102), a4 = fabs(k120 - k102), a5 = fabs(k111);
        const R l3 = w_s[0] + (R(1) - w_s[0]) * a3 / (lim + a3);
        const R l4 = w_d[0] + (R(1) - w_d[0]) * a4 / (lim + a4);
        w_s[0] = w_s[1] = w_s[2] = l3;
        w_d[0] = w_d[1] = w_d[2] = l4;
        w_xyz = w_xyz + (R(1) - w_xyz) * a5 / (lim + a5);
    }
    const R s1 = (k120 + k102) * (R(1) - w_s[0]), s2 = (k210 + k012) * (R(1) - w_s[1]),
            s3 = (k201 + k021) * (R(1) - w_s[2]);
    const R d1 = (k120 - k102) * (R(1) - w_d[0]), d2 = (k210 - k012) * (R(1) - w_d[1]),
            d3 = (k201 - k021) * (R(1) - w_d[2]);
    const R c111 = k111 * (R(1) - w_xyz);
    const R c120 = R(0.5) * (s1 + d1), c102 = R(0.5) * (s1 - d1);
    const R c210 = R(0.5) * (s2 + d2), c012 = R(0.5) * (s2 - d2);
    const R c201 = R(0.5) * (s3 + d3), c021 = R(0.5) * (s3 - d3);
    // fourth order
    R q1 = (C220 - R(2) * C202 + C022) * (R(1) - rate(17));
    R q2 = (C220 + C202 - R(2) * C022) * (R(1) - rate(18));
    R q3 = (C220 + C202 + C022) * (R(1) - rate(19));
    R C211s = C211 * (R(1) - rate(20)), C121s = C121 * (R(1) - rate(21)), C112s = C112 * (R(1) - rate(22));
    if (p.foc_limiter > 0.0) {
        // correction terms of the fourth-order polynomial cumulants from velocity-derivative
        // estimates of the pre-collision second-order cumulants (Geier et al. 2017, eq. 44-49;
        // fourth_order_correction.py:100-145)
        const R o1 = R(p.rates[4]), o2 = R(p.rates[9]);
        const R h = R(0.5) * irho;
        const R Dx = -o1 * h * (R(2) * k200 - k020 - k002) - o2 * h * (k200 + k020 + k002 - rho);
        const R Dy = Dx + R(3) * o1 * h * (k200 - k020);
        const R Dz = Dx + R(3) * o1 * h * (k200 - k002);
        const R g = (R(1) / o1 - R(0.5)) * rho;
        const R ca = g * R(p.foc_a), cb = g * R(p.foc_b) * R(-1.0 / 3.0) * R(-3) * o1 * irho;
        q1 += R(2.0 / 3.0) * R(p.rates[17]) * ca * (Dx - R(2) * Dy + Dz);
        q2 += R(2.0 / 3.0) * R(p.rates[17]) * ca * (Dx + Dy - R(2) * Dz);
        q3 += R(-4.0 / 3.0) * R(p.rates[19]) * ca * (Dx + Dy + Dz);
        C211s += R(p.rates[20]) * cb * k011;
        C121s += R(p.rates[20]) * cb * k101;
        C112s += R(p.rates[20]) * cb * k110;
    }
    const R C220s = (q3 + q1 + q2) * R(1.0 / 3.0);
    const R C202s = (q3 - q1) * R(1.0 / 3.0);
    const R C022s = (q3 - q2) * R(1.0 / 3.0);
    const R C221s = C221 * (R(1) - rate(23)), C212s = C212 * (R(1) - rate(24)), C122s = C122 * (R(1) - rate(25));
    const R C222s = C222 * (R(1) - rate(26));

    // ---- back to central moments (moment-cumulant relations, zero first order)
    K(2, 0, 0) = c200; K(0, 2, 0) = c020; K(0, 0, 2) = c002;
    K(1, 1, 0) = c110; K(1, 0, 1) = c101; K(0, 1, 1) = c011;
    K(1, 1, 1) = c111; K(2, 1, 0) = c210; K(2, 0, 1) = c201; K(1, 2, 0) = c120;
    K(0, 2, 1) = c021; K(1, 0, 2) = c102; K(0, 1, 2) = c012;
    const R k220s = C220s + (c200 * c020 + R(2) * c110 * c110) * irho;
    const R k202s = C202s + (c200 * c002 + R(2) * c101 * c101) * irho;
    const R k022s = C022s + (c020 * c002 + R(2) * c011 * c011) * irho;
    K(2, 2, 0) = k220s; K(2, 0, 2) = k202s; K(0, 2, 2) = k022s;
    K(2, 1, 1) = C211s + (c200 * c011 + R(2) * c110 * c101) * irho;
    K(1, 2, 1) = C121s + (c020 * c101 + R(2) * c110 * c011) * irho;
    K(1, 1, 2) = C112s + (c002 * c110 + R(2) * c101 * c011) * irho;
    K(1, 2, 2) = C122s + (c020 * c102 + c002 * c120 + R(2) * c110 * c012 + R(2) * c101 * c021 +
                          R(4) * c011 * c111) * irho;
    K(2, 1, 2) = C212s + (c200 * c012 + c002 * c210 + R(2) * c110 * c102 + R(4) * c101 * c111 +
                          R(2) * c011 * c201) * irho;
    K(2, 2, 1) = C221s + (c200 * c021 + c020 * c201 + R(4) * c110 * c111 + R(2) * c101 * c120 +
                          R(2) * c011 * c210) * irho;
    K(2, 2, 2) = C222s +
                 (c200 * C022s + c020 * C202s + c002 * C220s +
                  R(4) * (c110 * C112s + c101 * C121s + c011 * C211s)) * irho +
                 (R(2) * (c210 * c012 + c201 * c021 + c120 * c102) + R(4) * c111 * c111) * irho +
                 (c200 * c020 * c002 + R(2) * (c200 * c011 * c011 + c020 * c101 * c101 + c002 * c110 * c110) +
                  R(8) * c110 * c101 * c011) * irho * irho;
    // symmetric forcing, second half: first-order central moments become F/2
    if (cm_force) {
        K(1, 0, 0) = R(0.5) * R(p.force[0]);
        K(0, 1, 0) = R(0.5) * R(p.force[1]);
        K(0, 0, 1) = R(0.5) * R(p.force[2]);
    }
#undef K
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) k[a * 9 + b * 3 + c] -= bx[a] * by[b] * bz[c];
    chimera_backward(k, ux, 9, 3, 1);
    chimera_backward(k, uy, 3, 9, 1);
    chimera_backward(k, uz, 1, 9, 3);
#pragma unroll
    for (int i = 0; i < 27; ++i) f[i] = k[cube<27>(i)];
    return p.sgs == 1 ? om_sgs : R(p.rates[4]);
}

// D3Q27 central-moment method (methods/momentbased/centralmomentbasedmethod.py:296-394): the
// polynomial central moments of the method's groups (the cumulant groups, default_moment_sets.py:
// 110-148) about the equilibrium velocity relax towards rho times the central moments of a
// Gaussian of variance 1/3; the force model's population term (Simple, Luo, Guo) enters in
// central-moment space, scaled by (1 - omega/2) per moment for Guo (forcemodels.py:201-203,
// 261-263, 300-306).  Compressible, zero-centred storage with the lattice-weight background.
template <class R>
__device__ __forceinline__ R collide_cm(R (&f)[27], const Physics& p) {
    using L = Lat<27>;
    const bool guo = p.force_model == FM_GUO;
    const bool forced = p.force_model == FM_GUO || p.force_model == FM_LUO || p.force_model == FM_SIMPLE;
    const Macro<27, R> m = conserved<27, R>(f, p, guo);   // Guo: equilibrium velocity shift F / (2 rho)
    const R rho = m.rho;
    const R ux = m.ux, uy = m.uy, uz = m.uz;
    R k[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) k[cube<27>(i)] = f[i];
    chimera_forward(k, uz, 1, 9, 3);
    chimera_forward(k, uy, 3, 9, 1);
    chimera_forward(k, ux, 9, 3, 1);
    const R bx[3] = {R(1), -ux, R(1.0 / 3.0) + ux * ux};
    const R by[3] = {R(1), -uy, R(1.0 / 3.0) + uy * uy};
    const R bz[3] = {R(1), -uz, R(1.0 / 3.0) + uz * uz};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) k[a * 9 + b * 3 + c] += bx[a] * by[b] * bz[c];
    // central moments of the force model's population term about the same velocity
    R g[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) g[i] = R(0);
    if (forced) {
        const R Fx = R(p.force[0]), Fy = R(p.force[1]), Fz = R(p.force[2]);
#pragma unroll
        for (int i = 0; i < 27; ++i) {
            const R cF = R(L::cx(i)) * Fx + R(L::cy(i)) * Fy + R(L::cz(i)) * Fz;
            const R cu = R(L::cx(i)) * ux + R(L::cy(i)) * uy + R(L::cz(i)) * uz;
            const R uF = ux * Fx + uy * Fy + uz * Fz;
            g[cube<27>(i)] = p.force_model == FM_SIMPLE ? R(L::w(i)) * R(3) * cF
                                                        : R(L::w(i)) * (R(3) * (cF - uF) + R(9) * cu * cF);
        }
        chimera_forward(g, uz, 1, 9, 3);
        chimera_forward(g, uy, 3, 9, 1);
        chimera_forward(g, ux, 9, 3, 1);
    }
#define K(a, b, c) k[(a) * 9 + (b) * 3 + (c)]
#define G(a, b, c) g[(a) * 9 + (b) * 3 + (c)]
    // post = pre + omega (eq - pre) + corr * force, corr = 1 - omega/2 for Guo
    auto relax = [&](int idx, R pre, R eq, R frc) -> R {
        const R w = R(p.rates[idx]);
        return pre + w * (eq - pre) + (guo ? R(1) - R(0.5) * w : R(1)) * frc;
    };
    const R third = R(1.0 / 3.0);
    // first order: conserved (rate 0); the force term alone changes them
    const R p100 = K(1, 0, 0) + G(1, 0, 0), p010 = K(0, 1, 0) + G(0, 1, 0), p001 = K(0, 0, 1) + G(0, 0, 1);
    // second order
    const R c110 = relax(4, K(1, 1, 0), R(0), G(1, 1, 0));
    const R c101 = relax(5, K(1, 0, 1), R(0), G(1, 0, 1));
    const R c011 = relax(6, K(0, 1, 1), R(0), G(0, 1, 1));
    const R D1 = relax(7, K(2, 0, 0) - K(0, 2, 0), R(0), G(2, 0, 0) - G(0, 2, 0));
    const R D2 = relax(8, K(2, 0, 0) - K(0, 0, 2), R(0), G(2, 0, 0) - G(0, 0, 2));
    const R Sb = relax(9, K(2, 0, 0) + K(0, 2, 0) + K(0, 0, 2), rho, G(2, 0, 0) + G(0, 2, 0) + G(0, 0, 2));
    const R c200 = (Sb + D1 + D2) * third, c020 = c200 - D1, c002 = c200 - D2;
    // third order: sums and differences, xyz
    const R s1 = relax(10, K(1, 2, 0) + K(1, 0, 2), R(0), G(1, 2, 0) + G(1, 0, 2));
    const R s2 = relax(11, K(2, 1, 0) + K(0, 1, 2), R(0), G(2, 1, 0) + G(0, 1, 2));
    const R s3 = relax(12, K(2, 0, 1) + K(0, 2, 1), R(0), G(2, 0, 1) + G(0, 2, 1));
    const R d1 = relax(13, K(1, 2, 0) - K(1, 0, 2), R(0), G(1, 2, 0) - G(1, 0, 2));
    const R d2 = relax(14, K(2, 1, 0) - K(0, 1, 2), R(0), G(2, 1, 0) - G(0, 1, 2));
    const R d3 = relax(15, K(2, 0, 1) - K(0, 2, 1), R(0), G(2, 0, 1) - G(0, 2, 1));
    const R c111 = relax(16, K(1, 1, 1), R(0), G(1, 1, 1));
    // fourth order
    const R q1 = relax(17, K(2, 2, 0) - R(2) * K(2, 0, 2) + K(0, 2, 2), R(0),
                       G(2, 2, 0) - R(2) * G(2, 0, 2) + G(0, 2, 2));
    const R q2 = relax(18, K(2, 2, 0) + K(2, 0, 2) - R(2) * K(0, 2, 2), R(0),
                       G(2, 2, 0) + G(2, 0, 2) - R(2) * G(0, 2, 2));
    const R q3 = relax(19, K(2, 2, 0) + K(2, 0, 2) + K(0, 2, 2), rho * third, G(2, 2, 0) + G(2, 0, 2) + G(0, 2, 2));
    const R c211 = relax(20, K(2, 1, 1), R(0), G(2, 1, 1));
    const R c121 = relax(21, K(1, 2, 1), R(0), G(1, 2, 1));
    const R c112 = relax(22, K(1, 1, 2), R(0), G(1, 1, 2));
    // fifth and sixth order
    const R c221 = relax(23, K(2, 2, 1), R(0), G(2, 2, 1));
    const R c212 = relax(24, K(2, 1, 2), R(0), G(2, 1, 2));
    const R c122 = relax(25, K(1, 2, 2), R(0), G(1, 2, 2));
    const R c222 = relax(26, K(2, 2, 2), rho * R(1.0 / 27.0), G(2, 2, 2));
    K(0, 0, 0) = rho;
    K(1, 0, 0) = p100; K(0, 1, 0) = p010; K(0, 0, 1) = p001;
    K(1, 1, 0) = c110; K(1, 0, 1) = c101; K(0, 1, 1) = c011;
    K(2, 0, 0) = c200; K(0, 2, 0) = c020; K(0, 0, 2) = c002;
    K(1, 2, 0) = R(0.5) * (s1 + d1); K(1, 0, 2) = R(0.5) * (s1 - d1);
    K(2, 1, 0) = R(0.5) * (s2 + d2); K(0, 1, 2) = R(0.5) * (s2 - d2);
    K(2, 0, 1) = R(0.5) * (s3 + d3); K(0, 2, 1) = R(0.5) * (s3 - d3);
    K(1, 1, 1) = c111;
    K(2, 2, 0) = (q3 + q1 + q2) * third; K(2, 0, 2) = (q3 - q1) * third; K(0, 2, 2) = (q3 - q2) * third;
    K(2, 1, 1) = c211; K(1, 2, 1) = c121; K(1, 1, 2) = c112;
    K(2, 2, 1) = c221; K(2, 1, 2) = c212; K(1, 2, 2) = c122;
    K(2, 2, 2) = c222;
#undef K
#undef G
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) k[a * 9 + b * 3 + c] -= bx[a] * by[b] * bz[c];
    chimera_backward(k, ux, 9, 3, 1);
    chimera_backward(k, uy, 3, 9, 1);
    chimera_backward(k, uz, 1, 9, 3);
#pragma unroll
    for (int i = 0; i < 27; ++i) f[i] = k[cube<27>(i)];
    return R(p.rates[4]);
}

// D3Q27 cumulant when every cumulant of third and higher order relaxes with rate 1 (lbmpy's
// default for a single relaxation rate, methods/creationfunctions.py:638-652): those post-collision
// cumulants are zero, so only second-order pre-collision moments are needed.  The post-collision
// central moments are formed directly as deviations from the central moments of the lattice-weight
// background, Delta = kappa* - B(u) (B separable: B0 = 1, B1 = -u, B2 = 1/3 + u^2); the inverse
// transform of Delta gives the zero-centred populations with no O(1/3) cancellation.
//
// CLOSURE: the shear rate comes from an eddy viscosity nu_t(Pi_xx, Pi_yy, Pi_zz, Pi_xy, Pi_xz,
// Pi_yz, rho, ux, uy, uz) evaluated on the same non-equilibrium stress the Smagorinsky branch uses
// (the learned closure, lbm_closure.cuh), as omega = 1 / (tau0 + 3 nu_t).
template <class R, bool CLOSURE = false, class NU = int>
__device__ __forceinline__ R collide_cum_ho1(R (&f)[27], const Physics& p, const NU& nu_t = NU()) {
    // raw moments of f~ (no shift) on the velocity cube: m[a*9 + b*3 + c]
    R m[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) m[cube<27>(i)] = f[i];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const int base = a * 9 + b * 3;   // z lines
            const R fm = m[base], f0 = m[base + 1], fp = m[base + 2];
            m[base] = fm + f0 + fp; m[base + 1] = fp - fm; m[base + 2] = fp + fm;
        }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int base = a * 9 + c;       // y lines
            const R fm = m[base], f0 = m[base + 3], fp = m[base + 6];
            m[base] = fm + f0 + fp; m[base + 3] = fp - fm; m[base + 6] = fp + fm;
        }
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int base = b * 3 + c;       // x lines
            const R fm = m[base], f0 = m[base + 9], fp = m[base + 18];
            m[base] = fm + f0 + fp; m[base + 9] = fp - fm; m[base + 18] = fp + fm;
        }
#define M_(a, b, c) m[(a) * 9 + (b) * 3 + (c)]
    const R drho = M_(0, 0, 0);
    const R rho = R(1) + drho, irho = R(1) / rho;
    const bool cm_force = p.force_model == FM_CENTRAL;
    R ux = M_(1, 0, 0) * irho, uy = M_(0, 1, 0) * irho, uz = M_(0, 0, 1) * irho;
    const R hx = R(0.5) * R(p.force[0]), hy = R(0.5) * R(p.force[1]), hz = R(0.5) * R(p.force[2]);
    if (cm_force) { ux += hx * irho; uy += hy * irho; uz += hz * irho; }
    const R uxx = ux * ux, uyy = uy * uy, uzz = uz * uz;
    // second-order central moments of the full PDFs minus rho/3 (diagonal) -- small numbers:
    // kappa_200 = m~200 - 2 ux m~100 + ux^2 m~000 + (1/3 + ux^2), and rho/3 = 1/3 + drho/3
    const R third = R(1.0 / 3.0);
    const R a0 = M_(2, 0, 0) - R(2) * ux * M_(1, 0, 0) + uxx * drho + uxx - drho * third;
    const R b0 = M_(0, 2, 0) - R(2) * uy * M_(0, 1, 0) + uyy * drho + uyy - drho * third;
    const R c0 = M_(0, 0, 2) - R(2) * uz * M_(0, 0, 1) + uzz * drho + uzz - drho * third;
    const R k110 = M_(1, 1, 0) - ux * M_(0, 1, 0) - uy * M_(1, 0, 0) + ux * uy * drho + ux * uy;
    const R k101 = M_(1, 0, 1) - ux * M_(0, 0, 1) - uz * M_(1, 0, 0) + ux * uz * drho + ux * uz;
    const R k011 = M_(0, 1, 1) - uy * M_(0, 0, 1) - uz * M_(0, 1, 0) + uy * uz * drho + uy * uz;
#undef M_
    R om_sgs = R(0);
    if (CLOSURE || p.sgs == 1) {
        // Pi_neq from the central moments: raw second moments minus their equilibrium values
        const R pxx = a0 - ux * R(p.force[0]) * R(cm_force ? 1 : 0);
        const R pyy = b0 - uy * R(p.force[1]) * R(cm_force ? 1 : 0);
        const R pzz = c0 - uz * R(p.force[2]) * R(cm_force ? 1 : 0);
        const R fxy = cm_force ? R(0.5) * (ux * R(p.force[1]) + uy * R(p.force[0])) : R(0);
        const R fxz = cm_force ? R(0.5) * (ux * R(p.force[2]) + uz * R(p.force[0])) : R(0);
        const R fyz = cm_force ? R(0.5) * (uy * R(p.force[2]) + uz * R(p.force[1])) : R(0);
        const R pxy = k110 - fxy, pxz = k101 - fxz, pyz = k011 - fyz;
        if constexpr (CLOSURE) {
            om_sgs = R(1) / (R(p.tau0) + R(3) * nu_t(pxx, pyy, pzz, pxy, pxz, pyz, rho, ux, uy, uz));
        } else {
            const R s2 = pxx * pxx + pyy * pyy + pzz * pzz + R(2) * (pxy * pxy + pxz * pxz + pyz * pyz);
            const R pi = sqrt(R(2) * s2) * irho;
            const R tau0 = R(p.tau0);
            om_sgs = R(2) / (tau0 + sqrt(R(p.sgs_c18) * pi + tau0 * tau0));
        }
    }
    auto rate = [&](int idx) -> R {
        R r = R(p.rates[idx]);
        if ((CLOSURE || p.sgs == 1) && ((p.sgs_mask >> idx) & 1u)) r = om_sgs;
        return r;
    };
    const R w_xy = rate(4), w_xz = rate(5), w_yz = rate(6), w_d1 = rate(7), w_d2 = rate(8), w_b = rate(9);
    R D1 = (a0 - b0) * (R(1) - w_d1);
    R D2 = (a0 - c0) * (R(1) - w_d2);
    R Sd = (a0 + b0 + c0) * (R(1) - w_b);   // (sum of diagonal second cumulants) - rho
    if (p.galilean) {
        const R o1 = R(p.rates[7]), o2 = R(p.rates[9]);
        const R h = R(0.5) * irho;
        // c_xx = rho/3 + a0: 2cxx - cyy - czz = 2a0 - b0 - c0; cxx + cyy + czz - rho = a0 + b0 + c0
        const R Dx = -o1 * h * (R(2) * a0 - b0 - c0) - o2 * h * (a0 + b0 + c0);
        const R Dy = Dx + R(3) * o1 * h * (a0 - b0);
        const R Dz = Dx + R(3) * o1 * h * (a0 - c0);
        const R g1 = R(-3) * rho * (R(1) - R(0.5) * o1);
        const R g2 = R(-3) * rho * (R(1) - R(0.5) * o2);
        D1 += g1 * (uxx * Dx - uyy * Dy);
        D2 += g1 * (uxx * Dx - uzz * Dz);
        Sd += g2 * (uxx * Dx + uyy * Dy + uzz * Dz);
    }
    const R a = (Sd + D1 + D2) * third;
    const R b = a - D1, c = a - D2;
    const R cxy = k110 * (R(1) - w_xy), cxz = k101 * (R(1) - w_xz), cyz = k011 * (R(1) - w_yz);

    // Delta = kappa* - B(u), kappa* built from the post-collision cumulants (orders >= 3 zero)
    R d[27];
#define D_(x, y, z) d[(x) * 9 + (y) * 3 + (z)]
    const R bx2 = third + uxx, by2 = third + uyy, bz2 = third + uzz;
    D_(0, 0, 0) = drho;
    D_(1, 0, 0) = ux + (cm_force ? hx : R(0));
    D_(0, 1, 0) = uy + (cm_force ? hy : R(0));
    D_(0, 0, 1) = uz + (cm_force ? hz : R(0));
    D_(2, 0, 0) = a + drho * third - uxx;
    D_(0, 2, 0) = b + drho * third - uyy;
    D_(0, 0, 2) = c + drho * third - uzz;
    D_(1, 1, 0) = cxy - ux * uy;
    D_(1, 0, 1) = cxz - ux * uz;
    D_(0, 1, 1) = cyz - uy * uz;
    // third order: kappa* = 0, Delta = -B
    D_(1, 1, 1) = ux * uy * uz;
    D_(2, 1, 0) = bx2 * uy; D_(2, 0, 1) = bx2 * uz;
    D_(1, 2, 0) = by2 * ux; D_(0, 2, 1) = by2 * uz;
    D_(1, 0, 2) = bz2 * ux; D_(0, 1, 2) = bz2 * uy;
    // fourth order
    const R t9 = R(1.0 / 9.0);
    D_(2, 2, 0) = drho * t9 + (a + b) * third + (a * b + R(2) * cxy * cxy) * irho - (uxx + uyy) * third - uxx * uyy;
    D_(2, 0, 2) = drho * t9 + (a + c) * third + (a * c + R(2) * cxz * cxz) * irho - (uxx + uzz) * third - uxx * uzz;
    D_(0, 2, 2) = drho * t9 + (b + c) * third + (b * c + R(2) * cyz * cyz) * irho - (uyy + uzz) * third - uyy * uzz;
    D_(2, 1, 1) = cyz * third + (a * cyz + R(2) * cxy * cxz) * irho - bx2 * uy * uz;
    D_(1, 2, 1) = cxz * third + (b * cxz + R(2) * cxy * cyz) * irho - by2 * ux * uz;
    D_(1, 1, 2) = cxy * third + (c * cxy + R(2) * cxz * cyz) * irho - bz2 * ux * uy;
    // fifth order: kappa* = 0
    D_(2, 2, 1) = bx2 * by2 * uz;
    D_(2, 1, 2) = bx2 * bz2 * uy;
    D_(1, 2, 2) = by2 * bz2 * ux;
    // sixth order
    {
        const R i2 = irho * irho;
        const R ss = cxy * cxy + cxz * cxz + cyz * cyz;
        D_(2, 2, 2) = drho * (R(1.0 / 27.0)) + (a + b + c) * t9 + (a * b + b * c + a * c) * third * irho +
                      a * b * c * i2 + R(2.0 / 3.0) * ss * irho +
                      R(2) * (a * cyz * cyz + b * cxz * cxz + c * cxy * cxy) * i2 + R(8) * cxy * cxz * cyz * i2 -
                      (uxx + uyy + uzz) * t9 - (uxx * uyy + uxx * uzz + uyy * uzz) * third - uxx * uyy * uzz;
    }
#undef D_
    chimera_backward(d, ux, 9, 3, 1);
    chimera_backward(d, uy, 3, 9, 1);
    chimera_backward(d, uz, 1, 9, 3);
#pragma unroll
    for (int i = 0; i < 27; ++i) f[i] = d[cube<27>(i)];
    return (CLOSURE || p.sgs == 1) ? om_sgs : R(p.rates[4]);
}

// ------------------------------------------------------------------ equilibria (setter)
// Zero-centred equilibrium populations of the method at (rho, u) (macroscopic_value_kernels.py:29-45).
template <int Q, class R, int MK>
__device__ __forceinline__ void equilibrium(R (&f)[Q], R rho, R ux, R uy, R uz, const Physics& p) {
    using L = Lat<Q>;
    const R drho = rho - R(1);
    if (MK == MK_CUM || MK == MK_CM) {
        // product form: kappa = rho * Gaussian moments (variance 1/3), shifted by u
        const R phx[3] = {R(0.5) * (R(1.0 / 3.0) + ux * ux - ux), R(2.0 / 3.0) - ux * ux,
                          R(0.5) * (R(1.0 / 3.0) + ux * ux + ux)};
        const R phy[3] = {R(0.5) * (R(1.0 / 3.0) + uy * uy - uy), R(2.0 / 3.0) - uy * uy,
                          R(0.5) * (R(1.0 / 3.0) + uy * uy + uy)};
        const R phz[3] = {R(0.5) * (R(1.0 / 3.0) + uz * uz - uz), R(2.0 / 3.0) - uz * uz,
                          R(0.5) * (R(1.0 / 3.0) + uz * uz + uz)};
#pragma unroll
        for (int i = 0; i < Q; ++i)
            f[i] = rho * phx[L::cx(i) + 1] * phy[L::cy(i) + 1] * phz[L::cz(i) + 1] - R(L::w(i));
        return;
    }
    const R rf = p.compressible ? rho : R(1);
    const R uu[6] = {ux * ux, uy * uy, uz * uz, ux * uy, ux * uz, uy * uz};
    if (MK == MK_MRT) {
        // f = M^-1 m_eq with the MRT basis (identical to the population form of the same equilibrium)
        R meq[Q];
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            R lin = 0, quad = 0;
            lin = cmad(lin, L::mlin(k, 0), ux);
            lin = cmad(lin, L::mlin(k, 1), uy);
            lin = cmad(lin, L::mlin(k, 2), uz);
#pragma unroll
            for (int a = 0; a < 6; ++a) quad = cmad(quad, L::mquad(k, a), uu[a]);
            meq[k] = cmad(rf * (lin + quad), L::p0(k), drho);
        }
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            R s = 0;
#pragma unroll
            for (int k = 0; k < Q; ++k) s = cmad(s, L::Minv(i, k), meq[k]);
            f[i] = s;
        }
        return;
    }
    const bool cont = p.continuous_eq != 0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        R lin = 0, quad = 0;
        lin = cmad(lin, L::eqlin(true, i, 0), ux);
        lin = cmad(lin, L::eqlin(true, i, 1), uy);
        lin = cmad(lin, L::eqlin(true, i, 2), uz);
#pragma unroll
        for (int a = 0; a < 6; ++a)
            quad = cont ? cmad(quad, L::eqquad(true, i, a), uu[a]) : cmad(quad, L::eqquad(false, i, a), uu[a]);
        f[i] = drho * R(L::w(i)) + rf * (lin + quad);
    }
}

}  // namespace lbm
