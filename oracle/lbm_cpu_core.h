/*
 * lbm_cpu_core.h -- per-cell collision cores of lbm_cpu.c (test infrastructure only).
 *
 * Included twice by lbm_cpu.c: with VT = real for single cells, and with VT = a GCC vector of
 * reals (one value per x-adjacent cell) for the straight-line row path, the way lbmpy's CPU
 * backend vectorises its generated kernels over x.  Scalars (rates, force, table entries) mix
 * freely with VT values; SPLAT(v) makes a VT from a scalar.
 */

/* D3Q19/D3Q27 TRT in population space (methods/momentbased/momentbasedmethod.py:389-398) with the
 * delta-form equilibrium f_eq_i - w_i drho = rf (lin_i . u + quad_i . uu). */
ALWAYS_INLINE void CORE(trt_core)(VT* f, const int Q, const FN(consts)* k, const int comp) {
    VT drho = SPLAT(0), jx = SPLAT(0), jy = SPLAT(0), jz = SPLAT(0);
#pragma GCC unroll 27
    for (int i = 0; i < Q; ++i) {
        drho += f[i];
        if (DX[i] == 1) jx += f[i]; else if (DX[i] == -1) jx -= f[i];
        if (DY[i] == 1) jy += f[i]; else if (DY[i] == -1) jy -= f[i];
        if (DZ[i] == 1) jz += f[i]; else if (DZ[i] == -1) jz -= f[i];
    }
    const VT rho = (real)1 + drho;
    const VT rf = comp ? rho : SPLAT(1);
    const VT ir = (real)1 / rf;
    const VT ux = jx * ir, uy = jy * ir, uz = jz * ir;
    const VT uu[6] = {ux * ux, uy * uy, uz * uz, ux * uy, ux * uz, uy * uz};
    const real we = k->we, wo = k->wo;
#pragma GCC unroll 27
    for (int i = 0; i < Q; ++i) {
        const int j = INV[i];
        if (j < i) continue;
        VT quad = SPLAT(0);
#pragma GCC unroll 6
        for (int a = 0; a < 6; ++a) quad += k->quad[i][a] * uu[a];
        const VT feq_e = drho * k->w[i] + rf * quad;
        if (j == i) {
            f[i] += we * (feq_e - f[i]);
            continue;
        }
        const VT feq_o = rf * (k->lin[i][0] * ux + k->lin[i][1] * uy + k->lin[i][2] * uz);
        const VT fe = (real)0.5 * (f[i] + f[j]), fo = (real)0.5 * (f[i] - f[j]);
        const VT de = we * (feq_e - fe), dod = wo * (feq_o - fo);
        f[i] += de + dod;
        f[j] += de - dod;
    }
}

/* One line of the inverse chimera transform: central moments (k0, k1, k2) about u of the
 * populations (f-, f0, f+) on a velocity line -> those populations. */
ALWAYS_INLINE void CORE(line_back)(VT* g, int s, VT u) {
    const VT k0 = g[0], k1 = g[s], k2 = g[2 * s];
    const VT m1 = k1 + u * k0, m2 = k2 + (real)2 * u * k1 + u * u * k0;
    g[0] = (real)0.5 * (m2 - m1);
    g[s] = k0 - m2;
    g[2 * s] = (real)0.5 * (m2 + m1);
}

/* D3Q27 cumulant, orders >= 3 relaxed by 1 (methods/cumulantbased/cumulantbasedmethod.py:296-402),
 * symmetric CentralMoment forcing (forcemodels.py:213-233), optional Galilean correction. */
ALWAYS_INLINE void CORE(cum_core)(VT* f, const FN(consts)* kc, const int gal) {
    VT m[27];
#pragma GCC unroll 27
    for (int i = 0; i < 27; ++i) m[(DX[i] + 1) * 9 + (DY[i] + 1) * 3 + (DZ[i] + 1)] = f[i];
    /* raw moments of the zero-centred populations: per line (f-, f0, f+) -> (sum, f+ - f-, f+ + f-) */
#pragma GCC unroll 9
    for (int a = 0; a < 9; ++a) {              /* z lines */
        VT* g = m + 3 * a;
        const VT fm = g[0], f0 = g[1], fp = g[2];
        g[0] = fm + f0 + fp; g[1] = fp - fm; g[2] = fp + fm;
    }
#pragma GCC unroll 9
    for (int a = 0; a < 9; ++a) {              /* y lines */
        VT* g = m + 9 * (a / 3) + (a % 3);
        const VT fm = g[0], f0 = g[3], fp = g[6];
        g[0] = fm + f0 + fp; g[3] = fp - fm; g[6] = fp + fm;
    }
#pragma GCC unroll 9
    for (int a = 0; a < 9; ++a) {              /* x lines */
        VT* g = m + a;
        const VT fm = g[0], f0 = g[9], fp = g[18];
        g[0] = fm + f0 + fp; g[9] = fp - fm; g[18] = fp + fm;
    }
#define MM(x, y, z) m[(x) * 9 + (y) * 3 + (z)]
    const VT drho = MM(0, 0, 0), rho = (real)1 + drho, irho = (real)1 / rho;
    const real Fx = kc->F[0], Fy = kc->F[1], Fz = kc->F[2];
    /* velocity with the half-force shift of the CentralMoment model */
    const VT ux = (MM(1, 0, 0) + (real)0.5 * Fx) * irho;
    const VT uy = (MM(0, 1, 0) + (real)0.5 * Fy) * irho;
    const VT uz = (MM(0, 0, 1) + (real)0.5 * Fz) * irho;
    const real third = (real)1 / (real)3;
    /* second-order central moments of the full populations about u (the background w_i adds
     * 1/3 + u^2 on the diagonal and u_a u_b off it) */
    const VT kxx = MM(2, 0, 0) - (real)2 * ux * MM(1, 0, 0) + rho * ux * ux + third;
    const VT kyy = MM(0, 2, 0) - (real)2 * uy * MM(0, 1, 0) + rho * uy * uy + third;
    const VT kzz = MM(0, 0, 2) - (real)2 * uz * MM(0, 0, 1) + rho * uz * uz + third;
    const VT kxy = MM(1, 1, 0) - ux * MM(0, 1, 0) - uy * MM(1, 0, 0) + rho * ux * uy;
    const VT kxz = MM(1, 0, 1) - ux * MM(0, 0, 1) - uz * MM(1, 0, 0) + rho * ux * uz;
    const VT kyz = MM(0, 1, 1) - uy * MM(0, 0, 1) - uz * MM(0, 1, 0) + rho * uy * uz;
#undef MM
    /* relaxation of the second-order polynomial cumulants: shear (x^2-y^2, x^2-z^2, off-diagonal)
     * with omega, bulk (x^2+y^2+z^2, equilibrium rho) with omega_b */
    const real w1 = kc->we, w2 = kc->wo;
    VT dxy2 = (kxx - kyy) * ((real)1 - w1);
    VT dxz2 = (kxx - kzz) * ((real)1 - w1);
    VT sum = kxx + kyy + kzz + w2 * (rho - (kxx + kyy + kzz));
    if (gal) {
        /* velocity-gradient estimates from the non-equilibrium second moments and the correction
         * of the diagonal cumulants (Geier et al. 2015, eq. 58-63) */
        const VT h = (real)0.5 * irho;
        const VT gx = -w1 * h * ((real)2 * kxx - kyy - kzz) - w2 * h * (kxx + kyy + kzz - rho);
        const VT gy = gx + (real)3 * w1 * h * (kxx - kyy);
        const VT gz = gx + (real)3 * w1 * h * (kxx - kzz);
        const VT s1 = (real)-3 * rho * ((real)1 - (real)0.5 * w1);
        const VT s2 = (real)-3 * rho * ((real)1 - (real)0.5 * w2);
        dxy2 += s1 * (ux * ux * gx - uy * uy * gy);
        dxz2 += s1 * (ux * ux * gx - uz * uz * gz);
        sum += s2 * (ux * ux * gx + uy * uy * gy + uz * uz * gz);
    }
    const VT cxx = (sum + dxy2 + dxz2) * third;
    const VT cyy = cxx - dxy2, czz = cxx - dxz2;
    const VT cxy = kxy * ((real)1 - w1), cxz = kxz * ((real)1 - w1), cyz = kyz * ((real)1 - w1);
    /* post-collision central moments: cumulants of order >= 3 are zero */
    VT k[27];
#pragma GCC unroll 27
    for (int i = 0; i < 27; ++i) k[i] = SPLAT(0);
#define KK(x, y, z) k[(x) * 9 + (y) * 3 + (z)]
    KK(0, 0, 0) = rho;
    KK(2, 0, 0) = cxx; KK(0, 2, 0) = cyy; KK(0, 0, 2) = czz;
    KK(1, 1, 0) = cxy; KK(1, 0, 1) = cxz; KK(0, 1, 1) = cyz;
    KK(2, 2, 0) = (cxx * cyy + (real)2 * cxy * cxy) * irho;
    KK(2, 0, 2) = (cxx * czz + (real)2 * cxz * cxz) * irho;
    KK(0, 2, 2) = (cyy * czz + (real)2 * cyz * cyz) * irho;
    KK(2, 1, 1) = (cxx * cyz + (real)2 * cxy * cxz) * irho;
    KK(1, 2, 1) = (cyy * cxz + (real)2 * cxy * cyz) * irho;
    KK(1, 1, 2) = (czz * cxy + (real)2 * cxz * cyz) * irho;
    KK(2, 2, 2) = (cxx * cyy * czz + (real)2 * (cxx * cyz * cyz + cyy * cxz * cxz + czz * cxy * cxy) +
                   (real)8 * cxy * cxz * cyz) * irho * irho;
    /* symmetric forcing, second half */
    KK(1, 0, 0) = SPLAT((real)0.5 * Fx); KK(0, 1, 0) = SPLAT((real)0.5 * Fy); KK(0, 0, 1) = SPLAT((real)0.5 * Fz);
#undef KK
#pragma GCC unroll 9
    for (int a = 0; a < 9; ++a) CORE(line_back)(k + a, 9, ux);                      /* x */
#pragma GCC unroll 9
    for (int a = 0; a < 9; ++a) CORE(line_back)(k + 9 * (a / 3) + (a % 3), 3, uy);  /* y */
#pragma GCC unroll 9
    for (int a = 0; a < 9; ++a) CORE(line_back)(k + 3 * a, 1, uz);                  /* z */
#pragma GCC unroll 27
    for (int i = 0; i < 27; ++i) f[i] = k[(DX[i] + 1) * 9 + (DY[i] + 1) * 3 + (DZ[i] + 1)] - kc->w[i];
}
