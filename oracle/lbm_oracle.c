/*
 * lbm_oracle.c -- CPU oracle for the lbmpy stream-collide sweep.  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py load this library,
 * always as the checker.  The product (lbmpy_b200) never links or calls it.
 *
 * It restates, in plain C99 + OpenMP and in FP64, the arithmetic of lbmpy's generated sweep
 * (paths relative to src/lbmpy of mabau/lbmpy):
 *   - conserved quantities ..... methods/conservedquantitycomputation.py:218-249, 274-374
 *   - moment-space collision ... methods/momentbased/momentbasedmethod.py:320-416
 *                                (f* = M^-1 [m + D(m_eq - m) + forcing], SRT/TRT/MRT)
 *   - continuous equilibrium ... equilibrium/continuous_hydro_maxwellian.py:82-116, 192-235
 *   - force models ............. forcemodels.py:179-317 (Simple, Luo, Guo), :213-233 (CentralMoment)
 *   - cumulant collision ....... methods/cumulantbased/cumulantbasedmethod.py:296-402 with the
 *                                generating-function transform moment_transforms/cumulanttransforms.py:46-220
 *   - Galilean correction ...... methods/cumulantbased/galilean_correction.py:56-91
 *   - Smagorinsky .............. turbulence_models.py:25-84
 *   - PDF accessors ............ fieldaccess.py:66-181 (pull, push, AA, EsoTwist)
 *   - NoSlip / UBB ............. boundaries/boundaryconditions.py:128-139, 794-841 applied as
 *                                link kernels between steps (boundaries/boundaryhandling.py:15-199,
 *                                advanced_streaming/indexing.py:12-183)
 *   - periodicity .............. ghost-layer copies (advanced_streaming/communication.py:21-183)
 *   - getter / setter .......... macroscopic_value_kernels.py:14-61
 * The layout is lbmpy's: one ghost layer per active dimension, arbitrary element strides
 * (fzyx = x fastest, PDF index slowest, is the default).  Parity status: see oracle_spec.py.
 */
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define QMAX 27
#define TMAX 40
#define MLP_NIN 10
#define MLP_NH 32
#define MLP_NPARAM (MLP_NIN * MLP_NH + MLP_NH + MLP_NH * MLP_NH + MLP_NH + MLP_NH + 1 + 1)

typedef struct {
    int D, Q;
    int c[QMAX][3];
    int inv[QMAX];
    double w[QMAX];
    int kind;                 /* 0: moment based (SRT/TRT/MRT), 1: cumulant (D3Q27) */
    int compressible, zero_centered, delta_eq, eq_order;
    int nterms[QMAX];         /* moment (or polynomial cumulant) k = sum_t coef * x^a y^b z^c */
    int texp[QMAX][TMAX][3];
    double tcoef[QMAX][TMAX];
    double M[QMAX][QMAX];     /* moment-based: M[k][i]; cumulant: mono->poly matrix A[k][mono] */
    double Minv[QMAX][QMAX];
    double rate[QMAX];
    int force_model;          /* 0 none, 1 Guo, 2 CentralMoment, 3 Simple, 4 Luo */
    double F[3];
    int galilean;
    int sgs;                  /* 0 none, 1 Smagorinsky, 2 learned eddy viscosity (MLP) */
    double sgs_c;
    double shear_rate;
    float mlp[MLP_NPARAM];    /* sgs == 2: W1[10][32] b1[32] W2[32][32] b2[32] W3[32] b3 scale */
    int discrete_eq;          /* moment based: 1 = discrete Maxwellian (maxwellian_equilibrium.py:64-104,
                                 equilibrium/discrete_hydro_maxwellian.py:9-96), 0 = continuous */
    int ubb_adapt;            /* UBB: wall velocity shifted by -F / (2 rho_ref) (boundaryconditions.py:790-794) */
    double ubb_density;       /* UBB: prescribed wall density (compressible), 0: the fluid cell's (:824-830) */
    const double* ubb_link;   /* UBB: per-link velocities [cell][q][3] (interior cells, x fastest), or NULL */
    double fd_rho1;           /* density of FixedDensity cells of flag 7 (a second density) */
    const int* link_code;     /* flags 8-10: per-link source, dir | (ox+1)<<8 | (oy+1)<<10 | (oz+1)<<12,
                                 [cell][q] (interior cells, x fastest; q the link direction) */
    double* link_value;       /* flags 10, 11: per-link values [cell][q][2] (outflow state, Bouzidi q) */
    double foc_limiter;       /* > 0: fourth-order cumulant correction with this limiter */
} om_method;

typedef struct {
    int n[3];                 /* interior cells per dimension (n[2] = 1 in 2-D) */
    int g[3];                 /* ghost layers per dimension (g[2] = 0 in 2-D) */
    int64_t s[4];             /* element strides of x, y, z, q */
} om_grid;

enum { P_PULL = 0, P_PUSH = 1, P_AA = 2, P_ESOTWIST = 3, P_ESOPULL = 4, P_ESOPUSH = 5 };

/* Whether direction c sits at an even position of lbmpy's 'lehmann' ordering (stencils.py,
 * D2Q9 / D3Q19 / D3Q27 'lehmann'; used by fieldaccess.py:184-318 through _get_lehmann_stencil,
 * :371-388).  That ordering lists each direction right before its inverse, so the even ones are
 * the second of each pair; the rest population is at position 0. */
static int lehmann_even(const int c[3]) {
    static const int even[13][3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {-1, -1, 0}, {-1, 0, -1},
                                    {0, -1, -1}, {-1, 1, 0}, {-1, 0, 1}, {0, -1, 1}, {-1, -1, -1},
                                    {-1, -1, 1}, {-1, 1, -1}, {1, -1, -1}};
    int k;
    if (c[0] == 0 && c[1] == 0 && c[2] == 0) return 1;
    for (k = 0; k < 13; ++k)
        if (c[0] == even[k][0] && c[1] == even[k][1] && c[2] == even[k][2]) return 1;
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
static double ipow(double b, int e) { double r = 1.0; while (e-- > 0) r *= b; return r; }

/* Accessor table: offset and slot of the read (rw=0) or write (rw=1) of direction i.
 * fieldaccess.py:66-318.  parity 0 = EVEN, 1 = ODD (two-field patterns ignore it). */
static void accessor(const om_method* m, int pattern, int parity, int rw, int i, int off[3], int* slot) {
    const int* c = m->c[i];
    int d;
    switch (pattern) {
    case P_PULL:
        for (d = 0; d < 3; ++d) off[d] = rw == 0 ? -c[d] : 0;
        *slot = i; return;
    case P_PUSH:
        for (d = 0; d < 3; ++d) off[d] = rw == 0 ? 0 : c[d];
        *slot = i; return;
    case P_AA:
        if (parity == 0) { for (d = 0; d < 3; ++d) off[d] = 0; *slot = rw == 0 ? i : m->inv[i]; }
        else {
            for (d = 0; d < 3; ++d) off[d] = rw == 0 ? -c[d] : c[d];
            *slot = rw == 0 ? m->inv[i] : i;
        }
        return;
    case P_ESOTWIST:
        for (d = 0; d < 3; ++d) off[d] = rw == 0 ? (c[d] < 0 ? -c[d] : 0) : (c[d] > 0 ? c[d] : 0);
        if (parity == 0) *slot = rw == 0 ? i : m->inv[i];
        else *slot = rw == 0 ? m->inv[i] : i;
        return;
    case P_ESOPULL: {     /* fieldaccess.py:184-232: even-position directions stream on read */
        const int e = lehmann_even(c);
        for (d = 0; d < 3; ++d) off[d] = rw == 0 ? (e ? -c[d] : 0) : (e ? 0 : c[d]);
        if (parity == 0) *slot = rw == 0 ? i : m->inv[i];
        else *slot = rw == 0 ? m->inv[i] : i;
        return;
    }
    case P_ESOPUSH: {     /* fieldaccess.py:235-318: odd-position directions stream on read */
        const int e = lehmann_even(c);
        for (d = 0; d < 3; ++d) off[d] = rw == 0 ? (e ? 0 : -c[d]) : (e ? c[d] : 0);
        if (parity == 0) *slot = rw == 0 ? m->inv[i] : i;
        else *slot = rw == 0 ? i : m->inv[i];
        return;
    }
    }
}

static inline int64_t gidx(const om_grid* gr, int x, int y, int z) {
    return (int64_t)(x + gr->g[0]) * gr->s[0] + (int64_t)(y + gr->g[1]) * gr->s[1] +
           (int64_t)(z + gr->g[2]) * gr->s[2];
}

static inline int64_t fidx(const om_grid* gr, int x, int y, int z) {   /* flag arrays: no q */
    int ex = gr->n[0] + 2 * gr->g[0], ey = gr->n[1] + 2 * gr->g[1];
    return (int64_t)(x + gr->g[0]) + (int64_t)ex * ((y + gr->g[1]) + (int64_t)ey * (z + gr->g[2]));
}

/* ------------------------------ equilibrium moments -------------------------------------- */
/* 1-D Maxwellian moment <(u + cs Z)^n> as polynomial in u: coef[k] multiplies u^k. */
static void gauss1d(int n, double cs2, double coef[8]) {
    int k;
    for (k = 0; k < 8; ++k) coef[k] = 0.0;
    for (k = 0; k <= n; k += 2) {           /* k = power of the fluctuation */
        double binom = 1.0, df = 1.0; int j;
        for (j = 0; j < k; ++j) binom = binom * (n - j) / (j + 1);
        for (j = k - 1; j > 0; j -= 2) df *= j;
        coef[n - k] += binom * df * ipow(cs2, k / 2);
    }
}

/* Raw moment of the unit-density continuous Maxwellian, truncated to total order `order`
 * in u (order < 0: no truncation).  equilibrium/continuous_hydro_maxwellian.py:192-235. */
static double maxwell_raw(const int e[3], const double u[3], int order, double cs2) {
    double g[3][8]; int d, a, b, cc; double r = 0.0;
    for (d = 0; d < 3; ++d) gauss1d(e[d], cs2, g[d]);
    for (a = 0; a <= e[0]; ++a)
        for (b = 0; b <= e[1]; ++b)
            for (cc = 0; cc <= e[2]; ++cc) {
                if (order >= 0 && a + b + cc > order) continue;
                r += g[0][a] * g[1][b] * g[2][cc] * ipow(u[0], a) * ipow(u[1], b) * ipow(u[2], cc);
            }
    return r;
}

/* Equilibrium value of polynomial moment k in the method's storage convention. */
static double eq_moment(const om_method* m, int k, double rho, double drho, const double u[3]) {
    double pu = 0.0, p0 = 0.0, zero[3] = {0, 0, 0}, base; int t;
    if (m->discrete_eq && m->kind == 0) {
        /* moment k of the discrete populations w_i rho (1 + c.u/cs2 + (c.u)^2/(2 cs4) - u.u/(2 cs2))
         * (compressible) or w_i rho + w_i (...) (incompressible), minus w_i in delta form */
        double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2], r = 0.0; int i;
        for (i = 0; i < m->Q; ++i) {
            double cu = m->c[i][0] * u[0] + m->c[i][1] * u[1] + m->c[i][2] * u[2];
            double poly = 3.0 * cu + 4.5 * cu * cu - 1.5 * uu, fe;
            fe = m->compressible ? m->w[i] * rho * (1.0 + poly) : m->w[i] * (rho + poly);
            if (m->delta_eq) fe -= m->w[i];
            r += m->M[k][i] * fe;
        }
        return r;
    }
    for (t = 0; t < m->nterms[k]; ++t) {
        pu += m->tcoef[k][t] * maxwell_raw(m->texp[k][t], u, m->eq_order, 1.0 / 3.0);
        p0 += m->tcoef[k][t] * maxwell_raw(m->texp[k][t], zero, m->eq_order, 1.0 / 3.0);
    }
    base = m->compressible ? rho * pu : pu + drho * p0;   /* psi(rho,u) or psi(1,u)+psi(drho,0) */
    if (m->delta_eq) base -= p0;                            /* subtract psi(1, 0) */
    return base;
}

/* --------------------------------- conserved quantities ----------------------------------- */
static void conserved(const om_method* m, const double* f, double* rho, double* drho,
                      double* rho_ref, double u[3]) {
    double s = 0.0, j[3] = {0, 0, 0}; int i, d;
    for (i = 0; i < m->Q; ++i) {
        s += f[i];
        for (d = 0; d < 3; ++d) j[d] += m->c[i][d] * f[i];
    }
    if (m->zero_centered) { *drho = s; *rho = 1.0 + s; } else { *rho = s; *drho = s - 1.0; }
    *rho_ref = m->compressible ? *rho : 1.0;
    for (d = 0; d < 3; ++d) u[d] = j[d] / *rho_ref;
}

/* Population force vectors, forcemodels.py:179-211 (Simple), :235-271 (Luo). */
static void luo_terms(const om_method* m, const double u[3], double* out) {
    int i, d;
    for (i = 0; i < m->Q; ++i) {
        double cu = 0.0, cf = 0.0, t = 0.0;
        for (d = 0; d < 3; ++d) { cu += m->c[i][d] * u[d]; cf += m->c[i][d] * m->F[d]; }
        for (d = 0; d < 3; ++d) t += m->F[d] * ((m->c[i][d] - u[d]) * 3.0 + m->c[i][d] * cu * 9.0);
        out[i] = m->w[i] * t;
    }
}

/* -------------------------------- moment-based collision --------------------------------- */
static void collide_moment(const om_method* m, const double* f, double* fo, double* omega_out) {
    int Q = m->Q, i, k, d;
    double rho, drho, rho_ref, u[3], mom[QMAX], meq[QMAX], ms[QMAX], rates[QMAX], bg[QMAX];
    conserved(m, f, &rho, &drho, &rho_ref, u);
    if (m->force_model == 1 || m->force_model == 2)
        for (d = 0; d < 3; ++d) u[d] += m->F[d] / (2.0 * rho_ref);
    for (k = 0; k < Q; ++k) {
        double s = 0.0;
        for (i = 0; i < Q; ++i) s += m->M[k][i] * f[i];
        mom[k] = s;
        meq[k] = eq_moment(m, k, rho, drho, u);
        rates[k] = m->rate[k];
        bg[k] = 0.0;
    }
    if (m->zero_centered && !m->delta_eq) {     /* background shift (raw moment space) */
        for (k = 0; k < Q; ++k) {
            double s = 0.0;
            for (i = 0; i < Q; ++i) s += m->M[k][i] * m->w[i];
            bg[k] = s;
            mom[k] += s;
        }
    }
    if (m->sgs == 1) {                          /* turbulence_models.py:25-84 */
        double feq[QMAX], pi[3][3] = {{0}}, pn = 0.0, tau0, om;
        int a, b;
        for (i = 0; i < Q; ++i) {
            double s = 0.0;
            for (k = 0; k < Q; ++k) s += m->Minv[i][k] * (meq[k] - bg[k]);
            feq[i] = s;
        }
        for (i = 0; i < Q; ++i)
            for (a = 0; a < 3; ++a)
                for (b = 0; b < 3; ++b) pi[a][b] += m->c[i][a] * m->c[i][b] * (f[i] - feq[i]);
        for (a = 0; a < m->D; ++a)
            for (b = 0; b < m->D; ++b) pn += pi[a][b] * pi[a][b];
        pn = sqrt(2.0 * pn) / rho_ref;
        tau0 = 1.0 / m->shear_rate;
        om = 2.0 / (tau0 + sqrt(18.0 * m->sgs_c * m->sgs_c * pn + tau0 * tau0));
        for (k = 0; k < Q; ++k) if (m->rate[k] == m->shear_rate) rates[k] = om;
        if (omega_out) *omega_out = om;
    }
    for (k = 0; k < Q; ++k) ms[k] = mom[k] + rates[k] * (meq[k] - mom[k]);
    if (m->force_model == 1 || m->force_model == 3 || m->force_model == 4) {
        double pf[QMAX];
        if (m->force_model == 3) {
            for (i = 0; i < Q; ++i) {
                double cf = 0.0;
                for (d = 0; d < 3; ++d) cf += m->c[i][d] * m->F[d];
                pf[i] = m->w[i] * 3.0 * cf;
            }
        } else {
            luo_terms(m, u, pf);
        }
        for (k = 0; k < Q; ++k) {
            double s = 0.0;
            for (i = 0; i < Q; ++i) s += m->M[k][i] * pf[i];
            if (m->force_model == 1) s *= (1.0 - 0.5 * rates[k]);   /* Guo: (I - D/2) M Luo */
            ms[k] += s;
        }
    }
    for (k = 0; k < Q; ++k) ms[k] -= bg[k];
    for (i = 0; i < Q; ++i) {
        double s = 0.0;
        for (k = 0; k < Q; ++k) s += m->Minv[i][k] * ms[k];
        fo[i] = s;
    }
}

/* ------------------------------------ cumulant collision --------------------------------- */
/* Monomials (a,b,c), a,b,c in {0,1,2}, are indexed a*9 + b*3 + c. */
static int binom_small(int n, int k) { return (k < 0 || k > n) ? 0 : (n == 2 && k == 1) ? 2 : 1; }

/* Cumulants of a distribution from its normalised moments mm (mm[0] = 1):
 * multivariate moment-cumulant recursion, the derivative form of C = ln K. */
static void cumulants_from_moments(const double* mm, double* cc) {
    int order, a, b, c;
    cc[0] = 0.0;
    for (order = 1; order <= 6; ++order)
        for (a = 0; a <= 2; ++a) for (b = 0; b <= 2; ++b) for (c = 0; c <= 2; ++c) {
            int n[3] = {a, b, c}, j, np[3], k0, k1, k2; double s;
            if (a + b + c != order) continue;
            j = a > 0 ? 0 : (b > 0 ? 1 : 2);
            np[0] = a; np[1] = b; np[2] = c; np[j] -= 1;
            s = mm[a * 9 + b * 3 + c];
            for (k0 = 0; k0 <= np[0]; ++k0) for (k1 = 0; k1 <= np[1]; ++k1) for (k2 = 0; k2 <= np[2]; ++k2) {
                int kk[3] = {k0, k1, k2}, e[3];
                double coef;
                if (k0 == np[0] && k1 == np[1] && k2 == np[2]) continue;
                coef = binom_small(np[0], k0) * binom_small(np[1], k1) * binom_small(np[2], k2);
                e[0] = kk[0]; e[1] = kk[1]; e[2] = kk[2]; e[j] += 1;
                s -= coef * cc[e[0] * 9 + e[1] * 3 + e[2]] * mm[(np[0] - k0) * 9 + (np[1] - k1) * 3 + (np[2] - k2)];
            }
            (void)n;
            cc[a * 9 + b * 3 + c] = s;
        }
}

static void moments_from_cumulants(const double* cc, double* mm) {
    int order, a, b, c;
    mm[0] = 1.0;
    for (order = 1; order <= 6; ++order)
        for (a = 0; a <= 2; ++a) for (b = 0; b <= 2; ++b) for (c = 0; c <= 2; ++c) {
            int j, np[3], k0, k1, k2; double s = 0.0;
            if (a + b + c != order) continue;
            j = a > 0 ? 0 : (b > 0 ? 1 : 2);
            np[0] = a; np[1] = b; np[2] = c; np[j] -= 1;
            for (k0 = 0; k0 <= np[0]; ++k0) for (k1 = 0; k1 <= np[1]; ++k1) for (k2 = 0; k2 <= np[2]; ++k2) {
                int e[3] = {k0, k1, k2};
                double coef = binom_small(np[0], k0) * binom_small(np[1], k1) * binom_small(np[2], k2);
                e[j] += 1;
                s += coef * cc[e[0] * 9 + e[1] * 3 + e[2]] * mm[(np[0] - k0) * 9 + (np[1] - k1) * 3 + (np[2] - k2)];
            }
            mm[a * 9 + b * 3 + c] = s;
        }
}

/* Central moments (about u) of the lattice distribution g over the D3Q27 velocities. */
static void central_moments(const om_method* m, const double* g, const double u[3], double* km) {
    int a, b, c, i;
    for (a = 0; a <= 2; ++a) for (b = 0; b <= 2; ++b) for (c = 0; c <= 2; ++c) {
        double s = 0.0;
        for (i = 0; i < m->Q; ++i)
            s += g[i] * ipow(m->c[i][0] - u[0], a) * ipow(m->c[i][1] - u[1], b) * ipow(m->c[i][2] - u[2], c);
        km[a * 9 + b * 3 + c] = s;
    }
}

/* Populations from central moments about u: per-axis inverse of the 3-velocity moment map. */
static void populations_from_central(const om_method* m, const double* km, const double u[3], double* f) {
    double t[27], t2[27]; int a, b, c, i, v;
    /* work array t[(a|vx) * 9 + (b|vy) * 3 + (c|vz)]: transform axis by axis, x first. */
    memcpy(t, km, sizeof(t));
    for (int axis = 0; axis < 3; ++axis) {
        double uu = u[axis];
        for (a = 0; a < 3; ++a) for (b = 0; b < 3; ++b) {
            int idx[3], base, st;
            double k0, k1, k2, m0, m1, m2;
            if (axis == 0) { base = a * 3 + b; st = 9; }
            else if (axis == 1) { base = a * 9 + b; st = 3; }
            else { base = a * 9 + b * 3; st = 1; }
            (void)idx;
            k0 = t[base]; k1 = t[base + st]; k2 = t[base + 2 * st];
            m0 = k0; m1 = k1 + uu * k0; m2 = k2 + 2.0 * uu * k1 + uu * uu * k0;
            /* slots 0,1,2 of the axis now hold velocities -1, 0, +1 */
            t2[base] = 0.5 * (m2 - m1);
            t2[base + st] = m0 - m2;
            t2[base + 2 * st] = 0.5 * (m2 + m1);
        }
        memcpy(t, t2, sizeof(t));
    }
    for (i = 0; i < m->Q; ++i) {
        int idx = (m->c[i][0] + 1) * 9 + (m->c[i][1] + 1) * 3 + (m->c[i][2] + 1);
        f[i] = t[idx];
    }
    (void)c; (void)v;
}

/* Learned eddy viscosity: features of the pre-collision non-equilibrium stress P (3x3), density
 * and velocity, then a 10-32-32-1 perceptron (SiLU hidden units, softplus output times a fixed
 * scale), evaluated in FP64 with the FP32 parameters.  nu_t enters as omega = 1/(tau0 + 3 nu_t),
 * on the moments whose rate is the shear rate, as the Smagorinsky model does
 * (turbulence_models.py:25-84). */
static void mlp_features(const double P[3][3], double rho, const double u[3], double x[MLP_NIN]) {
    double s2 = 0.0, off2, tr, d[3][3], d2 = 0.0, dn, tr3 = 0.0, u2, uau = 0.0, mx = 0.0, pim;
    int a, b, c;
    for (a = 0; a < 3; ++a) for (b = 0; b < 3; ++b) s2 += P[a][b] * P[a][b];
    off2 = P[0][1] * P[0][1] + P[0][2] * P[0][2] + P[1][2] * P[1][2];
    tr = P[0][0] + P[1][1] + P[2][2];
    for (a = 0; a < 3; ++a) for (b = 0; b < 3; ++b) d[a][b] = P[a][b] - (a == b ? tr / 3.0 : 0.0);
    for (a = 0; a < 3; ++a) for (b = 0; b < 3; ++b) d2 += d[a][b] * d[a][b];
    dn = sqrt(d2);
    for (a = 0; a < 3; ++a) for (b = 0; b < 3; ++b) for (c = 0; c < 3; ++c) tr3 += d[a][b] * d[b][c] * d[c][a];
    u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    for (a = 0; a < 3; ++a) for (b = 0; b < 3; ++b) uau += u[a] * d[a][b] * u[b];
    for (a = 0; a < 3; ++a) if (fabs(d[a][a]) > mx) mx = fabs(d[a][a]);
    pim = sqrt(2.0 * s2) / rho;
    x[0] = log(pim + 1e-9);
    x[1] = 100.0 * pim;
    x[2] = tr / (sqrt(s2) + 1e-12);
    x[3] = sqrt(6.0) * tr3 / (d2 * dn + 1e-30);
    x[4] = 30.0 * sqrt(u2);
    x[5] = 1000.0 * (rho - 1.0);
    x[6] = uau / ((u2 + 1e-12) * dn + 1e-30);
    x[7] = off2 / (s2 + 1e-30);
    x[8] = mx / (dn + 1e-30);
    x[9] = 1000.0 * u2;
}

static double silu(double z) { return z / (1.0 + exp(-z)); }

double om_mlp_nu_t(const float* w, const double x[MLP_NIN]) {
    const float* W1 = w;
    const float* b1 = W1 + MLP_NIN * MLP_NH;
    const float* W2 = b1 + MLP_NH;
    const float* b2 = W2 + MLP_NH * MLP_NH;
    const float* W3 = b2 + MLP_NH;
    const float* b3 = W3 + MLP_NH;
    double h1[MLP_NH], y = b3[0];
    int i, j, k;
    for (k = 0; k < MLP_NH; ++k) {
        double z = b1[k];
        for (i = 0; i < MLP_NIN; ++i) z += x[i] * W1[i * MLP_NH + k];
        h1[k] = silu(z);
    }
    for (k = 0; k < MLP_NH; ++k) {
        double z = b2[k];
        for (j = 0; j < MLP_NH; ++j) z += h1[j] * W2[j * MLP_NH + k];
        y += silu(z) * W3[k];
    }
    return (double)b3[1] * (y > 20.0 ? y : log1p(exp(y)));
}

void om_mlp_features(const double* P6, double rho, const double* u, double* x) {
    double P[3][3] = {{P6[0], P6[3], P6[4]}, {P6[3], P6[1], P6[5]}, {P6[4], P6[5], P6[2]}};
    mlp_features(P, rho, u, x);
}

/* Index of the method's polynomial whose monomial row (M[k][.], monomials a*9 + b*3 + c) has exactly
 * the n given entries, or -1. */
static int poly_row(const om_method* m, int n, const int* mono, const double* coef) {
    int k, j, t;
    for (k = 0; k < m->Q; ++k) {
        int ok = 1;
        for (j = 0; j < 27 && ok; ++j) {
            double want = 0.0;
            for (t = 0; t < n; ++t) if (mono[t] == j) want = coef[t];
            if (m->M[k][j] != want) ok = 0;
        }
        if (ok) return k;
    }
    return -1;
}

#define MONO(a, b, c) ((a) * 9 + (b) * 3 + (c))

/* Fourth-order correction of the polynomial cumulant collision (Geier et al. 2017, eq. 44-49 and
 * 112-116; methods/cumulantbased/fourth_order_correction.py:21-237): the third-order groups relax
 * with limited rates, and the fourth-order polynomials PC1..PC6 receive correction terms built from
 * the velocity-derivative estimates of the second-order cumulants.  cmono: pre-collision monomial
 * cumulants (rho-scaled); cpoly / cpost: pre- / post-collision polynomial cumulants. */
static void fourth_order_correction(const om_method* m, double rho, const double* cmono, const double* cpoly,
                                    double* cpost) {
    static const double one = 1.0;
    const double p11[2] = {1.0, 1.0}, p1m[2] = {1.0, -1.0}, pc1[3] = {1.0, -2.0, 1.0},
                 pc2[3] = {1.0, 1.0, -2.0}, pc3[3] = {1.0, 1.0, 1.0};
    /* third-order groups: sums, differences (each of the three permutations), xyz */
    const int sums[3][2] = {{MONO(1, 2, 0), MONO(1, 0, 2)}, {MONO(2, 1, 0), MONO(0, 1, 2)},
                            {MONO(2, 0, 1), MONO(0, 2, 1)}};
    const int m4[3] = {MONO(2, 2, 0), MONO(2, 0, 2), MONO(0, 2, 2)};
    const int xy = MONO(1, 1, 0), xz = MONO(1, 0, 1), yz = MONO(0, 1, 1), x2 = MONO(2, 0, 0),
              y2 = MONO(0, 2, 0), z2 = MONO(0, 0, 2), xyz = MONO(1, 1, 1);
    const int bulk[3] = {x2, y2, z2};
    int ks[3], kd[3], k5, kp[6], j, kxy, kb;
    double w1, w2, w3, w4, w5, w6, w7, w8, lim, a, b, den, w11, w12, w22, dx, dy, dz, dxy, dxz, dyz, g, t;
    for (j = 0; j < 3; ++j) {
        ks[j] = poly_row(m, 2, sums[j], p11);
        kd[j] = poly_row(m, 2, sums[j], p1m);
    }
    k5 = poly_row(m, 1, &xyz, &one);
    kp[0] = poly_row(m, 3, m4, pc1);
    kp[1] = poly_row(m, 3, m4, pc2);
    kp[2] = poly_row(m, 3, m4, pc3);
    {
        const int p4 = MONO(2, 1, 1), p5 = MONO(1, 2, 1), p6 = MONO(1, 1, 2);
        kp[3] = poly_row(m, 1, &p4, &one);
        kp[4] = poly_row(m, 1, &p5, &one);
        kp[5] = poly_row(m, 1, &p6, &one);
    }
    kxy = poly_row(m, 1, &xy, &one);
    kb = poly_row(m, 3, bulk, pc3);
    w1 = m->rate[kxy];
    w2 = m->rate[kb];
    w6 = m->rate[kp[0]]; w7 = m->rate[kp[2]]; w8 = m->rate[kp[3]];
    /* limited third-order rates (fourth_order_correction.py:199-211) */
    lim = rho * m->foc_limiter;
    t = fabs(cmono[MONO(1, 2, 0)] + cmono[MONO(1, 0, 2)]);
    w3 = m->rate[ks[0]] + (1.0 - m->rate[ks[0]]) * t / (lim + t);
    t = fabs(cmono[MONO(1, 2, 0)] - cmono[MONO(1, 0, 2)]);
    w4 = m->rate[kd[0]] + (1.0 - m->rate[kd[0]]) * t / (lim + t);
    t = fabs(cmono[xyz]);
    w5 = m->rate[k5] + (1.0 - m->rate[k5]) * t / (lim + t);
    for (j = 0; j < 3; ++j) {          /* third-order equilibria are zero */
        cpost[ks[j]] = cpoly[ks[j]] - w3 * cpoly[ks[j]];
        cpost[kd[j]] = cpoly[kd[j]] - w4 * cpoly[kd[j]];
    }
    cpost[k5] = cpoly[k5] - w5 * cpoly[k5];
    /* a and b (eq. 115-116) */
    w11 = w1 * w1; w12 = w1 * w2; w22 = w2 * w2;
    den = (w1 - w2) * (w2 * (2.0 + 3.0 * w1) - 8.0 * w1);
    a = (4.0 * w11 + 2.0 * w12 * (w1 - 6.0) + w22 * (w1 * (10.0 - 3.0 * w1) - 4.0)) / den;
    b = (4.0 * w12 * (9.0 * w1 - 16.0) - 4.0 * w11 - 2.0 * w22 * (2.0 + 9.0 * w1 * (w1 - 2.0))) / (3.0 * den);
    /* velocity-derivative estimates from the pre-collision second-order cumulants */
    dx = -w1 / (2.0 * rho) * (2.0 * cmono[x2] - cmono[y2] - cmono[z2])
         - w2 / (2.0 * rho) * (cmono[x2] + cmono[y2] + cmono[z2] - rho);
    dy = dx + (3.0 * w1) / (2.0 * rho) * (cmono[x2] - cmono[y2]);
    dz = dx + (3.0 * w1) / (2.0 * rho) * (cmono[x2] - cmono[z2]);
    dxy = -3.0 * w1 / rho * cmono[xy];
    dxz = -3.0 * w1 / rho * cmono[xz];
    dyz = -3.0 * w1 / rho * cmono[yz];
    g = 1.0 / w1 - 0.5;
    cpost[kp[0]] += 2.0 / 3.0 * g * w6 * a * rho * (dx - 2.0 * dy + dz);
    cpost[kp[1]] += 2.0 / 3.0 * g * w6 * a * rho * (dx + dy - 2.0 * dz);
    cpost[kp[2]] += -4.0 / 3.0 * g * w7 * a * rho * (dx + dy + dz);
    cpost[kp[3]] += -1.0 / 3.0 * g * w8 * b * rho * dyz;
    cpost[kp[4]] += -1.0 / 3.0 * g * w8 * b * rho * dxz;
    cpost[kp[5]] += -1.0 / 3.0 * g * w8 * b * rho * dxy;
}

static void collide_cumulant(const om_method* m, const double* f, double* fo, double* omega_out,
                             int all_rates_one) {
    int Q = m->Q, i, k, d, n;
    double rho, drho, rho_ref, u[3], km[27], kbg[27], mm[27], cc[27], cmono[27], cpoly[27];
    double cpost[27], cmono_post[27], rates[27], half[3] = {0, 0, 0};
    conserved(m, f, &rho, &drho, &rho_ref, u);
    if (m->force_model == 2)
        for (d = 0; d < 3; ++d) { u[d] += m->F[d] / (2.0 * rho); half[d] = 0.5 * m->F[d]; }
    central_moments(m, f, u, km);
    if (m->zero_centered) {
        central_moments(m, m->w, u, kbg);
        for (n = 0; n < 27; ++n) km[n] += kbg[n];
    }
    /* conserved central moments exactly as lbmpy's simplified forward transform has them
     * (moment_transforms/centralmomenttransforms.py:268-291): kappa_000 = rho,
     * kappa_100 = -F/2, then the symmetric forcing adds +F/2 (forcemodels.py:222-230). */
    km[0] = rho;
    km[9] = -half[0] + half[0]; km[3] = -half[1] + half[1]; km[1] = -half[2] + half[2];
    for (n = 0; n < 27; ++n) mm[n] = km[n] / rho;
    cumulants_from_moments(mm, cc);
    for (n = 1; n < 27; ++n) cmono[n] = rho * cc[n];
    cmono[9] = rho * (u[0] + mm[9]); cmono[3] = rho * (u[1] + mm[3]); cmono[1] = rho * (u[2] + mm[1]);
    cmono[0] = rho * log(km[0]);
    for (k = 0; k < Q; ++k) {
        double s = 0.0;
        for (n = 0; n < 27; ++n) s += m->M[k][n] * cmono[n];
        cpoly[k] = s;
        rates[k] = all_rates_one ? 1.0 : m->rate[k];
    }
    if ((m->sgs == 1 || m->sgs == 2) && !all_rates_one) {
        /* f_neq = f - f_eq with f_eq = the rates-one collision (cumulantbasedmethod.py:220-240) */
        double feq[27], pi[3][3] = {{0}}, pn = 0.0, tau0, om; int a, b;
        collide_cumulant(m, f, feq, 0, 1);
        for (i = 0; i < Q; ++i)
            for (a = 0; a < 3; ++a)
                for (b = 0; b < 3; ++b) pi[a][b] += m->c[i][a] * m->c[i][b] * (f[i] - feq[i]);
        for (a = 0; a < 3; ++a) for (b = 0; b < 3; ++b) pn += pi[a][b] * pi[a][b];
        pn = sqrt(2.0 * pn) / rho;
        tau0 = 1.0 / m->shear_rate;
        if (m->sgs == 1) {
            om = 2.0 / (tau0 + sqrt(18.0 * m->sgs_c * m->sgs_c * pn + tau0 * tau0));
        } else {
            double x[MLP_NIN];
            mlp_features(pi, rho, u, x);
            om = 1.0 / (tau0 + 3.0 * om_mlp_nu_t(m->mlp, x));
        }
        for (k = 0; k < Q; ++k) if (m->rate[k] == m->shear_rate) rates[k] = om;
        if (omega_out) *omega_out = om;
    }
    {
        /* equilibrium cumulants of the compressible Maxwellian, rescaled by rho */
        double ceq[27];
        for (n = 0; n < 27; ++n) ceq[n] = 0.0;
        ceq[0] = rho * log(rho);
        ceq[9] = rho * u[0]; ceq[3] = rho * u[1]; ceq[1] = rho * u[2];
        ceq[18] = ceq[6] = ceq[2] = rho / 3.0;
        for (k = 0; k < Q; ++k) {
            double s = 0.0;
            for (n = 0; n < 27; ++n) s += m->M[k][n] * ceq[n];
            cpost[k] = cpoly[k] + rates[k] * (s - cpoly[k]);
        }
    }
    if (m->galilean && !all_rates_one) {
        /* galilean_correction.py:56-91, with the base (numeric) relaxation rates */
        int kxy = -1, kxz = -1, kb = -1;
        double o1, o2, cxx = cmono[18], cyy = cmono[6], czz = cmono[2], dx, dy, dz;
        for (k = 0; k < Q; ++k) {
            /* identify x^2-y^2, x^2-z^2, x^2+y^2+z^2 by their mono->poly rows */
            double r200 = m->M[k][18], r020 = m->M[k][6], r002 = m->M[k][2], other = 0.0;
            for (n = 0; n < 27; ++n) if (n != 18 && n != 6 && n != 2) other += fabs(m->M[k][n]);
            if (other != 0.0) continue;
            if (r200 == 1 && r020 == -1 && r002 == 0) kxy = k;
            if (r200 == 1 && r020 == 0 && r002 == -1) kxz = k;
            if (r200 == 1 && r020 == 1 && r002 == 1) kb = k;
        }
        o1 = m->rate[kxy]; o2 = m->rate[kb];
        dx = -o1 / (2.0 * rho) * (2.0 * cxx - cyy - czz) - o2 / (2.0 * rho) * (cxx + cyy + czz - rho);
        dy = dx + (3.0 * o1) / (2.0 * rho) * (cxx - cyy);
        dz = dx + (3.0 * o1) / (2.0 * rho) * (cxx - czz);
        cpost[kxy] += -3.0 * rho * (1.0 - o1 / 2.0) * (u[0] * u[0] * dx - u[1] * u[1] * dy);
        cpost[kxz] += -3.0 * rho * (1.0 - o1 / 2.0) * (u[0] * u[0] * dx - u[2] * u[2] * dz);
        cpost[kb] += -3.0 * rho * (1.0 - o2 / 2.0) * (u[0] * u[0] * dx + u[1] * u[1] * dy + u[2] * u[2] * dz);
    }
    if (m->foc_limiter > 0.0 && !all_rates_one) fourth_order_correction(m, rho, cmono, cpoly, cpost);
    for (n = 0; n < 27; ++n) {
        double s = 0.0;
        for (k = 0; k < Q; ++k) s += m->Minv[n][k] * cpost[k];
        cmono_post[n] = s;
    }
    /* back to central moments: K = exp(C - Xi.u); kappa_000 stays rho */
    for (n = 1; n < 27; ++n) cc[n] = cmono_post[n] / rho;
    cc[9] -= u[0]; cc[3] -= u[1]; cc[1] -= u[2];
    cc[0] = 0.0;
    moments_from_cumulants(cc, mm);
    for (n = 0; n < 27; ++n) km[n] = rho * mm[n];
    km[9] += half[0]; km[3] += half[1]; km[1] += half[2];
    if (all_rates_one) { km[9] -= half[0]; km[3] -= half[1]; km[1] -= half[2]; }
    populations_from_central(m, km, u, fo);
    if (m->zero_centered) for (i = 0; i < Q; ++i) fo[i] -= m->w[i];
}

/* Central-moment method (D3Q27, compressible): polynomial central moments about the equilibrium
 * velocity relaxed towards those of the continuous Maxwellian, forcing applied in central-moment
 * space (methods/momentbased/centralmomentbasedmethod.py:296-394, relax_central_moments;
 * forcemodels.py:201-203 Simple, :261-263 Luo, :300-306 Guo with (1 - omega/2)).  The equilibrium
 * central moments are rho times those of a Gaussian of variance 1/3 (independent of u; the
 * truncated raw Maxwellian moments give the same values, which tests/test_central_moment.py checks
 * symbolically). */
static void collide_central(const om_method* m, const double* f, double* fo) {
    int Q = m->Q, i, k, n, d;
    double rho, drho, rho_ref, u[3], km[27], kbg[27], keq[27], kf[27], post[27], mono[27], fpop[27] = {0};
    static const double g[3] = {1.0, 0.0, 1.0 / 3.0};
    conserved(m, f, &rho, &drho, &rho_ref, u);
    if (m->force_model == 1)                      /* Guo: equilibrium velocity shift F / (2 rho) */
        for (d = 0; d < 3; ++d) u[d] += m->F[d] / (2.0 * rho);
    central_moments(m, f, u, km);
    if (m->zero_centered) {
        central_moments(m, m->w, u, kbg);
        for (n = 0; n < 27; ++n) km[n] += kbg[n];
    }
    km[0] = rho;
    for (n = 0; n < 27; ++n) keq[n] = rho * g[n / 9] * g[(n / 3) % 3] * g[n % 3];
    for (n = 0; n < 27; ++n) kf[n] = 0.0;
    if (m->force_model == 1 || m->force_model == 3 || m->force_model == 4) {
        for (i = 0; i < Q; ++i) {
            double cu = 0.0, cf = 0.0, t = 0.0;
            for (d = 0; d < 3; ++d) { cu += m->c[i][d] * u[d]; cf += m->c[i][d] * m->F[d]; }
            if (m->force_model == 3) t = 3.0 * cf;                        /* Simple */
            else for (d = 0; d < 3; ++d) t += m->F[d] * ((m->c[i][d] - u[d]) * 3.0 + m->c[i][d] * cu * 9.0);
            fpop[i] = m->w[i] * t;
        }
        central_moments(m, fpop, u, kf);
    }
    for (k = 0; k < Q; ++k) {
        double pk = 0.0, pe = 0.0, pf = 0.0;
        for (n = 0; n < 27; ++n) { pk += m->M[k][n] * km[n]; pe += m->M[k][n] * keq[n]; pf += m->M[k][n] * kf[n]; }
        post[k] = pk + m->rate[k] * (pe - pk) + (m->force_model == 1 ? 1.0 - 0.5 * m->rate[k] : 1.0) * pf;
    }
    for (n = 0; n < 27; ++n) {
        double s = 0.0;
        for (k = 0; k < Q; ++k) s += m->Minv[n][k] * post[k];
        mono[n] = s;
    }
    populations_from_central(m, mono, u, fo);
    if (m->zero_centered) for (i = 0; i < Q; ++i) fo[i] -= m->w[i];
}

void om_collide(const om_method* m, const double* f, double* fo, double* omega_out) {
    if (m->kind == 1) collide_cumulant(m, f, fo, omega_out, 0);
    else if (m->kind == 2) collide_central(m, f, fo);
    else collide_moment(m, f, fo, omega_out);
}

/* ------------------------------------ equilibrium ---------------------------------------- */
void om_equilibrium(const om_method* m, double rho, const double uin[3], double* feq) {
    double u[3], rho_ref = m->compressible ? rho : 1.0; int d, i, k;
    for (d = 0; d < 3; ++d) u[d] = uin[d];
    if (m->force_model != 0)                   /* macroscopic_velocity_shift, forcemodels.py:592 */
        for (d = 0; d < 3; ++d) u[d] -= m->F[d] / (2.0 * rho_ref);
    if (m->kind == 1 || m->kind == 2) {      /* the Gaussian in central moments, shifted by u */
        double cc[27], mm[27], km[27];
        for (i = 0; i < 27; ++i) cc[i] = 0.0;
        cc[18] = cc[6] = cc[2] = 1.0 / 3.0;
        moments_from_cumulants(cc, mm);
        for (i = 0; i < 27; ++i) km[i] = rho * mm[i];
        populations_from_central(m, km, u, feq);
        if (m->zero_centered) for (i = 0; i < m->Q; ++i) feq[i] -= m->w[i];
        return;
    }
    {
        double meq[QMAX], bg[QMAX];
        for (k = 0; k < m->Q; ++k) {
            meq[k] = eq_moment(m, k, rho, rho - 1.0, u);
            bg[k] = 0.0;
            if (m->zero_centered && !m->delta_eq)
                for (i = 0; i < m->Q; ++i) bg[k] += m->M[k][i] * m->w[i];
        }
        for (i = 0; i < m->Q; ++i) {
            double s = 0.0;
            for (k = 0; k < m->Q; ++k) s += m->Minv[i][k] * (meq[k] - bg[k]);
            feq[i] = s;
        }
    }
}

/* ------------------------------------ field kernels -------------------------------------- */
static int interior(const om_grid* gr, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x < gr->n[0] && y < gr->n[1] && z < gr->n[2];
}

/* One stream-collide sweep over all interior cells whose flag is 0 (or every cell if flags
 * is NULL).  For in-place patterns src == dst.  omega_field (optional) receives the SGS rate. */
void om_sweep(const om_method* m, const om_grid* gr, int pattern, int parity,
              const double* src, double* dst, const uint8_t* flags, double* omega_field) {
    int roff[QMAX][3], rslot[QMAX], woff[QMAX][3], wslot[QMAX], i;
    for (i = 0; i < m->Q; ++i) {
        accessor(m, pattern, parity, 0, i, roff[i], &rslot[i]);
        accessor(m, pattern, parity, 1, i, woff[i], &wslot[i]);
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < gr->n[2]; ++z)
        for (int y = 0; y < gr->n[1]; ++y)
            for (int x = 0; x < gr->n[0]; ++x) {
                double f[QMAX], fo[QMAX], om = 0.0; int q;
                if (flags && flags[fidx(gr, x, y, z)] != 0) continue;
                for (q = 0; q < m->Q; ++q)
                    f[q] = src[gidx(gr, x + roff[q][0], y + roff[q][1], z + roff[q][2]) + rslot[q] * gr->s[3]];
                om_collide(m, f, fo, &om);
                for (q = 0; q < m->Q; ++q)
                    dst[gidx(gr, x + woff[q][0], y + woff[q][1], z + woff[q][2]) + wslot[q] * gr->s[3]] = fo[q];
                if (omega_field) omega_field[fidx(gr, x, y, z)] = om;
            }
}

/* Ghost-layer periodicity between two steps (advanced_streaming/communication.py:21-121):
 * 1) values the previous step wrote into ghost cells move to their periodic images,
 * 2) every ghost cell that is a periodic image of an interior cell gets all its slots copied. */
void om_periodic_sync(const om_method* m, const om_grid* gr, int pattern, int prev_parity,
                      const int periodic[3], double* f) {
    int woff[QMAX][3], wslot[QMAX], i;
    int lo[3], hi[3];
    for (i = 0; i < 3; ++i) { lo[i] = -gr->g[i]; hi[i] = gr->n[i] + gr->g[i]; }
    for (i = 0; i < m->Q; ++i) accessor(m, pattern, prev_parity, 1, i, woff[i], &wslot[i]);
    /* 1) write-back */
    for (int z = lo[2]; z < hi[2]; ++z) for (int y = lo[1]; y < hi[1]; ++y) for (int x = lo[0]; x < hi[0]; ++x) {
        int p[3] = {x, y, z}, w[3], d, ok = 1, q;
        if (interior(gr, x, y, z)) continue;
        for (d = 0; d < 3; ++d) {
            w[d] = p[d];
            if (p[d] < 0 || p[d] >= gr->n[d]) { if (!periodic[d]) ok = 0; w[d] = ((p[d] % gr->n[d]) + gr->n[d]) % gr->n[d]; }
        }
        if (!ok) continue;
        for (q = 0; q < m->Q; ++q) {
            int sx = x - woff[q][0], sy = y - woff[q][1], sz = z - woff[q][2];
            if (!interior(gr, sx, sy, sz)) continue;
            f[gidx(gr, w[0], w[1], w[2]) + wslot[q] * gr->s[3]] = f[gidx(gr, x, y, z) + wslot[q] * gr->s[3]];
        }
    }
    /* 2) fill */
    for (int z = lo[2]; z < hi[2]; ++z) for (int y = lo[1]; y < hi[1]; ++y) for (int x = lo[0]; x < hi[0]; ++x) {
        int p[3] = {x, y, z}, w[3], d, ok = 1, q;
        if (interior(gr, x, y, z)) continue;
        for (d = 0; d < 3; ++d) {
            w[d] = p[d];
            if (p[d] < 0 || p[d] >= gr->n[d]) { if (!periodic[d]) ok = 0; w[d] = ((p[d] % gr->n[d]) + gr->n[d]) % gr->n[d]; }
        }
        if (!ok) continue;
        for (q = 0; q < m->Q; ++q)
            f[gidx(gr, x, y, z) + q * gr->s[3]] = f[gidx(gr, w[0], w[1], w[2]) + q * gr->s[3]];
    }
}

/* Link boundary kernel between two steps.  flags over the ghost-layered domain:
 * 0 fluid, 1 NoSlip, 2 UBB (velocity ubb_u).  f_out / f_in proxies follow
 * advanced_streaming/indexing.py:12-183; NoSlip boundaryconditions.py:128-139,
 * UBB boundaryconditions.py:794-841. */
/* Outgoing population d of cell (x, y, z) as the previous step wrote it, the cell wrapped on periodic
 * axes (the ghost layers hold the same values after om_periodic_sync); 0 with *ok = 0 when the
 * location lies beyond the ghost layer of a non-periodic axis. */
static double f_out_at(const om_method* m, const om_grid* gr, const int periodic[3], int ooff[QMAX][3],
                       int oslot[QMAX], const double* f, int x, int y, int z, int d, int* ok) {
    /* the sweep wrote from the interior image of the cell, at the write offset, into a ghost cell
     * where that offset crosses a face: om_periodic_sync moves such values to the periodic image
     * and copies them back, except in ghost cells beyond a non-periodic face (edges and corners),
     * so the value is always found at the unwrapped write location of the wrapped cell */
    int c[3] = {x, y, z}, a;
    for (a = 0; a < 3; ++a) {
        if (a >= m->D) continue;
        if (periodic[a]) c[a] = ((c[a] % gr->n[a]) + gr->n[a]) % gr->n[a];
        c[a] += ooff[d][a];
        if (c[a] < -1 || c[a] > gr->n[a]) { *ok = 0; return 0.0; }
    }
    *ok = 1;
    return f[gidx(gr, c[0], c[1], c[2]) + oslot[d] * gr->s[3]];
}

/* Flags: 1 NoSlip, 2 UBB (velocity ubb_u), 6 / 7 FixedDensity (density fd_rho / m->fd_rho1),
 * 8 FreeSlip and 9 SimpleExtrapolationOutflow (copy from the cell and direction of the link code,
 * boundaryconditions.py:360-455, 844-889), 10 ExtrapolationOutflow (:894-1041), 11
 * NoSlipLinearBouzidi (:142-212).
 * FixedDensity (boundaryconditions.py:1044-1099): f_in(inv q) = 2 feq_even_q(rho_w, u) - f_out(q),
 * feq_even the part of the method's equilibrium that is even in u (the mean of directions q and
 * inv q), u from the fluid cell's outgoing populations with the density replaced by rho_w. */
void om_boundaries(const om_method* m, const om_grid* gr, int pattern, int prev_parity,
                   const uint8_t* flags, const double ubb_u[3], double fd_rho, const int periodic[3], double* f) {
    int ooff[QMAX][3], oslot[QMAX], ioff[QMAX][3], islot[QMAX], i;
    int next_parity = 1 - prev_parity;
    for (i = 0; i < m->Q; ++i) {
        accessor(m, pattern, prev_parity, 1, i, ooff[i], &oslot[i]);
        accessor(m, pattern, next_parity, 0, i, ioff[i], &islot[i]);
    }
    for (int z = 0; z < gr->n[2]; ++z) for (int y = 0; y < gr->n[1]; ++y) for (int x = 0; x < gr->n[0]; ++x) {
        int q;
        if (flags[fidx(gr, x, y, z)] != 0) continue;
        for (q = 1; q < m->Q; ++q) {
            int bx = x + m->c[q][0], by = y + m->c[q][1], bz = z + m->c[q][2], iq = m->inv[q];
            uint8_t fl = flags[fidx(gr, bx, by, bz)];
            double fout, val;
            if (fl == 0) continue;
            fout = f[gidx(gr, x + ooff[q][0], y + ooff[q][1], z + ooff[q][2]) + oslot[q] * gr->s[3]];
            val = fout;
            if (fl == 2) {
                double cu = 0.0, rho = 1.0, uw[3]; int k;
                for (k = 0; k < 3; ++k) uw[k] = ubb_u[k];
                if (m->ubb_link) {
                    const int64_t c = x + (int64_t)gr->n[0] * (y + (int64_t)gr->n[1] * z);
                    for (k = 0; k < 3; ++k) uw[k] = m->ubb_link[(c * m->Q + q) * 3 + k];
                }
                if (m->compressible) {
                    double s = 0.0;
                    for (k = 0; k < m->Q; ++k)
                        s += f[gidx(gr, x + ooff[k][0], y + ooff[k][1], z + ooff[k][2]) + oslot[k] * gr->s[3]];
                    rho = m->zero_centered ? 1.0 + s : s;
                    if (m->ubb_density > 0.0) rho = m->ubb_density;
                }
                if (m->ubb_adapt)      /* cqc.equilibrium_input_equations_from_init_values(velocity) */
                    for (k = 0; k < 3; ++k) uw[k] -= m->F[k] / (2.0 * rho);
                for (k = 0; k < 3; ++k) cu += m->c[q][k] * uw[k];
                val = fout - 6.0 * m->w[q] * cu * rho;
            } else if (fl >= 8 && fl <= 11 && (m->link_code || m->link_value)) {
                const int64_t c = x + (int64_t)gr->n[0] * (y + (int64_t)gr->n[1] * z);
                const int64_t li = c * m->Q + q;
                int ok = 1;
                if (fl <= 10 && m->link_code) {
                    const int code = m->link_code[li], d = code & 0xff;
                    const double w = f_out_at(m, gr, periodic, ooff, oslot, f, x + ((code >> 8) & 3) - 1,
                                              y + ((code >> 10) & 3) - 1, z + ((code >> 12) & 3) - 1, d, &ok);
                    val = ok ? w : fout;
                    if (fl == 10 && m->link_value) {
                        double* st = m->link_value + li * 2;
                        const double cc = sqrt(1.0 / 3.0), fin = cc * st[0] + (1.0 - cc) * st[1];
                        st[0] = val;
                        st[1] = fin;
                        val = fin;
                    }
                } else if (fl == 11 && m->link_value) {
                    const double qd = m->link_value[li * 2];
                    if (qd >= 0.5) {
                        const double finv =
                            f[gidx(gr, x + ooff[iq][0], y + ooff[iq][1], z + ooff[iq][2]) + oslot[iq] * gr->s[3]];
                        val = 0.5 * (fout + finv * (2.0 * qd - 1.0)) / qd;
                    } else if (qd > 0.0) {
                        const double d2 = f_out_at(m, gr, periodic, ooff, oslot, f, x - m->c[q][0], y - m->c[q][1],
                                                   z - m->c[q][2], q, &ok);
                        val = 2.0 * qd * fout + (1.0 - 2.0 * qd) * (ok ? d2 : fout);
                    }
                }
            } else if (fl == 6 || fl == 7) {
                double j[3] = {0.0, 0.0, 0.0}, u[3], feq[QMAX]; int k, d;
                const double rw = fl == 6 ? fd_rho : m->fd_rho1;
                for (k = 0; k < m->Q; ++k) {
                    const double fk = f[gidx(gr, x + ooff[k][0], y + ooff[k][1], z + ooff[k][2]) + oslot[k] * gr->s[3]];
                    for (d = 0; d < 3; ++d) j[d] += m->c[k][d] * fk;
                }
                for (d = 0; d < 3; ++d) u[d] = m->compressible ? j[d] / rw : j[d];
                om_equilibrium(m, rw, u, feq);
                val = feq[q] + feq[iq] - fout;
            }
            f[gidx(gr, x + ioff[iq][0], y + ioff[iq][1], z + ioff[iq][2]) + islot[iq] * gr->s[3]] = val;
        }
    }
}

/* Equilibrium initialisation through the write accessor of prev_parity
 * (macroscopic_value_kernels.py:29-45).  rho: n0*n1*n2, u: 3*n0*n1*n2 (x fastest). */
void om_set_equilibrium(const om_method* m, const om_grid* gr, int pattern, int prev_parity,
                        const double* rho, const double* u, double* f) {
    int woff[QMAX][3], wslot[QMAX], i;
    int64_t nc = (int64_t)gr->n[0] * gr->n[1] * gr->n[2];
    for (i = 0; i < m->Q; ++i) accessor(m, pattern, prev_parity, 1, i, woff[i], &wslot[i]);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < gr->n[2]; ++z) for (int y = 0; y < gr->n[1]; ++y) for (int x = 0; x < gr->n[0]; ++x) {
        int64_t c = x + (int64_t)gr->n[0] * (y + (int64_t)gr->n[1] * z);
        double uu[3] = {u[c], u[nc + c], u[2 * nc + c]}, feq[QMAX]; int q;
        om_equilibrium(m, rho[c], uu, feq);
        for (q = 0; q < m->Q; ++q)
            f[gidx(gr, x + woff[q][0], y + woff[q][1], z + woff[q][2]) + wslot[q] * gr->s[3]] = feq[q];
    }
}

/* Density and velocity from the values the previous step wrote (macroscopic_value_kernels.py:48-61). */
void om_get_macroscopic(const om_method* m, const om_grid* gr, int pattern, int prev_parity,
                        const double* f, double* rho, double* u) {
    int woff[QMAX][3], wslot[QMAX], i;
    int64_t nc = (int64_t)gr->n[0] * gr->n[1] * gr->n[2];
    for (i = 0; i < m->Q; ++i) accessor(m, pattern, prev_parity, 1, i, woff[i], &wslot[i]);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < gr->n[2]; ++z) for (int y = 0; y < gr->n[1]; ++y) for (int x = 0; x < gr->n[0]; ++x) {
        int64_t c = x + (int64_t)gr->n[0] * (y + (int64_t)gr->n[1] * z);
        double g[QMAX], r, dr, rr, uu[3]; int q, d;
        for (q = 0; q < m->Q; ++q)
            g[q] = f[gidx(gr, x + woff[q][0], y + woff[q][1], z + woff[q][2]) + wslot[q] * gr->s[3]];
        conserved(m, g, &r, &dr, &rr, uu);
        if (m->force_model != 0) for (d = 0; d < 3; ++d) uu[d] += m->F[d] / (2.0 * rr);
        rho[c] = r;
        for (d = 0; d < 3; ++d) u[d * nc + c] = uu[d];
    }
}

/* The whole time loop of lbmpy's manual in-place loop (test_periodic_pipe_with_force.py:129-150)
 * or LatticeBoltzmannStep.time_step (lbstep.py:271-282) for two-field patterns:
 * periodicity, boundaries, sweep, (swap).  *parity is the parity of the last completed step
 * and is updated.  For two-field patterns a and b are swapped by pointer; returns 1 if the
 * result ends up in b. */
int om_run(const om_method* m, const om_grid* gr, int pattern, int* parity, int steps,
           const int periodic[3], const uint8_t* flags, const double ubb_u[3], double fd_rho, double* a,
           double* b) {
    int t, inplace = (pattern == P_AA || pattern == P_ESOTWIST || pattern == P_ESOPULL || pattern == P_ESOPUSH),
        swapped = 0;
    double *src = a, *dst = b;
    for (t = 0; t < steps; ++t) {
        om_periodic_sync(m, gr, pattern, *parity, periodic, src);
        if (flags) om_boundaries(m, gr, pattern, *parity, flags, ubb_u, fd_rho, periodic, src);
        *parity = inplace ? 1 - *parity : *parity;
        om_sweep(m, gr, pattern, *parity, src, inplace ? src : dst, flags, 0);
        if (!inplace) { double* tmp = src; src = dst; dst = tmp; swapped ^= 1; }
    }
    return swapped;
}

/* FP64 sums over fluid cells of rho, rho_ref*u (momentum) and rho*|u|^2/2. out[5]. */
void om_reduce(const om_method* m, const om_grid* gr, int pattern, int prev_parity, const double* f,
               const uint8_t* flags, double* out) {
    int woff[QMAX][3], wslot[QMAX], i;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
    for (i = 0; i < m->Q; ++i) accessor(m, pattern, prev_parity, 1, i, woff[i], &wslot[i]);
#pragma omp parallel for collapse(2) reduction(+ : s0, s1, s2, s3, s4)
    for (int z = 0; z < gr->n[2]; ++z) for (int y = 0; y < gr->n[1]; ++y) for (int x = 0; x < gr->n[0]; ++x) {
        double g[QMAX], r, dr, rr, uu[3]; int q, d;
        if (flags && flags[fidx(gr, x, y, z)] != 0) continue;
        for (q = 0; q < m->Q; ++q)
            g[q] = f[gidx(gr, x + woff[q][0], y + woff[q][1], z + woff[q][2]) + wslot[q] * gr->s[3]];
        conserved(m, g, &r, &dr, &rr, uu);
        if (m->force_model != 0) for (d = 0; d < 3; ++d) uu[d] += m->F[d] / (2.0 * rr);
        s0 += r; s1 += rr * uu[0]; s2 += rr * uu[1]; s3 += rr * uu[2];
        s4 += 0.5 * r * (uu[0] * uu[0] + uu[1] * uu[1] + uu[2] * uu[2]);
    }
    out[0] = s0; out[1] = s1; out[2] = s2; out[3] = s3; out[4] = s4;
}

int om_sizeof_method(void) { return (int)sizeof(om_method); }

/* Threads of the OpenMP loops that follow (small grids run faster on one thread). */
void om_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#else
    (void)n;
#endif
}

/* The accessor table of one pattern / parity: read (rw = 0) or write (rw = 1) offset off[3*i..]
 * and slot slot[i] of every direction i. */
void om_accessor_table(const om_method* m, int pattern, int parity, int rw, int* off, int* slot) {
    int i;
    for (i = 0; i < m->Q; ++i) accessor(m, pattern, parity, rw, i, off + 3 * i, slot + i);
}
