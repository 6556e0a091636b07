/*
 * lbm_cpu.c -- closed-form CPU sweeps in the style of lbmpy's generated OpenMP kernels.
 * TEST INFRASTRUCTURE ONLY: the CPU baseline that bench.py times and the fast checker that the
 * long-run tests use.  The product (lbmpy_b200) never links or calls it.
 *
 * lbmpy's CPU backend emits one loop nest per method: OpenMP over the outer dimension, the x loop
 * innermost over an fzyx (SoA) field, and per cell a straight-line block of assignments that sympy
 * simplified for the numeric relaxation rates (creationfunctions.py:543-582 with
 * `target=Target.CPU, openmp=True`).  This file restates two such kernels by hand, each compiled
 * for FP64 and FP32 arithmetic and storage (REAL):
 *
 *   ocpu_trt_pull_*   D3Q19/D3Q27 TRT, pull streaming, two fields; equilibrium tables supplied by
 *                     the caller (continuous or discrete Maxwellian, delta form,
 *                     equilibrium/continuous_hydro_maxwellian.py:82-116), population-space
 *                     collision (methods/momentbased/momentbasedmethod.py:389-398);
 *   ocpu_cum_aa_*     D3Q27 cumulant with every cumulant of order >= 3 relaxed by 1 (lbmpy's
 *                     rates for one relaxation rate, methods/creationfunctions.py:638-652), AA in
 *                     place (fieldaccess.py:134-159), Galilean correction
 *                     (methods/cumulantbased/galilean_correction.py:56-91) and the symmetric
 *                     CentralMoment force (forcemodels.py:213-233), zero-centred storage.
 *
 * Periodic axes wrap their indices; NoSlip (flag 1) and one UBB (flag 2) are halfway bounce-back
 * links into the ghost layer (boundaries/boundaryconditions.py:128-139, 794-841), folded into the
 * read of the fluid cell next to them.  Field element (x, y, z, q), ghost-inclusive coordinates:
 * x + y*sy + z*sz + q*sq.  Flags: uint8, x + (nx+2)*(y + (ny+2)*z).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL double
#define SUFFIX f64
#endif
#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUFFIX)

typedef REAL real;

#ifndef OCPU_TYPES
#define OCPU_TYPES
typedef struct {
    int q;                    /* 19 or 27 */
    int c[27][3];             /* directions, lbmpy's 'walberla' order */
    int inv[27];
    double w[27];
    double eq_lin[27][3];     /* TRT: f_eq_i - w_i drho = rf * (lin_i . u + quad_i . (uxx uyy uzz uxy uxz uyz)) */
    double eq_quad[27][6];
    double omega_even, omega_odd; /* TRT rates; cumulant: omega_even = shear rate, omega_odd = bulk rate */
    int compressible;
    int galilean;
    double force[3];          /* cumulant: CentralMoment force */
    double ubb[3];            /* wall velocity of flag 2 */
    int n[3];                 /* interior cells */
    int64_t sy, sz, sq;       /* element strides (x stride 1) */
    int periodic[3];
} ocpu_params;

static inline int cube_index(const int c[3]) { return (c[0] + 1) * 9 + (c[1] + 1) * 3 + (c[2] + 1); }

/* lbmpy's 'walberla' order of D3Q27 (stencils.py:220-227); its first 19 entries are D3Q19's
 * (:193-199), with the same inverses.  The row kernels below use these compile-time tables, as
 * lbmpy's generated code has the directions as constants. */
static const int DX[27] = {0, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1};
static const int DY[27] = {0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, -1, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
static const int DZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1};
static const int INV[27] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 16, 15, 18, 17, 12, 11, 14, 13,
                            26, 25, 24, 23, 22, 21, 20, 19};

/* 1 when the caller's direction table is the compile-time one. */
int FN(ocpu_tables_match)(const ocpu_params* p) {
    int i;
    for (i = 0; i < p->q; ++i)
        if (p->c[i][0] != DX[i] || p->c[i][1] != DY[i] || p->c[i][2] != DZ[i] || p->inv[i] != INV[i]) return 0;
    return 1;
}
#endif

#define ALWAYS_INLINE static inline __attribute__((always_inline))

/* Offset (elements) of the neighbour of (x, y, z) at direction d in {-1, 0, 1}^3, periodic axes
 * wrapped; on a non-periodic axis the neighbour may be the ghost layer. */
ALWAYS_INLINE int FN(wrap)(int v, int n, int periodic) {
    if (periodic) {
        if (v < 0) v += n;
        else if (v >= n) v -= n;
    }
    return v;
}

ALWAYS_INLINE int64_t FN(nbr)(const ocpu_params* p, int x, int y, int z, int dx, int dy, int dz) {
    const int xx = FN(wrap)(x + dx, p->n[0], p->periodic[0]);
    const int yy = FN(wrap)(y + dy, p->n[1], p->periodic[1]);
    const int zz = FN(wrap)(z + dz, p->n[2], p->periodic[2]);
    return (int64_t)(xx + 1) + (int64_t)(yy + 1) * p->sy + (int64_t)(zz + 1) * p->sz;
}

ALWAYS_INLINE int FN(flag_at)(const ocpu_params* p, const uint8_t* fl, int x, int y, int z, int dx, int dy, int dz) {
    const int xx = FN(wrap)(x + dx, p->n[0], p->periodic[0]);
    const int yy = FN(wrap)(y + dy, p->n[1], p->periodic[1]);
    const int zz = FN(wrap)(z + dz, p->n[2], p->periodic[2]);
    return fl[(xx + 1) + (int64_t)(p->n[0] + 2) * ((yy + 1) + (int64_t)(p->n[1] + 2) * (zz + 1))];
}

/* Method constants in the arithmetic type, loaded once per sweep. */
typedef struct {
    real w[27], lin[27][3], quad[27][6];
    real we, wo;              /* TRT even / odd rates; cumulant shear / bulk rates */
    real F[3];
    int compressible, galilean;
} FN(consts);

static void FN(load_consts)(const ocpu_params* p, FN(consts)* k) {
    int i, a;
    for (i = 0; i < 27; ++i) {
        k->w[i] = (real)p->w[i];
        for (a = 0; a < 3; ++a) k->lin[i][a] = (real)p->eq_lin[i][a];
        for (a = 0; a < 6; ++a) k->quad[i][a] = (real)p->eq_quad[i][a];
    }
    k->we = (real)p->omega_even;
    k->wo = (real)p->omega_odd;
    for (a = 0; a < 3; ++a) k->F[a] = (real)p->force[a];
    k->compressible = p->compressible;
    k->galilean = p->galilean;
}

/* Collision cores: once on scalars (single cells), once on 32-byte vectors of x-adjacent cells. */
typedef real FN(vreal) __attribute__((vector_size(32), aligned(sizeof(real))));
#define VLEN ((int)(32 / sizeof(real)))
#define VT real
#define CORE(name) CAT(name, CAT(s, SUFFIX))
#define SPLAT(v) ((real)(v))
#include "lbm_cpu_core.h"
#undef VT
#undef CORE
#undef SPLAT
#define VT FN(vreal)
#define CORE(name) CAT(name, CAT(v, SUFFIX))
#define SPLAT(v) ((VT){0} + (real)(v))
#include "lbm_cpu_core.h"
#undef VT
#undef CORE
#undef SPLAT
#define SCORE(name) CAT(name, CAT(s, SUFFIX))
#define VCORE(name) CAT(name, CAT(v, SUFFIX))

/* Rows (y, z) whose cells x in [1, nx-2] have no boundary cell among their neighbours: those
 * cells take the straight-line path with the row's constant offsets.  1 byte per row. */
static unsigned char* FN(fast_rows)(const ocpu_params* p, const uint8_t* flags) {
    const int nx = p->n[0], ny = p->n[1], nz = p->n[2];
    unsigned char* fast = (unsigned char*)malloc((size_t)ny * nz);
    int z;
    if (fast == NULL) return NULL;
#pragma omp parallel for schedule(static)
    for (z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y) {
            int ok = nx >= 3;
            for (int dz = -1; dz <= 1 && ok && flags; ++dz)
                for (int dy = -1; dy <= 1 && ok; ++dy)
                    for (int x = 0; x < nx && ok; ++x)
                        if (FN(flag_at)(p, flags, x, y, z, 0, dy, dz) & 7) ok = 0;
            fast[(size_t)y + (size_t)ny * z] = (unsigned char)ok;
        }
    return fast;
}

/* Row offsets of the neighbour rows: dy[1 + cy] * sy + dz[1 + cz] * sz, periodic axes wrapped. */
static void FN(row_offsets)(const ocpu_params* p, int y, int z, int64_t oy[3], int64_t oz[3]) {
    int d;
    for (d = -1; d <= 1; ++d) {
        oy[d + 1] = (int64_t)(FN(wrap)(y + d, p->n[1], p->periodic[1]) - y) * p->sy;
        oz[d + 1] = (int64_t)(FN(wrap)(z + d, p->n[2], p->periodic[2]) - z) * p->sz;
    }
}

/* ------------------------------------------------------------------ TRT, pull, two fields */
/* One cell on the general path: wrapped indices, bounce-back read for wall neighbours. */
ALWAYS_INLINE void FN(trt_cell_general)(const ocpu_params* p, const FN(consts)* k, const int Q, const real* src,
                                        real* dst, const uint8_t* flags, int x, int y, int z) {
    const int64_t cell = (int64_t)(x + 1) + (int64_t)(y + 1) * p->sy + (int64_t)(z + 1) * p->sz;
    if (flags && (FN(flag_at)(p, flags, x, y, z, 0, 0, 0) & 7)) return;
    real f[27];
    for (int i = 0; i < Q; ++i) {
        const int fl = flags ? FN(flag_at)(p, flags, x, y, z, -DX[i], -DY[i], -DZ[i]) & 7 : 0;
        if (fl == 0) {
            f[i] = src[FN(nbr)(p, x, y, z, -DX[i], -DY[i], -DZ[i]) + (int64_t)i * p->sq];
        } else {   /* halfway bounce-back: this cell's own outgoing inv(i) */
            real v = src[cell + (int64_t)INV[i] * p->sq];
            if (fl == 2) {
                real rho = 1;
                if (p->compressible)
                    for (int q = 0; q < Q; ++q) rho += src[cell + (int64_t)q * p->sq];
                v += (real)6 * k->w[i] *
                     ((real)DX[i] * (real)p->ubb[0] + (real)DY[i] * (real)p->ubb[1] + (real)DZ[i] * (real)p->ubb[2]) *
                     rho;
            }
            f[i] = v;
        }
    }
    SCORE(trt_core)(f, Q, k, k->compressible);
    for (int i = 0; i < Q; ++i) dst[cell + (int64_t)i * p->sq] = f[i];
}

/* The straight-line path: one row segment, every offset a row constant (lbmpy's inner loop),
 * VLEN cells per vector operation. */
ALWAYS_INLINE void FN(trt_row)(const FN(consts)* k, const int Q, const real* restrict src, real* restrict dst,
                               int64_t row, int x0, int x1, const int64_t* ro, int64_t sq, const int comp) {
    int x = x0;
    for (; x + VLEN <= x1; x += VLEN) {
        FN(vreal) f[27];
#pragma GCC unroll 27
        for (int i = 0; i < Q; ++i) memcpy(&f[i], src + row + x + ro[i], sizeof(FN(vreal)));
        VCORE(trt_core)(f, Q, k, comp);
#pragma GCC unroll 27
        for (int i = 0; i < Q; ++i) memcpy(dst + row + x + (int64_t)i * sq, &f[i], sizeof(FN(vreal)));
    }
    for (; x < x1; ++x) {
        real f[27];
        for (int i = 0; i < Q; ++i) f[i] = src[row + x + ro[i]];
        SCORE(trt_core)(f, Q, k, comp);
        for (int i = 0; i < Q; ++i) dst[row + x + (int64_t)i * sq] = f[i];
    }
}

ALWAYS_INLINE void FN(trt_pull_q)(const ocpu_params* p, const int Q, const real* src, real* dst,
                                  const uint8_t* flags, const unsigned char* fast) {
    const int nx = p->n[0], ny = p->n[1], nz = p->n[2];
    FN(consts) k;
    FN(load_consts)(p, &k);
    int z;
#pragma omp parallel for schedule(static) collapse(2)
    for (z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y) {
            if (fast[(size_t)y + (size_t)ny * z]) {
                int64_t oy[3], oz[3], ro[27];
                FN(row_offsets)(p, y, z, oy, oz);
                for (int i = 0; i < Q; ++i) ro[i] = -DX[i] + oy[1 - DY[i]] + oz[1 - DZ[i]] + (int64_t)i * p->sq;
                const int64_t row = 1 + (int64_t)(y + 1) * p->sy + (int64_t)(z + 1) * p->sz;
                if (k.compressible) FN(trt_row)(&k, Q, src, dst, row, 1, nx - 1, ro, p->sq, 1);
                else FN(trt_row)(&k, Q, src, dst, row, 1, nx - 1, ro, p->sq, 0);
                FN(trt_cell_general)(p, &k, Q, src, dst, flags, 0, y, z);
                FN(trt_cell_general)(p, &k, Q, src, dst, flags, nx - 1, y, z);
            } else {
                for (int x = 0; x < nx; ++x) FN(trt_cell_general)(p, &k, Q, src, dst, flags, x, y, z);
            }
        }
}

void FN(ocpu_trt_pull)(const ocpu_params* p, const real* src, real* dst, const uint8_t* flags) {
    unsigned char* fast = FN(fast_rows)(p, flags);
    if (fast == NULL) return;
    if (p->q == 19) FN(trt_pull_q)(p, 19, src, dst, flags, fast);
    else FN(trt_pull_q)(p, 27, src, dst, flags, fast);
    free(fast);
}

/* ------------------------------------------------------------------ D3Q27 cumulant, AA */
/* AA accessors (fieldaccess.py:134-159): EVEN reads f[x](i) and writes f[x](inv i); ODD reads
 * f[x - c_i](inv i) and writes f[x + c_i](i).  A fluid cell whose neighbour x - c_i is a wall
 * reads instead where the previous step wrote this cell's direction inv(i). */
ALWAYS_INLINE void FN(cum_cell_general)(const ocpu_params* p, const FN(consts)* k, real* f, const uint8_t* flags,
                                        int parity, int x, int y, int z) {
    if (flags && (FN(flag_at)(p, flags, x, y, z, 0, 0, 0) & 7)) return;
    const int64_t cell = FN(nbr)(p, x, y, z, 0, 0, 0);
    real g[27];
    for (int i = 0; i < 27; ++i) {
        const int j = INV[i];
        const int fl = flags ? FN(flag_at)(p, flags, x, y, z, -DX[i], -DY[i], -DZ[i]) & 7 : 0;
        if (fl == 0) {
            g[i] = parity == 0 ? f[cell + (int64_t)i * p->sq]
                               : f[FN(nbr)(p, x, y, z, -DX[i], -DY[i], -DZ[i]) + (int64_t)j * p->sq];
        } else {
            /* previous step ODD wrote direction j of x at x + c_j (slot j); EVEN at x (slot i) */
            g[i] = parity == 0 ? f[FN(nbr)(p, x, y, z, -DX[i], -DY[i], -DZ[i]) + (int64_t)j * p->sq]
                               : f[cell + (int64_t)i * p->sq];
        }
    }
    SCORE(cum_core)(g, k, k->galilean);
    for (int i = 0; i < 27; ++i) {
        if (parity == 0) f[cell + (int64_t)INV[i] * p->sq] = g[i];
        else f[FN(nbr)(p, x, y, z, DX[i], DY[i], DZ[i]) + (int64_t)i * p->sq] = g[i];
    }
}

/* The straight-line path.  Within one sweep every location is read and written by one cell
 * only (the AA pattern's property), so the cells of a row are independent and VLEN of them go
 * through one vector operation. */
ALWAYS_INLINE void FN(cum_row)(const FN(consts)* k, real* f, int64_t row, int x0, int x1, const int64_t* ro,
                               const int64_t* wo, const int gal) {
    int x = x0;
    for (; x + VLEN <= x1; x += VLEN) {
        FN(vreal) g[27];
#pragma GCC unroll 27
        for (int i = 0; i < 27; ++i) memcpy(&g[i], f + row + x + ro[i], sizeof(FN(vreal)));
        VCORE(cum_core)(g, k, gal);
#pragma GCC unroll 27
        for (int i = 0; i < 27; ++i) memcpy(f + row + x + wo[i], &g[i], sizeof(FN(vreal)));
    }
    for (; x < x1; ++x) {
        real g[27];
        for (int i = 0; i < 27; ++i) g[i] = f[row + x + ro[i]];
        SCORE(cum_core)(g, k, gal);
        for (int i = 0; i < 27; ++i) f[row + x + wo[i]] = g[i];
    }
}

void FN(ocpu_cum_aa)(const ocpu_params* p, real* f, const uint8_t* flags, int parity) {
    const int nx = p->n[0], ny = p->n[1], nz = p->n[2];
    unsigned char* fast = FN(fast_rows)(p, flags);
    if (fast == NULL) return;
    FN(consts) k;
    FN(load_consts)(p, &k);
    int z;
#pragma omp parallel for schedule(static) collapse(2)
    for (z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y) {
            if (fast[(size_t)y + (size_t)ny * z]) {
                int64_t oy[3], oz[3], ro[27], wo[27];
                FN(row_offsets)(p, y, z, oy, oz);
                for (int i = 0; i < 27; ++i) {
                    if (parity == 0) {
                        ro[i] = (int64_t)i * p->sq;
                        wo[i] = (int64_t)INV[i] * p->sq;
                    } else {
                        ro[i] = -DX[i] + oy[1 - DY[i]] + oz[1 - DZ[i]] + (int64_t)INV[i] * p->sq;
                        wo[i] = DX[i] + oy[1 + DY[i]] + oz[1 + DZ[i]] + (int64_t)i * p->sq;
                    }
                }
                const int64_t row = 1 + (int64_t)(y + 1) * p->sy + (int64_t)(z + 1) * p->sz;
                if (k.galilean) FN(cum_row)(&k, f, row, 1, nx - 1, ro, wo, 1);
                else FN(cum_row)(&k, f, row, 1, nx - 1, ro, wo, 0);
                FN(cum_cell_general)(p, &k, f, flags, parity, 0, y, z);
                FN(cum_cell_general)(p, &k, f, flags, parity, nx - 1, y, z);
            } else {
                for (int x = 0; x < nx; ++x) FN(cum_cell_general)(p, &k, f, flags, parity, x, y, z);
            }
        }
    free(fast);
}

/* `steps` sweeps; pull alternates a -> b -> a and returns 1 when the result is in b. */
int FN(ocpu_run_trt_pull)(const ocpu_params* p, real* a, real* b, const uint8_t* flags, int steps) {
    int t, in_b = 0;
    for (t = 0; t < steps; ++t) {
        if (in_b) FN(ocpu_trt_pull)(p, b, a, flags);
        else FN(ocpu_trt_pull)(p, a, b, flags);
        in_b ^= 1;
    }
    return in_b;
}

/* `steps` AA sweeps starting at `parity`; returns the parity of the next step. */
int FN(ocpu_run_cum_aa)(const ocpu_params* p, real* f, const uint8_t* flags, int parity, int steps) {
    int t;
    for (t = 0; t < steps; ++t) {
        FN(ocpu_cum_aa)(p, f, flags, parity);
        parity ^= 1;
    }
    return parity;
}

int FN(ocpu_sizeof_params)(void) { return (int)sizeof(ocpu_params); }
