// Shared definitions of the B200 lattice Boltzmann sweep: lattice traits, PDF storage
// conversions and the by-value argument block every kernel receives.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "lbm_tables.h"

namespace lbm {

enum StoreType : int { ST_F64 = 0, ST_F32 = 1, ST_F16 = 2, ST_BF16 = 3, ST_E3M12 = 4 };
// SRT/TRT | raw-moment MRT | cumulant | cumulant with every order >= 3 relaxed by 1 | with a learned
// closure | D3Q27 central moments
enum MethodKind : int { MK_POP = 0, MK_MRT = 1, MK_CUM = 2, MK_CUM1 = 3, MK_CUM1_MLP = 4, MK_CM = 5 };
enum PatternKind : int {
    PAT_PULL = 0, PAT_AA_EVEN = 1, PAT_AA_ODD = 2, PAT_ESO_EVEN = 3, PAT_ESO_ODD = 4,
    PAT_PUSH = 5, PAT_EPULL_EVEN = 6, PAT_EPULL_ODD = 7, PAT_EPUSH_EVEN = 8, PAT_EPUSH_ODD = 9
};

// Whether direction (x, y, z) sits at an even position of lbmpy's 'lehmann' ordering (stencils.py,
// D3Q19 / D3Q27 'lehmann', which lists each direction right before its inverse; the rest
// population is at position 0).  EsoPull / EsoPush (fieldaccess.py:184-318) stream the even ones
// on one side of the collision and the odd ones on the other.
LBM_HD constexpr bool lehmann_even(int x, int y, int z) {
    return (x == 0 && y == 0 && z == 0) || (x == -1 && y == 0 && z == 0) || (x == 0 && y == -1 && z == 0) ||
           (x == 0 && y == 0 && z == -1) || (x == -1 && y == -1 && z == 0) || (x == -1 && y == 0 && z == -1) ||
           (x == 0 && y == -1 && z == -1) || (x == -1 && y == 1 && z == 0) || (x == -1 && y == 0 && z == 1) ||
           (x == 0 && y == -1 && z == 1) || (x == -1 && y == -1 && z == -1) || (x == -1 && y == -1 && z == 1) ||
           (x == -1 && y == 1 && z == -1) || (x == 1 && y == -1 && z == -1);
}
enum ForceKind : int { FM_NONE = 0, FM_GUO = 1, FM_CENTRAL = 2, FM_SIMPLE = 3, FM_LUO = 4 };

// Cell flags (uint8, ghost-layered domain): low 4 bits = cell type, bit 7 = fluid cell with at
// least one boundary neighbour.  Type 0 fluid, 1 NoSlip, 2..5 UBB number (type - 2),
// 6 / 7 FixedDensity with the plan's first / second density, 8 FreeSlip, 9 SimpleExtrapolation-
// Outflow, 10 ExtrapolationOutflow, 11 NoSlipLinearBouzidi (the last four read per-link data).
constexpr int FLAG_TYPE_MASK = 15;
constexpr int FLAG_NEAR_WALL = 128;
constexpr int FLAG_NOSLIP = 1;
constexpr int FLAG_UBB0 = 2;
constexpr int MAX_UBB = 4;
constexpr int FLAG_FIXED_DENSITY = 6;
constexpr int FLAG_FIXED_DENSITY1 = 7;
constexpr int FLAG_FREE_SLIP = 8;
constexpr int FLAG_SIMPLE_OUTFLOW = 9;
constexpr int FLAG_OUTFLOW = 10;
constexpr int FLAG_BOUZIDI = 11;

// Per-link code of FreeSlip and the outflow conditions: the incoming population is the outgoing
// population `dir` of the cell at offset (ox, oy, oz) in {-1, 0, 1}^3 from the fluid cell:
// code = dir | (ox + 1) << 8 | (oy + 1) << 10 | (oz + 1) << 12.
LBM_HD constexpr int link_dir(int code) { return code & 0xff; }
LBM_HD constexpr int link_off(int code, int axis) { return ((code >> (8 + 2 * axis)) & 3) - 1; }

LBM_HD constexpr bool flag_is_ubb(int t) { return t >= FLAG_UBB0 && t < FLAG_UBB0 + MAX_UBB; }
LBM_HD constexpr bool flag_is_fixed_density(int t) { return t == FLAG_FIXED_DENSITY || t == FLAG_FIXED_DENSITY1; }

template <int Q> struct Lat;

template <> struct Lat<19> {
    static constexpr int Q = 19;
    LBM_HD static constexpr int cx(int i) { return lbm_tables::q19_cx(i); }
    LBM_HD static constexpr int cy(int i) { return lbm_tables::q19_cy(i); }
    LBM_HD static constexpr int cz(int i) { return lbm_tables::q19_cz(i); }
    LBM_HD static constexpr int inv(int i) { return lbm_tables::q19_inv(i); }
    LBM_HD static constexpr int pair(int p) { return lbm_tables::q19_pair(p); }   // p < (Q - 1) / 2
    LBM_HD static constexpr double w(int i) { return lbm_tables::q19_w(i); }
    LBM_HD static constexpr double eqlin(bool cont, int i, int a) {
        return cont ? lbm_tables::q19_eqlin_cont(i, a) : lbm_tables::q19_eqlin_disc(i, a);
    }
    LBM_HD static constexpr double eqquad(bool cont, int i, int a) {
        return cont ? lbm_tables::q19_eqquad_cont(i, a) : lbm_tables::q19_eqquad_disc(i, a);
    }
    LBM_HD static constexpr double M(int k, int i) { return lbm_tables::q19_mrt_M(k, i); }
    LBM_HD static constexpr bool Meven(int k) { return lbm_tables::q19_mrt_even(k) != 0; }
    LBM_HD static constexpr double fT(int k, int a) { return lbm_tables::q19_mrt_fT(k, a); }
    LBM_HD static constexpr double fB(int k, int a) { return lbm_tables::q19_mrt_fB(k, a); }
    LBM_HD static constexpr double fS(int k) { return lbm_tables::q19_mrt_fS(k); }
    LBM_HD static constexpr double Minv(int i, int k) { return lbm_tables::q19_mrt_Minv(i, k); }
    LBM_HD static constexpr double p0(int k) { return lbm_tables::q19_mrt_p0(k); }
    LBM_HD static constexpr double mlin(int k, int a) { return lbm_tables::q19_mrt_lin(k, a); }
    LBM_HD static constexpr double mquad(int k, int a) { return lbm_tables::q19_mrt_quad(k, a); }
};

template <> struct Lat<27> {
    static constexpr int Q = 27;
    LBM_HD static constexpr int cx(int i) { return lbm_tables::q27_cx(i); }
    LBM_HD static constexpr int cy(int i) { return lbm_tables::q27_cy(i); }
    LBM_HD static constexpr int cz(int i) { return lbm_tables::q27_cz(i); }
    LBM_HD static constexpr int inv(int i) { return lbm_tables::q27_inv(i); }
    LBM_HD static constexpr int pair(int p) { return lbm_tables::q27_pair(p); }   // p < (Q - 1) / 2
    LBM_HD static constexpr double w(int i) { return lbm_tables::q27_w(i); }
    LBM_HD static constexpr double eqlin(bool cont, int i, int a) {
        return cont ? lbm_tables::q27_eqlin_cont(i, a) : lbm_tables::q27_eqlin_disc(i, a);
    }
    LBM_HD static constexpr double eqquad(bool cont, int i, int a) {
        return cont ? lbm_tables::q27_eqquad_cont(i, a) : lbm_tables::q27_eqquad_disc(i, a);
    }
    LBM_HD static constexpr double M(int k, int i) { return lbm_tables::q27_mrt_M(k, i); }
    LBM_HD static constexpr bool Meven(int k) { return lbm_tables::q27_mrt_even(k) != 0; }
    LBM_HD static constexpr double fT(int k, int a) { return lbm_tables::q27_mrt_fT(k, a); }
    LBM_HD static constexpr double fB(int k, int a) { return lbm_tables::q27_mrt_fB(k, a); }
    LBM_HD static constexpr double fS(int k) { return lbm_tables::q27_mrt_fS(k); }
    LBM_HD static constexpr double Minv(int i, int k) { return lbm_tables::q27_mrt_Minv(i, k); }
    LBM_HD static constexpr double p0(int k) { return lbm_tables::q27_mrt_p0(k); }
    LBM_HD static constexpr double mlin(int k, int a) { return lbm_tables::q27_mrt_lin(k, a); }
    LBM_HD static constexpr double mquad(int k, int a) { return lbm_tables::q27_mrt_quad(k, a); }
};

// ------------------------------------------------------------------ storage conversions
template <class S, class R> struct Conv;
template <class R> struct Conv<double, R> {
    __device__ __forceinline__ static R ld(const double* p) { return (R)*p; }
    __device__ __forceinline__ static void st(double* p, R v) { *p = (double)v; }
};
template <class R> struct Conv<float, R> {
    __device__ __forceinline__ static R ld(const float* p) { return (R)*p; }
    __device__ __forceinline__ static void st(float* p, R v) { *p = (float)v; }
};
template <class R> struct Conv<__half, R> {
    __device__ __forceinline__ static R ld(const __half* p) { return (R)__half2float(*p); }
    __device__ __forceinline__ static void st(__half* p, R v) { *p = __float2half_rn((float)v); }
};
template <class R> struct Conv<__nv_bfloat16, R> {
    __device__ __forceinline__ static R ld(const __nv_bfloat16* p) { return (R)__bfloat162float(*p); }
    __device__ __forceinline__ static void st(__nv_bfloat16* p, R v) { *p = __float2bfloat16_rn((float)v); }
};

// e3m12: a 16-bit float for zero-centred PDFs, which stay far below 1 in magnitude: sign, 3 exponent
// bits and 12 mantissa bits, scaled by 16.  Code (s, E, M) holds (-1)^s (1 + M/4096) 2^(E-12) for
// E = 1..7 and (-1)^s M 2^-23 for E = 0 (gradual underflow), so |value| < 1/16 with a relative step
// of 2^-12 (IEEE half: 2^-10) down to 2^-11, and an absolute step of 2^-23 below.  Larger
// magnitudes saturate.  The bits are those of the FP32 number value * 2^-115 shifted right by 11:
// decoding is an integer shift and one FP32 multiply (the FP32 subnormal range carries E = 0),
// encoding one multiply, rounding to nearest even on the dropped 11 bits, and a clamp.
struct e3m12 {
    uint16_t bits;
};

#ifdef __CUDACC__   // device intrinsics; host-only builds of the collision code do not store e3m12
__device__ __forceinline__ float e3m12_decode(unsigned h) {
    const unsigned b = ((h & 0x7fffu) << 11) | ((h & 0x8000u) << 16);
    return __fmul_rn(__uint_as_float(b), 0x1p115f);
}

__device__ __forceinline__ unsigned e3m12_encode(float v) {
    const unsigned b = __float_as_uint(__fmul_rn(v, 0x1p-115f));
    const unsigned mag = b & 0x7fffffffu;
    const unsigned c = min((mag + 0x3ffu + ((mag >> 11) & 1u)) >> 11, 0x7fffu);
    return c | ((b >> 16) & 0x8000u);
}

template <class R> struct Conv<e3m12, R> {
    __device__ __forceinline__ static R ld(const e3m12* p) { return (R)e3m12_decode(p->bits); }
    __device__ __forceinline__ static void st(e3m12* p, R v) { p->bits = (uint16_t)e3m12_encode((float)v); }
};
#endif

// ------------------------------------------------------------------ kernel arguments
struct Physics {
    double rates[27];      // per moment (MRT), per polynomial cumulant, or [omega+, omega-] (SRT/TRT)
    double force[3];
    int force_model;
    int compressible;
    int continuous_eq;     // SRT/TRT equilibrium: continuous Maxwellian (1) or discrete (0)
    int sgs;               // 0 none, 1 Smagorinsky
    double sgs_c18;        // 18 * C^2
    double tau0;           // 1 / shear rate
    uint32_t sgs_mask;     // moments (or TRT parts) whose rate is the shear rate
    int galilean;
    double ubb[MAX_UBB][3];
    double fixed_density;  // wall density of FixedDensity cells of type 6 (0: none)
    double fixed_density1; // wall density of FixedDensity cells of type 7 (0: none)
    double ubb_density[MAX_UBB];  // prescribed wall density of UBB number u (0: the fluid cell's density)
    unsigned ubb_link_mask;       // bit u: UBB number u takes per-link velocities (SweepArgs::ubb_link_vel)
    unsigned ubb_adapt_mask;      // bit u: the wall velocity is shifted by -F / (2 rho_ref)
    double foc_limiter;           // > 0: fourth-order cumulant correction with this limiter
    double foc_a, foc_b;          // its parameters a and b (Geier et al. 2017, eq. 115-116)
};

struct Grid {
    int nx, ny, nz;        // interior cells
    int sy, sz;            // element strides of y and z (x stride is 1)
    unsigned sq;           // element stride between PDF slots (Q * sq < 2^32, checked by the host)
    int periodic;          // bit 0 x, bit 1 y, bit 2 z
    const uint8_t* flags;  // (nx+2)*(ny+2)*(nz+2), x fastest, or nullptr
    int fsy, fsz;          // flag strides
    // Bit y + ny*z set: interior row (y, z) holds a cell whose flag is non-zero (a boundary cell
    // or a fluid cell next to one).  nullptr: every row may.  Sweeps skip the flag loads of the
    // other rows, so that a fluid cell's populations are not held up behind its flag.
    const uint32_t* rowmask;
};

struct SweepArgs {
    Grid g;
    Physics p;
    const void* src;
    void* dst;
    float* omega_out;      // optional per-cell effective shear rate (interior, x fastest)
    int zc;                // closure sweep: consecutive z-planes per thread (next plane prefetched to L2)
    int stage_probe;       // staged sweep: before its last tile each CTA also waits on a barrier that
                           // nothing arrives at (exercises the bounded wait and the status report)
    unsigned long long stage_wait_ns;   // staged sweep: bound of each barrier wait (0: 1 s)
    const void* ubb_rho;   // compressible moving walls: previous-step density of the cells next to them
    unsigned* status;      // device status word of the plan (STATUS_* bits), or nullptr
    // Per-link boundary data: block index of each interior cell (x fastest, -1: none) and, per
    // block and link direction q (pointing from the fluid cell to the wall, lbmpy's `dir`):
    // the UBB velocity ubb_link_vel[(block * Q + q) * 3 + k], the code link_code[block * Q + q]
    // (FreeSlip, outflows) and two values link_value[(block * Q + q) * 2 + k] (Bouzidi: q;
    // ExtrapolationOutflow: the previous outgoing and interpolated populations, updated by the
    // sweep that reads them).
    const int* ubb_block;
    const double* ubb_link_vel;
    const int* link_code;
    double* link_value;
};

// Whether interior row (y, z) may hold a cell with a non-zero flag.
__device__ __forceinline__ bool row_flagged(const Grid& g, int y, int z) {
    if (g.rowmask == nullptr) return true;
    const unsigned r = unsigned(y) + unsigned(g.ny) * unsigned(z);
    return (g.rowmask[r >> 5] >> (r & 31u)) & 1u;
}

// Neighbour offsets in elements for c in {-1, 0, +1} along each axis, with periodic wrap.
struct NbrOffsets {
    int dx[3], dy[3], dz[3];
    __device__ __forceinline__ void init(const Grid& g, int x, int y, int z) {
        dx[1] = 0; dy[1] = 0; dz[1] = 0;
        dx[0] = (x == 0 && (g.periodic & 1)) ? g.nx - 1 : -1;
        dx[2] = (x == g.nx - 1 && (g.periodic & 1)) ? -(g.nx - 1) : 1;
        dy[0] = ((y == 0 && (g.periodic & 2)) ? g.ny - 1 : -1) * g.sy;
        dy[2] = ((y == g.ny - 1 && (g.periodic & 2)) ? -(g.ny - 1) : 1) * g.sy;
        dz[0] = ((z == 0 && (g.periodic & 4)) ? g.nz - 1 : -1) * g.sz;
        dz[2] = ((z == g.nz - 1 && (g.periodic & 4)) ? -(g.nz - 1) : 1) * g.sz;
    }
    __device__ __forceinline__ int off(int cx, int cy, int cz) const {
        return dx[cx + 1] + dy[cy + 1] + dz[cz + 1];
    }
};

}  // namespace lbm
