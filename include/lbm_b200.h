/*
 * lbm_b200.h -- C ABI of the B200 lattice Boltzmann sweep (liblbmb200.so).
 *
 * The library replaces the kernels that lbmpy generates and JIT-compiles through pystencils
 * (paths relative to src/lbmpy of mabau/lbmpy).  Every entry point returns 0 on success and a
 * non-zero LBM_E_* status otherwise; lbm_last_error() then holds a message.  All pointers
 * passed as PDF / flag / macroscopic fields are device pointers owned by the caller; the
 * library borrows them for the duration of the call.  Kernels are enqueued on `stream`
 * (a cudaStream_t, NULL = legacy default stream) and the calls return without waiting,
 * except lbm_reduce_conserved, which waits for its result.
 *
 * PDF field layout (lbmpy's, creationfunctions.py:605-618 and updatekernels.py:146-163):
 * interior domain nx*ny*nz plus one ghost layer per side, PDF index q in lbmpy's 'walberla'
 * direction order (stencils.py:193-227).  Element (x, y, z, q) with x, y, z in [0, n+2)
 * (ghost-inclusive coordinates) lives at  base + x + y*sy + z*sz + q*sq  elements; the x stride
 * must be 1 and sy, sz, sq are passed in `strides` = {1, sy, sz, sq}.
 *
 * Flag field (optional): uint8 over the ghost-inclusive domain, x fastest, contiguous:
 * index x + (nx+2)*(y + (ny+2)*z).  Low 4 bits: 0 fluid, 1 NoSlip, 2..5 UBB number 0..3,
 * 6 / 7 FixedDensity (density `fixed_density` / `fixed_density1` of the plan);
 * bit 7 marks fluid cells with a boundary neighbour (lbm_flags_finalize sets it).
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    LBM_OK = 0,
    LBM_E_INVALID = 1,      /* argument rejected on the host (shape, stride, dtype, null pointer) */
    LBM_E_CUDA = 2,         /* a CUDA call failed */
    LBM_E_UNSUPPORTED = 3,  /* method / pattern / dtype combination not built */
    LBM_E_DEVICE = 4        /* pointer or plan used on a different device than the plan's */
};

enum { LBM_STENCIL_D3Q19 = 19, LBM_STENCIL_D3Q27 = 27 };
/* CENTRAL_MOMENT: D3Q27 polynomial central moments relaxed about the equilibrium velocity
 * (methods/momentbased/centralmomentbasedmethod.py:296-394), compressible, force models Guo / Luo /
 * Simple applied in central-moment space; rates in the cumulant method's canonical order. */
enum { LBM_METHOD_SRT = 0, LBM_METHOD_TRT = 1, LBM_METHOD_MRT = 2, LBM_METHOD_CUMULANT = 3,
       LBM_METHOD_CENTRAL_MOMENT = 4 };
/* E3M12: 16-bit float for zero-centred PDFs (sign, 3 exponent, 12 mantissa bits, scaled by 16;
 * |value| < 1/16, relative step 2^-12, saturating); no lbmpy counterpart (lbmpy stores FP64 / FP32). */
enum { LBM_DTYPE_F64 = 0, LBM_DTYPE_F32 = 1, LBM_DTYPE_F16 = 2, LBM_DTYPE_BF16 = 3, LBM_DTYPE_E3M12 = 4 };
/* pull / push: two fields; AA, EsoTwist, EsoPull, EsoPush: in place (fieldaccess.py:66-318).
 * Push, EsoPull and EsoPush are built for FP64 / FP32 storage. */
enum { LBM_PATTERN_PULL = 0, LBM_PATTERN_AA = 1, LBM_PATTERN_ESOTWIST = 2, LBM_PATTERN_PUSH = 3,
       LBM_PATTERN_ESOPULL = 4, LBM_PATTERN_ESOPUSH = 5 };
enum { LBM_FORCE_NONE = 0, LBM_FORCE_GUO = 1, LBM_FORCE_CENTRAL_MOMENT = 2, LBM_FORCE_SIMPLE = 3,
       LBM_FORCE_LUO = 4 };
enum { LBM_SGS_NONE = 0, LBM_SGS_SMAGORINSKY = 1, LBM_SGS_MLP = 2 };

/* Everything a sweep needs, resolved on the host by the lbmpy-compatible front end
 * (LBMConfig.__post_init__, creationfunctions.py:347-484, and create_lb_method, :773-868). */
typedef struct LbmPlanDesc {
    int32_t stencil;            /* LBM_STENCIL_* */
    int32_t method;             /* LBM_METHOD_* */
    int32_t store_dtype;        /* LBM_DTYPE_*: PDF storage; arithmetic is FP64 for F64, else FP32 */
    int32_t pattern;            /* LBM_PATTERN_* */
    int32_t compressible;
    int32_t continuous_equilibrium; /* SRT/TRT: 1 continuous Maxwellian (lbmpy default), 0 discrete */
    double rates[27];           /* SRT: {w, w}; TRT: {w+, w-}; MRT / cumulant: one per moment in the
                                   canonical order of the method's moment (cumulant) basis */
    int32_t force_model;        /* LBM_FORCE_* */
    double force[3];
    int32_t galilean_correction;
    int32_t sgs;                /* LBM_SGS_* */
    double sgs_constant;
    double shear_rate;          /* rate whose moments the SGS model adapts */
    uint32_t sgs_mask;          /* bit k: moment k (SRT/TRT: bit0 even, bit1 odd) uses the shear rate */
    double ubb_velocity[4][3];  /* wall velocity of UBB numbers 0..3 */
    int32_t dims[3];            /* interior cells nx, ny, nz */
    int32_t periodic[3];
    double fixed_density;       /* wall density of FixedDensity cells (flag type 6); 0: none
                                   (boundaries/boundaryconditions.py:1044-1099) */
    double fixed_density1;      /* wall density of FixedDensity cells of flag type 7 (a second outlet
                                   or inlet density, create_channel(pressure_difference=...),
                                   scenarios.py:137-142); 0: none */
    double ubb_density[4];      /* prescribed wall density of UBB number u for compressible methods;
                                   0: the fluid cell's density (UBB(density=...),
                                   boundaries/boundaryconditions.py:824-830) */
    uint32_t ubb_adapt_mask;    /* bit u: UBB number u shifts its wall velocity by -F/(2 rho_ref)
                                   (UBB(adapt_velocity_to_force=True), :790-794) */
    double fourth_order_limiter; /* CUMULANT: > 0 applies the fourth-order correction (Geier et al.
                                   2017; LBMConfig(fourth_order_correction=...),
                                   methods/cumulantbased/fourth_order_correction.py:21-237) with this
                                   limiter (lbmpy: 1e6 for True).  The rates of the third-order groups
                                   (canonical 10-16) are then derived from the shear rate (rates[4])
                                   and the bulk rate (rates[9]), those of orders 4-6 are 1. */
} LbmPlanDesc;

typedef struct LbmPlan LbmPlan;

/* Validates `desc` and prepares a plan on the current CUDA device.
 * Replaces create_lb_function's code generation (creationfunctions.py:543-559). */
int lbm_plan_create(const LbmPlanDesc* desc, LbmPlan** out);
int lbm_plan_destroy(LbmPlan* plan);

/* Updates the physical parameters (rates, force, UBB velocities) of an existing plan without
 * rebuilding it; the pystencils kernel took these as kernel keyword arguments
 * (lbstep.py:269,280 `run_kernel(..., **kernel_params)`). */
int lbm_plan_update(LbmPlan* plan, const LbmPlanDesc* desc);

/* One fused stream-collide sweep.  Replaces the compiled kernel create_lb_function returns
 * (creationfunctions.py:543-559), called as kernel(src=..., dst=...) by
 * LatticeBoltzmannStep.time_step (lbstep.py:271-282), together with the boundary handling
 * (boundaries/boundaryhandling.py:15-155) and periodic synchronisation it runs before the
 * sweep.  Two-field pull / push: src != dst.  In-place AA / EsoTwist / EsoPull / EsoPush:
 * src == dst and `parity` is the parity of THIS step (0 = EVEN, 1 = ODD;
 * advanced_streaming/utility.py:18-38).
 * omega_out (optional, float32, nx*ny*nz x-fastest) receives the effective shear rate. */
int lbm_sweep(const LbmPlan* plan, const void* src, void* dst, const int64_t strides[4],
              const uint8_t* flags, int parity, float* omega_out, void* stream);

/* Device status word of the plan, OR-ed by its sweeps since the last clear: 0 when every sweep
 * ran to completion, LBM_STATUS_STAGE_TIMEOUT when a staged sweep gave up waiting for a
 * shared-memory stage (its CTA left the rest of its cells un-updated).  Synchronises the device.
 * lbmpy's generated kernels have no such word; it is the only way a sweep that must bound its
 * waits reports that it stopped early.  clear != 0 resets it after reading. */
#define LBM_STATUS_STAGE_TIMEOUT 1u
int lbm_plan_status(LbmPlan* plan, uint32_t* status, int clear);

/* Which kernel lbm_sweep runs for these arguments: one cell per thread, two or four x-adjacent
 * cells per thread, the row-staged sweep (shared-memory stages filled by bulk copies), or the
 * pipelined z-column sweep (a column of cells per thread, the next cell's loads in flight during
 * the current collision; D3Q27 cumulant FP32).  All give lbmpy's update; the choice follows
 * storage type, method, alignment and the environment overrides LBM_B200_PAIR / LBM_B200_QUAD /
 * LBM_B200_STAGED ("0" never, "1" when applicable) and LBM_B200_ZPIPE (cells per thread, >= 2).
 * Diagnostic: lbmpy has one generated kernel per configuration and no such query. */
#define LBM_VARIANT_CELL 0
#define LBM_VARIANT_PAIR 1
#define LBM_VARIANT_QUAD 2
#define LBM_VARIANT_STAGED 3
#define LBM_VARIANT_ZPIPE 4
int lbm_sweep_variant(const LbmPlan* plan, const void* src, const void* dst, const int64_t strides[4],
                      int parity, const float* omega_out, int* variant);

/* Runs `steps` sweeps; for pull / push the fields alternate a->b->a..., for in-place patterns
 * `a` is updated starting at parity `first_parity`.  Sets *result_in_b for pull. */
int lbm_run(const LbmPlan* plan, void* a, void* b, const int64_t strides[4], const uint8_t* flags,
            int first_parity, int steps, int* result_in_b, void* stream);

/* Equilibrium initialisation through the write accessor of the previous step
 * (macroscopic_value_kernels.py:29-45, compile_macroscopic_values_setter :170-242).
 * rho / u element type: double (for every storage type; the equilibrium is evaluated in FP64).
 * rho_strides: x, y, z; u_strides: x, y, z, component (elements). */
int lbm_set_equilibrium(const LbmPlan* plan, void* pdfs, const int64_t strides[4], const void* rho,
                        const int64_t rho_strides[3], const void* u, const int64_t u_strides[4],
                        int prev_parity, void* stream);

/* Density and velocity from the values the previous step wrote
 * (macroscopic_value_kernels.py:48-61, compile_macroscopic_values_getter :88-167).
 * rho / u element type: double for F64 storage, float otherwise; either may be NULL. */
int lbm_get_macroscopic(const LbmPlan* plan, const void* pdfs, const int64_t strides[4], void* rho,
                        const int64_t rho_strides[3], void* u, const int64_t u_strides[4],
                        int prev_parity, void* stream);

/* FP64 sums over fluid cells: out[0] mass, out[1..3] momentum (rho_ref * u incl. the force
 * shift), out[4] kinetic energy.  No lbmpy counterpart (lbmpy reduces on the host through
 * pystencils' data handling, lbstep.py:400); waits for the result. */
int lbm_reduce_conserved(const LbmPlan* plan, const void* pdfs, const int64_t strides[4],
                         const uint8_t* flags, int prev_parity, double out[5], void* stream);

/* Same sums as lbm_reduce_conserved, for callers that cannot allocate device memory: it takes
 * the plan description instead of a plan and keeps its partial sums in a static device array of
 * 2048 x 5 doubles (80 KiB per GPU, resident until exit), calling no cudaMalloc / cudaFree.
 * No counterpart in the reference.  Fails with LBM_E_INVALID if the launch would need more than
 * 2048 partial sums (more than 512 SMs).  Calls that overlap on the GPU share the array and race.
 * The first call on a device resolves the array's address and, with lazy module loading, may
 * load the library's module there (reserving the 80 KiB array and the code): make it at start-up.
 * Waits for its result, so it cannot be captured into a CUDA graph. */
int lbm_reduce_conserved_noalloc(const LbmPlanDesc* desc, const void* pdfs, const int64_t strides[4],
                                 const uint8_t* flags, int prev_parity, double out[5], void* stream);

/* Per-link data of the boundary conditions that differ from link to link.  No single lbmpy
 * counterpart: lbmpy keeps such data in the index array of each boundary kernel
 * (boundaries/boundaryhandling.py:15-199), filled by the boundary's init callback:
 *   UBB(velocity=callback)          the wall velocity of each link (boundaryconditions.py:747-799,
 *                                   geometry.py:36-86);
 *   FreeSlip, SimpleExtrapolationOutflow, ExtrapolationOutflow (flag types 8, 9, 10): the cell and
 *                                   direction the incoming population is copied from
 *                                   (:360-455, :844-889, :894-1041), packed as
 *                                   dir | (ox+1) << 8 | (oy+1) << 10 | (oz+1) << 12;
 *   ExtrapolationOutflow            its two stored populations per link (pdf, pdf_nd), which the
 *                                   sweep reads and updates;
 *   NoSlipLinearBouzidi (type 11)   the wall distance q of each link (:142-212), in value [0].
 * Links are grouped by fluid cell: cell_block (int32 per interior cell, x fastest) gives the block
 * of the cell's links or -1; entry [b][q] belongs to the link from that cell in direction q
 * (towards the boundary cell).  All arrays are device memory owned by the caller and kept by the
 * plan until it is given other tables (or NULL to detach). */
typedef struct LbmLinkTables {
    const int32_t* cell_block;
    int64_t n_blocks;
    const double* ubb_velocity;  /* [n_blocks][Q][3], read for the UBB numbers in ubb_mask; may be NULL if 0 */
    uint32_t ubb_mask;           /* bit u: UBB number u takes its velocity from ubb_velocity */
    const int32_t* link_code;    /* [n_blocks][Q] or NULL */
    double* link_value;          /* [n_blocks][Q][2] or NULL; ExtrapolationOutflow's entries are updated */
} LbmLinkTables;
int lbm_plan_set_links(LbmPlan* plan, const LbmLinkTables* tables);

/* Sets bit 7 on every fluid cell of `flags` (device, layout above) that has a boundary
 * neighbour along the plan's stencil, honouring periodicity.  Replaces the link-list setup of
 * LatticeBoltzmannBoundaryHandling (boundaries/boundaryhandling.py:15-155).
 * It also records, in the plan, which interior rows (y, z) hold a non-zero flag; the plan's
 * sweeps given this same `flags` pointer skip the flag loads of the other rows.  Call it again
 * (with every plan that sweeps the field) after changing the field's contents. */
int lbm_flags_finalize(const LbmPlan* plan, uint8_t* flags, void* stream);

/* ---- Learned eddy-viscosity closure ----
 * sgs = LBM_SGS_MLP replaces the closed-form eddy viscosity of lbmpy's Smagorinsky model
 * (turbulence_models.py:25-84: omega = 2 / (tau0 + sqrt(18 C^2 Pi + tau0^2))) by a 10-32-32-1
 * perceptron evaluated per cell inside the D3Q27 cumulant sweep: omega = 1 / (tau0 + 3 nu_t) on
 * the moments in sgs_mask.  No lbmpy counterpart beyond that hook.  Parameter block: 1442 FP32
 * values, W1[10][32] b1[32] W2[32][32] b2[32] W3[32] b3 scale (nu_t = scale * softplus(y)). */

/* Uploads the parameters (host memory) that every closure sweep on the current device reads;
 * one set per device and process, ordered on `stream` before later launches.  A one-block kernel
 * on the same stream then packs them into the FP16 fragment layout the FP32 sweep reads. */
int lbm_closure_set_weights(const float* params, int n, void* stream);
/* Features of n cells from their state, SoA [10][n] device arrays: Pi_xx Pi_yy Pi_zz Pi_xy
 * Pi_xz Pi_yz (pre-collision non-equilibrium stress), rho, ux, uy, uz -> feats [10][n]. */
int lbm_closure_features(const float* state, int64_t n, float* feats, void* stream);
/* nu_t of n samples (feats [10][n]) with device parameters `params`. */
int lbm_mlp_forward(const float* params, const float* feats, int64_t n, float* nu, void* stream);

typedef struct LbmMlp LbmMlp;
/* Trainer state: partial-gradient scratch for up to max_blocks blocks. */
int lbm_mlp_create(int max_blocks, LbmMlp** out);
int lbm_mlp_destroy(LbmMlp* trainer);
/* loss = sum_n w_n (nu_n - t_n)^2 * inv_wsum and its gradient (1442 floats, the scale entry 0);
 * weight may be NULL (all 1); loss (one double, device) may be NULL.  Deterministic. */
int lbm_mlp_loss_grad(LbmMlp* trainer, const float* params, const float* feats, const float* target,
                      const float* weight, int64_t n, double inv_wsum, float* grad, double* loss, void* stream);
/* One Adam step (bias-corrected, step counts from 1) on the trained parameters, in place. */
int lbm_mlp_adam(const float* grad, float* params, float* m1, float* m2, double lr, double beta1, double beta2,
                 double eps, int step, void* stream);

/* ---- Batched domains: many independent fields of uneven size in one persistent launch ----
 * No single lbmpy counterpart: lbmpy runs one LatticeBoltzmannStep (lbstep.py:18-450) per
 * domain; a batch replaces a loop over such steps.  Every domain owns a ghost-layered field at
 * `offset` elements into each of the two shared buffers (pull ping-pongs between them; in-place
 * patterns use buffer a only), its flags at `flags_offset` bytes into the shared flag buffer
 * (-1: none; same layout as for lbm_sweep), and its own relaxation rates and UBB velocities.
 * Everything else (stencil, method, dtype, pattern, force, SGS) comes from `common`, whose
 * dims, periodic, rates and ubb_velocity are ignored. */
typedef struct LbmDomainDesc {
    int32_t dims[3];
    int32_t periodic[3];
    int64_t strides[4];         /* {1, sy, sz, sq} elements */
    int64_t offset;             /* element offset of the field in buffer a and in buffer b */
    int64_t flags_offset;       /* byte offset into the flag buffer, or -1 */
    double rates[27];
    double ubb_velocity[4][3];
} LbmDomainDesc;

typedef struct LbmBatch LbmBatch;

/* How the persistent launch walks the domains: blocks of tile_x x tile_y threads
 * (tile_x * tile_y <= 256), each thread updating up to cells_z cells along z, and
 * blocks_per_sm x (number of SMs) blocks striding over the tiles (0: one block per tile). */
typedef struct LbmBatchTiling {
    int32_t tile_x, tile_y, cells_z, blocks_per_sm;
} LbmBatchTiling;

/* Validates every domain (bounds inside buffers of buffer_elems elements and a flag buffer of
 * flags_bytes bytes, no two domains overlapping), marks the near-wall cells of every domain's
 * flags in place (as lbm_flags_finalize), uploads the per-domain arguments and the tile table.
 * In-place patterns take buffer_b == NULL or buffer_a.  The buffers stay owned by the caller. */
int lbm_batch_create(const LbmPlanDesc* common, const LbmDomainDesc* domains, int n_domains, void* buffer_a,
                     void* buffer_b, int64_t buffer_elems, uint8_t* flags, int64_t flags_bytes,
                     const LbmBatchTiling* tiling, LbmBatch** out);
/* One sweep of every domain.  Pull: parity 0 reads a and writes b, parity 1 the reverse.
 * AA: the parity of this step.  Makes no host-side check or synchronisation, so it can be
 * captured in a CUDA graph. */
int lbm_batch_sweep(const LbmBatch* batch, int parity, void* stream);
/* info = {tiles, blocks launched, interior cells over all domains, thread slots (tiles x tile
 * cells)}. */
int lbm_batch_info(const LbmBatch* batch, int64_t info[4]);
int lbm_batch_destroy(LbmBatch* batch);

/* ---------------------------------------------------------------- sparse (list-based) domains
 * Replaces lbmpy's sparse kernels (sparse/update_rule_sparse.py:22-52 create_lb_update_rule_sparse,
 * :55-67 create_macroscopic_value_getter_sparse, :70-85 create_macroscopic_value_setter_sparse).
 * The cells are a list of n_cells (n_fluid fluid cells first, then boundary cells); PDF i of list
 * cell c is element c + i * n_cells of a PDF list.  `index` holds, for direction i = 1..Q-1 and
 * fluid cell c, at index[(i - 1) * n_fluid + c], the element that cell c pulls population i from
 * (lbmpy's SparseLbMapper.create_index_array (sparse/mapping.py:100-156), transposed from
 * [n_fluid][Q-1] to [Q-1][n_fluid]); n_cells * Q must fit 32 bits.  The plan gives the stencil,
 * method, rates, force, dtype (FP64 / FP32) and must use the pull pattern; its dims and flags
 * play no part.  Boundary cells are neither read nor written by the sweep. */
int lbm_sparse_sweep(const LbmPlan* plan, const void* src, void* dst, const uint32_t* index, int64_t n_fluid,
                     int64_t n_cells, void* stream);
/* Equilibrium of the fluid cells from rho[c] and u[k * n_fluid + c] (FP64 device arrays); the
 * velocity enters unshifted by the force, as lbmpy's sparse setter builds it. */
int lbm_sparse_set_equilibrium(const LbmPlan* plan, void* pdfs, const double* rho, const double* u,
                               int64_t n_fluid, int64_t n_cells, void* stream);
/* Velocity bounce-back on a PDF list before a sparse sweep (replaces the kernel lbmpy builds from
 * SparseLbBoundaryMapper(UBB(...)), sparse/mapping.py:157-247): link k is the fluid cell
 * links[n_links + k] with the direction links[k] (1..Q-1) pointing into the boundary cell
 * links[2 * n_links + k]; slot inv(d) of the boundary cell receives
 * f(c, d) - 6 w_d rho (c_d . velocity), rho the cell's density for compressible plans, else 1.
 * Directions outside 1..Q-1 are skipped. */
int lbm_sparse_ubb(const LbmPlan* plan, void* pdfs, const uint32_t* links, int64_t n_links, int64_t n_cells,
                   const double velocity[3], void* stream);
/* Density and velocity of the fluid cells into rho[c] and u[k * n_fluid + c] (FP64; either may
 * be NULL). */
int lbm_sparse_get_macroscopic(const LbmPlan* plan, const void* pdfs, double* rho, double* u, int64_t n_fluid,
                               int64_t n_cells, void* stream);

/* Staged sweep (LBM_VARIANT_STAGED): bound of each wait on a stage barrier, in ns (0: the default
 * of 1 s).  A wait that runs out makes the sweep set LBM_STATUS_STAGE_TIMEOUT in the plan's
 * status word (lbm_plan_status), leave the remaining cells of that CTA unswept and return.
 * probe != 0 makes every CTA also wait, before its last tile, on a barrier that nothing arrives
 * at, so that the bounded wait and the status report can be tested; 0 restores normal sweeps.
 * No lbmpy counterpart. */
int lbm_plan_set_stage_wait(LbmPlan* plan, uint64_t wait_ns, int probe);

/* ---------------------------------------------------------------- slab decomposition
 * Ghost-plane exchange of a z-slab (waLBerla-style block communication that lbmpy describes with
 * get_communication_slices, advanced_streaming/communication.py:122-183, for the z faces).  A job
 * copies slots slots[0..n_slots) of z-plane z (ghost-inclusive index, whole plane of
 * nx_ext x ny_ext cells including the x/y ghost layers) between the PDF field and `buffer`, where
 * element (k, y, x) sits at (k * ny_ext + y) * nx_ext + x: unpack == 0 packs the field into the
 * buffer, unpack != 0 the reverse.  One launch runs every job; jobs must not write the same
 * elements.  The field has Q = q slots of elem_size bytes (2, 4 or 8), nz_ext planes and the
 * fzyx element strides {1, sy, sz, sq}. */
#define LBM_HALO_MAX_JOBS 4
typedef struct LbmHaloJob {
    int32_t z;
    int32_t unpack;
    int32_t n_slots;
    int32_t slots[27];
    void* buffer;
} LbmHaloJob;
int lbm_halo_copy(void* pdfs, const int64_t strides[4], int32_t q, int32_t nx_ext, int32_t ny_ext, int32_t nz_ext,
                  int32_t elem_size, const LbmHaloJob* jobs, int32_t n_jobs, void* stream);

/* Copies the message of the last failed call on this thread into buf (NUL-terminated). */
int lbm_last_error(char* buf, size_t n);

/* Library version, for the loader's sanity check. */
int lbm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H */
