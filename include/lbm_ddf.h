/*
 * lbm_ddf.h — C ABI of the B200 double-distribution lattice Boltzmann engine
 * for 3D Rayleigh–Bénard convection (D3Q27 velocity populations f, D3Q27
 * temperature populations g).
 *
 * It replaces the single-GPU run surface of Summer536/LBM_DDF src/:
 *   - the compile-time fields of src/parameters.h:5-31      -> lbm_params
 *   - the derived globals of src/globals.cu:13-23            -> lbm_derive
 *   - initialize() / init_arrays, src/initial.cu:3-241       -> lbm_create,
 *     lbm_init_rest, lbm_init_conduction, lbm_init_temperature
 *   - the restart reader, src/initial.cu:110-205             -> lbm_load_ref_state
 *   - the six launches and two copies of one step,
 *     src/main.cu:27-46                                      -> lbm_step
 *   - output_nu / diag_flow / output_profile / output_flow /
 *     output_fg, src/output.cu:3-419 (src/rb3d.h:64-68)      -> lbm_get_observables,
 *     lbm_get_profile, lbm_store_ref_state
 *
 * Conventions, unlike the reference's exit(EXIT_FAILURE) on any error
 * (src/rb3d.h:71-79): every call returns an int status, LBM_OK (0) or a
 * negative LBM_ERR_*; lbm_last_error() gives a message for the calling
 * thread.  Cases are opaque handles owned by the library.  Host buffers are
 * owned by the caller.  `stream` arguments are cudaStream_t values (NULL is
 * the legacy default stream); calls that return host data synchronise that
 * stream.  One case must not be used from two host threads at once.
 *
 * Axes and layout follow the reference: x fastest, then y, then z; node
 * idx = (iz*LY + iy)*LX + ix; population ip of a reference-layout array at
 * ip*N + idx; y is vertical with the hot plate below iy = 0 and the cold
 * plate above iy = LY-1 (halfway walls).
 */
#ifndef LBM_DDF_H
#define LBM_DDF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_DDF_ABI_VERSION 3

/* status codes */
#define LBM_OK 0
#define LBM_ERR_ARG (-1)       /* bad argument or unsupported combination */
#define LBM_ERR_CUDA (-2)      /* a CUDA runtime call failed */
#define LBM_ERR_NOMEM (-3)     /* device or host allocation failed */
#define LBM_ERR_DIVERGED (-4)  /* NaN/Inf found in the state */
#define LBM_ERR_STATE (-5)     /* call not valid in the case's current state */

/* side walls (x and z faces) */
#define LBM_SIDES_WALL 0       /* closed box: no-slip, adiabatic (reference src/streaming.cu:59-124,183-250) */
#define LBM_SIDES_PERIODIC 1   /* x and z periodic; only the y plates are walls */

/* population storage in HBM; arithmetic is FP64 for F64 and FP32 otherwise */
#define LBM_STORE_F64 0
#define LBM_STORE_F32 1
#define LBM_STORE_F16S 2       /* FP16 of f_i/w_i and g_i/w_i - t0, stored as (f, g) pairs */
#define LBM_STORE_BF16S 3      /* BF16 of the same shifted values, stored as (f, g) pairs */

/* step kernels (same results, different data movement) */
#define LBM_KERNEL_AUTO 0      /* NODE (measured the fastest on B200) */
#define LBM_KERNEL_NODE 1      /* one node per thread, any grid and side-wall mode (16-bit
                                  storage with BGK collision: each node's update split
                                  over two warps, each taking half the populations) */
#define LBM_KERNEL_ROW 2       /* whole x-rows staged by bulk copies; FP32 or FP64 storage,
                                  periodic sides, 32 <= LX <= 256, LX*element size a
                                  multiple of 16 bytes */

/* collision models */
#define LBM_COLLISION_BGK 0          /* the reference's BGK (src/collision.cu:3-88); default */
#define LBM_COLLISION_REGULARIZED 1  /* regularised BGK (Latt and Chopard 2006): the relaxed
                                        non-equilibrium part projected on its second (f) and
                                        first (g) Hermite moments; same equilibria and force */

/* Run surface of src/parameters.h:8-26 plus the engine's own choices. */
typedef struct lbm_params {
    int32_t lx, ly, lz;        /* LX, LY, LZ (>= 2, 3, 2); y vertical */
    int32_t sides;             /* LBM_SIDES_* */
    int32_t storage;           /* LBM_STORE_* */
    int32_t device;            /* CUDA device ordinal */
    double rayleigh;           /* RAYLEIGH */
    double prandtl;            /* PRANDTL */
    double t_hot, t_cold;      /* T_HOT, T_COLD */
    double gravity, beta;      /* GRAVITY, BETA */
} lbm_params;

/* Derived parameters, src/globals.cu:13-23. */
typedef struct lbm_derived {
    double visc;               /* LY*sqrt(g*beta*dT*LY*Pr/Ra) */
    double tau;                /* 3*visc + 0.5 */
    double u0;                 /* sqrt(g*beta*dT*LY), free-fall velocity */
    double diff;               /* visc / Pr */
    double tauc;               /* 3*diff + 0.5 */
    double t0;                 /* (T_hot + T_cold) / 2 */
} lbm_derived;

/* Observables of the macroscopic fields at the current step.  u is the
 * reference's stored velocity sum(c f) + F/2 (src/macrovar.cu:28-30). */
typedef struct lbm_observables {
    int64_t step;              /* steps taken since the state was set */
    double nu_bulk;            /* 1 + <u_y T> LY / (kappa dT)      src/output.cu:228-233 */
    double nu_top, nu_bottom;  /* -<dT/dy>_plate LY / dT          src/output.cu:236-256 */
    double ke;                 /* 0.5 <|u|^2> */
    double re;                 /* sqrt(<|u|^2>) LY / visc */
    double ux_mean, uy_mean, uz_mean, phi_mean;  /* src/output.cu:24-34 */
    int32_t diverged;          /* 1 if any node had a NaN/Inf moment */
    int32_t reserved;
} lbm_observables;

/* One simulation case: its state and reduction buffers on p->device.  Calls
 * on one case come from one host thread at a time, and its GPU work runs in
 * the order of the streams it is given: work of one case enqueued on two
 * streams that may run at once races (the state, and the reduction rows of
 * lbm_step_observed, are the case's own).  Different cases are independent. */
typedef struct lbm_case lbm_case;

/* Message of the last failing call on this host thread ("" if none). */
const char *lbm_last_error(void);
int lbm_abi_version(void);

/* src/globals.cu:13-23.  Fails with LBM_ERR_ARG for a bad grid or parameters. */
int lbm_derive(const lbm_params *p, lbm_derived *out);

/* Device bytes a case with these parameters holds (populations, carried
 * temperature, reduction scratch), for admission against a memory budget.
 * The first lbm_step_observed call adds the rows of its in-kernel reduction
 * (13 doubles per 32 nodes, under 4 bytes per node) and one lbm_observables
 * per step of the longest call made. */
int lbm_case_bytes(const lbm_params *p, uint64_t *bytes);

/* Allocates a case on p->device (replaces the cudaMalloc calls of
 * src/initial.cu:5-18).  The state is undefined until an init or load call. */
int lbm_create(const lbm_params *p, lbm_case **out);
int lbm_destroy(lbm_case *c);

/* The init calls write the state with a kernel on `stream` and return once
 * it is written (like the reference's synchronous initialize()), so the
 * case can then be stepped on any stream. */

/* init_arrays, src/initial.cu:208-241: rho = 0, u = 0, phi = 0.5. */
int lbm_init_rest(lbm_case *c, void *stream);

/* Seeded conduction state: T = T_hot - (T_hot-T_cold)*iy/(LY-1) (the profile
 * of Parallel/initial.cu:89) + amplitude*(2u-1), u uniform in [0,1) from
 * splitmix64(splitmix64(seed) + idx); zero velocity; f = 0 and g_i = w_i T
 * (equilibria); carried previous temperature = T. */
int lbm_init_conduction(lbm_case *c, uint64_t seed, double amplitude, void *stream);

/* The same state from the caller's temperature field: zero velocity, f = 0,
 * g_i = w_i T and carried previous temperature = T, with T[idx] (idx =
 * (iz*LY + iy)*LX + ix, the reference's node order) copied from `temperature`
 * — host (pinned or pageable) or device memory, in the carried-temperature
 * type: double for F64 storage, float otherwise.  Memory the device can read
 * (its own, or page-locked host memory from cudaHostAlloc) is read by the
 * initialising kernel itself, the PCIe transfer overlapping the writes of the
 * populations; other memory is copied in first.  Returns with the state
 * written.  With the T that
 * lbm_init_conduction forms it gives that call's state bit for bit in F64
 * storage.  The reference starts from its rest state (init_arrays) or a
 * restart file only. */
int lbm_init_temperature(lbm_case *c, const void *temperature, void *stream);

/* Restart state from host FP64 arrays in the reference's file layout
 * (%09d.dat = rho,ux,uy,uz,phi and fg%09d.dat = f,g; src/initial.cu:110-205).
 * The engine keeps f, g and the previous-step temperature; the latter is
 * recovered from uy - sum(c_y f) = g*beta*(phi_prev - t0)/2.  rho, ux, uz
 * and phi are recomputed from f and g, as the reference's own files hold. */
int lbm_load_ref_state(lbm_case *c, const double *rho, const double *ux, const double *uy,
                       const double *uz, const double *phi, const double *f, const double *g);

/* Current state in the same layout: what output_flow and output_fg would
 * write at this step (src/output.cu:67-146, 379-419).  Any pointer may be
 * NULL to skip that field. */
int lbm_store_ref_state(lbm_case *c, double *rho, double *ux, double *uy, double *uz,
                        double *phi, double *f, double *g);

/* nsteps fused time steps (src/main.cu:27-46), enqueued on `stream`;
 * asynchronous. */
int lbm_step(lbm_case *c, int32_t nsteps, void *stream);

/* Device-side reduction of the observables at the current step; waits for
 * `stream`.  Returns LBM_ERR_DIVERGED (with *out filled) if a NaN/Inf was found. */
int lbm_get_observables(lbm_case *c, lbm_observables *out, void *stream);

/* Vertical profile at the current step, src/output.cu:336-368: for each iy,
 * out[5*iy + 0..4] = <ux>, <uy>, <uz>, <phi>, phi_rms over the xz plane.
 * out holds 5*LY doubles; waits for `stream`. */
int lbm_get_profile(lbm_case *c, double *out, void *stream);

/* Native checkpoint: the device state exactly as held (populations in the
 * case's storage format and current AA layout, the carried temperature, the
 * layout flag and the step count), for resuming a case later or evicting it
 * from HBM.  It has no counterpart in the reference, whose only checkpoint is
 * the FP64 restart pair above.  lbm_checkpoint_bytes gives the size;
 * lbm_save_state / lbm_restore_state copy to / from caller memory
 * (page-locked host memory makes the copies asynchronous) on `stream`;
 * save returns once the copy is enqueued, so the caller synchronises
 * `stream` before reading the buffer.  Restore needs a case created with the
 * same parameters. */
int lbm_checkpoint_bytes(const lbm_case *c, uint64_t *bytes);
int lbm_save_state(lbm_case *c, void *host, uint64_t bytes, void *stream);
int lbm_restore_state(lbm_case *c, const void *host, uint64_t bytes, void *stream);

/* Observables without allocating: the lbm_get_observables reduction over
 * populations the caller holds in memory of its own, for callers that may
 * not allocate device memory through this library (while a stream is being
 * captured, under a fixed HBM budget, or on a thread that must not block on
 * cudaMalloc / cudaFree).  No counterpart in the reference.
 *   f, g      27 population rows each, row k at base + k*pop_stride elements,
 *             in p->storage's format and in the layout `swapped` names
 *             (0 natural, 1 swapped; a case's layout is swapped after an odd
 *             number of steps from an init or load).  For F16S / BF16S the
 *             engine interleaves the two: one array of (f, g) pairs, row k
 *             at f + 2*k*pop_stride elements, node j's f at element 2j and
 *             its g at 2j + 1; g must be f + 1 element and pop_stride below
 *             477,218,589 (nine rows of pairs are indexed in 32 bits), else
 *             LBM_ERR_ARG; for F64 and F32, pop_stride is at most 2^40;
 *   phi_prev  previous-step temperature per node (double for F64, else float);
 *   out_dev   DEVICE memory for one lbm_observables, written on `stream`.
 * Enqueues two kernels on `stream` and returns without synchronising; the
 * caller reads out_dev after the stream.  The block partial sums go to a
 * fixed array inside the library (1184 rows of 13 doubles, 123 KB, held by
 * every GPU that loads the library until the process exits); the reduction
 * never runs more than 1184 blocks, so the array covers every grid the C ABI
 * accepts (fewer than 2^31 nodes).  Each call overwrites every row it reads,
 * so nothing has to be cleared between calls, but calls whose kernels
 * overlap on the GPU (other streams, other host threads) race on the array.
 * The first call on a device looks up the array's address; make that first
 * call before any stream capture.  It knows nothing of a case's history, so
 * for the state right after lbm_init_rest (step 0) it reports the mean
 * temperature from sum(g) = 0.5 - 2^-54 where lbm_get_observables reports
 * the rest state's stored 0.5. */
int lbm_observables_noalloc(const lbm_params *p, const void *f, const void *g, const void *phi_prev,
                            uint64_t pop_stride, int32_t swapped, int64_t step,
                            lbm_observables *out_dev, void *stream);

/* Device self-check of the division identity the FP64 path uses for its
 * constant divisors (a / b from the correctly rounded reciprocal with one
 * Markstein correction): counts, over n random dividends, the results that
 * differ from the GPU's correctly rounded division by `divisor`.  A
 * diagnostic with no counterpart in the reference; expected result 0. */
int lbm_selfcheck_division(int device, double divisor, uint64_t n, uint64_t seed, uint64_t *mismatches);

/* Advances nsteps steps and returns, in out[0 .. nsteps) (host memory), the
 * observables of every state the steps started from: out[i] is the state
 * after (initial step count + i) steps, as lbm_get_observables would report
 * it then.  Each step kernel reduces them from the moments it computes
 * anyway (in every storage format; for 16-bit BGK, half of each warp pair
 * of the split kernel), so the per-step observables cost no extra read of
 * the state (lbm_get_observables reads all populations once).  Call
 * lbm_get_observables for the state after the last step.  Node kernel only
 * (LBM_ERR_ARG if the case's step kernel is set to ROW); synchronises
 * `stream`; LBM_ERR_DIVERGED if any entry saw a NaN/Inf (all entries are
 * written).  The sums' order differs from lbm_get_observables', so results
 * agree to rounding.  No counterpart in the reference (src/main.cu runs
 * output_nu on stored fields every NNUOUT steps). */
int lbm_step_observed(lbm_case *c, int32_t nsteps, lbm_observables *out, void *stream);

/* lbm_step_observed without waiting: enqueues the steps and the copy of
 * their observables into out[0 .. nsteps) on `stream` and returns, so a
 * host loop keeps the GPU busy while it reads earlier entries.  `out` is
 * page-locked host memory (an asynchronous copy; pageable memory works but
 * the copy then blocks) or device memory; it is valid once the stream has
 * passed the call (synchronise it, or record an event after the call and
 * wait on that).  The caller checks out[i].diverged.  Successive calls on
 * one case reuse one device buffer in stream order, so they run on one
 * stream (or the caller orders the streams). */
int lbm_step_observed_async(lbm_case *c, int32_t nsteps, lbm_observables *out, void *stream);

/* Chooses the step kernel of a case (LBM_KERNEL_*); LBM_ERR_ARG if the case
 * cannot use it.  lbm_get_step_kernel reports the one lbm_step launches. */
int lbm_set_step_kernel(lbm_case *c, int32_t kind);
int lbm_get_step_kernel(const lbm_case *c, int32_t *kind);

/* Test hook of the row-staged kernel's bounded wait: its steps announce
 * `bytes` (a multiple of 16, at most 4096; 0 turns the hook off) more on
 * their shared-memory barrier than their bulk copies bring, so the copies
 * all land but the wait gives up, after one second, as it would if a copy
 * never arrived.  The kernel then sets the case's error flag and leaves
 * the step undone; the next lbm_get_observables returns LBM_ERR_CUDA ("a
 * step kernel gave up waiting ...") and the CUDA context stays usable.
 * The state after such a step is unspecified.  No counterpart in the
 * reference, which has no bounded waits. */
int lbm_debug_row_wait_extra_bytes(lbm_case *c, uint32_t bytes);

/* Chooses the collision model of a case (LBM_COLLISION_*; BGK at creation),
 * in effect from its next step.  The regularised model runs on the node
 * kernel (and in batches); LBM_ERR_ARG if the case's step kernel is set to
 * ROW.  No counterpart in the reference, which has BGK only. */
int lbm_set_collision(lbm_case *c, int32_t model);
int lbm_get_collision(const lbm_case *c, int32_t *model);

/* ---- batches: many cases advanced together ------------------------------
 * No counterpart in the reference, which runs one case per process.  A batch
 * holds cases (any grids, Ra, Pr) of one storage format, periodic sides, on
 * one device; it does not own them.  lbm_batch_step advances every member
 * by nsteps in one kernel launch per step (a CUDA graph of the launches is
 * captured on first use of a step count and replayed); each member's step
 * count and layout advance as with lbm_step, and a member's result is the
 * same alone or in any mix; members may differ in collision model.  A case
 * belongs to at most one batch.  Members stay usable with the single-case
 * calls that read them (observables, profile, store, save) on the same
 * stream; the calls that change a case's state or settings (init, load,
 * lbm_step, restore, lbm_set_collision) return LBM_ERR_STATE for a member
 * until it is removed.  Destroying a member removes it from its batch.  A
 * case right after lbm_init_rest must take its first step alone (its first
 * step uses the rest state's phi = 0.5). */
typedef struct lbm_batch lbm_batch;
int lbm_batch_create(int device, int32_t storage, lbm_batch **out);
int lbm_batch_destroy(lbm_batch *b);
int lbm_batch_add(lbm_batch *b, lbm_case *c);
int lbm_batch_remove(lbm_batch *b, lbm_case *c);
int lbm_batch_size(const lbm_batch *b, int32_t *members, uint64_t *nodes);
int lbm_batch_step(lbm_batch *b, int32_t nsteps, void *stream);
/* Observables of every member at its current step (as lbm_get_observables
 * would report each), enqueued on `stream` into out[0 .. members) in the
 * order the members were added (removals close the gaps), then returns
 * without synchronising: out (page-locked host memory for an asynchronous
 * copy, or device memory) is valid once the stream passes the call, and the
 * caller checks out[i].diverged.  Call it on the stream the batch steps on,
 * so it sees the steps enqueued before it.  It replaces one synchronising
 * lbm_get_observables per member (the reference reduces its one case on the
 * host, src/output.cu:148-280). */
int lbm_batch_observables(lbm_batch *b, lbm_observables *out, void *stream);
/* Launch shape: blocks of 128 or 256 threads, each tile 4 x block nodes of
 * one member; blocks_per_sm > 0 runs that many persistent blocks per SM
 * walking the tile list, 0 one block per tile; use_graph replays captured
 * graphs for multi-step calls. */
int lbm_batch_set_config(lbm_batch *b, int32_t block, int32_t blocks_per_sm, int32_t use_graph);
int lbm_batch_get_config(const lbm_batch *b, int32_t *block, int32_t *blocks_per_sm, int32_t *use_graph);
/* How a batch step is launched.  LBM_BATCH_TILES (the default): one
 * persistent kernel per group of members walks every member's tiles (the
 * launch shape above).  LBM_BATCH_PER_CASE: each member's own single-case
 * step kernel (the one lbm_step launches, its parameters in the constant
 * bank), the members spread over 8 streams forked from and joined to the
 * batch's stream, so in a captured graph they run as parallel branches;
 * results are bitwise those of lbm_step.  Both give every member the same
 * state. */
#define LBM_BATCH_TILES 0
#define LBM_BATCH_PER_CASE 1
int lbm_batch_set_launch(lbm_batch *b, int32_t launch);
int lbm_batch_get_launch(const lbm_batch *b, int32_t *launch);
/* Times every launch (the tile walk's shapes and the per-case launch) on
 * 2 x steps_per_trial real steps of the batch (all compute identical
 * per-node arithmetic for a member, so the steps count), keeps the fastest
 * and reports it (lbm_batch_get_launch tells which launch won);
 * steps_per_trial must be even. */
int lbm_batch_autotune(lbm_batch *b, int32_t steps_per_trial, void *stream, int32_t *block,
                       int32_t *blocks_per_sm, double *best_ms_per_step);

/* Parameters and step count of a case. */
int lbm_get_params(const lbm_case *c, lbm_params *p, lbm_derived *d, int64_t *step);

#ifdef __cplusplus
}
#endif

#endif
