/* cavity.h -- C ABI of the B200 lattice-Boltzmann step for the 2D
 * differentially heated cavity (drop-in for bbrangeo/cfd_cavity's step).
 *
 * The reference exposes its step through the Rust type
 * `uniform::solver::CavitySolver` (src/uniform/solver.rs:35-104); it has no
 * FFI of its own.  Each entry point below replaces one method of that type,
 * or one direct field access its callers make, and names the reference
 * interface it stands for.  A Rust caller binds them with `extern "C"`
 * declarations of the same names and #[repr(C)] mirrors of the structs.
 *
 * Conventions
 *  - Every function returns an int status (CAV_OK = 0) and never aborts or
 *    traps; cav_last_error() gives a one-line message for the last failure
 *    on a handle.  The reference panics or exit()s instead
 *    (src/uniform/solver.rs:130-132, 152-154, 236-240; src/main.rs:209-276).
 *  - Host arrays are caller-owned, row-major k = iy*nx + ix (the reference
 *    index, src/uniform/solver.rs:224-226), FP64, copied synchronously.
 *  - Populations cross the ABI in the reference's AoS layout [k][9]; the
 *    direction order is D2Q9 rest, E, N, NE, NW, W, S, SW, SE
 *    (c_{i+4} = -c_i for i = 1..4).
 *  - One handle is driven by one host thread at a time; it owns one CUDA
 *    stream and all of its device buffers.  Results are deterministic (no
 *    floating-point atomics).
 */
#ifndef CAVITY_B200_H
#define CAVITY_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define CAV_OK 0
#define CAV_ERR_ARG 1      /* invalid argument or size                       */
#define CAV_ERR_TAU 2      /* tau+ or tau_t too close to 1/2 (solver.rs:152-154) */
#define CAV_ERR_DIVERGED 3 /* non-finite field (post.rs:406-411, main.rs:230-275) */
#define CAV_ERR_MAXU 4     /* max|u| above the 0.10 guard (main.rs:46, 209-228) */
#define CAV_ERR_TIMEOUT 5  /* a bounded device wait gave up                 */
#define CAV_ERR_CUDA 6     /* CUDA runtime error                             */
#define CAV_ERR_STATE 7    /* call not valid in the handle's current state   */
#define CAV_ERR_NOMEM 8    /* device allocation failed                       */
#define CAV_ERR_IO 9       /* snapshot file missing, unwritable or malformed */

/* ---- enumerations -------------------------------------------------------- */
/* Storage precision of the populations (arithmetic: FP64 for CAV_PREC_F64,
 * FP32 otherwise; every reduced format stores f_i - w_i). */
#define CAV_PREC_F64 0  /* FP64 f and g                                        */
#define CAV_PREC_F32 1  /* FP32 f - w and g                                    */
#define CAV_PREC_F16 2  /* binary16 f - w and g (scaled by 2^15)               */
#define CAV_PREC_BF16 3 /* bfloat16 f - w and g                                */
#define CAV_PREC_F16G 4 /* binary16 f - w, 16-bit fixed-point g               */
/* The same three 16-bit encodings with stochastic rounding of every value
 * the collision writes (unbiased; the random bits are a hash of seed, step
 * and node, so results are reproducible). */
#define CAV_PREC_F16SR 5
#define CAV_PREC_BF16SR 6
#define CAV_PREC_F16GSR 7

/* Initial temperature field. */
#define CAV_INIT_LINEAR 0 /* linear theta + noise, CavitySolver::new (solver.rs:159-176) */
#define CAV_INIT_ZERO 1   /* theta = 0 + noise (benchmark configurations)     */

/* Debug phases: the pub(crate) methods the reference tests call
 * (src/uniform/tests.rs:154-169). */
#define CAV_PHASE_COLLIDE 0     /* collide(step)               solver.rs:421-540 */
#define CAV_PHASE_STREAM 1      /* stream()                    solver.rs:838-913 */
#define CAV_PHASE_BOUNCE_BACK 2 /* apply_bounce_back()         solver.rs:920-946 */
#define CAV_PHASE_THERMAL_BC 3  /* apply_thermal_boundary_conditions() :951-988 */
#define CAV_PHASE_MACRO 4       /* update_macroscopic()        solver.rs:298-367 */
#define CAV_PHASE_NOSLIP 5      /* enforce_wall_velocity()     solver.rs:992-1009 */
/* step_arg + 1 passes of the fused step kernel's stream + boundary code with
 * the collision replaced by the identity, then macroscopic + no-slip: checks
 * the streaming / bounce-back / thermal-BC index maps of the production
 * kernel against stream() + apply_thermal_boundary_conditions() bit for bit. */
#define CAV_PHASE_FUSED_IDENTITY 6
/* step_arg steps of the fused step kernel's plane-channel variant: periodic
 * in y, bounce-back walls at x = 0 and nx-1 without the wall-velocity
 * override or thermal boundary conditions, body force rho * beta_eff along
 * +y in the TRT + Guo collision (Cs from the parameters), then the REF state
 * of the channel.  The reference's Poiseuille test of the forcing
 * (src/uniform/tests.rs:246-376) turned by 90 degrees; start it from
 * init_from_fields with rho = 1, u = 0, T = 1 (the first collision's force
 * is rho * beta_eff * T). */
#define CAV_PHASE_CHANNEL 7

/* ---- parameters ------------------------------------------------------------ */
/* Arguments of CavitySolver::new (src/uniform/solver.rs:108) plus the
 * B200-side choices.  Fill with cav_default_params() first. */
typedef struct cav_params {
    int32_t nx, ny;          /* nodes in x (width) and y (height)             */
    double ra, pr, cs, pr_t; /* Rayleigh, Prandtl, Smagorinsky Cs, turbulent Pr */
    double utarget;          /* velocity target of the nu calibration         */
    uint64_t seed;           /* xorshift64* seed of the initial noise         */
    int32_t jobs;            /* accepted for API parity; unused on the GPU    */
    double alpha_mult;       /* alpha multiplier                              */
    double nu_start_mult;    /* initial viscosity multiplier (spin-up ramp)   */
    int32_t has_nu_override; /* 1: use nu_override (the reference's --nu)     */
    double nu_override;
    int32_t init_mode;       /* CAV_INIT_*                                    */
    double noise_amp;        /* amplitude of the uniform noise (ref: 1e-3)    */
    int32_t geq_order;       /* 2: quadratic g equilibrium (default), 1: linear */
    const double* t_hot_profile; /* [ny] hot-wall theta per row, or NULL (+0.5) */
    double t_cold;           /* cold-wall theta (-0.5)                        */
    int32_t precision;       /* CAV_PREC_*                                    */
    int32_t device;          /* CUDA device ordinal                           */
} cav_params;

/* Solver scalars the reference callers read as pub fields
 * (src/main.rs:131-145: sim.nu, sim.alpha, sim.lbm.tau, ...). */
typedef struct cav_info {
    double nu, alpha, alpha_phys, beta_eff, lz, lx, tau, tau_t;
    int64_t time_step, spin_up_steps;
    int32_t nx, ny, pitch, precision;
} cav_info;

/* Diagnostics of the current state (src/uniform/post.rs, src/main.rs:168-276),
 * reduced on the device in FP64 with a fixed-order tree. */
typedef struct cav_diag_out {
    double nusselt_hot;           /* post.rs:68-78  (2nd link, Lz scale)   */
    double nusselt_cold;          /* post.rs:100-111                        */
    double nusselt_hot_wall_link; /* post.rs:87-97  (1st link)              */
    double total_mass;            /* solver.rs:1012-1014  sum rho           */
    double total_f_mass;          /* solver.rs:1018-1020  sum f             */
    double max_u;                 /* main.rs:209-214  max(|ux|,|uy|)        */
    double max_uy;                /* post.rs:153-155                        */
    double nu_t_max;              /* main.rs:172-175                        */
    double y_plus_hot;            /* post.rs:182-199                        */
    double nusselt_volume;        /* post.rs:117-134                        */
    int32_t finite;               /* post.rs:406-411  (1 = all finite, rho > 0) */
} cav_diag_out;

typedef struct cav_handle cav_handle;

/* Library version string. */
const char* cav_version(void);
/* Default parameters: the reference CLI defaults (src/cli.rs:94-130),
 * FP64 storage. */
int cav_default_params(cav_params* p);
/* CavitySolver::new (src/uniform/solver.rs:108-210). */
int cav_create(const cav_params* p, cav_handle** out);
int cav_destroy(cav_handle* h);
/* Message of the last failure on h (or of the last failed cav_create when h is NULL). */
const char* cav_last_error(const cav_handle* h);
/* CavitySolver::init_from_fields (src/uniform/solver.rs:232-262). */
int cav_init_from_fields(cav_handle* h, const double* rho, const double* ux, const double* uy,
                         const double* t);
/* n x CavitySolver::step (src/uniform/solver.rs:279-293). */
int cav_step(cav_handle* h, int64_t n);
/* Reads lbm.{rho,ux,uy,temperature}, nu_t, fy_node (any pointer may be NULL). */
int cav_get_fields(cav_handle* h, double* rho, double* ux, double* uy, double* t, double* nu_t,
                   double* fy);
/* Writes lbm.{rho,ux,uy,temperature} and fy_node (NULL = leave unchanged). */
int cav_set_fields(cav_handle* h, const double* rho, const double* ux, const double* uy,
                   const double* t, const double* fy);
/* Reads / writes lbm.f and lbm.g, AoS [k][9] (NULL = skip). */
int cav_get_populations(cav_handle* h, double* f, double* g);
int cav_set_populations(cav_handle* h, const double* f, const double* g);
/* Solver scalars (pub fields, src/uniform/solver.rs:35-104). */
int cav_get_info(cav_handle* h, cav_info* out);
/* Sets time_step (the spin-up ramps read it; solver.rs:67, 433). */
int cav_set_time_step(cav_handle* h, int64_t t);
/* Diagnostics of the current state. */
int cav_diag(cav_handle* h, cav_diag_out* out);
/* Guards of the driver loop (src/main.rs:209-276): CAV_ERR_MAXU when
 * max|u| > max_u_abort, CAV_ERR_DIVERGED when a field is not finite. */
int cav_check_guards(cav_handle* h, double max_u_abort);
/* One pub(crate) phase (CAV_PHASE_*); step_arg is collide's step index. */
int cav_debug_phase(cav_handle* h, int32_t phase, int64_t step_arg);

/* TimeAverager (src/uniform/post.rs:11-57) kept on the device in FP64.
 * cav_sample = averager.accumulate(&sim) (src/main.rs:279-281). */
int cav_sample(cav_handle* h);
int cav_reset_means(cav_handle* h);
/* means of ux, uy, T, nu_t, |u|^2 (post.rs:52-56); *n_samples may be NULL. */
int cav_get_means(cav_handle* h, double* ux, double* uy, double* t, double* nu_t, double* uu,
                  int64_t* n_samples);
/* nusselt_from_mean on the mean temperature (src/main.rs:740-753). */
int cav_nusselt_from_mean(cav_handle* h, int32_t hot, double* out);

/* Per-step Nusselt accumulation: while enabled, every completed step adds the
 * instantaneous nusselt_hot / nusselt_cold of the new state (post.rs:68-111)
 * to FP64 accumulators on the device. */
int cav_nu_accumulate(cav_handle* h, int32_t enable);
int cav_nu_accumulated(cav_handle* h, double* nu_hot_mean, double* nu_cold_mean, int64_t* n);

/* Blocks until all work queued on the handle's stream has finished. */
int cav_sync(cav_handle* h);
/* The handle's CUDA stream (cudaStream_t), for callers that time or order
 * their own work against the step (no counterpart in the reference). */
int cav_get_stream(cav_handle* h, void** stream);
/* Number of kernels the handle has launched so far (graph replays count
 * every kernel they contain; no counterpart in the reference). */
int cav_launch_count(cav_handle* h, int64_t* n);
/* Kernel of the fused step (no counterpart in the reference):
 * CAV_STEP_NODE one node per thread; CAV_STEP_PAIR two x-adjacent nodes per
 * thread, each plane one 32-bit word (16-bit formats only);
 * CAV_STEP_PAIR_SPLIT the same node pairs with the f and g halves of each
 * pair's work on two warps (twice the warps, each a shorter chain: for
 * cavities too small to fill the GPU).  Default for the 16-bit formats:
 * CAV_STEP_PAIR_SPLIT up to 70 000 nodes, CAV_STEP_PAIR above; FP64 / FP32:
 * CAV_STEP_NODE.  All give the same bits; CAV_ERR_ARG for a pair kernel on
 * FP64 / FP32. */
#define CAV_STEP_NODE 0
#define CAV_STEP_PAIR 1
#define CAV_STEP_PAIR_SPLIT 2
int cav_set_step_kernel(cav_handle* h, int32_t kernel);
int cav_get_step_kernel(cav_handle* h, int32_t* kernel);

/* ---- snapshots and restart ------------------------------------------------ */
/* CAVSNAP1 files of the reference (src/uniform/snapshot.rs:10-131): rho, ux,
 * uy, T in FP64, written atomically (temporary file + rename, as
 * write_snapshot_atomic).  Host-only, no device needed:
 *   cav_snapshot_write_fields  write_snapshot_atomic of caller arrays;
 *   cav_snapshot_read_fields   read_snapshot: call with NULL arrays to get
 *                              nx, ny, then with [nx*ny] arrays. */
int cav_snapshot_write_fields(const char* path, int64_t nx, int64_t ny, const double* rho, const double* ux,
                              const double* uy, const double* t);
int cav_snapshot_read_fields(const char* path, int64_t* nx, int64_t* ny, double* rho, double* ux, double* uy,
                             double* t);
/* The cavity's fields to a CAVSNAP1 file (the driver's --snapshot-every). */
int cav_snapshot_write(cav_handle* h, const char* path);
/* The driver's --restart (src/main.rs, solver.rs:232-262): read a CAVSNAP1
 * file, interpolate it bilinearly onto this cavity's grid when the sizes
 * differ (interpolate_field, snapshot.rs:102-131) and set the populations
 * to the equilibria of the fields (init_from_fields), all on the device;
 * the time step restarts at 0. */
int cav_restart_from_snapshot(cav_handle* h, const char* path);

/* ---- dynamic mixed-scale subgrid model (--dynamic-smag) ------------------ */
/* set_dynamic_sgs (src/uniform/solver.rs:215-220): on = 1 computes nu_t and
 * alpha_t per node before every collision with the dynamic mixed-scale model
 * (compute_dynamic_sgs, :562-828) instead of Cs^2 |S| and nu_t / Pr_t.
 * Reference defaults: smag_alpha 0.5, nu_sm_min -0.1, eta_test 2.0
 * (src/cli.rs:118-120).  A step then runs the model's four kernels, the
 * collision and the streaming as separate launches (no graph replay). */
int cav_set_dynamic_sgs(cav_handle* h, int32_t on, double smag_alpha, double nu_sm_min, double eta_test);
/* out4 = cs_dyn_mean, cs_dyn_max, kappa_dyn_mean, kappa_dyn_max of the last
 * evaluation (the driver's progress line, src/main.rs:181-182); zeros before
 * the first dynamic step. */
int cav_dynamic_sgs_stats(cav_handle* h, double* out4);

/* ---- adjoint: gradients of the time-averaged hot-wall Nusselt number ------ */
/* No counterpart in the reference (it has no gradients).  Objective
 * J = mean over s in [window_start, n_steps] of nusselt_hot (post.rs:68-78)
 * of the state after s steps.  Runs the forward from step 0 (the handle must
 * be fresh: just created or re-initialised with cav_init_from_fields),
 * storing the state every checkpoint_every steps, then the hand-written
 * adjoint backwards with checkpoint-and-recompute.  FP32 or FP64 storage.
 * The handle ends at step n_steps, exactly as after cav_step(h, n_steps). */
typedef struct cav_adjoint_spec {
    int64_t n_steps;          /* N                                          */
    int64_t window_start;     /* first state of the average (1 <= ws <= N)  */
    int32_t checkpoint_every; /* forward states kept every this many steps  */
} cav_adjoint_spec;
typedef struct cav_adjoint_result {
    double objective;  /* J                                                 */
    double grad_cs;    /* dJ/dCs                                            */
    double forward_ms; /* forward pass with checkpoints (device time)       */
    double reverse_ms; /* recomputation + adjoint sweep (device time)       */
    int64_t checkpoints;
} cav_adjoint_result;
/* grad_theta[ny] = dJ/dtheta_w[iy] for the hot-wall profile (cav_params.
 * t_hot_profile; rows 0 and ny-1 are never used by the boundary condition
 * and get 0). */
int cav_adjoint_run(cav_handle* h, const cav_adjoint_spec* spec, double* grad_theta, cav_adjoint_result* res);

/* ---- batches: many cavities, one launch per step ------------------------- */
/* No single counterpart in the reference, which runs one cavity per process
 * (src/main.rs:42-443); a batch is n CavitySolver::new + lockstep step()
 * calls.  Cavities may differ in size, Ra, Cs, seeds and wall profiles but
 * share one precision and one device.  Each cavity of a batch evolves
 * bit-identically to the same cavity created with cav_create. */
typedef struct cav_batch cav_batch;
/* kernel and the fields it uses (the others are ignored):
 *   0  persistent grid of ctas_per_sm x #SMs CTAs over 32-column x
 *      rows_per_item tiles, one thread per node;
 *   1, 2  TMA-staged shared-memory tiles in shape 1 or 2 (taller),
 *      ctas_per_sm persistent CTAs per SM (at most its resident CTAs);
 *   3  one CTA per 32-column x rows_per_item item (1, 2, 4 or 8 rows), one
 *      thread per node;
 *   4  the same items, two rows per thread on packed FP32x2 arithmetic
 *      (2, 4 or 8 rows; FP64 runs it as 3);
 *   5  one CTA per 64-column x rows_per_item item (1, 2, 4 or 8 rows), two
 *      x-adjacent nodes per thread, each plane one 32-bit word (16-bit
 *      formats; FP64 and FP32 run it as 3);
 *   6  the same node-pair body on TMA-staged shared-memory tiles of 64
 *      columns x rows_per_item rows (4 or 8), ctas_per_sm persistent CTAs per
 *      SM (16-bit formats; FP64 and FP32 run it as 3).
 * Default: kernel 3, 4 rows. */
typedef struct cav_batch_tuning {
    int32_t rows_per_item; /* item / tile height in rows                     */
    int32_t ctas_per_sm;   /* resident CTAs per SM of the persistent kernels */
    int32_t kernel;        /* 0..6, above                                    */
} cav_batch_tuning;
int cav_batch_create(const cav_params* params, int32_t n, cav_batch** out);
int cav_batch_destroy(cav_batch* b);
const char* cav_batch_last_error(const cav_batch* b);
/* n lockstep steps of every cavity (one kernel launch per step). */
int cav_batch_step(cav_batch* b, int64_t n);
int cav_batch_get_fields(cav_batch* b, int32_t i, double* rho, double* ux, double* uy, double* t,
                         double* nu_t, double* fy);
int cav_batch_get_populations(cav_batch* b, int32_t i, double* f, double* g);
int cav_batch_diag(cav_batch* b, int32_t i, cav_diag_out* out);
int cav_batch_info(cav_batch* b, int32_t* n_cavities, int64_t* total_nodes, int64_t* time_step);
/* Tile / grid shape: set by hand, or chosen by timing candidates on a twin
 * batch (the batch's own state is not advanced); the choice is cached per
 * grid class (precision + multiset of cavity sizes) for later batches. */
int cav_batch_get_tuning(cav_batch* b, cav_batch_tuning* t);
int cav_batch_set_tuning(cav_batch* b, const cav_batch_tuning* t);
int cav_batch_autotune(cav_batch* b, int32_t trial_steps, cav_batch_tuning* chosen);
int cav_batch_sync(cav_batch* b);
/* Test of the tile kernel's bounded waits (no counterpart in the reference):
 * with on = 1 the tile kernel arms its barriers but issues no copy, every
 * wait gives up after about a second and the next cav_batch_sync returns
 * CAV_ERR_TIMEOUT (the steps of those launches are lost); on = 0 restores
 * the copies.  Nothing is left in flight, the device stays usable. */
int cav_batch_debug_stall_copies(cav_batch* b, int32_t on);
int cav_batch_get_stream(cav_batch* b, void** stream);
int cav_batch_launch_count(cav_batch* b, int64_t* n);

/* ---- block-refined (octree) cavity: src/octree/ ------------------------- */
/* Replaces octree::solver::CavitySolver (src/octree/solver.rs:284-1206):
 *   cav_octree_create   CavitySolver::new (solver.rs:284-471), init_cavity
 *                       (:504-578)
 *   cav_octree_step     n x step_cavity (:647-947)
 *   cav_octree_diag     nusselt_hot / nusselt_hot_link0 / nusselt_cold /
 *                       nusselt_hot_fine (src/octree/cavity.rs:672-741),
 *                       max_u_all (solver.rs:1005-1016), noise_stats
 *                       (:954-1003), check_finite_levels (cavity.rs:751)
 *   cav_octree_check_guards  check_guards (solver.rs:1019-1038)
 *   cav_octree_get_level     the LbmLevel fields (src/octree/lbm.rs:19-53)
 * Levels are numbered 0 = coarse L0, 1 / 2 = hot / cold L1 blocks,
 * 3 / 4 = hot / cold L2 strips (levels = 3).  Populations cross the ABI as
 * the reference's AoS [k][9] FP64, k = b * nx + a. */
enum {
    CAV_OCT_F64 = 0,     /* FP64 everywhere (bit-identical to the FP64 oracle) */
    CAV_OCT_F32 = 1,     /* FP32 arithmetic and storage                        */
    CAV_OCT_F32_F16 = 2, /* FP32 arithmetic, FP32 L0, binary16 (stochastic
                            rounding) L1 / L2 populations                      */
    CAV_OCT_F32_F16G = 3 /* as CAV_OCT_F32_F16 with the L1 / L2 g populations
                            in 16-bit fixed point (CAV_PREC_F16GSR's format)   */
};
typedef struct cav_octree_params {
    int32_t nx0, ny0;      /* coarse grid                                       */
    int32_t bl_width;      /* L1 block width in coarse cells (--bl-width)       */
    double ra, pr, utarget;
    uint64_t seed;
    int32_t jobs;          /* accepted for signature parity; unused             */
    int32_t odd_exact;     /* xi_odd = tau-_f / tau-_c / 2 instead of 1/2       */
    int32_t levels;        /* 2 or 3                                            */
    double nu_start_mult;  /* viscosity ramp start multiplier (>= 1)            */
    int32_t has_nu_override;
    double nu_override;
    int32_t precision;     /* CAV_OCT_*                                         */
    int32_t device;
    /* Extension (no counterpart in the reference octree, which has no fixed
     * Smagorinsky model): cs > 0 adds nu_t = cs^2 |S| on every level, with
     * the uniform solver's collision and the level's lattice spacing.
     * cs = 0 (default) is the reference. */
    double cs, pr_t;
} cav_octree_params;
typedef struct cav_octree_info {
    double nu, alpha, beta_eff_coarse;
    double tau_plus[3];                       /* L0, L1, L2                     */
    double xi_even, xi_odd, xi_thermal;       /* interface L0 / L1              */
    double xi_even_sub, xi_odd_sub, xi_thermal_sub; /* interface L1 / L2        */
    int64_t time_step, spin_up_steps, n_nodes_total;
    int32_t levels, precision;
    int32_t nx[5], ny[5];                     /* per level (0 when absent)      */
    int32_t n_ghosts, n_coincident;           /* L1 blocks, summed over both    */
    int32_t n_ghosts_sub, n_coincident_sub;   /* L2 strips, summed over both    */
} cav_octree_info;
typedef struct cav_octree_diag_out {
    double nu_hot, nu_hot_link0, nu_cold; /* coarse, 2nd / 1st link, x Lx      */
    double nu_hot_fine;                   /* hot L1 block, x lx_coarse         */
    double max_u;                         /* all levels, max(|ux|, |uy|)       */
    double mass;                          /* mean coarse rho                   */
    double max_rho_dev, max_rho_dev_ifaces;
    double finite;                        /* 1.0 when every field is finite    */
    double y_plus_fine;                   /* post.rs:182-199 formula on the
                                             finest hot-wall level (the
                                             reference octree has no y+)       */
} cav_octree_diag_out;
typedef struct cav_octree cav_octree;
int cav_octree_default_params(cav_octree_params* p);
int cav_octree_create(const cav_octree_params* p, cav_octree** out);
int cav_octree_destroy(cav_octree* h);
const char* cav_octree_last_error(const cav_octree* h);
int cav_octree_step(cav_octree* h, int64_t n_coarse_steps);
int cav_octree_get_info(cav_octree* h, cav_octree_info* out);
/* Any output pointer may be NULL.  rho, ux, uy, t: [nx*ny]; f, g: [nx*ny][9]. */
int cav_octree_get_level(cav_octree* h, int32_t level, double* rho, double* ux, double* uy, double* t,
                         double* f, double* g);
/* Overwrites the given parts of a level's state (NULL = keep); the next step
 * starts with the collision of that state, as the reference's would. */
int cav_octree_set_level(cav_octree* h, int32_t level, const double* rho, const double* ux,
                         const double* uy, const double* t, const double* f, const double* g);
/* Restart injection of one level (set_from_snapshot, src/octree/solver.rs:
 * 1080-1168, same grid): the level's fields become rho, ux, uy, t [nx*ny],
 * its populations feq / geq of them, then its no-slip is applied to the
 * stored velocity.  Call it for every level, then cav_octree_set_time_step(h,
 * 0) as the reference does (the ramps restart). */
int cav_octree_restart_level(cav_octree* h, int32_t level, const double* rho, const double* ux,
                             const double* uy, const double* t);
int cav_octree_set_time_step(cav_octree* h, int64_t t);
/* OCTSNAP1 files (src/octree/snapshot.rs:58-170): every level's rho, ux, uy,
 * T and the step, written atomically; the restart (set_from_snapshot,
 * src/octree/solver.rs:1080-1168) requires the same level layout (else
 * CAV_ERR_ARG) and restarts the time step at 0. */
int cav_octree_snapshot_write(cav_octree* h, const char* path, uint64_t step);
int cav_octree_restart_from_snapshot(cav_octree* h, const char* path);
/* One coupling on the current state: 0 = coarse_to_fine L0 -> L1,
 * 1 = fine_to_coarse L1 -> L0 + moment refresh, 2 / 3 = the same between L1
 * and L2 (src/octree/interface.rs:137-206). */
int cav_octree_couple(cav_octree* h, int32_t which);
int cav_octree_diag(cav_octree* h, cav_octree_diag_out* out);
/* check_guards: CAV_OK, CAV_ERR_MAXU (max_u > max_u_abort) or
 * CAV_ERR_DIVERGED (a non-finite field). */
int cav_octree_check_guards(cav_octree* h, double max_u_abort);
int cav_octree_sync(cav_octree* h);
int cav_octree_get_stream(cav_octree* h, void** stream);
int cav_octree_launch_count(cav_octree* h, int64_t* n);
/* The fine levels' (L1, L2) step kernel, same results bit for bit:
 *   CAV_OCT_LEVEL_NODE one thread per node;
 *   CAV_OCT_LEVEL_FG   the default: a node's f and g halves on two threads
 *                      exchanging u, v, u^2 and T through shared memory
 *                      (shifted formats without the fixed-Cs extension and
 *                      outside the dynamic model; the rest run one thread
 *                      per node). */
#define CAV_OCT_LEVEL_NODE 0
#define CAV_OCT_LEVEL_FG 1
int cav_octree_set_level_kernel(cav_octree* h, int32_t kind);
int cav_octree_get_level_kernel(cav_octree* h, int32_t* kind);
/* set_dynamic_sgs (src/octree/solver.rs:476-481): on = 1 runs the dynamic
 * mixed-scale model on every level before each of its collisions
 * (compute_dynamic_sgs_level, src/octree/smag.rs:144-416) and rescales the
 * interfaces with the mean effective relaxation times (step_cavity,
 * solver.rs:690-711, 808-829).  CAV_ERR_ARG for smag_alpha outside [0, 1],
 * eta_test < 1, a non-finite nu_sm_min, or on = 1 with cs != 0. */
int cav_octree_set_dynamic_sgs(cav_octree* h, int32_t on, double smag_alpha, double nu_sm_min, double eta_test);
/* out14: cs_dyn_mean, cs_dyn_max, kappa_dyn_mean, kappa_dyn_max (the L0
 * model of the last step), nu_t_max (all levels), then the rescaling factors
 * in use: xi A (even, odd, thermal), xi B of the hot strip, of the cold strip
 * (0 with levels = 2).  Before the first dynamic step: zeros and the
 * molecular factors. */
int cav_octree_dynamic_stats(cav_octree* h, double* out14);
/* nu_t_pre and alpha_t_pre of a level as last computed (CAV_ERR_STATE if the
 * model was never enabled); either pointer may be NULL. */
int cav_octree_get_nu_t(cav_octree* h, int32_t level, double* nu_t, double* alpha_t);

/* ---- diagnostics without device allocation ------------------------------ */
/* No counterpart in the reference.  The diagnostics of cav_diag computed on a
 * cavity state that lives in the caller's own device memory, for callers that
 * cannot let the library allocate device memory: a framework whose allocator
 * has already reserved the device memory it may use, or a loop that cannot
 * afford the device-wide synchronisation cudaMalloc / cudaFree may cause.
 * This entry point allocates nothing.  Its reduction scratch is a static
 * device array of CAV_NOALLOC_MAX_ROWS x 8 doubles (512 KiB), held by every
 * GPU that loads the library until the process exits; larger ny is rejected
 * with CAV_ERR_ARG.
 *  - Inputs: device pointers to dense FP64 arrays, k = iy*nx + ix: rho, ux,
 *    uy, t, nu_t [nx*ny] and the f populations f [nx*ny][9] (direction order
 *    of this header); nu = molecular viscosity (for y+), lz = ny - 1.
 *  - Output: out, a device pointer to 11 doubles in the field order of
 *    cav_diag_out, the last being 1.0 when every field is finite (else 0.0).
 *  - Runs asynchronously on `stream` (a cudaStream_t; NULL = default stream).
 *  - Every call looks up the scratch's device address on the current device
 *    (nothing is cached, so a device reset between calls is harmless); the
 *    first call on a device may load the library's device code there, so
 *    make that first call before any stream capture on that device.
 *  - A CUDA error already pending when the call starts is returned as
 *    CAV_ERR_CUDA without launching, and left pending for the caller.
 *  - All calls on a device share the scratch: calls whose kernels can overlap
 *    on the GPU race on it, so order them (same stream, or an event).
 * Rejections return CAV_ERR_ARG / CAV_ERR_CUDA and print one line on stderr. */
#define CAV_NOALLOC_MAX_ROWS 8192
int cav_diag_noalloc(const double* rho, const double* ux, const double* uy, const double* t,
                     const double* nu_t, const double* f, int32_t nx, int32_t ny, double nu, double lz,
                     double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CAVITY_B200_H */
