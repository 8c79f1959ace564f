/*
 * sgh_b200.h -- C ABI of libsgh_b200.so, the B200 (sm_100a) time-step engine of
 * the spectral-Galerkin laser heat solver.
 *
 * The reference solver has no native code: its time step is Python driving a
 * MathBackend plugin (backends/base.py:38-81, registered through
 * backends/_registry.py:45-110) whose kernel module exposes the functions
 * listed in physics/spectral_cpu_kernels.py and physics/spectral_gpu_kernels.py.
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions
 *   - Every function returns an int status: SGH_OK (0) or a negative SGH_ERR_*
 *     code; sgh_last_error() gives a message. Nothing aborts or traps.
 *   - Device memory is owned by the caller: the plan reports how many bytes of
 *     workspace it needs and the caller binds a device buffer of that size.
 *   - Streams are passed as void* (a cudaStream_t; NULL = legacy default).
 *   - Arrays are C-ordered [z][y][x] (x contiguous), FP64 unless stated.
 *   - One plan = one cuboid instance; a plan is used from one host thread.
 */
#ifndef SGH_B200_H
#define SGH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SGH_ABI_VERSION 3

/* status codes */
#define SGH_OK               0
#define SGH_ERR_INVALID     -1   /* bad argument or configuration            */
#define SGH_ERR_CUDA        -2   /* a CUDA runtime call failed               */
#define SGH_ERR_STATE       -3   /* plan not bound / called out of order     */
#define SGH_ERR_UNSUPPORTED -4   /* valid request this build does not handle */
#define SGH_ERR_WORKSPACE   -5   /* workspace too small or misaligned        */

/* step status (sgh_step_out.status) */
#define SGH_STEP_CONVERGED   0   /* Picard residual fell below the tolerance */
#define SGH_STEP_CAPPED      1   /* hit max_picard_iter                      */
#define SGH_STEP_NONFINITE   2   /* residual became NaN/Inf; loop stopped    */
#define SGH_STEP_TC_TIMEOUT  3   /* mixed plan: a bounded tensor-core wait ran
                                    out; the step's results are not trusted  */

/* property-expression opcodes (postfix program, see sgh_program) */
enum {
  SGH_OP_CONST = 1, SGH_OP_T = 2, SGH_OP_ADD = 3, SGH_OP_SUB = 4, SGH_OP_MUL = 5,
  SGH_OP_DIV = 6, SGH_OP_POW = 7, SGH_OP_NEG = 8,
  SGH_OP_SQRT = 16, SGH_OP_EXP = 17, SGH_OP_LOG = 18, SGH_OP_LOG2 = 19, SGH_OP_LOG10 = 20,
  SGH_OP_SIN = 21, SGH_OP_COS = 22, SGH_OP_TAN = 23, SGH_OP_ASIN = 24, SGH_OP_ACOS = 25,
  SGH_OP_ATAN = 26, SGH_OP_SINH = 27, SGH_OP_COSH = 28, SGH_OP_TANH = 29,
  SGH_OP_ASINH = 30, SGH_OP_ACOSH = 31, SGH_OP_ATANH = 32, SGH_OP_FABS = 33,
  SGH_OP_CEIL = 34, SGH_OP_FLOOR = 35, SGH_OP_TRUNC = 36, SGH_OP_LOG1P = 37,
  SGH_OP_EXPM1 = 38, SGH_OP_ATAN2 = 48
};
#define SGH_MAX_PROGRAM 64
#define SGH_MAX_CONSTS  32
#define SGH_MAX_STACK   16

/* One property branch p(T) as a postfix program. SGH_OP_CONST is followed by
 * the index of its value in consts[]. Replaces the generated CUDA-C of
 * core/property_expr.py:285-297 (PropertyExpr.to_c_source). */
typedef struct {
  int32_t n_ops;
  int32_t n_consts;
  int32_t ops[SGH_MAX_PROGRAM];
  double consts[SGH_MAX_CONSTS];
} sgh_program;

#define SGH_PRECISION_FP64  0
/* Single-instance plans only: every contraction in FP32 arithmetic on the CUDA
 * cores (operands rounded to FP32, FP32 products and sums) and the modal
 * iterates rounded to FP32 -- the FP32 arm of a precision study. */
#define SGH_PRECISION_FP32  2

/* Everything one instance needs; mirrors SimulationContext
 * (core/parameters.py:482-682) as consumed by SpectralSolver.initialize
 * (solvers/spectral.py:125-217). */
typedef struct {
  int32_t nx, ny, nz;
  /* SGH_PRECISION_FP64, or SGH_PRECISION_MIXED: every DCT contraction of the
   * step as split-BF16 products on the tensor cores (hi/lo operands, three
   * products, FP32 accumulation) and the modal iterates rounded to FP32 at
   * every write; the latent source across the solidus-liquidus band, the
   * property correction, the face fluxes, the Picard norms and the
   * coefficient tables stay FP64. SGH_PRECISION_FP32: the same with FP32
   * contractions on the CUDA cores instead. */
  int32_t precision;
  double Lx, Ly, Lz;          /* domain size, m                              */
  double dt;                  /* corrected step, s                           */
  /* material: reference constants of the propagators (MaterialParams)      */
  double k, rho, cp;
  double L_f, T_solidus, T_liquidus;
  double Pa, R_v, T_boil, dH_LV, T0;
  double h_top, h_bottom;
  /* temperature-dependent model (MaterialModel); has_model = model present  */
  int32_t has_model;          /* model is not None                           */
  int32_t model_constant;     /* model.is_constant                           */
  int32_t k_constant;         /* model.k.is_constant (k(T) = solid branch)   */
  int32_t pad0;
  sgh_program k_solid, k_liquid, rho_solid, rho_liquid, c_solid, c_liquid;
  /* beam (LaserParams + LaserProfile)                                      */
  double r_x, r_y, absorptivity;
  double order;               /* super-Gaussian order (2 = Gaussian)        */
  double area_factor;         /* f of I0 = A P / (f r_x r_y)                */
  int32_t cell_integrated;
  /* Picard controls (solvers/spectral.py:107-123)                          */
  int32_t max_iter;
  double omega, tol;
  /* Tile policy of the FP64 axis passes of a plan (no reference
   * counterpart): a pass uses 2 x 4 register tiles when that grid has at
   * least this many CTAs, else 1 x 1 tiles; 0 = the built-in default (132).
   * Chosen per (nx, ny, nz) by the autotuner (autotune.py). Batches ignore it. */
  int32_t axis_min_ctas;
  /* 0: passes large enough run on the FP64 tensor cores (mma.sync .f64);
   * 1: every pass runs on the CUDA-core FP64 kernels (for comparison). */
  int32_t axis_cuda_cores;
  /* Laser-following refined sub-box (FineMeshParams, core/parameters.py:391-410;
   * FineMeshState, physics/spectral_state.py:166-239). box = 1 selects box
   * mode: the latent-heat source is evaluated on a fine box of
   * box_refinement cells per coarse cell that follows the laser in x and y
   * and spans the top box_size[2] metres in z. box = 0 is grid mode. */
  int32_t box;
  int32_t box_refinement;
  double box_size[3];         /* Lx_box, Ly_box, Lz_box, m                   */
} sgh_config;

/* Laser state of one step (LaserState, core/laser.py:150-167). */
typedef struct {
  double x, y, power, vx, vy;
  int32_t is_on;
  int32_t flags;              /* SGH_LASER_* bits; 0 for float64 states      */
} sgh_laser;

/* x, y, vx and vy are float32 values, as a G-code path reports them
 * (io_utils/gcode_path.py:91-119). The reference then forms the warm-start
 * shift v*dt/dx, the box-history shift and the box window position x/dx in
 * float32 arithmetic (solvers/spectral.py:303-305, physics/spectral_ops.py:
 * 300-302, physics/spectral_helpers.py:74); with this bit the library does the
 * same, so G-code-driven steps match it to rounding. */
#define SGH_LASER_F32 1

/* Metrics of one step (solvers/spectral.py:536-542), written on the device. */
typedef struct {
  double T_surface_max;
  double P_laser;
  double picard_rel_err;
  int32_t n_iter;             /* n_evap_iter                                 */
  int32_t converged;          /* picard_converged                            */
  int32_t status;             /* SGH_STEP_*                                  */
  int32_t flags;              /* SGH_STEP_FLAG_* (box mode)                  */
} sgh_step_out;

/* sgh_step_out.flags: the latent-heat source of the step reaches a face of
 * the fine box with more than 1% of its peak magnitude, so the melt pool
 * extends past the box (SpectralSolver._check_latent_box_truncation,
 * solvers/spectral.py:545-586). The x and y flags are raised only for an
 * axis on which the box is narrower than the domain. */
#define SGH_STEP_FLAG_BOX_FLOOR  1
#define SGH_STEP_FLAG_BOX_X      2
#define SGH_STEP_FLAG_BOX_Y      4

/* named workspace buffers (sgh_plan_buffer) */
enum {
  SGH_BUF_MODES = 0,      /* (nz,ny,nx) committed modes a                      */
  SGH_BUF_K = 1,          /* (nz,ny,nx) exp(-alpha lam dt)                     */
  SGH_BUF_KK = 2,         /* (nz,ny,nx) phi_1 / (rho c)                        */
  SGH_BUF_T_PREV = 3,     /* (nz,ny,nx) previous converged temperature         */
  SGH_BUF_Q_EVAP_OLD = 4, /* (ny,nx) previous evaporation flux                 */
  SGH_BUF_Q_MODES = 5,    /* (nz,ny,nx) latent modes of the last iteration     */
  SGH_BUF_SURFACE = 6,    /* (ny,nx) top-surface temperature after the step    */
  SGH_BUF_SCRATCH = 7,    /* (nz,ny,nx) general scratch                        */
  /* box mode only */
  SGH_BUF_BOX_T_PREV = 8, /* (nz_box,ny_box,nx_box) FineMeshState.T_prev       */
  SGH_BUF_BOX_Q_PREV = 9, /* (nz_box,ny_box,nx_box) FineMeshState.Q_prev       */
  SGH_BUF_BOX_BX = 10,    /* (nx_fine_total, nx) B_fine_full[0] transposed     */
  SGH_BUF_BOX_BY = 11,    /* (ny_fine_total, ny) B_fine_full[1] transposed     */
  SGH_BUF_BOX_BZ = 12     /* (nz_box + 1, nz) B_fine_full[2] transposed, then
                             the top-surface weights Ct                      */
};

/* Geometry of the fine box of a box-mode plan (FineMeshState.__init__,
 * physics/spectral_state.py:189-227). */
typedef struct {
  int32_t n_box[3];           /* nx_box, ny_box, nz_box                      */
  int32_t n_fine_total[3];    /* n_fine_totals (x, y over the domain; z over
                                 the box depth)                              */
  double d_fine[3];           /* dx_fine, dy_fine, dz_fine                   */
  double dV_fine;
  double z0;                  /* Lz - Lz_box: height of the box floor        */
} sgh_box_geom;

typedef struct sgh_plan sgh_plan;

int sgh_abi_version(void);
const char* sgh_last_error(void);

/* Validate a configuration and create a plan (no device memory is allocated).
 * Replaces SpectralSolverState.__init__ (physics/spectral_state.py:352-365). */
int sgh_plan_create(const sgh_config* cfg, sgh_plan** out);
int sgh_plan_destroy(sgh_plan* plan);

/* Bytes of device workspace the plan needs (256-byte aligned base). */
int sgh_plan_workspace_bytes(const sgh_plan* plan, uint64_t* bytes);

/* Bind caller-owned workspace, build the tables on the device (grid, DCT
 * matrices, K/KK as precompute_K_KK, physics/spectral_state.py:374-421) and
 * capture the step graph. Leaves the state at the initial condition.
 * The stream is synchronised before return. */
int sgh_plan_bind(sgh_plan* plan, void* workspace, uint64_t bytes, void* stream);

/* Device pointer and size of a named workspace buffer (SGH_BUF_*). */
int sgh_plan_buffer(const sgh_plan* plan, int32_t which, void** ptr, uint64_t* bytes);

/* Kernels launched per step: *pre before the Picard loop (including the
 * launch-setup kernel), *per_iter per Picard iteration, *post after it. A step
 * with n iterations launches pre + n * per_iter + post kernels. No reference
 * counterpart (launch accounting for benchmarks). */
int sgh_plan_launch_counts(const sgh_plan* plan, int32_t* pre, int32_t* per_iter, int32_t* post);

/* Initial condition: a = 0, a[0,0,0] = T0 sqrt(Lx Ly Lz), T_prev = T0, no
 * evaporation or latent history (solvers/spectral.py:176-202). Async. */
int sgh_state_reset(sgh_plan* plan, void* stream);

/* One time step: SpectralSolver.step (solvers/spectral.py:219-543). Copies the
 * host laser state in, replays the step graph (device-resident Picard loop,
 * no host sync per iteration) and copies the metrics back; returns after the
 * stream has drained. */
int sgh_step(sgh_plan* plan, const sgh_laser* laser, sgh_step_out* out, void* stream);

/* The same step as sgh_step with the same kernels launched one by one on the
 * stream and the Picard loop driven from the host (one device->host read of
 * the stop flag per iteration) -- the reference's own control flow
 * (solvers/spectral.py:386-499). For profilers that cannot see kernels inside
 * conditional graph nodes, and for debugging. */
int sgh_step_eager(sgh_plan* plan, const sgh_laser* laser, sgh_step_out* out, void* stream);

/* n_steps time steps back to back, laser states read from a device table and
 * metrics written to a device table; asynchronous. */
int sgh_run(sgh_plan* plan, const sgh_laser* lasers_dev, int32_t n_steps,
            sgh_step_out* outs_dev, void* stream);

/* Orthonormal 3-D DCT over the plan's (nz,ny,nx) grid, device to device:
 * kind 2 = DCT_II, kind 3 = IDCT_II (physics/spectral_cpu_kernels.py:374-389).
 * Uses the plan's scratch buffers; in and out may alias. Async. */
int sgh_dct3d(sgh_plan* plan, int32_t kind, const double* in, double* out, void* stream);

/* Top (top = 1) or bottom (top = 0) surface temperature of modes (nz,ny,nx)
 * into out (ny,nx): reconstruct_surface_temperature /
 * reconstruct_bottom_temperature (physics/spectral_ops.py:210-231). Async. */
int sgh_surface_temperature(sgh_plan* plan, const double* modes, int32_t top,
                            double* out, void* stream);

/* modes = sqrt(dV) * DCT_II(field) over the plan's grid: project_volume
 * (physics/spectral_ops.py:94-102); also SpectralSolver.set_state
 * (solvers/spectral.py:588-619). Async. */
int sgh_project_volume(sgh_plan* plan, const double* field, double* modes, void* stream);

/* field = IDCT_II(modes) / sqrt(dV): reconstruct_volume
 * (physics/spectral_ops.py:83-91). Async. */
int sgh_reconstruct_volume(sgh_plan* plan, const double* modes, double* field, void* stream);

/* Warm-start flags of the instance state, for checkpoints: bit 0 = the
 * latent modes of the previous step are present (grid mode,
 * SpectralSolver._Q_latent_modes_prev is not None, solvers/spectral.py:328),
 * bit 1 = the box history is present (FineMeshState.T_prev is not None,
 * physics/spectral_ops.py:182-194). sgh_state_flags copies them to the host
 * and synchronises the stream; sgh_state_set_flags writes them (async). */
#define SGH_STATE_HAVE_Q_MODES   1
#define SGH_STATE_HAVE_BOX       2
int sgh_state_flags(sgh_plan* plan, int32_t* flags, void* stream);
int sgh_state_set_flags(sgh_plan* plan, int32_t flags, void* stream);

/* Box mode. Geometry of the fine box (host values, no device work);
 * SGH_ERR_STATE for a grid-mode plan. */
int sgh_box_geometry(const sgh_plan* plan, sgh_box_geom* out);

/* Start indices (x, y) of the box window of the last step on the fine grid
 * (_calculate_subgrid_indices, physics/spectral_helpers.py:49-85, as applied
 * by FineMeshState.update, physics/spectral_state.py:229-237). Copies from
 * the device and synchronises the stream. Both are -1 before the first
 * step, when the window bases are still zero as in the reference. */
int sgh_box_window(sgh_plan* plan, int32_t* i0, void* stream);

/* Picard history of the plan's last step (the per-iteration record of
 * SpectralSolver.step with track_picard_history, solvers/spectral.py:470-481):
 * out[2 k] = rms of the residual a_raw - a_old and out[2 k + 1] = the relative
 * residual of iteration k, for k < min(*n_iter, cap, SGH_PICARD_HISTORY_MAX);
 * *n_iter = the step's iteration count. The record is written on the device by
 * the convergence test; this call copies it to the host array out (2 cap
 * doubles) and returns after the stream has drained. */
#define SGH_PICARD_HISTORY_MAX 4096
int sgh_picard_history(sgh_plan* plan, double* out, int32_t cap, int32_t* n_iter, void* stream);

/* out (nz_box, ny_box, nx_box) = the temperature of modes on the fine box at
 * the current window: reconstruct_temperature_box
 * (physics/spectral_ops.py:173-179). Async. */
int sgh_box_temperature(sgh_plan* plan, const double* modes, double* out, void* stream);

/* modes = dV_fine * the contraction of field_box (nz_box, ny_box, nx_box)
 * against the window bases: project_box_to_modes
 * (physics/spectral_ops.py:53-74). Async. */
int sgh_box_project(sgh_plan* plan, const double* field_box, double* modes, void* stream);

/* Plan-free orthonormal DCT over every axis of a C-ordered FP64 array of
 * ndim = 1..3 dimensions (shape[0] slowest): kind 2 = DCT_II, kind 3 =
 * IDCT_II (physics/spectral_cpu_kernels.py:374-389, any shape). The caller
 * passes device scratch of sgh_dctn_workspace_bytes() bytes (256-byte aligned).
 * in and out may alias. Async. */
int sgh_dctn_workspace_bytes(int32_t ndim, const int32_t* shape, uint64_t* bytes);
int sgh_dctn(int32_t kind, int32_t ndim, const int32_t* shape, const double* in, double* out,
             void* workspace, uint64_t bytes, void* stream);

/* ------------------------------------------------------------------------
 * Batched instances (many cuboids of uneven sizes, one launch per stage).
 *
 * A batch holds n slots, each with its own sgh_config (shape and physics).
 * One batch step advances every active slot by one time step: laser/face
 * forcing, the Picard loop and the commit run as batched kernels over all
 * slots inside one CUDA graph, and a slot whose Picard loop has converged
 * stays frozen while the others iterate, so each slot's result equals the
 * result of stepping it alone. Supported physics: what the face-space
 * Picard form covers -- laser, evaporation, no convection, no latent heat,
 * no temperature-dependent model; other configurations are rejected with
 * SGH_ERR_UNSUPPORTED. No reference counterpart: the reference steps one
 * instance per solver (solvers/spectral.py:219-543).
 * ------------------------------------------------------------------------ */
#define SGH_PRECISION_MIXED 1   /* FP32 modes and K/KK (computed in FP64); face contractions in
                                   split-BF16 on the tensor cores; FP64 faces and norms */

typedef struct sgh_batch sgh_batch;

typedef struct {
  int32_t active;     /* 1 while the slot still has steps to run          */
  int32_t step;       /* steps done since sgh_batch_slot_start            */
  int32_t n_steps;    /* steps requested                                  */
  int32_t iters;      /* Picard iterations summed over the steps done     */
  sgh_step_out last;  /* metrics of the last step                         */
} sgh_batch_slot_info;

int sgh_batch_create(const sgh_config* cfgs, int32_t n, int32_t precision, sgh_batch** out);

/* Tile policy of a batch's kernels (no reference counterpart: the reference
 * steps one instance with library transforms). vol_unroll: z-planes whose
 * loads one round of the volume pass issues before their arithmetic (2, 4 or
 * 8; 0 = 4). vol_vec: columns per thread of the volume pass (1, 2, or 4 with
 * FP32 modes; 0 = the widest; a width that does not divide every slot's face
 * falls back to 1). The reserved fields must be 0. Chosen per grid mix by the
 * autotuner; set before sgh_batch_bind. */
typedef struct {
  int32_t vol_unroll;
  int32_t vol_vec;
  int32_t reserved[6];
} sgh_batch_policy;
int sgh_batch_set_policy(sgh_batch* batch, const sgh_batch_policy* policy);
int sgh_batch_destroy(sgh_batch* batch);
int sgh_batch_workspace_bytes(const sgh_batch* batch, uint64_t* bytes);
/* Bind workspace, build per-slot tables, capture the batch step graph. All
 * slots start inactive. Synchronises the stream. */
int sgh_batch_bind(sgh_batch* batch, void* workspace, uint64_t bytes, void* stream);
/* (Re)start a slot: initial condition, laser table (n_steps entries, device),
 * optional per-step metrics table (device, may be NULL). Async. */
int sgh_batch_slot_start(sgh_batch* batch, int32_t slot, const sgh_laser* lasers_dev, int32_t n_steps,
                         sgh_step_out* outs_dev, void* stream);
/* Stop a slot (it is skipped by later steps). Async. */
int sgh_batch_slot_stop(sgh_batch* batch, int32_t slot, void* stream);
/* Resume a slot from state the caller has written into its buffers
 * (SGH_BUF_MODES and SGH_BUF_Q_EVAP_OLD of sgh_batch_buffer, e.g. copied out
 * of a slot of the same configuration in this or another batch after a step):
 * it continues at entry `step` of its laser table (n_steps entries, device)
 * with the same results as if it had never stopped. This is the per-request
 * state the reference keeps between steps (modes and the evaporation warm
 * start, solvers/spectral.py:502-512; its modes.h5 layout,
 * io_utils/spectral_fs_io.py:207-241), used for preemption and to move
 * requests between batches. Async. */
int sgh_batch_slot_resume(sgh_batch* batch, int32_t slot, const sgh_laser* lasers_dev, int32_t n_steps,
                          int32_t step, sgh_step_out* outs_dev, void* stream);
/* n_steps batch steps (each active slot advances until its table ends). Async. */
int sgh_batch_step(sgh_batch* batch, int32_t n_steps, void* stream);
/* One batch step with the same kernels launched one by one and the Picard
 * loop driven from the host (for profilers and debugging). Synchronous. */
int sgh_batch_step_eager(sgh_batch* batch, void* stream);
/* Per-slot status (n entries) into a host array; synchronises the stream. */
int sgh_batch_status(const sgh_batch* batch, sgh_batch_slot_info* out, void* stream);
/* Device pointer / size of a slot buffer: SGH_BUF_MODES, SGH_BUF_K, SGH_BUF_KK
 * (element type FP64 or FP32 by precision), SGH_BUF_Q_EVAP_OLD, SGH_BUF_SURFACE (FP64). */
int sgh_batch_buffer(const sgh_batch* batch, int32_t slot, int32_t which, void** ptr, uint64_t* bytes);
/* *err = nonzero once a tensor-core wait of a mixed-precision batch expired
 * (the affected face pass wrote no results). Synchronises the stream. */
int sgh_batch_error(const sgh_batch* batch, int32_t* err, void* stream);
/* Bound of the tensor-core data waits of the batch's face transforms: at most
 * `polls` mbarrier polls (0 = the default, 2^22) before the CTA records the
 * error flag, waits for its copies and MMAs in flight (always with the
 * default bound), frees its tensor memory and returns without results.
 * stall_test = 1 makes every face-transform CTA first wait, with that bound,
 * on a barrier that nothing completes -- a wait that can only run out -- so a
 * test can drive the error path without a fault (needs polls > 0); 0 for
 * normal stepping. No reference counterpart: the reference has no bounded
 * device waits. Synchronises the stream. */
int sgh_batch_set_wait_limit(sgh_batch* batch, uint32_t polls, int32_t stall_test, void* stream);
/* Kernels per batch step: *pre + n_iter * *per_iter + *post, n_iter = the
 * largest iteration count over the active slots. */
int sgh_batch_launch_counts(const sgh_batch* batch, int32_t* pre, int32_t* per_iter, int32_t* post);
/* The step's volume pass by itself, over every active slot: the modal commit
 * a <- K a + KK Ct sigma (solvers/spectral.py:502-512 with
 * spectral_cpu_kernels.py:83-91), fused with the next step's face sums. For
 * timing and profiling the memory-bound pass of a batch; the slots' modes
 * advance as in a commit. Async. */
int sgh_batch_volume_pass(sgh_batch* batch, void* stream);

/* Orthonormal 2-D DCT-II (kind 2) or DCT-III (kind 3) of an (ny, nx) FP64
 * face with both contractions on the tensor cores (tcgen05) in split-BF16
 * form: each operand is split into BF16 hi + lo, three products per k-step
 * accumulate in FP32 (relative error ~1e-5). The face contraction of the
 * mixed-precision step; no reference counterpart (the reference's
 * DCT_II / IDCT_II, physics/spectral_cpu_kernels.py:374-389, are FP64/FP32).
 * After completion the first int32 of the workspace is 0, or nonzero when a
 * tensor-core wait expired (the output is then not written). Async. */
int sgh_dct2_bf16x3_workspace_bytes(int32_t ny, int32_t nx, uint64_t* bytes);
int sgh_dct2_bf16x3(int32_t kind, int32_t ny, int32_t nx, const double* in, double* out, void* workspace,
                    uint64_t bytes, void* stream);

/* sgh_dctn without a workspace argument, for callers that hold device arrays
 * but cannot allocate device memory themselves -- for example a plain
 * ctypes/FFI host that has no CUDA array library to allocate with, or an
 * application whose memory manager owns the whole device and allows no other
 * allocation. No counterpart in the reference (its DCT_II / IDCT_II allocate
 * freely through NumPy/CuPy).
 *
 * Same transform, arguments and result as sgh_dctn. Its scratch is a fixed
 * array inside the library's device module, SGH_NOALLOC_SCRATCH_BYTES bytes
 * on every GPU that loads the library, held until the process exits; it calls
 * no cudaMalloc/cudaFree and no allocating library routine. An array whose
 * sgh_dctn_workspace_bytes() exceeds that size is rejected with
 * SGH_ERR_WORKSPACE (about 10^6 elements for a 3-D array).
 *
 * Every call looks up the scratch's device address on the current device
 * (cudaGetSymbolAddress, which allocates nothing) and runs sgh_dctn on it; the
 * first call on a device may load the library's device module there, so make
 * that first call before any stream capture. All calls share the one scratch array: calls that overlap
 * on the GPU (different streams, or several threads) race and must be
 * serialised by the caller. The scratch keeps the previous call's contents;
 * this transform writes every scratch element it reads, so none needs
 * clearing. Async. */
#define SGH_NOALLOC_SCRATCH_BYTES (16ull << 20)
int sgh_dctn_noalloc(int32_t kind, int32_t ndim, const int32_t* shape, const double* in, double* out,
                     void* stream);

/* ---- output reconstruction on the device -------------------------------- */

/* Node-centred temperature of FP64 modes (nz, ny, nx) on a cuboid of size
 * Lx x Ly x Lz: out[l][k][j] = sum a[p][n][m] C_m cos(pi m j / nx)
 * C_n cos(pi n k / ny) C_p cos(pi p l / nz) for j = 0..nx, k = 0..ny,
 * l = 0..nz, with C_0 = sqrt(1/L), C_m = sqrt(2/L); out is C-ordered
 * (nz+1, ny+1, nx+1) (the reference returns its transpose). Replaces
 * reconstruct_temperature_DCT (physics/spectral_helpers.py:146-204), which
 * evaluates the same series as a weighted DCT-I on the host. workspace:
 * sgh_nodal_workspace_bytes() bytes, caller-owned, 8-byte aligned. Async. */
int sgh_nodal_workspace_bytes(int32_t nx, int32_t ny, int32_t nz, uint64_t* bytes);
int sgh_nodal_temperature(int32_t nx, int32_t ny, int32_t nz, double Lx, double Ly, double Lz,
                          const double* modes, double* out, void* workspace, uint64_t bytes, void* stream);

/* Temperature of FP64 modes at n_points points coords[3 i + 0..2] = (x, y, z),
 * each clipped to the domain: out[i] = sum a[p][n][m] C_m cos(pi m x / Lx)
 * C_n cos(pi n y / Ly) C_p cos(pi p z / Lz). Replaces
 * reconstruct_temperature_volume_at_points (physics/spectral_helpers.py:206-248),
 * the point evaluation behind save_temp_profiles (:251-333). coords and out
 * are device arrays; workspace: sgh_points_workspace_bytes() bytes. Async. */
/* Temperature along a line parallel to axis (0 = x, 1 = y, 2 = z) at the fixed
 * position (x, y, z) of the other two axes (the axis's own entry is ignored),
 * at n_points positions coords (device, along the axis); every coordinate is
 * clipped to the domain. The same values as sgh_points_temperature on those
 * points, as the profiles of save_temp_profiles (physics/spectral_helpers.py:251-333)
 * need them, but the modes are reduced once per line (two one-row axis passes)
 * instead of once per point. out (n_points). Async. */
int sgh_line_workspace_bytes(int32_t nx, int32_t ny, int32_t nz, uint64_t* bytes);
int sgh_line_temperature(int32_t nx, int32_t ny, int32_t nz, double Lx, double Ly, double Lz,
                         const double* modes, int32_t axis, double x, double y, double z, int32_t n_points,
                         const double* coords, double* out, void* workspace, uint64_t bytes, void* stream);

int sgh_points_workspace_bytes(int32_t nx, int32_t ny, int32_t nz, int32_t n_points, uint64_t* bytes);
int sgh_points_temperature(int32_t nx, int32_t ny, int32_t nz, double Lx, double Ly, double Lz,
                           const double* modes, int32_t n_points, const double* coords, double* out,
                           void* workspace, uint64_t bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SGH_B200_H */
