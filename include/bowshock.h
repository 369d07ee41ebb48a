/*
 * bowshock_b200 C ABI: the steady 2D axisymmetric finite-volume Euler solve on
 * NVIDIA B200 (sm_100a), as a drop-in for the engines behind bowshock's
 * `SteadyEngine` / `EngineFactory` plug-in boundary
 * (src/analysis/verified-drag.ts:22-37).
 *
 * Conventions (the reference's, src/grid/structured.ts:1-50 and
 * src/engine-cpu/euler2d.ts:99-113):
 *   - a block of ni x nj cells between (ni + 1) x (nj + 1) nodes; node (i, j)
 *     at i + j (ni + 1), cell (i, j) at i + j ni;
 *   - x is axial and y radial (y >= 0) in axisymmetric geometry;
 *   - primitive states are (rho, u, v, p), conserved ones (rho, rho u, rho v, E),
 *     four values per cell, cell c at 4 c.
 *
 * Ownership: the caller owns every host array; the library copies inputs in
 * and results out and keeps no caller pointer after a call returns. The
 * library owns its device memory until the matching *_destroy.
 *
 * Errors: every entry point returns a bs_status; BS_OK is 0. The message of
 * the last failure on the calling thread is bs_last_error().
 *
 * Threading: an engine or batch runs one operation at a time; a call that
 * overlaps another on the same object returns BS_BUSY. Distinct objects may
 * be used from different threads; each owns its CUDA stream.
 */
#ifndef BOWSHOCK_B200_H
#define BOWSHOCK_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define BS_API __attribute__((visibility("default")))
#else
#define BS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference throws RangeError (BS_INVALID_ARGUMENT),
 * NonPhysicalStateError (BS_NON_PHYSICAL, src/solver/errors.ts:2),
 * GpuMemoryLimitError / GpuExecutionError (BS_MEMORY_LIMIT / BS_EXECUTION,
 * src/engine-gpu/gpu-common.ts:7-17); ExclusiveRunner's overlapping-call
 * error becomes BS_BUSY (gpu-common.ts:122-140); a solve that does not reach
 * its tolerance within its step budget returns BS_NOT_CONVERGED (the
 * driver's IterationStalled, src/analysis/verified-drag.ts:202). */
typedef enum bs_status {
  BS_OK = 0,
  BS_INVALID_ARGUMENT = 1,
  BS_NON_PHYSICAL = 2,
  BS_MEMORY_LIMIT = 3,
  BS_EXECUTION = 4,
  BS_NOT_CONVERGED = 5,
  BS_BUSY = 6,
  BS_GRID_QUALITY = 7
} bs_status;

typedef enum bs_geometry { BS_PLANAR = 0, BS_AXISYMMETRIC = 1 } bs_geometry;

/* Face fluxes available on the GPU (src/engine-gpu/euler2d-gpu.ts:235-239). */
typedef enum bs_flux { BS_FLUX_HLLC = 0, BS_FLUX_RUSANOV = 1 } bs_flux;

/* LIMITERS (src/scheme/limiters.ts:87-94). */
typedef enum bs_limiter {
  BS_LIMITER_FIRST_ORDER = 0,
  BS_LIMITER_MINMOD = 1,
  BS_LIMITER_VAN_LEER = 2,
  BS_LIMITER_VAN_ALBADA = 3,
  BS_LIMITER_MONOTONIZED_CENTRAL = 4,
  BS_LIMITER_UNLIMITED_CENTRAL = 5
} bs_limiter;

/* Reconstruction (src/scheme/reconstruction.ts:43). */
typedef enum bs_reconstruction {
  BS_RECON_PER_VARIABLE = 0,
  BS_RECON_SHARED = 1,
  BS_RECON_SHARED_SCALED = 2
} bs_reconstruction;

/* RUNGE_KUTTA_STAGES (src/solver/runge-kutta.ts:17-28). */
typedef enum bs_integrator {
  BS_FORWARD_EULER = 0,
  BS_SSPRK2 = 1,
  BS_SSPRK3 = 2
} bs_integrator;

typedef enum bs_time_stepping { BS_TIME_LOCAL = 0, BS_TIME_GLOBAL = 1 } bs_time_stepping;

/* BoundaryCondition2D kinds (src/engine-cpu/euler2d.ts:34-56); the fitted
 * shock's 'faceStates' is not on this path. */
typedef enum bs_bc_kind {
  BS_BC_INFLOW = 0,
  BS_BC_OUTFLOW = 1,
  BS_BC_WALL = 2,
  BS_BC_FAR_FIELD = 3,
  BS_BC_PERIODIC = 4,
  /* States outside each face given per face, with an optional flux imposed
   * per face ('faceStates', src/engine-cpu/euler2d.ts:42, 356-390): the
   * fitted shock's sides (bs_fit_*); batches and engines refuse it. */
  BS_BC_FACE_STATES = 5
} bs_bc_kind;

/* Side (src/engine-cpu/euler2d.ts:32). */
typedef enum bs_side { BS_IMIN = 0, BS_IMAX = 1, BS_JMIN = 2, BS_JMAX = 3 } bs_side;

/* Primitive2D (src/scheme/flux.ts:331-336). */
typedef struct bs_primitive {
  double rho, u, v, p;
} bs_primitive;

typedef struct bs_boundary {
  int32_t kind;       /* bs_bc_kind */
  int32_t reserved;   /* zero */
  bs_primitive state; /* inflow / far-field free stream; ignored otherwise */
} bs_boundary;

/* Euler2DConfig (src/engine-cpu/euler2d.ts:58-81) without the grid nodes,
 * which are passed beside it, and without the manufactured-solution source
 * (the GPU engine refuses sources, src/analysis/gpu-engine.ts:21). */
typedef struct bs_config {
  int32_t ni, nj;
  int32_t geometry;       /* bs_geometry */
  int32_t flux;           /* bs_flux */
  int32_t limiter;        /* bs_limiter */
  int32_t reconstruction; /* bs_reconstruction */
  int32_t integrator;     /* bs_integrator */
  int32_t time_stepping;  /* bs_time_stepping */
  double gamma;
  double cfl;             /* explicit CFL number, in (0, 1] */
  bs_boundary boundaries[4]; /* indexed by bs_side */
} bs_config;

/* BoundaryFaceFlux (src/engine-cpu/euler2d.ts:99-113): midpoint, outward
 * unit normal, area (per radian when axisymmetric) and the flux per unit area
 * along the outward normal [mass, x momentum, y momentum, energy]. */
typedef struct bs_face_flux {
  double x, y, nx, ny, area;
  double flux[4];
} bs_face_flux;

/* Outcome of a steady solve. */
typedef struct bs_solve_result {
  int32_t status;          /* bs_status of this solve */
  int32_t steps;           /* steps taken by this solve */
  double residual;         /* final RMS density residual, FP64 */
  double initial_residual; /* residual of the state the solve started from */
  double drag;             /* forebody pressure drag coefficient, FP64 */
} bs_solve_result;

typedef struct bs_engine bs_engine;

/* Arithmetic of a GPU solve. BS_PRECISION_FP64 (the default): the state and
 * the residual that decides convergence in FP64, the LU-SGS operator, the
 * time steps and the grid metrics in FP32 - the FP32 field alone cannot
 * reach an RMS density residual of 1e-6 (its rounding floor is near 1e-5).
 * BS_PRECISION_FP32: every field quantity in FP32 with gamma rounded to
 * FP32, the reference GPU engine's arithmetic
 * (src/engine-gpu/euler2d-gpu.ts:129-146). */
typedef enum bs_precision { BS_PRECISION_FP32 = 32, BS_PRECISION_FP64 = 64 } bs_precision;

/* Message of the last failure on this thread ("" if none). */
BS_API const char *bs_last_error(void);

/* Library version string. */
BS_API const char *bs_version(void);

/* Number of CUDA devices the library can use (0 without a GPU). */
BS_API bs_status bs_device_count(int32_t *count);

/* The device this thread's engines and batches are created on (default 0);
 * objects stay on the device they were created on. */
BS_API bs_status bs_set_device(int32_t device);

/* The measured FP64 fused multiply-add rate of the current device: a grid
 * that fills every SM, each thread running 8 independent FMA chains of
 * `iterations` steps, timed by CUDA events after one warm-up launch. The
 * denominator of the flux kernels' FP64 fraction (their residual is FP64
 * arithmetic). No counterpart in the reference. */
BS_API bs_status bs_fp64_fma_rate(int32_t iterations, double *tflops, double *ms);

/* ---- single-grid engine: Euler2D / GpuEuler2D --------------------------- */

/* new Euler2D(config) / GpuEuler2D.create (src/engine-cpu/euler2d.ts:318,
 * src/engine-gpu/euler2d-gpu.ts:217): validates the configuration
 * (src/solver/config.ts:35-55), computes the grid metrics in FP64
 * (src/grid/structured.ts:94-168) and uploads them as FP32. x and y hold the
 * (ni + 1)(nj + 1) nodes. The state starts undefined until set. */
BS_API bs_status bs_engine_create(const bs_config *config, const double *x, const double *y,
                           bs_engine **out);

/* bs_engine_create with an explicit bs_precision. */
BS_API bs_status bs_engine_create_ex(const bs_config *config, const double *x, const double *y,
                              int32_t precision, bs_engine **out);

/* GpuEuler2D.destroy (src/engine-gpu/euler2d-gpu.ts:673). */
BS_API bs_status bs_engine_destroy(bs_engine *engine);

/* Cell centroids in FP64 (GridMetrics.centroidX/Y, src/grid/structured.ts:48-49),
 * ni nj each, for evaluating an initial field on the host. */
BS_API bs_status bs_engine_centroids(bs_engine *engine, double *cx, double *cy);

/* setCellPrimitives / setInitialCondition (src/engine-gpu/euler2d-gpu.ts:412-459):
 * four primitives per cell; resets the step count. The energy uses gamma
 * rounded to FP32, as the reference GPU does. Returns BS_NON_PHYSICAL, with
 * nothing uploaded, if a state has rho <= 0, p <= 0 or a non-finite value. */
BS_API bs_status bs_engine_set_primitives(bs_engine *engine, const double *primitives);

/* iterate(count) (src/engine-cpu/euler2d.ts:554-560): explicit SSP-RK steps
 * with the configured integrator and time stepping. BS_NON_PHYSICAL if a
 * cell became non-physical (the state then holds the failing step). */
BS_API bs_status bs_engine_iterate(bs_engine *engine, int32_t steps);

/* setImplicitCfl (src/engine-gpu/euler2d-gpu.ts:681-692): the CFL number the
 * next implicit step starts from (1 after create). */
BS_API bs_status bs_engine_set_implicit_cfl(bs_engine *engine, double cfl);

/* iterateImplicit with LU-SGS sweeps (src/engine-cpu/euler2d.ts:581-589,
 * implicitCorrection :878-1105, applyImplicitUpdate :816-847): each step uses
 * the current CFL number, which then grows by `growth` up to `cfl_max`
 * (src/engine-gpu/shaders/euler2d-implicit.wgsl:232-237). growth = 1 with
 * bs_engine_set_implicit_cfl(cfl_max) is the CPU engine's fixed-CFL form.
 * The sweeps run as anti-diagonal wavefronts on the GPU. */
BS_API bs_status bs_engine_iterate_implicit(bs_engine *engine, int32_t steps, double cfl_max,
                                     double omega, double growth);

/* densityResidualNorm (src/engine-cpu/euler2d.ts:480-491): RMS over the
 * interior cells of R_rho / V, the residual evaluated on the GPU from the
 * FP32 state and accumulated in FP64. */
BS_API bs_status bs_engine_density_residual_norm(bs_engine *engine, double *norm);

/* residualVector (src/engine-cpu/euler2d.ts:456-472): the residual of the
 * current state, four FP64 values per cell, evaluated on the GPU. */
BS_API bs_status bs_engine_residual(bs_engine *engine, double *residual);

/* Local time step of every cell (computeTimeSteps, src/engine-cpu/euler2d.ts:1183-1205),
 * evaluated on the GPU and stored as FP32; ni nj values. */
BS_API bs_status bs_engine_time_steps(bs_engine *engine, double *dt);

/* boundaryFluxes(side) (src/engine-cpu/euler2d.ts:499-525): wall-face fluxes
 * evaluated on the GPU in FP64 from the FP32 state; `out` holds ni (j sides)
 * or nj (i sides) entries. */
BS_API bs_status bs_engine_boundary_fluxes(bs_engine *engine, int32_t side, bs_face_flux *out);

/* forebodyPressureDrag over the jMin faces (src/analysis/forces.ts:19-30),
 * computed and reduced in FP64 on the GPU. */
BS_API bs_status bs_engine_forebody_drag(bs_engine *engine, double p_inf, double q_inf,
                                  double base_radius, double *drag);

/* readState (src/engine-gpu/euler2d-gpu.ts:549-571): the FP32 conserved
 * state, four values per cell. */
BS_API bs_status bs_engine_read_state(bs_engine *engine, float *conserved);

/* cells() (src/analysis/verified-drag.ts:26-27, gpuPrimitive2D
 * euler2d-gpu.ts:136-146): primitives in FP64 recovered from the FP32 state
 * with gamma rounded to FP32. */
BS_API bs_status bs_engine_read_primitives(bs_engine *engine, double *primitives);

/* Steps taken since the state was last set. */
BS_API bs_status bs_engine_steps(bs_engine *engine, int64_t *steps);

/* Iterate until the FP64 RMS density residual is at most `tolerance` times
 * the residual of the starting state (relative = 1) or at most `tolerance`
 * (relative = 0), checking every `check_every` steps, up to `max_steps`.
 * method 0 = explicit (config integrator), 1 = LU-SGS at fixed `cfl` and
 * `omega`. The convergence test runs on the GPU in FP64; the host reads one
 * word per check. Fills `result` (drag with p = 1, q = gamma M^2 / 2 taken
 * from the jMin-side free stream is not known here, so result->drag is 0;
 * use bs_engine_forebody_drag). Returns BS_NOT_CONVERGED if the budget ran
 * out first. */
BS_API bs_status bs_engine_solve(bs_engine *engine, int32_t method, double cfl, double omega,
                          double tolerance, int32_t relative, int32_t max_steps,
                          int32_t check_every, bs_solve_result *result);
/* As bs_batch_set_anderson, for the engine's later bs_engine_solve and
 * bs_engine_iterate_accelerated calls. */
BS_API bs_status bs_engine_set_anderson(bs_engine *engine, int32_t depth, int32_t plain_steps);

/* LU-SGS steps as bs_engine_iterate_implicit (the CFL number growing by
 * `growth` up to `cfl_max` from its current value), with the Anderson
 * acceleration of bs_engine_set_anderson and its history kept from one call
 * to the next: plain steps until plain_steps have been taken since the state
 * or the settings were last set, accelerated ones after (solveTransonic's
 * steps, src/analysis/transonic-flow.ts:151-245: the history forgotten when
 * |f|^2 exceeds 100 times its least value, a non-physical accelerated state
 * replaced by the plain step). Without acceleration (depth 0) it is
 * bs_engine_iterate_implicit. */
BS_API bs_status bs_engine_iterate_accelerated(bs_engine *engine, int32_t steps, double cfl_max,
                                               double omega, double growth);
/* The times the acceleration forgot its history since it was last reset. */
BS_API bs_status bs_engine_anderson_restarts(bs_engine *engine, int32_t *restarts);

/* The metrics the residual reads: 32 (FP32, the default) or 64 (two-float:
 * each face normal, face area, cell volume and planar area as its FP32 value
 * plus the FP32 low part of the FP64 value, about 48 bits, as the reference's
 * two-float engine holds them, src/engine-gpu/euler2d-two-float.ts:1-8,
 * 584-605). The steady state is then that of the FP64 residual to about
 * 1e-12 instead of FP32 metric rounding (a drag error near 1e-6 of its value
 * on the far-field domains of transonic flow); the LU-SGS operator and the
 * time steps keep FP32 metrics. Costs 24 more bytes per cell of device
 * memory and of residual traffic. Engines of precision 32 refuse 64. */
BS_API bs_status bs_engine_set_metric_precision(bs_engine *engine, int32_t bits);

/* Polls each bounded wait of the engine's later LU-SGS sweeps makes before it
 * gives up (-1 restores the default of 2^22; 0 makes the first wait give up
 * at once). A sweep that gives up drains its copies in flight under the
 * default bound, leaves the case's state as it was before the step, and the
 * call that ran it returns BS_EXECUTION; the engine stays usable. For tests
 * of that path; the reference detects a GPU step that did not complete by
 * its step ledger instead (src/engine-gpu/time-loop.ts:125-150). */
BS_API bs_status bs_engine_set_sweep_wait_limit(bs_engine *engine, int32_t polls);

/* ---- an LU-SGS step that allocates nothing -------------------------------- */

/* One LU-SGS step (residual and diagonal pass, forward and backward wavefront
 * sweeps, update) of one case whose FP64 state and grid metrics the caller
 * keeps in its own device memory; no counterpart in the reference. For
 * callers that cannot let a library allocate device memory: applications
 * that hand out all GPU memory from their own pool (cudaMalloc would bypass
 * their budget, and cudaMalloc/cudaFree synchronise the device) and solver
 * loops that must not allocate once running. All scratch lives in one static
 * device array of the library (about 11.6 MB), reserved on every GPU that
 * loads it until the process exits: at most 65536 cells (ni nj) and 512
 * cells across (nj); larger grids return BS_INVALID_ARGUMENT. The first
 * call on a device looks up the array's device address with that device
 * current; after cudaDeviceReset that address is stale and the entry point
 * must not be called again in the process. Each call waits for `stream` (it
 * reads back the residual and the status), so no call may be made while that
 * stream is being captured. Every call shares the array, so calls that
 * overlap on the GPU race: order them. A sweep that gives up waiting for its
 * records returns BS_EXECUTION and leaves the state as it was. Device inputs (layout as the engine's,
 * device/layout.cuh): iface (ni + 1) nj float4 (nx, ny, area, 0), jface
 * ni (nj + 1) float4, cells ni nj float2 (volume, planar area); the state as
 * four FP64 arrays of ni nj, updated in place. `stream` is a cudaStream_t
 * (NULL for the default stream). On return, *residual is the RMS density
 * residual of the state the step started from and *non_physical is 1 if a
 * cell became non-physical. */
BS_API bs_status bs_lusgs_step_static(const bs_config *config, const float *iface,
                                      const float *jface, const float *cells, double *rho,
                                      double *mu, double *mv, double *e, double cfl, double omega,
                                      void *stream, double *residual, int32_t *non_physical);

/* ---- batches: many cases of uneven size in one set of launches ------------ */

typedef struct bs_batch bs_batch;

/* A batch of n independent cases (their own grids, configurations and free
 * streams) solved together: every kernel launch covers all active cases, and
 * a case stops when its own residual reaches the tolerance. configs[k] with
 * nodes x[k], y[k] as in bs_engine_create. The cases share one time
 * integrator. */
BS_API bs_status bs_batch_create(int32_t n, const bs_config *configs, const double *const *x,
                                 const double *const *y, int32_t precision, bs_batch **out);
BS_API bs_status bs_batch_destroy(bs_batch *batch);
BS_API bs_status bs_batch_size(bs_batch *batch, int32_t *n);

/* As bs_engine_set_primitives, for case `c`. */
BS_API bs_status bs_batch_set_primitives(bs_batch *batch, int32_t c, const double *primitives);

/* Every case from its own jMax/iMin inflow state (the free stream). */
BS_API bs_status bs_batch_set_free_stream(bs_batch *batch);

/* `steps` explicit steps (each case's own integrator, CFL and time stepping)
 * of the batch's active cases, as bs_engine_iterate per case; the
 * verified-drag driver (src/analysis/verified-drag.ts:258-299) iterates a
 * family of grids this way between drag checks. */
BS_API bs_status bs_batch_iterate(bs_batch *batch, int32_t steps);

/* Which cases bs_batch_iterate advances: flags[c] != 0 active, 0 frozen
 * (a case whose drag has settled). bs_batch_solve sets its own. */
BS_API bs_status bs_batch_set_active(bs_batch *batch, const int32_t *flags);

/* Case c's display field per cell into out (ni nj doubles, cell (i, j) at
 * i + j ni), computed on the GPU from the current state: the compute half of
 * the reference's flow view (src/render/flow-fields.ts:36-117; drawing it is
 * graphics, not done here). field: 0 schlieren (|grad rho| by Green-Gauss in
 * the plane, times `length` over the free stream's density), 1 Mach number,
 * 2 pressure coefficient against `free`, 3 density over the free stream's. */
BS_API bs_status bs_batch_flow_field(bs_batch *batch, int32_t c, int32_t field, const bs_primitive *free,
                                     double length, double *out);

/* As bs_engine_solve for every case at once; results[k] for case k. Returns
 * BS_OK when the call ran; each case's outcome is in its result. */
BS_API bs_status bs_batch_solve(bs_batch *batch, int32_t method, double cfl, double omega,
                                double tolerance, int32_t relative, int32_t max_steps,
                                int32_t check_every, bs_solve_result *results);

/* Anderson acceleration of the LU-SGS steps of later bs_batch_solve calls
 * (method 1): after `plain_steps` plain steps, x <- x + f - (dX + dF) gamma
 * with the last `depth` differences of the iterates and of their LU-SGS
 * corrections f, gamma minimising |f - dF gamma| (AndersonMixing,
 * src/solver/anderson.ts:20-123, applied as src/analysis/transonic-flow.ts:
 * 183-206 applies it: the history is forgotten after a non-physical
 * accelerated state, which is replaced by the plain update, and when |f|^2
 * exceeds 100 times its smallest value since the last restart). depth 0 (the
 * default) keeps plain steps; at most 16. The steady state, and the residual
 * test that stops a case, are those of the plain steps. */
BS_API bs_status bs_batch_set_anderson(bs_batch *batch, int32_t depth, int32_t plain_steps);
/* As bs_engine_set_metric_precision, for every case of the batch. */
BS_API bs_status bs_batch_set_metric_precision(bs_batch *batch, int32_t bits);
/* The tile shape of the batch's residual passes and explicit stages: -1 the
 * default (16 x 15 cells on 256 threads, four resident CTAs asked for on
 * launches of four waves or more), 0 .. 7 the autotuner's choices: 16 x 15
 * on 256 threads with one or four resident CTAs asked for, 16 x 15 on 512,
 * 8 x 15 and 16 x 7 on 256 (about one face per thread), 24 x 15 on 384 (the
 * least halo), 8 x 15 on 128, 16 x 15 on 256 with two resident CTAs asked
 * for. Every shape computes the same residual, cell
 * for cell; bs_batch_autotune picks the fastest. FP32 batches keep -1. No
 * counterpart in the reference (its passes are one dispatch per face
 * direction, src/engine-gpu/shaders/euler2d.wgsl:316-367). */
BS_API bs_status bs_batch_set_tile_shape(bs_batch *batch, int32_t shape);
/* The batch's lanes and tile shape as set or tuned, with the shape's cells
 * along i and j and its threads. */
BS_API bs_status bs_batch_tuning(bs_batch *batch, int32_t *lanes, int32_t *shape, int32_t *tile_i,
                                 int32_t *tile_j, int32_t *threads);
/* Sets the number of lanes (concurrent groups of cases, each on its own
 * stream), 1 .. min(cases, 64), as bs_batch_autotune would choose it: for a
 * caller that applies a choice it tuned before on a batch of the same kind. */
BS_API bs_status bs_batch_set_lanes(bs_batch *batch, int32_t lanes);
/* How the batch's LU-SGS steps apply their update: 1 (the default) inside
 * the next step's residual pass as it reads each cell, halo cells included
 * (two launches a step); 0 by a separate kernel after each sweep (three
 * launches, less work a step). Both give the same state bit for bit;
 * bs_batch_autotune picks the faster. No counterpart in the reference. */
BS_API bs_status bs_batch_set_update_mode(bs_batch *batch, int32_t fused);
/* The update mode as set or tuned. */
BS_API bs_status bs_batch_update_mode(bs_batch *batch, int32_t *fused);
/* As bs_engine_set_sweep_wait_limit, for the batch's later LU-SGS sweeps; a
 * solve reports a case whose sweep gave up as BS_EXECUTION in its result. */
BS_API bs_status bs_batch_set_sweep_wait_limit(bs_batch *batch, int32_t polls);
/* Per case, the times the last solve's acceleration forgot its history. */
BS_API bs_status bs_batch_anderson_restarts(bs_batch *batch, int32_t *restarts);

/* As bs_engine_forebody_drag, for case `c`. */
BS_API bs_status bs_batch_forebody_drag(bs_batch *batch, int32_t c, double p_inf, double q_inf,
                                        double base_radius, double *drag);
/* As bs_engine_read_primitives / bs_engine_density_residual_norm, for case c. */
BS_API bs_status bs_batch_read_primitives(bs_batch *batch, int32_t c, double *primitives);
BS_API bs_status bs_batch_density_residual_norms(bs_batch *batch, double *norms);

/* Device time (CUDA events on the batch's stream) and kernel launches of the
 * last bs_batch_solve. */
BS_API bs_status bs_batch_last_solve_timing(bs_batch *batch, double *device_ms,
                                            int64_t *launches);

/* Times each kernel of the solve's step on the batch's current state:
 * `iterations` steps of `method`, a CUDA event pair around every launch on
 * the batch's stream. ms[k] (three values) is the mean duration of kernel k
 * per launch: method 1 (LU-SGS): k = 0 residual/diagonal pass, 1 wavefront
 * sweeps, 2 update; method 0 (explicit): k = 0 the first stage, 1 a later
 * stage, 2 zero. The state advances by `iterations` steps. */
BS_API bs_status bs_batch_kernel_times(bs_batch *batch, int32_t method, double cfl,
                                       double omega, int32_t iterations, double *ms);

/* ---- grids and exact solutions (host, FP64) ------------------------------ */

/* Nose shapes (NoseShape, src/geometry/nose.ts:13-34). */
typedef enum bs_nose_kind {
  BS_NOSE_CONICAL = 0,
  BS_NOSE_OGIVE = 1,     /* parameter: ogive parameter, 1 = tangent ogive */
  BS_NOSE_ELLIPSOID = 2,
  BS_NOSE_POWER = 3,     /* parameter: exponent in (0, 1] */
  BS_NOSE_PARABOLIC = 4, /* parameter: K in [0, 1] */
  BS_NOSE_HAACK = 5      /* parameter: C in [0, 1/3]; 0 = Von Karman */
} bs_nose_kind;

/* Body (src/geometry/body.ts:8-13): a nose followed by a cylinder. */
typedef struct bs_body {
  int32_t nose_kind;
  int32_t reserved;
  double parameter;
  double nose_length;
  double base_radius;
  double cylinder_length;
} bs_body;

/* BodyGridOptions (src/grid/body-grid.ts:27-45), plus `ni`: when > 0 the
 * grid gets exactly ni columns (refinement must be 1), apportioned to the
 * upstream, nose and cylinder intervals by the generator's own density. */
typedef struct bs_body_grid_options {
  int32_t nj;
  int32_t refinement;
  int32_t ni;
  int32_t flags;  /* BS_GRID_UNGATED: skip the quality gates (blunt grids only) */
  double mach;
  double gamma;
} bs_body_grid_options;

/* Skip the quality gates of a C-topology grid, as the reference does for the
 * captured solution of a two-scale (Haack) nose, whose grids fail them
 * (src/grid/blunt-grid.ts:47-51, tests/grid/blunt-grid.test.ts:133-137). */
#define BS_GRID_UNGATED 1

typedef struct bs_grid bs_grid;

/* bodyGrid (src/grid/body-grid.ts:76-181): the H-topology grid of a sharp
 * nose; BS_GRID_QUALITY if it fails the quality gates
 * (src/grid/quality.ts:24-38). */
BS_API bs_status bs_body_grid(const bs_body *body, const bs_body_grid_options *options, bs_grid **out);

/* bluntBodyGrid (src/grid/blunt-grid.ts:159-540): the C-topology grid of a
 * blunt nose (ellipsoid, Haack / Von Karman, power series) or of a sharp one
 * whose bow shock detaches. iMin is the axis ahead of the tip (a symmetry
 * line: give it a wall condition), jMin the body, jMax the outer boundary,
 * iMax the outflow plane. options->ni > 0 asks for exactly ni columns. */
BS_API bs_status bs_blunt_body_grid(const bs_body *body, const bs_body_grid_options *options,
                                    bs_grid **out);

/* bluntBodyGrid with BluntGridOptions.outerBoundary (src/grid/blunt-grid.ts:42,
 * 296-331): the outer boundary is the polyline of the n_outer points given
 * (at least two, the first on the axis, y strictly increasing outwards),
 * linear between them and continued by its last segment; the lines and
 * their spacing are placed as for the generator's own boundary. n_outer = 0
 * is bs_blunt_body_grid. A two-scale nose's fitted family is built on such a
 * boundary (secondCapture, src/analysis/fitted-flow.ts:624-672). */
BS_API bs_status bs_blunt_body_grid_bounded(const bs_body *body, const bs_body_grid_options *options,
                                            const double *outer_x, const double *outer_y,
                                            int32_t n_outer, bs_grid **out);

/* transonicGrid's options (TransonicGridOptions and TRANSONIC_SPACING,
 * src/grid/transonic-grid.ts:39-126): the refinement (1, 2, 4, ...), the far
 * boundaries' distance in body radii (rounded up to whole base cells), the
 * cylinder solved behind the nose in calibers, and the base grid's spacings
 * in body radii, each 0 for the default (wall 0.05, growth 0.2, tip 0.05,
 * shoulder 0.02, nose 0.2, nose_growth 0.1). */
typedef struct bs_transonic_grid_options {
  int32_t refinement;
  int32_t nested;  /* 1: cut back or continue the grid to nested_far_field / nested_cylinder */
  double far_field;
  double cylinder;
  double wall, growth, tip, shoulder, nose, nose_growth;
  /* The nested domain (TransonicGridOptions.nested): far boundaries and
   * cylinder, 0 for the grid's own; every node it shares with the grid is
   * the same. Sharp noses only. */
  double nested_far_field, nested_cylinder;
} bs_transonic_grid_options;

/* transonicGrid (src/grid/transonic-grid.ts:128-460): for flow from Mach 1 to
 * about 1.2, the H grid of a sharp nose and a long cylinder (jMin the axis
 * ahead of the tip and the body, jMax the far radius, iMin the far boundary
 * upstream, iMax the plane ending the cylinder: give the far sides a
 * far-field condition), optionally cut back or continued to a nested domain;
 * or the C grid of a blunt nose meeting the body tangentially (jMin the body
 * from the stagnation point, iMin the axis ahead of it: a wall, jMax a
 * quarter circle about the stagnation point continued at the far radius,
 * iMax the plane ending the cylinder). Every base cell divides into
 * refinement^2 cells of the refined grid. */
BS_API bs_status bs_transonic_grid(const bs_body *body, const bs_transonic_grid_options *options,
                                   bs_grid **out);
/* TransonicGrid's fields (src/grid/transonic-grid.ts:84-101) of a grid from
 * bs_transonic_grid: the shoulder's column, the base grid's cells across, the
 * far radius, the upstream boundary's x, the end of the cylinder and the
 * topology (1: C, 0: H); the tip's column is bs_grid_info's i_tip. */
BS_API bs_status bs_grid_transonic_info(const bs_grid *grid, int32_t *i_shoulder, int32_t *base_nj,
                                        double *far_radius, double *x_upstream, double *x_end,
                                        int32_t *c_topology);

/* rampGrid (src/grid/shapes.ts:30-52): a channel whose lower wall turns by
 * `angle` at x_corner. */
BS_API bs_status bs_ramp_grid(int32_t ni, int32_t nj, double x_min, double x_corner, double x_max,
                       double height, double angle, bs_grid **out);

BS_API bs_status bs_grid_dims(const bs_grid *grid, int32_t *ni, int32_t *nj);
/* Node coordinates, (ni + 1)(nj + 1) each. */
BS_API bs_status bs_grid_nodes(const bs_grid *grid, double *x, double *y);
/* BodyGrid.iTip and outerAngle (src/grid/body-grid.ts:47-54). */
BS_API bs_status bs_grid_info(const bs_grid *grid, int32_t *i_tip, double *outer_angle);
/* BluntGrid.twoScale (src/grid/blunt-grid.ts:553): 1 for a C grid whose
 * generator's boundary is sized for the tip's blunt part, narrower than the
 * body (Haack and power-series noses, and sharp tips whose shock detaches);
 * 0 for spheres, ellipsoids and every H grid. */
BS_API bs_status bs_grid_two_scale(const bs_grid *grid, int32_t *two_scale);
BS_API bs_status bs_grid_destroy(bs_grid *grid);

/* GridQuality (src/grid/quality.ts:6-21, gridQuality :75-128). */
typedef struct bs_grid_quality {
  double min_angle, min_wall_angle, max_size_ratio, max_aspect_ratio, min_area;
} bs_grid_quality;
BS_API bs_status bs_grid_quality_of(int32_t ni, int32_t nj, const double *x, const double *y,
                             bs_grid_quality *out);

/* ConeFlow (src/validation/taylor-maccoll.ts:23-36). */
typedef struct bs_cone_flow {
  double shock_angle, post_shock_mach, post_shock_pressure_ratio, surface_mach,
      surface_pressure_ratio, surface_pressure_coefficient;
} bs_cone_flow;

/* taylorMaccoll (src/validation/taylor-maccoll.ts:153-216); BS_INVALID_ARGUMENT
 * if the shock detaches. */
BS_API bs_status bs_taylor_maccoll(double mach, double cone_angle, double gamma, double tolerance,
                            bs_cone_flow *out);

/* ObliqueShock / NormalShock (src/validation/gas-dynamics.ts:29-96). */
typedef struct bs_shock {
  double beta, pressure_ratio, density_ratio, downstream_mach;
} bs_shock;
BS_API bs_status bs_oblique_shock(double mach, double theta, double gamma, bs_shock *out);
BS_API bs_status bs_normal_shock(double mach, double gamma, bs_shock *out);

/* The Taylor-Maccoll flow on rays between the cone and its shock
 * (coneFlowField, src/validation/taylor-maccoll.ts:227-275): for each of the
 * n polar angles, the speed over the maximum speed and the flow angle; the
 * cone solution itself in *flow. BS_INVALID_ARGUMENT if a ray lies outside
 * the conical flow or the shock detaches. */
BS_API bs_status bs_cone_flow_field(double mach, double cone_angle, double gamma, double tolerance,
                                    int32_t n, const double *polar, double *speed, double *flow_angle,
                                    bs_cone_flow *flow);

/* The state behind a shock of outward normal (nx, ny) met by the free stream
 * at relative normal Mach number `mach`, the shock's speed along the normal
 * and the post-shock normal velocity (shockState,
 * src/solver/shock-fitting.ts:50-78). */
typedef struct bs_fitted_shock {
  bs_primitive state;
  double speed, normal_velocity, mach;
} bs_fitted_shock;
BS_API bs_status bs_shock_state(const bs_primitive *free, double gamma, double mach, double nx, double ny,
                                bs_fitted_shock *out);
/* The shock consistent with the flow behind it (compatibleShock,
 * src/solver/shock-fitting.ts:87-111): behind-state density, sound speed,
 * pressure and normal velocity extrapolated to the face. */
BS_API bs_status bs_compatible_shock(const bs_primitive *free, double gamma, double nx, double ny, double rho,
                                     double a, double p, double un, bs_fitted_shock *out);

/* The body's radius at axial position x (bodyRadius, src/geometry/body.ts:25-28),
 * for n positions. */
BS_API bs_status bs_body_radius(const bs_body *body, int32_t n, const double *x, double *r);
/* The nose profile's slope dr/dx at the tip (infinite for a blunt tip) and at
 * the base (noseTipSlope / noseBaseSlope, src/geometry/nose.ts:145-196). */
BS_API bs_status bs_nose_slopes(const bs_body *body, double *tip, double *base);

/* ---- the fitted bow shock (fitShock, src/solver/shock-fitting.ts:170-314) ---
 *
 * One case whose jMax side is its bow shock: a curve of nodes on straight
 * lines from the body (origin (line_x, line_y), unit direction (line_dx,
 * line_dy), ni + 1 lines), node j of line i at fraction
 * fractions[i (nj + 1) + j] of the line's height heights[i]. Every step, on
 * the GPU: the shock compatible with the flow in the two cells below each
 * jMax face fills that face's ghosts and imposes its flux; one explicit step
 * (config: SSP-RK with local time steps; iMin the inflow plane's face states,
 * i_min_states 4 primitives per face, or the axis as a wall; jMin the wall;
 * iMax outflow; jMax BS_BC_FACE_STATES); each node moves along its line by
 * the shock's speed times half the top cell's height over its fastest signal;
 * the grid is rebuilt and the flow interpolated along the lines. first_node:
 * 0 keeps the first node ('fixed', a sharp tip), 1 keeps the shock normal to
 * the axis ('symmetry'). initial: 4 primitives per cell, cell (i, j) at
 * i + j ni. A fit is not re-entrant (BS_BUSY). */
typedef struct bs_fit bs_fit;
BS_API bs_status bs_fit_create(const bs_config *config, const double *line_x, const double *line_y,
                               const double *line_dx, const double *line_dy, const double *fractions,
                               const double *heights, const bs_primitive *free, const double *i_min_states,
                               int32_t first_node, const double *initial, bs_fit **out);
BS_API bs_status bs_fit_destroy(bs_fit *fit);
BS_API bs_status bs_fit_iterate(bs_fit *fit, int32_t steps);
/* The largest shock speed of the last move over the free stream's sound
 * speed, and the density residual of the current flow (its shock boundary
 * applied) over the larger of the starting flow's and the free stream's on
 * the first grid. */
BS_API bs_status bs_fit_check(bs_fit *fit, double *max_speed, double *residual);
/* Steps in checks of check_every until both fall below their tolerances
 * (*converged 1) or max_iterations steps are taken. */
BS_API bs_status bs_fit_solve(bs_fit *fit, double speed_tolerance, double residual_tolerance,
                              int32_t max_iterations, int32_t check_every, int32_t *iterations,
                              int32_t *converged, double *max_speed, double *residual);
BS_API bs_status bs_fit_heights(bs_fit *fit, double *heights);
BS_API bs_status bs_fit_nodes(bs_fit *fit, double *x, double *y);
BS_API bs_status bs_fit_read_primitives(bs_fit *fit, double *primitives);
/* The jMin wall's fluxes, ni faces, as bs_engine_boundary_fluxes. */
BS_API bs_status bs_fit_wall_fluxes(bs_fit *fit, bs_face_flux *out);
/* The forebody pressure drag of the jMin wall (FP64 on the GPU), as
 * bs_engine_forebody_drag. */
BS_API bs_status bs_fit_forebody_drag(bs_fit *fit, double p_inf, double q_inf, double base_radius,
                                      double *drag);

/* The column positions of a sharp nose's fitted grid (sharpFitProblem,
 * src/analysis/fitted-flow.ts:380-395): from x0 to the end of the body, with
 * the nose's end as a breakpoint, spaced `aspect` times the geometric mean of
 * the wall and outer cell heights under the tip cone's shock line at angle
 * beta, nj cells across (refined). At most `capacity` positions. */
BS_API bs_status bs_sharp_fit_columns(const bs_body *body, double beta, double x0, int32_t nj,
                                      int32_t refinement, double aspect, double density, int32_t capacity,
                                      double *out, int32_t *n_out);

/* Node positions along a line of breakpoints by an integrated density
 * (columnPositions, src/grid/spacing.ts:31-71): `total` > 0 asks for exactly
 * that many intervals. Writes at most `capacity` positions, their count in
 * *n_out (BS_INVALID_ARGUMENT if more are needed). */
typedef double (*bs_density_fn)(double x, void *user);
BS_API bs_status bs_column_positions(int32_t n_breakpoints, const double *breakpoints, bs_density_fn density,
                                     void *user, int32_t refinement, int32_t total, int32_t capacity,
                                     double *out, int32_t *n_out);

/* Autotuning of a batch (no counterpart in the reference): times `steps`
 * steps of `method` (0 explicit, 1 LU-SGS with cfl, omega) from the current
 * state with 1, 2, 4, ... up to 64 lanes (concurrent groups of cases, each on
 * its own stream) and keeps the fastest for later solves; *lanes is the
 * choice and *ms_per_step its time. The state is unchanged. */
BS_API bs_status bs_batch_autotune(bs_batch *batch, int32_t method, int32_t steps, double cfl, double omega,
                                   int32_t *lanes, double *ms_per_step);

/* ---- learned warm start (no counterpart in the reference) -----------------
 *
 * The tensor-core GEMM under the warm-start network, exposed for testing:
 * C (m x n, FP32, row-major) = A (m x k) . B (n x k)^T with A and B bf16,
 * row-major, on the device; n a multiple of 64, k a multiple of 64, 16-byte
 * aligned pointers. With `accumulate`, C += A B^T with K split over `splits`
 * CTAs per tile (FP32 atomics); otherwise splits must be 1. `stream` is a
 * cudaStream_t (NULL: default stream); the call returns after the GEMM. */
BS_API bs_status bs_gemm_bf16(const void *a, const void *b, float *c, int32_t m, int32_t n, int32_t k,
                              int32_t splits, int32_t accumulate, void *stream);
/* The same GEMM (no split, C stored) launched `iterations` times back to back
 * on the default stream after one warm-up; *ms = CUDA-event milliseconds per
 * launch. */
BS_API bs_status bs_gemm_bf16_time(const void *a, const void *b, float *c, int32_t m, int32_t n, int32_t k,
                                   int32_t iterations, float *ms);

/* The warm-start network: a GELU MLP from one grid cell's sample to its
 * steady primitive state, trained with Adam on solved cases, all on the GPU
 * (BF16 weights and activations, FP32 accumulation and master weights).
 *
 * A sample is 10 floats: the cell centroid (x, r) in body diameters and 8
 * case values (nose family one-hot over conical, ogive, parabolic, ellipsoid,
 * haack; fineness / 5; body length / 8; Mach / 5). A target or prediction is
 * 4 floats: log(rho / rho_inf), u / u_inf, v / u_inf, log(p / p_inf).
 * Inside, the sample becomes 74 features (x / 8, r / 4, the case values, and
 * sin and cos of pi 2^(7k/15) x / 8 and r / 4, k = 0..15), padded to 128.
 *
 * Parameters, flat, layer by layer: W (out x in, row-major) then b (out);
 * in = 128 for the first layer, out = 128 for the last (only its first 4
 * outputs are used; the other rows stay zero). One call at a time per network
 * (BS_BUSY otherwise). */
typedef struct bs_mlp bs_mlp;

/* hidden_layers of width 256 (width must be 256); `batch` (a multiple of
 * 128) samples per training step and per inference pass; weights drawn from
 * `seed`. */
BS_API bs_status bs_mlp_create(int32_t hidden_layers, int32_t width, int32_t batch, uint64_t seed,
                               bs_mlp **out);
BS_API bs_status bs_mlp_destroy(bs_mlp *net);
BS_API bs_status bs_mlp_param_count(const bs_mlp *net, int64_t *out);
BS_API bs_status bs_mlp_get_params(bs_mlp *net, float *out);
BS_API bs_status bs_mlp_set_params(bs_mlp *net, const float *params);
/* The training set: n samples (n x 10) and targets (n x 4), copied to the
 * device. */
BS_API bs_status bs_mlp_set_data(bs_mlp *net, int64_t n, const float *samples, const float *targets);
/* `steps` Adam steps (learning rate lr) on random batches of the training
 * set drawn from `seed`; losses[s] (if not NULL) is step s's mean squared
 * error over the batch's 4 outputs. */
BS_API bs_status bs_mlp_train(bs_mlp *net, int32_t steps, float lr, uint64_t seed, float *losses);
/* Loss and parameter gradients (flat, as the parameters) over n <= batch
 * given samples, without changing the network. */
BS_API bs_status bs_mlp_loss_grad(bs_mlp *net, int32_t n, const float *samples, const float *targets,
                                  float *loss, float *grads);
/* Predictions (n x 4) for n samples (n x 10). */
BS_API bs_status bs_mlp_predict(bs_mlp *net, int64_t n, const float *samples, float *out);

#ifdef __cplusplus
}
#endif

#endif /* BOWSHOCK_B200_H */
