/*
 * dsmc.h - C ABI of the B200 DSMC engine.
 *
 * This is the drop-in boundary.  The reference solver exposes argument-less
 * C++ functions over global state (include/Simulation.h:4,
 * include/Initialization.h:4-5, include/Boundary.h:3-21, include/Geometry.h:14-22,
 * include/Collision.h:4-6, include/Sampling.h:7-8).  Here the same operations
 * take an explicit context, plain pointers and sizes; every call returns an
 * int status and no exception crosses the boundary.  The C++ surface with the
 * reference's own names (dsmc_reference_api.h) is a thin layer on top of
 * these entry points.
 *
 * A context holds one or more independent cases (a batched ensemble).  All
 * particle and cell storage lives in device memory owned by the context;
 * host buffers are only touched by the explicit upload/download calls.
 *
 * Units are SI throughout, as in the reference.
 */
#ifndef DSMC_H
#define DSMC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------
 * The reference aborts with MPI error codes; the same numbers are returned
 * here (Geometry.cpp:82,120,157; MPIManager.cpp:628,792;
 * Initialization.cpp:218).                                                 */
enum {
    DSMC_OK = 0,
    DSMC_ERR_ARGUMENT = 2,        /* invalid argument or parameter           */
    DSMC_ERR_OUT_OF_DOMAIN = 20,  /* particle outside the grid (Geometry.cpp:66-86) */
    DSMC_ERR_CELL_OVERFLOW = 22,  /* > max_particles_in_cell (Geometry.cpp:142-161) */
    DSMC_ERR_EXCHANGE = 30,       /* particle outside the domain at exchange  */
    DSMC_ERR_CAPACITY = 31,       /* particle slots exhausted (Boundary.cpp:73-80,
                                     MPIManager.cpp:782-796)                 */
    DSMC_ERR_BAD_CLL = 40,        /* CLL coefficient outside [0, 1]
                                     (Initialization.cpp:211-220, Boundary.cpp:247-250) */
    DSMC_ERR_CUDA = 50,           /* a CUDA runtime call failed              */
    DSMC_ERR_NO_DEVICE = 51,      /* no CUDA device                          */
    DSMC_ERR_TIMEOUT = 60,        /* a bounded device-side wait gave up      */
    DSMC_ERR_STATE = 61,          /* call out of order (e.g. step before init) */
    DSMC_ERR_UNSUPPORTED = 62,    /* feature not available in this build     */
    DSMC_ERR_TOO_LARGE = 63       /* input beyond a fixed maximum size       */
};

/* WallModel, same enumerator order as the reference (include/Boundary.h:3). */
enum {
    DSMC_WALL_DIFFUSE = 0,
    DSMC_WALL_SPECULAR = 1,
    DSMC_WALL_CLL = 2
};

/* Storage precision of particle positions and velocities.  Hit times, inflow
 * counts, cell indices and every moment accumulator are FP64 in both.     */
enum {
    DSMC_FP64 = 0,
    DSMC_FP32 = 1
};

/* One case.  Field names follow the reference globals they replace
 * (Geometry.cpp:11-24, Initialization.cpp:11-31, Boundary.cpp:11-13).     */
typedef struct dsmc_params {
    double x1, x2, y1, y2;   /* domain bounds X1 X2 Y1 Y2 [m]              */
    double dz;               /* thickness DZ [m]                           */
    double dl;               /* inflow strip width DL [m]                  */
    int32_t nx, ny;          /* grid NX NY                                 */
    double box_x, box_y;     /* obstacle centre BoxX BoxY [m]              */
    double box_width, box_height;
    double dt;               /* Dt [s]                                     */
    int32_t n_step;          /* NStep                                      */
    int32_t first_sampling_step; /* FirstSamplingStep                      */
    int32_t sampling_period; /* SamplingPeriod                             */
    int32_t wall_model;      /* DSMC_WALL_*  (WallInteraction)             */
    double npc_free;         /* NPCFree                                    */
    double molar_mass;       /* MolarMass [kg/mol]                         */
    double ma_free;          /* MaFree                                     */
    double n_free;           /* NFree [1/m^3]                              */
    double t_free;           /* TFree [K]                                  */
    double attack_angle;     /* AttackAngle [deg]                          */
    double t_wall;           /* Tw [K]                                     */
    double d_ref;            /* DRef [m]                                   */
    double viscosity_index;  /* ViscosityIndex (omega)                     */
    double t_ref;            /* Tref [K]                                   */
    double cll_normal;       /* CLLNormalAccommodation                     */
    double cll_tangential;   /* CLLTangentialAccommodation                 */
    uint64_t seed;           /* Philox key of this case                    */
    int32_t precision;       /* DSMC_FP64 or DSMC_FP32                     */
    int32_t reserved1;       /* must be 0                                  */
    int32_t max_particles_in_cell; /* 0: unlimited; >0: report
                                DSMC_ERR_CELL_OVERFLOW above it as the
                                reference's MAX_PCL_IN_CELL does            */
    int32_t reserved0;
    int64_t capacity;        /* particle slots; 0 = sized automatically    */
} dsmc_params;

/* Derived constants computed by Setup() (Initialization.cpp:221-265). */
typedef struct dsmc_derived {
    double molecule_mass;    /* MoleculeMass                               */
    double p_free;           /* PFree                                      */
    double u_free;           /* UFree                                      */
    double ux_free, uy_free; /* UxFree UyFree                              */
    double dx, dy, dv;       /* DX DY DV                                   */
    double weight;           /* Weight                                     */
    double sigma_ref;        /* SigmaRef                                   */
    double omega;            /* Omega = 2 omega - 1                        */
    double cr_ref;           /* CrRef                                      */
    double mft_free;         /* MFTFree                                    */
    double mfp_free;         /* MFPFree                                    */
    double kn_free;          /* KnFree                                     */
    double sc_max;           /* SCMax of Collision.cpp:23                  */
} dsmc_derived;

/* Run-time counters of one case. */
typedef struct dsmc_counters {
    int64_t np;                   /* NP after the last completed stage     */
    int64_t step;                 /* Step                                  */
    int64_t sample_step;          /* SampleStep                            */
    int64_t collisions_last_step; /* NC returned by CollideParticles       */
    int64_t collisions_total;
    int64_t drag_collision_count; /* DragCollisionCount                    */
    int64_t particle_steps;       /* sum of NP over completed steps        */
    double drag_impulse_total;    /* DragImpulseTotal                      */
    double time;                  /* Time                                  */
    double sample_time;           /* SampleTime                            */
    double drag_sampling_time;    /* DragSamplingTime                      */
    /* The impacts of the moves made while DragSamplingTime runs (steps after
     * FirstSamplingStep): the window the mean drag force is taken over.  The
     * reference's totals above count every step.                         */
    int64_t drag_collision_count_window;
    double drag_impulse_window;
} dsmc_counters;

/* Drag diagnostics of a run (Simulation.cpp:210-237, code the reference
 * keeps commented out): mean force = impulse / DragSamplingTime and
 * Cd = mean force / (0.5 NFree MoleculeMass UFree^2 BoxHeight DZ).        */
typedef struct dsmc_drag {
    double sampling_time;    /* DragSamplingTime, s                          */
    double rho_free;         /* NFree * MoleculeMass, kg/m^3                 */
    double area_ref;         /* BoxHeight * DZ, m^2                          */
    /* The reference's expression: DragImpulseTotal over all steps divided by
     * the sampling time.                                                  */
    double mean_force_total; /* N                                            */
    double cd_total;
    int64_t box_collisions;  /* DragCollisionCount                           */
    /* The same over the sampling window only (the physical mean force).    */
    double mean_force;       /* N                                            */
    double cd;
    int64_t box_collisions_window;
} dsmc_drag;

/* Moments of one cell, laid out exactly as the reference's CELL
 * (include/Cell.h:4-10), 17 doubles.                                       */
typedef struct dsmc_cell {
    double count_np;
    double count_v[3];
    double count_vv[3][3];
    double count_v2v[3];
    double count_nc;
} dsmc_cell;

typedef struct dsmc_ctx dsmc_ctx;

/* ---- host-only helpers (no device needed) ------------------------------ */

/* Reference defaults: Initialization.cpp:11-31, Geometry.cpp:11-24,
 * Boundary.cpp:11-13 (CLL 0.8/0.8 walls). */
void dsmc_default_params(dsmc_params *p);

/* Setup() (Initialization.cpp:210-288): validates the case and fills *d.
 * Returns DSMC_ERR_BAD_CLL for CLL coefficients outside [0, 1]. */
int dsmc_setup(const dsmc_params *p, dsmc_derived *d);

/* WallModelName() (Boundary.cpp:15-24); NULL for an unknown model. */
const char *dsmc_wall_model_name(int wall_model);

const char *dsmc_status_string(int status);

/* Fills `out` from the counters of one case.  DSMC_ERR_STATE when no
 * sampling time has elapsed yet (the reference would divide by zero).      */
int dsmc_drag_report(const dsmc_params *p, const dsmc_derived *d, const dsmc_counters *c,
                     dsmc_drag *out);

/* Printing() (Sampling.cpp:36-268): writes <dir>/<wall>/DSMC2D_Field.plt and
 * .json from a gathered field of nx*ny cells in x-major order (k*ny + l),
 * exactly in the reference format.  `sample_step` is SampleStep. */
int dsmc_write_field(const dsmc_params *p, const dsmc_derived *d, int64_t sample_step,
                     const dsmc_cell *cells, const char *results_dir);

/* ---- context ------------------------------------------------------------ */

/* Creates a context of n_cases (1 to 65535) independent cases on the current
 * CUDA device.  `derived` may be NULL (computed by dsmc_setup) or an array of n_cases
 * overrides.  `cuda_stream` is a cudaStream_t to launch on, or NULL for a
 * stream owned by the context. */
int dsmc_ctx_create(const dsmc_params *cases, const dsmc_derived *derived, int n_cases,
                    void *cuda_stream, dsmc_ctx **out);
int dsmc_ctx_destroy(dsmc_ctx *ctx);

/* InitialConditions() (Initialization.cpp:290-313) for every case, followed
 * by the cell sort that leaves particles ordered by cell.  Clears the device
 * error word of a previous run (and so does dsmc_init_warm). */
int dsmc_init_cold(dsmc_ctx *ctx);

/* Warm start (no counterpart in the reference): instead of the uniform
 * freestream of InitialConditions, every case is filled from the local
 * Maxwellian of a given field, e.g. a surrogate's prediction or the
 * converged field of a neighbouring case.  `host_field` holds 4 doubles per
 * cell, cells x-major (k*ny + l) and cases one after another: number
 * density n [1/m^3], velocity ux, uy [m/s], temperature T [K].  A cell gets
 * floor(n DV / W) + Bernoulli(rest) particles, uniform in the cell, with
 * velocity (ux, uy, 0) plus Gaussians of variance k T / m (each cell's own
 * random stream); those inside the box are dropped.  Counters and moments
 * start from zero as after InitialConditions.  DSMC_ERR_CAPACITY when a
 * case's particles exceed its capacity. */
int dsmc_init_warm(dsmc_ctx *ctx, const double *host_field);
/* The same from 7 doubles per cell: n, ux, uy and the temperature tensor
 * Txx, Tyy, Tzz, Txy [K] (m <(v - u)(v - u)> / k, as Printing's Tx, Ty and
 * the moments give it): the velocities are Gaussians with that covariance,
 * which keeps the anisotropy of shock layers and wakes. */
int dsmc_init_warm_tensor(dsmc_ctx *ctx, const double *host_field);
/* The same from 8 doubles per cell: n, alpha, ux_r, uy_r, Txx_r, Tyy_r,
 * Tzz_r, Txy_r.  Each particle belongs with probability alpha to the case's
 * freestream Maxwellian (UxFree, UyFree, TFree) and otherwise to the
 * Gaussian of mean (ux_r, uy_r, 0) with that temperature tensor (an
 * isotropic T_r: Txx_r = Tyy_r = Tzz_r = T_r, Txy_r = 0): a two-population
 * gas such as the mix of freestream and wall-reflected molecules ahead of a
 * body in a rarefied flow, whose distribution no single Maxwellian
 * matches. */
int dsmc_init_warm_mixture(dsmc_ctx *ctx, const double *host_field);

/* Runs n_steps complete time steps (Simulation.cpp:138-199) for every case:
 * move, boundary conditions, indexing, collisions, sampling.  Launched as
 * CUDA graphs; returns after enqueueing.  Errors raised on the device are
 * reported by the next dsmc_synchronize(). */
int dsmc_step(dsmc_ctx *ctx, int n_steps);

/* dsmc_step with the counters of every step read back without stopping the
 * device: after step k, the counters of case i (as dsmc_get_counters would
 * return them then) are copied asynchronously into
 * host_out[k * n_cases + i].  No counterpart in the reference (which prints
 * its progress from the host); the values are complete once
 * dsmc_synchronize() returns, and the copies overlap the steps only when
 * host_out is page-locked. */
int dsmc_step_read(dsmc_ctx *ctx, int n_steps, dsmc_counters *host_out);

/* The stages of one step, for callers of the per-function surface.  They
 * must be called in this order; dsmc_stage_end_step advances Step. */
int dsmc_stage_move(dsmc_ctx *ctx);      /* MoveParticles (Boundary.cpp:284-328) */
int dsmc_stage_boundary(dsmc_ctx *ctx);  /* BoundaryConditions (Boundary.cpp:94-203) */
int dsmc_stage_index(dsmc_ctx *ctx);     /* Indexing (Geometry.cpp:37-170)          */
int dsmc_stage_collide(dsmc_ctx *ctx);   /* CollideParticles (Collision.cpp:45-56)  */
int dsmc_stage_sample(dsmc_ctx *ctx);    /* Sampling (Sampling.cpp:14-31), in sampling steps */
int dsmc_stage_end_step(dsmc_ctx *ctx);  /* Step++, Time += Dt (Simulation.cpp:160-161) */

/* Waits for queued work and returns the first device-side error, if any. */
int dsmc_synchronize(dsmc_ctx *ctx);

int dsmc_get_counters(dsmc_ctx *ctx, int case_index, dsmc_counters *out);

/* Accumulated moments of one case, nx*ny cells x-major, as GatherGlobalField
 * (MPIManager.cpp:305-499) returns them.  The expanded moments are gathered
 * on the device into the context's changed-cell list buffer (between steps,
 * when it is large enough) or else a temporary stream-ordered allocation,
 * then copied to host_out: directly when host_out is page-locked, otherwise
 * through two pinned chunks of the context. */
int dsmc_get_fields(dsmc_ctx *ctx, int case_index, dsmc_cell *host_out);
/* dsmc_get_fields without any allocation.  No counterpart in the reference:
 * it exists for callers that cannot allocate device memory at read-out time,
 * for example an application whose device memory is already reserved by its
 * own pool, or a monitor that must not stall the device (cudaFree
 * synchronizes it).  dsmc_get_fields may stage
 * the expanded moments in a temporary device buffer; this variant stages them in
 * one static device array of DSMC_FIELDS_NOALLOC_MAX_CELLS cells (8.9 MB,
 * held by every GPU that loads the library until the process exits).
 *   - A case with more cells returns DSMC_ERR_TOO_LARGE and touches nothing.
 *   - The first call on a device looks up the array's device address (with
 *     the context's device current); make that first call before any stream
 *     capture begins.
 *   - All calls share the array and return only after the copy to host_out
 *     completed.  Calls from several host threads that overlap on the GPU
 *     race on the array: serialize them.  Every element the call reads is
 *     written by the same call, so no clearing is needed. */
#define DSMC_FIELDS_NOALLOC_MAX_CELLS 65536
int dsmc_get_fields_noalloc(dsmc_ctx *ctx, int case_index, dsmc_cell *host_out);

/* Same, into device memory (17 doubles per cell), e.g. for an all-reduce. */
int dsmc_get_fields_device(dsmc_ctx *ctx, int case_index, double *device_out);
/* Replaces the accumulators of a case (e.g. after a replica all-reduce). */
int dsmc_set_fields_device(dsmc_ctx *ctx, int case_index, const double *device_in,
                           int64_t sample_step);

/* Particle state of one case in slot order, as FP64 host arrays. */
int dsmc_download_particles(dsmc_ctx *ctx, int case_index, double *x, double *y, double *vx,
                            double *vy, double *vz, int64_t capacity, int64_t *n_out);
/* Replaces the particle state of one case and re-sorts it by cell. */
int dsmc_upload_particles(dsmc_ctx *ctx, int case_index, const double *x, const double *y,
                          const double *vx, const double *vy, const double *vz, int64_t n);
/* Cell start offsets (nx*ny + 1 entries) of the last sort. */
int dsmc_get_cell_starts(dsmc_ctx *ctx, int case_index, int32_t *host_out);

/* Population edits between steps (ctx idle: after InitialConditions or a
 * completed step; DSMC_ERR_STATE otherwise), for the reference-named
 * GenerateNewParticles and RemoveParticlesInsideBox of callers that build
 * their own inflow or initial state.  Both remove with the reference's
 * swap-with-last loop and then re-sort by cell, as the reference's next
 * Indexing would order the particles; NP changes accordingly.
 *
 * GenerateNewParticles' particles (Boundary.cpp:60-92) joining the case:
 * n FP64 particles in device arrays are appended after its NP particles;
 * those outside [X1, X2] x [Y1, Y2] are removed as BoundaryConditions'
 * removal (Boundary.cpp:181-202) would remove them.  DSMC_ERR_CAPACITY when
 * NP + n exceeds the case's slots. */
int dsmc_append_particles_device(dsmc_ctx *ctx, int case_index, const double *x,
                                 const double *y, const double *vx, const double *vy,
                                 const double *vz, int64_t n);
/* RemoveParticlesInsideBox (Geometry.cpp:231-247). */
int dsmc_remove_inside_box(dsmc_ctx *ctx, int case_index);
/* BinaryCollisionsInCell(CellVolume, NPC, IPC) (Collision.cpp:21-44) on the
 * particles of case case_index at slots ipc[0, n) (host array of slot
 * indices into the current cell-sorted population, as dsmc_download_particles
 * orders it); draws from stream (kind, step, entity).  Valid between steps
 * and after the step's Indexing; *n_collisions receives NC. */
int dsmc_collide_list(dsmc_ctx *ctx, int case_index, double cell_volume, int32_t n,
                      const int32_t *ipc, uint32_t kind, uint32_t step, uint32_t entity,
                      int32_t *n_collisions);

/* Checkpoint of every case of an idle context (between steps) in one file:
 * the run counters, the particles in slot order and the sampled moments.
 * The reference has none (its RunSimulation cannot resume).  Loading it
 * into a context created with the same parameters (NStep aside), cases and
 * precision resumes the run: the next steps are bit-identical to the uninterrupted
 * run's (the random streams are keyed by the step), except the order of the
 * atomic drag-impulse sums.  DSMC_ERR_ARGUMENT for a file that is not a
 * checkpoint of such a context; DSMC_ERR_STATE in the middle of a step.    */
int dsmc_checkpoint_save(dsmc_ctx *ctx, const char *path);
int dsmc_checkpoint_load(dsmc_ctx *ctx, const char *path);

/* Launch shapes (no counterpart in the reference): the CTAs per SM of the
 * step's kernels whose grids are tunable, in the order and with the names
 * of dsmc_get_kernel_times; max_ctas_per_sm is what fits on an SM (0 for a
 * kernel with a fixed grid).  Every kernel gives the same results for any
 * shape, so tuning never changes a run's particles or moments. */
int dsmc_get_launch_config(dsmc_ctx *ctx, int32_t *ctas_per_sm, int32_t *max_ctas_per_sm,
                           int max_kernels, int *n_kernels, const char **names_out);
/* Sets the shapes of the first n kernels (entries <= 0 are kept; values are
 * capped at the maximum); the step's CUDA graphs are rebuilt at the next
 * dsmc_step. */
int dsmc_set_launch_config(dsmc_ctx *ctx, const int32_t *ctas_per_sm, int n);
/* Autotuner: for each tunable kernel in turn, times steps_per_trial steps
 * (CUDA events around the kernel) for each candidate shape (the maximum,
 * its half and quarter, 1, 2, 4, 8, 16 CTAs per SM) and keeps the fastest.
 * The trial steps are real steps of the run (it advances); re-initialise
 * afterwards for a run from step 0 with the tuned shapes. */
int dsmc_autotune(dsmc_ctx *ctx, int steps_per_trial);

/* How dsmc_step runs the steps of every case of the context (no counterpart
 * in the reference, whose ranks loop over MoveParticles .. Sampling):
 *   DSMC_STEP_GRAPH       one CUDA graph launch per step, the step's kernels
 *                         as its nodes (the default);
 *   DSMC_STEP_PERSISTENT  ONE cooperative kernel for all n_steps steps of a
 *                         dsmc_step call, launched as the kernel node of a
 *                         CUDA graph: every CTA stays resident and the
 *                         stages of a step are separated by grid barriers.
 * Both give identical particles, cell lists, counters and moments.  The
 * persistent grid is ctas_per_sm x SMs CTAs (0: the most that fit); every
 * barrier wait is bounded (about 2 s), after which the launch ends and
 * DSMC_ERR_TIMEOUT is reported.  DSMC_ERR_UNSUPPORTED when the device has
 * no cooperative launch; DSMC_ERR_STATE in the middle of a staged step.
 * dsmc_set_profiling's per-kernel timing always uses the graph sequence. */
enum { DSMC_STEP_GRAPH = 0, DSMC_STEP_PERSISTENT = 1 };
int dsmc_set_step_mode(dsmc_ctx *ctx, int mode, int ctas_per_sm);
/* The mode, the persistent grid's CTAs per SM and their maximum (0 without
 * cooperative launch), and whether persistent launches go through CUDA
 * graphs (1) or, where the driver refuses graphs of cooperative kernels,
 * are launched directly (0). */
int dsmc_get_step_mode(dsmc_ctx *ctx, int *mode, int *ctas_per_sm, int *max_ctas_per_sm,
                       int *graph_launch);
/* Device time of each phase of the persistent step (the stages between two
 * grid barriers: plan, move+inject, move_near, dead_scan, holes, tail,
 * cell_scan+tile_scan, olist+collide_select, cell_fix, scatter,
 * collide_pairs, sample), summed over the persistent steps run since the
 * last reset, in milliseconds, with the phase names; reset != 0 zeroes the
 * sums after reading them. */
int dsmc_get_phase_times(dsmc_ctx *ctx, double *ms_out, int max_phases, int *n_phases,
                         const char **names_out, int reset);
/* Test of the bounded grid-barrier wait: one CTA waits at a barrier that
 * one more CTA would have to reach (none does) and gives up after wait_ns
 * nanoseconds.  Returns DSMC_ERR_TIMEOUT, the status the kernel reported;
 * the context's own error word is untouched and it stays usable. */
int dsmc_grid_sync_probe(dsmc_ctx *ctx, int64_t wait_ns);

/* Per-kernel device time of the stages, for profiling.  When enabled,
 * dsmc_step brackets every kernel with CUDA events; dsmc_get_kernel_times
 * returns the summed milliseconds per kernel since the last reset and the
 * kernel names. */
int dsmc_set_profiling(dsmc_ctx *ctx, int enabled);
int dsmc_get_kernel_times(dsmc_ctx *ctx, double *ms_out, int64_t *launches_out, int max_kernels,
                          int *n_kernels, const char **names_out);

/* ---- unit kernels (parity tests of single device functions) ------------
 * Pointers are device pointers of n elements. */

/* IntersectBox (Geometry.cpp:179-229) over a batch of segments. */
int dsmc_k_intersect(const dsmc_params *p, int64_t n, const double *x, const double *y,
                     const double *dx, const double *dy, int32_t *hit, double *t_hit,
                     double *nx, double *ny, void *cuda_stream);

/* InsideBox (Geometry.cpp:173-177) over a batch of points; inside[i] = 0/1. */
int dsmc_k_inside_box(const dsmc_params *p, int64_t n, const double *x, const double *y,
                      int32_t *inside, void *cuda_stream);

/* One wall interaction per element (Boundary.cpp:205-282) with the case's
 * wall model; element i draws from stream (kind, step, entity[i]).  v is
 * 3*n doubles, (vx, vy, vz) per element, updated in place. */
int dsmc_k_scatter(const dsmc_params *p, const dsmc_derived *d, int64_t n, double *v,
                   const double *nx, const double *ny, uint32_t kind, uint32_t step,
                   const uint32_t *entity, void *cuda_stream);

/* GenerateNewParticles(X1, Y1, X2, Y2, Ngas, Ugasx, Ugasy, Tgas, MoveFlag)
 * (Boundary.cpp:60-92) on the rectangle rect = {X1, Y1, X2, Y2} (host
 * array), drawing from stream (kind, step, entity): the count (floor plus a
 * Bernoulli draw when the mean Ngas V / Weight exceeds 20, else a Poisson
 * draw), then per particle a uniform position and a Maxwellian velocity
 * around (Ugasx, Ugasy, 0) at Tgas, pre-moved by Dt when move_flag is 1.
 * The count is returned in *n_out (host; the call waits for it on the
 * stream); the particles are written to the device arrays x .. vz, which
 * hold `capacity` elements: DSMC_ERR_CAPACITY (nothing written) when the
 * count exceeds it.  d, when given, replaces the derived constants (Weight,
 * MoleculeMass, Dt come from p otherwise). */
int dsmc_k_inject(const dsmc_params *p, const dsmc_derived *d, const double *rect, double n_gas,
                  double ux_gas, double uy_gas, double t_gas, int move_flag, uint32_t kind,
                  uint32_t step, uint32_t entity, int64_t capacity, double *x, double *y,
                  double *vx, double *vy, double *vz, int64_t *n_out, void *cuda_stream);

/* BinaryCollisionsInCell(CellVolume, NPC, IPC) (Collision.cpp:21-44) for
 * n_lists independent lists: list l is IPC = ipc[list_start[l],
 * list_start[l + 1]) (indices into vx, vy, vz), or the particles
 * list_start[l] .. list_start[l + 1] - 1 themselves when ipc is NULL; it
 * draws from stream (kind, step, entity[l]) (entity NULL: l) and its NC is
 * written to n_collisions[l] (may be NULL).  Lists must not share particles.
 * All pointers are device pointers. */
int dsmc_k_collide(const dsmc_params *p, const dsmc_derived *d, double cell_volume,
                   int32_t n_lists, const int32_t *list_start, const int32_t *ipc, double *vx,
                   double *vy, double *vz, uint32_t kind, uint32_t step, const uint32_t *entity,
                   int32_t *n_collisions, void *cuda_stream);

/* ElasticCollision(V1, V2, Cr) (Collision.cpp:7-19) per pair i: v1, v2 are
 * 3*n doubles updated in place, cr[i] the relative speed; pair i draws from
 * stream (kind, step, entity[i]) (entity NULL: i). */
int dsmc_k_elastic(const dsmc_params *p, int64_t n, double *v1, double *v2, const double *cr,
                   uint32_t kind, uint32_t step, const uint32_t *entity, void *cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* DSMC_H */
