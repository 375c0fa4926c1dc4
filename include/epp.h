/*
 * epp.h -- C ABI of libepp.so, the B200 (sm_100a) SPH time-step backend for
 * EtherParallelParticles.jl.
 *
 * The reference reaches its device through three Julia entry points that take a
 * particle system, a domain, a neighbour system and a user closure:
 *   Algorithm.search!       src/Algorithm/NeighbourSearch.jl:323-347 (static_search! :349-377)
 *   Algorithm.interaction!  src/Algorithm/Action.jl:140-152 (static_interaction! :154-181)
 *   Algorithm.selfaction!   src/Algorithm/Action.jl:53-67 (static_selfaction! :69-93)
 * plus the host<->device mirror Class.syncto!/asyncto!
 *   src/Class/ParticleSystem/ParticleSystem.jl:275-307, ParticleSystemBase.jl:33-50.
 * Closures cannot cross a C ABI, so the actions are named bundles (EPP_ACTION_*)
 * and the search criteria are named (EPP_CRITERION_*).  The property matrices keep
 * the reference's layout: column-major, leading dimension = capacity, one column per
 * scalar (vectors take dim consecutive columns), 1-based particle and cell ids.
 *
 * Conventions: every function returns an epp_status (0 = EPP_OK).  Nothing throws,
 * aborts or traps.  Errors detected on the device set bits of a status word that
 * epp_synchronize returns.  A context is not thread-safe; use one per host thread.
 * All work is queued on the context's own CUDA stream; host buffers are borrowed
 * only for the duration of the call.  The library owns all device memory.
 */
#ifndef EPP_H
#define EPP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EPP_ABI_VERSION 4
#define EPP_MAX_TAGS 16

typedef enum epp_status {
    EPP_OK = 0,
    EPP_ERR_INVALID_ARGUMENT = 1,
    EPP_ERR_CUDA = 2,
    EPP_ERR_OUT_OF_MEMORY = 3,
    EPP_ERR_UNSUPPORTED_ACTION = 4,
    EPP_ERR_UNSUPPORTED_CRITERION = 5,
    EPP_ERR_STATE = 6,          /* call order: e.g. interaction! before any search! */
    EPP_ERR_DEVICE_STATUS = 7,  /* a device-side check failed; see the status word */
    EPP_ERR_BUDGET = 8,         /* HBM budget of the context or server exceeded */
    EPP_ERR_NO_DEVICE = 9,
    EPP_ERR_CAPACITY = 10       /* more particles than the context's capacity */
} epp_status;

/* Bits of the device status word (accumulated until read by epp_synchronize). */
#define EPP_STATUS_KILLED             (1u << 0) /* particles left the domain (info, as reference) */
#define EPP_STATUS_NEIGHBOUR_OVERFLOW (1u << 1) /* a list exceeded max_neighbour_number */
#define EPP_STATUS_CELL_OVERFLOW      (1u << 2) /* a cell exceeded max_cell_particles */
#define EPP_STATUS_NONFINITE          (1u << 3) /* NaN/Inf in density or velocity */
#define EPP_STATUS_SPIN_TIMEOUT       (1u << 4) /* a bounded device wait gave up */
#define EPP_STATUS_BAD_TAG            (1u << 5) /* tag outside 1..n_tags */
#define EPP_STATUS_QUEUE              (1u << 6) /* persistent work queue inconsistency */

/* Search criteria: src/Algorithm/NeighbourSearch.jl:141-164 */
#define EPP_CRITERION_DEFAULT  0 /* dr^2 <= gap^2                       (:141-151) */
#define EPP_CRITERION_SYMMETRY 1 /* dr^2 <= (2 harmonic(h_i, h_j))^2    (:153-164) */

/* Named actions.  The dam-break bundle restates example/collapse_dry/same/main.jl:74-126
 * with the physics substitutions of the benchmark cases (Wendland C2, Tait EOS,
 * artificial viscosity, symplectic Euler). */
#define EPP_ACTION_NONE                  0 /* defaultSelfaction!  Action.jl:27-35 */
#define EPP_ACTION_DAMBREAK_CONTINUITY   1 /* search! action: kernel cache + continuity  main.jl:74-90 */
#define EPP_ACTION_DAMBREAK_DENSITY      2 /* selfaction!: rho += drho dt, V = m/rho, p = eos  main.jl:92-105 */
#define EPP_ACTION_DAMBREAK_MOMENTUM     3 /* interaction!: pressure + artificial viscosity  main.jl:107-118 */
#define EPP_ACTION_DAMBREAK_INTEGRATE    4 /* selfaction!: gravity, sAccelerate!, sMove!  main.jl:120-126 */
#define EPP_ACTION_ZERO_DVELOCITY        5 /* selfaction!: dVelocity = 0 (test helper, ActionTest.jl:66-69) */
#define EPP_ACTION_COUNT_NEIGHBOURS      6 /* interaction!: dVelocity += 1 per neighbour (ActionTest.jl:71-75) */
#define EPP_ACTION_KERNEL_FILTER         7 /* interaction!: iFilter, fluid-fluid: wv += W V_j, wv_rho += W m_j
                                            * (main.jl:128-134, Filter.jl:10-23) */
#define EPP_ACTION_KERNEL_FILTER_SELF    8 /* selfaction!: sFilter, fluid: rho = (wv_rho + W0 m)/(wv + W0 V),
                                            * V = m/rho, p = eos (main.jl:136-144, Filter.jl:25-38) */
#define EPP_ACTION_EXTRAPOLATE_PRESSURE  9 /* interaction!: wall i, fluid j: iExtrapolatePressure!
                                            * wv += W V_j, wv_p += W V_j (max(p_j, p0) + max(rho_j g.r_ij, p0))
                                            * (Pressure.jl:85-131; p0 and g of the physics) */
#define EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF 10 /* selfaction!: wall: sExtrapolatePressure! p = wv_p / wv,
                                                * or p0 without fluid neighbours (Pressure.jl:133-150) */

/* epp_search flags */
#define EPP_SEARCH_EMIT_LIST 1 /* keep per-particle neighbour lists for epp_download */

/* Viscosity forms */
#define EPP_VISCOSITY_REFERENCE 0 /* artificial, Viscosity.jl:28-52 as written: extra 1/(rho_i rho_j) */
#define EPP_VISCOSITY_MONAGHAN  1 /* artificial, textbook Monaghan: divide by the mean density only */
#define EPP_VISCOSITY_CLASSIC   2 /* physical, iClassicViscosity! (Viscosity.jl:10-26) with mu */

/* Smoothing kernels (src/SPH/Kernel/: WendlandC2.jl, CubicSpline.jl, Gaussian.jl, WendlandC4.jl) */
#define EPP_KERNEL_WENDLAND_C2  0
#define EPP_KERNEL_CUBIC_SPLINE 1
#define EPP_KERNEL_GAUSSIAN     2
#define EPP_KERNEL_WENDLAND_C4  3

/* Equations of state */
#define EPP_EOS_TAIT   0 /* p = rho0 c0^2 / gamma ((rho/rho0)^gamma - 1) + p0 (benchmark) */
#define EPP_EOS_LINEAR 1 /* p = c0^2 (rho - rho0) + p0 (main.jl:64) */

/* Time integration of the fluid */
#define EPP_MOTION_SYMPLECTIC       0 /* sAccelerate! + sMove!: u += du dt, x += u dt (Motion.jl:17-51) */
#define EPP_MOTION_ACCELERATE_MOVE  1 /* sAccelerateMove!: x += (u + du dt/2) dt, u += du dt (Motion.jl:61-75) */

/* Pressure term of a pair (Pressure.jl:24-83); DEFAULT is the dam break's choice per pair type:
 * CLASSIC for fluid-fluid (main.jl:109), BALANCED for fluid-wall (main.jl:113) */
#define EPP_PRESSURE_DEFAULT          0
#define EPP_PRESSURE_CLASSIC          1 /* iClassicPressure!: p_i / rho_i^2 + p_j / rho_j^2 */
#define EPP_PRESSURE_BALANCED         2 /* iBalancedPressure!: (p_i + p_j) / (rho_i rho_j) */
#define EPP_PRESSURE_DENSITY_WEIGHTED 3 /* iDensityWeightedPressure!: 2 (p_i rho_i + p_j rho_j) /
                                         * ((rho_i + rho_j) rho_i rho_j) */

/* Wall pressure in epp_step */
#define EPP_WALL_PRESSURE_EOS         0 /* p = eos(rho) like the fluid (main.jl:99-102) */
#define EPP_WALL_PRESSURE_EXTRAPOLATE 1 /* after each density update, EXTRAPOLATE_PRESSURE(_SELF) */

typedef struct epp_domain {
    int32_t dim;      /* 2 (Domain2D, src/Class/Domain/Domain2D.jl:28-67) or 3 (new) */
    float gap;        /* cell size; the reference uses 2h */
    float first[3];   /* lower corner */
    float last[3];    /* upper corner */
} epp_domain;

typedef struct epp_physics {
    float dt;             /* time step (fixed, as the reference: main.jl:68) */
    float rho0;           /* reference density */
    float c0;             /* speed of sound */
    float p0;             /* background pressure added by the EOS */
    int32_t gamma;        /* Tait exponent, integer (7) */
    float gravity[3];
    float alpha;          /* artificial viscosity alpha (Viscosity.jl:36) */
    float beta;           /* artificial viscosity beta (reference default 0.1, Viscosity.jl:37) */
    int32_t viscosity;    /* EPP_VISCOSITY_* */
    int32_t fluid_tag;    /* 1 in the reference example */
    int32_t wall_tag;     /* 2 in the reference example */
    int32_t kahan;        /* 1: compensated (Kahan) position update; 0: sMove! as written */
    /* Zero in each field below is the benchmark physics (Wendland C2, Tait, symplectic Euler, no
     * filter, the dam break's pressure terms, no tensile correction, wall pressure from the EOS);
     * the reference example (example/collapse_dry/same/main.jl) is CUBIC_SPLINE, LINEAR,
     * EPP_VISCOSITY_CLASSIC with mu = 1e-3, ACCELERATE_MOVE and filter_interval = 20. */
    int32_t kernel;           /* EPP_KERNEL_* */
    int32_t eos;              /* EPP_EOS_* */
    float mu;                 /* dynamic viscosity of EPP_VISCOSITY_CLASSIC */
    int32_t motion;           /* EPP_MOTION_* */
    int32_t filter_interval;  /* epp_step: kernel filter after the search of every k-th step
                               * (steps counted from 1 after epp_upload, main.jl:180-183); 0 = never */
    int32_t pressure_ff;      /* EPP_PRESSURE_* of fluid-fluid pairs */
    int32_t pressure_fw;      /* EPP_PRESSURE_* of fluid-wall pairs */
    int32_t tensile;          /* 1: iPressureCorrection (Pressure.jl:10-22) on both: the pressure term
                               * grows by |term| 0.01 W(r) / W((gap_i + gap_j) / 2); needs the gap column */
    int32_t wall_pressure;    /* EPP_WALL_PRESSURE_* */
    float cfl;                /* 0: every step takes dt (the reference's fixed step, main.jl:68).
                               * > 0: each epp_step step takes dt = cfl h_min / (c0 + max|v|) of the
                               * state it starts from: max|v| and h_min (smallest H) over the alive
                               * fluid particles, per instance in a batch with the instance's c0,
                               * reduced in FP64 on the device inside the step (no host round trip)
                               * and rounded once to FP32.  At rest, cfl = 0.1 gives the reference's
                               * dt = 0.1 h / c0.  The per-call selfaction!(DAMBREAK_DENSITY) takes
                               * the same dt of the current state; INTEGRATE reuses it. */
} epp_physics;

typedef struct epp_config {
    epp_domain domain;
    int32_t n_capacity;            /* rows of the property matrices (at most 2^28: EPP_ERR_CAPACITY) */
    int32_t max_neighbour_number;  /* list capacity for EPP_SEARCH_EMIT_LIST (reference: 50) */
    int32_t max_cell_particles;    /* reference bucket capacity; only checked (0 = unchecked) */
    int32_t n_tags;                /* adjacency matrix is n_tags x n_tags, tags are 1-based */
    int32_t adjacency[EPP_MAX_TAGS * EPP_MAX_TAGS]; /* row-major [tag_i-1][tag_j-1] */
    int32_t device;                /* CUDA ordinal */
    int64_t hbm_budget_bytes;      /* 0 = unlimited; creation fails with EPP_ERR_BUDGET above it */
    int32_t n_instances;           /* batch: independent 2D systems on the same domain (0 or 1 = one);
                                    * particles carry their instance in the `instance` column and
                                    * never interact across instances */
} epp_config;

/* 0-based column indices into the caller's property matrices; -1 = absent.
 * Vector properties occupy dim consecutive columns starting at the index. */
typedef struct epp_column_map {
    /* int_properties_ */
    int32_t tag, is_movable, n_count, n_index;
    /* float_properties_ */
    int32_t position, velocity, dvelocity, mass, volume, density, ddensity, pressure, gap, h;
    int32_t n_rvec, n_r, n_w, n_dw, n_hinv;
    int32_t instance;   /* int column: 0-based instance of a batch (-1: all in instance 0) */
} epp_column_map;

typedef struct epp_integrals {
    double mass_total;      /* sum m over alive particles */
    double mass_fluid;      /* sum m over alive fluid particles */
    double kinetic;         /* sum 1/2 m |v|^2 (fluid) */
    double potential;       /* sum -m g.x (fluid) */
    double internal;        /* sum m e(rho), Tait internal energy (fluid) */
    double max_speed;       /* max |v| (fluid) */
    double cfl_dt;          /* cfl h_min / (c0 + max|v|) (cfl of the physics, 0.1 when it is 0): the
                             * CFL time step of this state, in FP64 (epp_step rounds it to FP32) */
    int64_t n_alive;
    int64_t n_pairs;        /* directed active neighbour pairs of the last search */
} epp_integrals;

typedef struct epp_ctx epp_ctx;

/* Library */
int32_t epp_abi_version(void);
int32_t epp_device_count(int32_t* count);

/* Context lifetime */
int32_t epp_create(const epp_config* config, epp_ctx** out);
int32_t epp_destroy(epp_ctx* ctx);
const char* epp_last_error(const epp_ctx* ctx);

/* Host <-> device in the reference layout (Class.asyncto!, ParticleSystem.jl:292-307).
 * int_props / float_props are column-major with leading dimension ld_int / ld_float.
 * is_alive and cell_index are the base_.is_alive_ / base_.cell_index_ vectors (cell ids
 * 1-based, 0 = not binned).  Download writes only mapped columns; neighbour columns are
 * written when the last search used EPP_SEARCH_EMIT_LIST. */
int32_t epp_upload(epp_ctx* ctx, int32_t n_particles, const int32_t* is_alive,
                   const int32_t* cell_index, const int32_t* int_props, int64_t ld_int,
                   const float* float_props, int64_t ld_float, const epp_column_map* map);
int32_t epp_download(epp_ctx* ctx, int32_t* is_alive, int32_t* cell_index, int32_t* int_props,
                     int64_t ld_int, float* float_props, int64_t ld_float,
                     const epp_column_map* map);

/* Algorithm layer.  Each call is asynchronous on the context stream.
 *   epp_search      replaces Algorithm.search!       (NeighbourSearch.jl:323-347)
 *   epp_interaction replaces Algorithm.interaction!  (Action.jl:140-152)
 *   epp_selfaction  replaces Algorithm.selfaction!   (Action.jl:53-67) */
int32_t epp_search(epp_ctx* ctx, int32_t criterion, int32_t action, const epp_physics* phys,
                   int32_t flags);
int32_t epp_interaction(epp_ctx* ctx, int32_t action, const epp_physics* phys);
int32_t epp_selfaction(epp_ctx* ctx, int32_t action, const epp_physics* phys);

/* The whole dam-break time step of main.jl:166-182 (density update, momentum,
 * integrate, search + continuity), fused into 6 kernels and replayed as a CUDA graph.
 * Requires one prior epp_search with EPP_ACTION_DAMBREAK_CONTINUITY (main.jl:157-164). */
int32_t epp_step(epp_ctx* ctx, int32_t n_steps, const epp_physics* phys);

/* FP64 reductions of the current state. */
int32_t epp_get_integrals(epp_ctx* ctx, const epp_physics* phys, epp_integrals* out);

/* The same reductions without blocking: epp_integrals_async enqueues them for the current state
 * (their copy to the host included) on a second stream of the context, once the work queued
 * before has finished, and returns a ticket; epp_integrals_wait(ticket) waits for them and fills
 * `out`.  The next epp_step runs beside them (it reads the state they reduce and writes the
 * other buffer set); any other call that could change that state waits for them first.  At most
 * EPP_INTEGRALS_SLOTS tickets may be outstanding (EPP_ERR_STATE beyond). */
#define EPP_INTEGRALS_SLOTS 4
int32_t epp_integrals_async(epp_ctx* ctx, const epp_physics* phys, int64_t* ticket);
int32_t epp_integrals_wait(epp_ctx* ctx, int64_t ticket, epp_integrals* out);

/* Parity access to the cell list: counts[n_cells] per cell, offsets[n_cells+1] exclusive
 * scan, sorted_ids[n_alive] 1-based particle ids in cell order (within a cell by id).
 * Any pointer may be NULL. */
int32_t epp_cell_stats(epp_ctx* ctx, int32_t* counts, int32_t* offsets, int32_t* sorted_ids,
                       int32_t* n_cells);

/* Parity access to the neighbour lists the default pair passes (family 0) read, as the search pass
 * built them at the last epp_search or epp_step: counts[row] = nCount of the particle in caller row
 * `row` (0 for particles not alive), and ids[k * ld + row] for k < min(counts[row], max_nb) = the
 * 1-based id of its k-th neighbour in list order (stencil rows, then cell order, then id order
 * inside a cell).  A particle with more neighbours than a list keeps (64 in 2D, 160 in 3D; its
 * pair passes read its stencil instead) has its ids left as they were.  ids may be NULL.
 * Replaces reading the nCount / nIndex columns of the reference's particle system after search!
 * (NeighbourSearch.jl:166-227). */
int32_t epp_neighbour_lists(epp_ctx* ctx, int32_t* counts, int32_t* ids, int64_t ld, int32_t max_nb);

/* Waits for the context stream; returns EPP_ERR_DEVICE_STATUS when a device check failed
 * (bits in *device_status, which is then cleared). device_status may be NULL. */
int32_t epp_synchronize(epp_ctx* ctx, uint32_t* device_status);

/* Time stepping: next_dt[k] = the dt the next step of instance k takes under `phys` (phys->dt, the
 * instance's dt, or with phys->cfl > 0 the CFL dt of the current state, computed on the device);
 * sim_time[k] = simulated time advanced by epp_step since the last epp_upload (the sum of the dt
 * of every step taken).  n = the context's instances (1 without a batch); either array may be
 * NULL.  No reference counterpart: main.jl:165-206 keeps t on the host with its fixed dt. */
int32_t epp_step_dt(epp_ctx* ctx, const epp_physics* phys, int32_t n, float* next_dt, double* sim_time);

/* Device time of the last epp_step call (ms, CUDA events on the context stream). */
int32_t epp_last_step_timing(epp_ctx* ctx, float* ms_total);

/* Directed active pairs found by all searches of this context so far (the numerator of the
 * pair-interactions/s metric; each step's search counts its pairs once). */
int32_t epp_pairs_total(epp_ctx* ctx, int64_t* out);

/* Optional dv/dt output of the fused step (momentum sum + gravity, before integration), for
 * per-step force comparisons.  epp_get_accel writes out[a * n + row] for a < dim. */
int32_t epp_set_accel_output(epp_ctx* ctx, int32_t enable);
int32_t epp_get_accel(epp_ctx* ctx, float* out, int32_t n);

/* Batch: per-instance time step and speed of sound (Tait B = rho0 c0^2 / gamma per instance);
 * they override phys.dt / phys.c0 of epp_step for instance k = 0..n-1. */
int32_t epp_set_instance_physics(epp_ctx* ctx, int32_t n, const float* dt, const float* c0);
/* Batch: FP64 integrals of every instance, out[0..n_instances). */
int32_t epp_get_instance_integrals(epp_ctx* ctx, const epp_physics* phys, epp_integrals* out, int32_t n);

/* Pair-pass kernel family (batches of more than one instance use family 0): 0 (default) = one
 * warp tile of 32 particles per warp, neighbours filtered once per step into a per-particle
 * neighbour list that the momentum pass reuses; 1 = one warp per occupied cell with a compacted
 * pair queue; 2, 4, 8, 16 or 32 = that many lanes of a warp per particle.  Chosen by the
 * autotuner; results change only at the FP32 rounding level (neighbour sets are identical).
 * In 2D, family 0's search pass tests each particle's own stencil-row windows (cells cx-1 .. cx+1
 * of each stencil row, staged per warp in shared memory) and runs the search action (continuity
 * and the density preview) in the same pass; EPP_TUNING_LISTS selects family 0 with the lockstep
 * warp-tile search and a separate continuity pass instead (the 3D form): the same neighbour lists,
 * sums equal to FP32 rounding. */
#define EPP_TUNING_LISTS 64
int32_t epp_set_tuning(epp_ctx* ctx, int32_t lanes_per_particle);
/* Threads per block of the family-0 search and list passes: 128 (default), 64 or 32.  Smaller
 * blocks spread a small system over more SMs; results do not change (the per-particle order is
 * independent of the block size).  Chosen by the autotuner. */
int32_t epp_set_block_threads(epp_ctx* ctx, int32_t threads);

/* Queue the context's work on a caller-owned cudaStream_t (passed as void*; NULL restores the
 * context's own stream).  Lets a host application order it with its own work and events. */
int32_t epp_set_stream(epp_ctx* ctx, void* stream);

/* Serving support (no reference counterpart: the reference runs one simulation per process).
 * epp_context_bytes: device bytes epp_create would allocate for this configuration, without
 * allocating (the optional neighbour-list emission and dv/dt output are extra); a server admits
 * simulations against an HBM budget with it.  Context memory comes from the stream-ordered
 * allocator, so creating or destroying a context does not synchronise the device.
 * epp_query: *done = 1 when every call queued on the context has finished on the device, 0 while
 * work is pending; never blocks. */
int32_t epp_context_bytes(const epp_config* cfg, int64_t* bytes);
int32_t epp_query(epp_ctx* ctx, int32_t* done);
/* Recreate the context's own stream with a CUDA stream priority (lower value = scheduled first;
 * clamped to the device's range, the value used returned in *applied).  A server gives short
 * runs the higher priorities so they finish first while long runs fill the remaining SMs. */
int32_t epp_set_priority(epp_ctx* ctx, int32_t priority, int32_t* applied);

/* Native serving loop (no reference counterpart: the reference runs one simulation per
 * process).  The same loop as the Python serving module, behind the C ABI so that a Julia or C
 * host can use it: each submitted simulation (a dam-break state in the reference layout, its
 * physics and step count) waits in a FIFO queue; epp_server_poll admits from the head while the
 * resident contexts' epp_context_bytes stay within the budget (a request that can never fit
 * fails with EPP_ERR_BUDGET), gives each admitted run its own context and a stream priority by
 * size, keeps `ahead` chunks of `chunk_steps` steps queued on every resident stream (refilled
 * when epp_query reports it drained), and retires a run after its last step with its FP64
 * integrals (and, if asked at submit, its final state).  Every run uses the plain path's kernels
 * and graphs, so its result equals the same simulation run alone.  A server is not thread-safe:
 * drive it from one host thread.
 *   epp_server_submit   copies the state (the caller's arrays may be reused at once); the
 *                       initial search and all steps run later, inside epp_server_poll
 *   epp_server_poll     one non-blocking pass of the loop; counts of waiting, resident, finished
 *   epp_server_drain    polls until every submitted request has finished or failed
 *   epp_server_result   a finished request's integrals, device status, and seconds from submit
 *                       to admission and to completion; EPP_ERR_STATE while it is not finished,
 *                       the request's own error code if it failed
 *   epp_server_download its final state (submit with keep_state = 1), written like epp_download
 *                       into arrays of the submitted layout */
typedef struct epp_server epp_server;
typedef struct epp_server_stats {
    int64_t submitted, completed, failed;
    int64_t peak_resident_bytes;
    int32_t max_concurrent;
    int32_t waiting, active;
} epp_server_stats;
int32_t epp_server_create(int32_t device, int64_t budget_bytes, int32_t max_active, int32_t chunk_steps,
                          int32_t ahead, epp_server** out);
int32_t epp_server_destroy(epp_server* server);
/* Co-batching (off by default): at admission the waiting requests that can share the head's cell
 * grid (2D, the same domain, tags, column map, step count, keep_state and physics apart from dt
 * and c0; no instance column of their own) join it, up to batch_max, as the instances of one
 * batch context: one launch per pass for all of them.  Each keeps its own dt and c0; its state
 * equals the request run alone, its FP64 integrals agree to rounding (another summation order). */
int32_t epp_server_set_co_batch(epp_server* server, int32_t enabled, int32_t batch_max);
int32_t epp_server_submit(epp_server* server, const epp_config* config, int32_t n_particles,
                          const int32_t* is_alive, const int32_t* cell_index, const int32_t* int_props,
                          int64_t ld_int, const float* float_props, int64_t ld_float,
                          const epp_column_map* map, const epp_physics* phys, int32_t n_steps,
                          int32_t keep_state, int64_t* request_id);
int32_t epp_server_poll(epp_server* server, epp_server_stats* stats);
int32_t epp_server_drain(epp_server* server, epp_server_stats* stats);
int32_t epp_server_result(epp_server* server, int64_t request_id, epp_integrals* integrals,
                          uint32_t* device_status, double* admit_s, double* done_s);
int32_t epp_server_download(epp_server* server, int64_t request_id, int32_t* is_alive, int32_t* cell_index,
                            int32_t* int_props, int64_t ld_int, float* float_props, int64_t ld_float);

/* One dam-break step launched kernel by kernel (no graph) with CUDA events between the
 * kernels; stage_ms[0 .. EPP_PROFILE_STAGES-1] = momentum+integrate+bin, scan, scatter,
 * rank+gather, search (neighbour lists), continuity (0 for pair-pass families that fuse the
 * search and continuity into one kernel).  Same results as epp_step(ctx, 1, phys). */
#define EPP_PROFILE_STAGES 6
int32_t epp_profile_step(epp_ctx* ctx, const epp_physics* phys, float* stage_ms);

/* Cell-list build that allocates nothing, for callers that must not call cudaMalloc while they
 * drive the library (a host application that owns a fixed device pool, or one that is in the
 * middle of a step where a device allocation would synchronise or is not allowed).  It has no
 * counterpart in the reference.  It runs the bin + count + scan + counting sort of epp_search's
 * cell-list build as one call on caller-owned device buffers.
 *   pos         device, column-major positions: x at pos[i], y at pos[n + i], z at pos[2n + i]
 *   counts      device [n_cells] or NULL;  offsets  device [n_cells + 1] or NULL
 *   sorted_ids  device [n]: 1-based particle ids in cell order, by id inside a cell (the first
 *               *n_alive entries are set; particles outside the domain are left out)
 *   n_alive     host: number of particles inside the domain
 *   stream      cudaStream_t (NULL = default stream); the call waits for it before returning
 * All intermediate arrays live in one static device array of this library (see
 * epp_noalloc_limits: up to 2^20 particles and 2^20 cells, about 29 MB, held by every GPU that
 * loads the library until the process exits).  Larger inputs return EPP_ERR_CAPACITY.  Every call
 * shares that array, so calls that overlap on the GPU (other streams, other host threads) race;
 * serialise them.  The first call on a device looks up the array's device address for that
 * device (cudaGetSymbolAddress), so make it before any stream capture; that look-up is guarded,
 * so first calls from several host threads are safe.  It calls no cudaMalloc, cudaFree or other
 * allocating routine.  A domain of more than 2^20 cells (checked axis by axis, before anything
 * runs on the GPU) returns EPP_ERR_CAPACITY; a device-side inconsistency returns
 * EPP_ERR_DEVICE_STATUS. */
int32_t epp_cell_sort_noalloc(const epp_domain* domain, int32_t n, const float* pos, int32_t* counts,
                              int32_t* offsets, int32_t* sorted_ids, int32_t* n_alive, void* stream);
int32_t epp_noalloc_limits(int32_t* max_particles, int32_t* max_cells, int64_t* scratch_bytes);

#ifdef __cplusplus
}
#endif

#endif /* EPP_H */
