/*
 * lbm_b200.h — C ABI of the B200 lattice-Boltzmann time-step library.
 *
 * This is the drop-in boundary for the time-step hot path of LBMengine.jl
 * (GPU module).  The reference has no FFI layer of its own: its boundary is
 * the exported Julia API (src/LBMengine.jl:27-41) and the fields of
 * `LBMmodel` / `LBMparticle` (src/gpu/structs.jl:52-95).  Each entry point
 * below names the reference function whose effect it reproduces; a Julia
 * shim binds them with `ccall` (lbmengine.jl_b200/julia/LBMengineB200.jl), a
 * Python mirror binds them with ctypes (lbmengine.jl_b200/lbmengine/_capi.py).
 *
 * Conventions
 *   - Every function returns an int status: 0 = LBM_OK, < 0 = error.  The
 *     message of the last failure is returned by lbm_last_error(h) (or by
 *     lbm_last_global_error() when no handle exists yet).
 *   - All caller buffers are HOST memory owned by the caller, FP64, in the
 *     reference's column-major order: scalar fields (N...) with x fastest,
 *     vector fields (N..., d) and populations (N..., Q) with the component /
 *     direction index slowest.  Cell index = x + nx*(y + ny*z).
 *   - The library owns all device memory; a handle is not thread-safe and
 *     issues all its work on one CUDA stream.
 *   - Lattice units follow the reference's GPU module: the time step equals
 *     the lattice parameter (dt == dx, src/gpu/initMethods.jl:475-492) and the
 *     lattice speed is 1.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define LBM_OK               0
#define LBM_ERR_INVALID     -1  /* bad argument (mirrors the reference's @assert / error sites) */
#define LBM_ERR_CUDA        -2  /* CUDA runtime failure */
#define LBM_ERR_OOM         -3  /* device allocation failed */
#define LBM_ERR_UNSUPPORTED -4  /* valid in the reference, not supported by this build */
#define LBM_ERR_NUMERIC     -5  /* NaN/Inf or non-positive density detected on device */
#define LBM_ERR_TIMEOUT     -6  /* a bounded device wait gave up */
#define LBM_ERR_STATE       -7  /* call not valid in the handle's current state */
#define LBM_ERR_NO_DEVICE   -8  /* no CUDA device / extension not usable */

/* ---- enumerations ------------------------------------------------------ */
/* velocity sets, src/gpu/misc.jl:195-272 */
#define LBM_D2Q9   9
#define LBM_D3Q15 15
#define LBM_D3Q19 19
#define LBM_D3Q27 27

/* collision model, src/gpu/fluids.jl:58-101 */
#define LBM_BGK 0
#define LBM_TRT 1

/* population storage on the device (the reference stores FP64 everywhere) */
#define LBM_STORE_F32  0   /* shifted FP32: (f_i/w_i - rho0) */
#define LBM_STORE_F16  1   /* shifted FP16: (f_i/w_i - rho0) * store_scale */
#define LBM_STORE_BF16 2   /* shifted BF16: (f_i/w_i - rho0) * store_scale */
#define LBM_STORE_F64  3   /* shifted FP64 (high-precision reference runs) */

/* particle kinds, src/gpu/initMethods.jl:7 (addBead!) and :91 (addSquirmer!) */
#define LBM_BEAD     0
#define LBM_SQUIRMER 1

/* force modes, src/gpu/initMethods.jl:636-654 */
#define LBM_FORCE_NONE    0
#define LBM_FORCE_UNIFORM 1   /* constant vector, zeroed on wall nodes */
#define LBM_FORCE_FIELD   2   /* (N..., d) field, zeroed on wall nodes */

/* ---- model configuration: the resolved keyword set of modelInit ---------
 * Replaces modelInit(; ...) src/gpu/initMethods.jl:440-702.  Keyword
 * resolution (tau from viscosity, default limits, walls from a Julia
 * function, ...) is done by the host shim; this struct carries the result. */
typedef struct lbm_config {
    int32_t dims;              /* 2 or 3 */
    int32_t lattice;           /* LBM_D2Q9 / LBM_D3Q15 / LBM_D3Q19 / LBM_D3Q27 */
    int64_t n[3];              /* nodes per axis; n[2] == 1 when dims == 2 */
    const double* coords[3];   /* node coordinates per axis (length n[a]), or NULL */
    double x0[3];              /* used when coords[a] == NULL: x = x0[a] + i*dx */
    double dx;                 /* lattice parameter == time step */
    double tau;                /* relaxation time (relaxationTimeRatio * dt); tau+ for TRT */
    double tau_minus;          /* TRT tau- (kineticParameter*c_s^2*dt^2/nu + dt/2), ignored for BGK */
    int32_t collision;         /* LBM_BGK / LBM_TRT */
    int32_t compressible;      /* isFluidCompressible (src/gpu/fluids.jl:50-51) */
    int32_t force_mode;        /* LBM_FORCE_* */
    int32_t storage;           /* LBM_STORE_* */
    double force[3];           /* uniform force density (force_mode == LBM_FORCE_UNIFORM) */
    const double* force_field; /* (N..., d) (force_mode == LBM_FORCE_FIELD) */
    const uint8_t* wall_mask;  /* (N...) solid wall nodes, or NULL (no bounce-back walls) */
    const double* wall_velocity; /* (N..., d) moving-wall velocity, or NULL */
    const double* rho_init;    /* (N...) initial density, or NULL -> rho_uniform */
    const double* u_init;      /* (N..., d) initial velocity, or NULL -> u_uniform */
    double rho_uniform;        /* initial density when rho_init == NULL */
    double u_uniform[3];       /* initial velocity when u_init == NULL */
    double rho_ref;            /* shift density rho0 of the stored populations (0 -> 1.0) */
    double store_scale;        /* power-of-two scale for F16/BF16 storage (0 -> default 2^12) */
    int32_t device;            /* CUDA device ordinal; < 0: the calling thread's current device */
    int32_t schedule;          /* LBM_SCHEDULE_*: how the kernels of a tick are launched */
    int32_t particle_rules;    /* LBM_RULES_*: which of the reference's two modules the particle update follows */
    int32_t rounding;          /* LBM_ROUND_*: rounding of the F16/BF16 stores */
} lbm_config;

/* Rounding of the populations stored in F16/BF16 (FP32/FP64 ignore it).
 *   STOCHASTIC (default)  the fraction below the kept bits is rounded up when
 *                         it exceeds a dither that is a hash of the cell and of
 *                         kept bits of the node's values, so the rounding
 *                         errors of a uniform region have zero mean instead
 *                         of adding up tick after tick (a uniformly forced
 *                         fluid otherwise drifts by ~1e-3 of its velocity
 *                         within a few hundred ticks); deterministic, costs
 *                         three integer operations per stored value
 *   NEAREST               round to nearest even */
#define LBM_ROUND_STOCHASTIC 0
#define LBM_ROUND_NEAREST 1

/* Particle update rules.  The reference has two implementations of the
 * particle update, picked when the package loads (src/LBMengine.jl:10-24):
 *   GPU_MODULE  moveParticles! of src/gpu/particles.jl:7-92 (the default):
 *               v += dt F/m and R += dt v only with coupleForces, Rodrigues
 *               rotation of the swimming direction with coupleTorques;
 *   CPU_MODULE  moveParticles! of src/cpu/particles.jl:48-100: v += dP/m and
 *               w += dL/I from the summed momentum inputs, R += dt v whenever
 *               v != 0 (whatever coupleForces says), the swimming direction
 *               never rotates, and the node (slip) velocity is the CPU
 *               module's bulkVelocity (:21-46).
 * The fluid step is the same in both (src/gpu/fluids.jl:132-226 and
 * src/cpu/fluids.jl:377-461). */
#define LBM_RULES_GPU_MODULE 0
#define LBM_RULES_CPU_MODULE 1

/* Kernel schedule of a tick.  Results do not depend on it (the per-node
 * arithmetic is the same).
 *   STREAM      bulk -> fix-up in stream order, particle update on a side
 *               stream overlapping the next bulk pass (AUTO: the default)
 *   PERSISTENT  one persistent kernel per tick over a work queue of bulk
 *               tiles, fix-up blocks and particle updates (vector bulk kernel
 *               with rows of at most 256 nodes; otherwise STREAM)
 * (value 2 is reserved) */
#define LBM_SCHEDULE_AUTO 0
#define LBM_SCHEDULE_STREAM 1
#define LBM_SCHEDULE_PERSISTENT 3

/* ---- particle parameters: the resolved keyword set of addBead!/addSquirmer!
 * Replaces src/gpu/initMethods.jl:7-89 and :91-222.  The shim resolves B1/B2
 * from swimmingSpeed/slipSpeed/beta and normalises and signs the swimming
 * direction (:133-173); the library computes the mass exactly as the
 * reference does (node count of an origin-centred sphere, :108) and the
 * moment of inertia (:117-127). */
typedef struct lbm_particle_params {
    int32_t kind;              /* LBM_BEAD / LBM_SQUIRMER */
    int32_t couple_forces;     /* coupleForces */
    int32_t couple_torques;    /* coupleTorques */
    int32_t reserved;
    double radius;
    double mass_density;
    double position[3];
    double velocity[3];
    double angular_velocity[3];   /* 2D: angular_velocity[0] is the scalar omega */
    double swimming_direction[3]; /* squirmer only; already normalised and signed */
    double B1, B2;                /* squirmer only */
} lbm_particle_params;

/* ---- particle state (read back) ----------------------------------------
 * Mirrors LBMparticle (src/gpu/structs.jl:85-95) after a tick. */
typedef struct lbm_particle_state {
    int32_t id;                /* 1-based, as LBMparticle.id */
    int32_t kind;
    int32_t couple_forces;
    int32_t couple_torques;
    double radius;
    double inverse_mass;
    double inverse_inertia;
    double B1, B2;
    double position[3];
    double velocity[3];
    double angular_velocity[3];   /* 2D: [0] */
    double swimming_direction[3];
    double last_force[3];      /* momentum-exchange force of the last tick (forceInput before reset) */
    double last_torque[3];     /* 2D: [0] */
} lbm_particle_state;

typedef struct lbm_info {
    int32_t dims, lattice, q, storage;
    int64_t n[3];
    int64_t cells;
    int64_t tick;
    double time;
    int32_t num_particles;
    int32_t bytes_per_population;  /* storage bytes of one population value */
    int64_t device_bytes;          /* device memory held by the handle */
    int32_t bulk_kernel;           /* LBM_BULK_*: the stream-collide kernel lbm_step launches */
    int32_t bulk_threads;          /* its threads per CTA */
    int32_t bulk_stages;           /* shared-memory ring buffers (TMA kernel), else 0 */
    int32_t reserved;
} lbm_info;

/* Bulk stream-collide kernel of a tick (results do not depend on it).
 *   SCALAR  one node per thread (FP64 storage, per-node force fields, rows
 *           that are not a multiple of 4 nodes or wider than 2048)
 *   VECTOR  four x-nodes per thread, vector loads and stores
 *   TMA     as VECTOR, with the loads issued as bulk copies by the Tensor
 *           Memory Accelerator through a ring of shared-memory buffers; for
 *           x-rows of 4*2^k <= 128 nodes
 * lbm_set_bulk_kernel(h, kind, threads, stages): AUTO (the default) is
 * VECTOR; threads per CTA and ring buffers of the TMA kernel
 * (0: chosen by the library).  LBM_ERR_UNSUPPORTED where the kind or shape
 * does not apply. */
#define LBM_BULK_AUTO 0
#define LBM_BULK_VECTOR 1
#define LBM_BULK_TMA 2
#define LBM_BULK_SCALAR 3

typedef struct lbm_handle lbm_handle;

/* Library identity. */
int32_t lbm_abi_version(void);
const char* lbm_build_info(void);

/* modelInit(; ...)  src/gpu/initMethods.jl:440-702 (with findInitialConditions
 * :417-438 and the initial hydroVariablesUpdate! src/gpu/fluids.jl:32). */
int lbm_create(const lbm_config* cfg, lbm_handle** out);

/* addBead! / addSquirmer!  src/gpu/initMethods.jl:7-89 / :91-222, including
 * the initial-setup moveParticles! (src/gpu/particles.jl:7-92).
 * *id_out receives the 1-based particle id. */
int lbm_add_particle(lbm_handle* h, const lbm_particle_params* p, int32_t* id_out);

/* LBMpropagate!(model; ticks = nsteps)  src/gpu/fluids.jl:228-264: nsteps
 * calls of tick! (:132-226), each = collision + streaming + bounce-back +
 * moving walls + Ladd coupling + hydro update + particle update. */
int lbm_step(lbm_handle* h, int64_t nsteps);

/* model.massDensity (N...) and model.fluidVelocity (N..., d) after the last
 * tick (hydroVariablesUpdate!, src/gpu/fluids.jl:32-37).  Either may be NULL. */
int lbm_get_fields(lbm_handle* h, double* rho, double* u);

/* viscousStressTensor(model) (src/cpu/fluids.jl:507-520; the GPU module's
 * copy is commented out, src/gpu/fluids.jl:272-285): sigma_ab =
 * -(1 - dt/(2 tau)) sum_i c_ia c_ib (f_i - f_eq_i) at the current rho and u,
 * as (N..., d, d) FP64 column-major, entry (a, b) of cell c at
 * sigma[c + N*(a + d*b)], computed on the device. */
int lbm_get_stress(lbm_handle* h, double* sigma);

/* Output of LBMpropagate!(...) with the :saveData scheme (src/gpu/fluids.jl:243-259).
 *
 * lbm_record_trajectories: from now on the particle update records, after
 * every tick, each particle's position, velocity and angular velocity
 * (writeParticleTrajectory, src/gpu/aux.jl:319-356) into a device ring of
 * `capacity` ticks (0: stop); no host synchronisation per tick, so stepping
 * stays graph-replayed.  Adding a particle restarts the ring.
 * lbm_read_trajectories: the ticks recorded since the last read, oldest
 * first, as out[(t * P + p) * 9 + k] (k: position 0-2, velocity 3-5,
 * angular velocity 6-8; 2D angular velocity at 6); *ticks = how many (with
 * out == NULL only the count).  They are the last *ticks ticks of the model.
 * LBM_ERR_STATE if more ticks than the ring holds passed since the last read.
 *
 * lbm_write_fluid_csv: writeTrajectories (src/gpu/aux.jl:271-317), the file
 * `fluidTrj_<tick>.csv` of the reference: per node tick, time, id_*,
 * coordinate_*, massDensity, fluidVelocity_*, f1..fQ, numbers printed as
 * Julia prints them.  The fields are read back at once; the file is
 * formatted and written by a host thread while the caller steps on.
 * lbm_output_flush waits for it (and reports a failed write); the next
 * lbm_write_fluid_csv and lbm_destroy wait too. */
int lbm_record_trajectories(lbm_handle* h, int64_t capacity);
int lbm_read_trajectories(lbm_handle* h, double* out, int64_t capacity, int64_t* ticks);
int lbm_write_fluid_csv(lbm_handle* h, const char* path);
int lbm_output_flush(lbm_handle* h);

/* Global sums over the lattice in FP64, on the device in a fixed order:
 * mass = sum of rho, momentum = sum of rho u (the momentum density of
 * hydroVariablesUpdate!, with the Guo half force; wall nodes contribute
 * zero), in lattice units (multiply by dx^d for physical units).  No
 * counterpart in the reference; for conservation checks. */
int lbm_get_totals(lbm_handle* h, double* mass, double* momentum);

/* model.distributions (N..., Q), FP64. */
int lbm_get_distributions(lbm_handle* h, double* f);

/* Overwrite the populations (N..., Q) from the host (checkpoint restore). */
int lbm_set_distributions(lbm_handle* h, const double* f);

/* model.particles[...] state; writes min(capacity, P) entries, *count = P. */
int lbm_get_particles(lbm_handle* h, lbm_particle_state* out, int32_t capacity, int32_t* count);

/* Overwrite position / velocity / angular velocity / swimming direction of
 * particle `id` (1-based) and re-voxelise it (moveParticles! initialSetup). */
int lbm_set_particle(lbm_handle* h, int32_t id, const lbm_particle_state* s);

/* Report the momentum-exchange force (last_force) of particle `id` even when
 * it is not coupled to forces, without applying it: the drag on a held
 * particle.  No counterpart in the reference, which accumulates no force for
 * an uncoupled particle (src/gpu/fluids.jl:198-202); off by default. */
int lbm_record_force(lbm_handle* h, int32_t id, int32_t on);

/* ---- particle-particle interactions (molecularDynamicsTick!,
 * src/gpu/particles.jl:100-197; set-up src/gpu/initMethods.jl:224-414) ------
 * Every tick, after the hydrodynamic update and before the particles move,
 * each interaction adds its forces to the force input of its particles, from
 * their positions before the move; the particle update then applies force
 * input and momentum exchange together (coupled particles only).  The list
 * replaces any previous one; pair interactions (Lennard-Jones, WCA, dipoles)
 * come as one entry per pair, in the reference's order (the pairs (i, j),
 * i < j, of each interaction, interactions in the order they were added).
 * Parameters p[]:
 *   LINEAR        bond: p0 equilibrium displacement, p1 stiffness
 *   BISTABLE      p0 trap radius, p1 a, p2 b (force (a (d-R)^3 - b (d-R)) r^)
 *   POLAR         three particles id1-id2-id3: p0 equilibrium angle, p1 stiffness
 *   LENNARD_JONES p0 epsilon, p1 sigma, p2 cutoff (a WCA potential: cutoff 2^(1/6) sigma)
 *   DIPOLE        p0 dipole constant, p1..p3 magnetic field (the front end evaluates
 *                 a time-dependent field and sets the list again)
 * Not with the CPU module's particle rules (the CPU module has no
 * interactions), the persistent tick schedule (the tick runs in stream order
 * instead), batches or lbm_adjoint. */
#define LBM_INTERACTION_LINEAR 0
#define LBM_INTERACTION_BISTABLE 1
#define LBM_INTERACTION_POLAR 2
#define LBM_INTERACTION_LENNARD_JONES 3
#define LBM_INTERACTION_DIPOLE 4
typedef struct lbm_interaction {
    int32_t kind;
    int32_t id1, id2, id3;  /* 1-based particle ids (id3: POLAR only) */
    double p[4];
} lbm_interaction;
int lbm_set_interactions(lbm_handle* h, const lbm_interaction* list, int32_t n);

/* particle.boundaryConditionsParams.solidRegion (N...) as 0/1 bytes
 * (getSphere, src/gpu/aux.jl:206-215), for particle `id` (1-based). */
int lbm_get_mask(lbm_handle* h, int32_t id, uint8_t* mask);

/* Boundary links of particle `id`: the (cell, direction) pairs of
 * streamingInvasionRegions (bounceBackPrep, src/gpu/aux.jl:187-198), i.e.
 * fluid cells x with x - c_dir solid, as 0-based cell index and 0-based
 * direction index, sorted by (direction, cell).  They are read from the
 * particle's device link list, the one the boundary fix-up uses.  With
 * cells == NULL only the count is returned in *n. */
int lbm_get_links(lbm_handle* h, int32_t id, int64_t* cells, int8_t* dirs, int64_t capacity, int64_t* n);

int lbm_get_info(lbm_handle* h, lbm_info* info);

/* Choose the bulk stream-collide kernel (LBM_BULK_*, see lbm_info). */
int lbm_set_bulk_kernel(lbm_handle* h, int32_t kind, int32_t threads, int32_t stages);

/* Device-time profile of the most recent lbm_step call (CUDA events on the
 * handle's stream; with profiling on, event nodes are captured around every
 * kernel of the step graph).  No counterpart in the reference, which has no
 * tracing (only a `verbose` progress print, src/gpu/fluids.jl:229-253). */
typedef struct lbm_profile {
    double total_ms;        /* device time of the whole lbm_step call */
    double bulk_ms;         /* mean duration of one bulk stream-collide launch (of the whole tick
                               kernel where bulk, fix-up and particles run as one persistent kernel) */
    double fixup_ms;        /* mean duration of one boundary-link fix-up launch (0 if none) */
    double particles_ms;    /* mean duration of one particle-update launch (0 if none) */
    int64_t steps;          /* ticks in the call */
    int64_t launches;       /* kernel launches enqueued by the call */
    int64_t profiled_steps; /* ticks whose kernels were bracketed by events */
    int64_t bulk_cells;     /* lattice nodes updated by the bulk kernel per tick */
    int64_t fixup_entries;  /* nodes the boundary fix-up visits per tick (particle link nodes + wall-link nodes) */
} lbm_profile;

/* level 0: off; 1: device time of each lbm_step call; 2: also per-kernel
 * durations (event nodes around every kernel of the step graph) */
int lbm_set_profiling(lbm_handle* h, int32_t level);
int lbm_get_profile(lbm_handle* h, lbm_profile* out);

/* Mean device duration of one launch of a single kernel of the tick
 * (0: bulk stream-collide over all tiles, 1: boundary-link fix-up, 2:
 * particle update, 3: the persistent tick kernel that runs all three as one
 * launch; LBM_ERR_STATE where that kernel does not apply), from CUDA events
 * around `launches` back-to-back launches on the handle's stream.  The model
 * state is saved before and restored after, so the simulation is
 * unaffected.  No counterpart in the reference. */
#define LBM_KERNEL_BULK 0
#define LBM_KERNEL_FIXUP 1
#define LBM_KERNEL_PARTICLES 2
#define LBM_KERNEL_TICK 3
int lbm_time_kernel(lbm_handle* h, int32_t kernel, int32_t launches, double* avg_ms);

/* Failure detection.  No counterpart in the reference, whose only checks are
 * the @assert / error sites of its keyword handling
 * (src/gpu/initMethods.jl:472-473,514,533,540,556).
 *   - Every bulk stream-collide pass tests the density it forms at each node
 *     and raises LBM_ERR_NUMERIC from lbm_step (or lbm_batch_step) when it
 *     is not finite or below -1e-3 (wall nodes hold zero density, as in the
 *     reference, so zero itself cannot be told apart from a failure).
 *   - Every wait inside the persistent tick kernel (LBM_SCHEDULE_PERSISTENT)
 *     gives up after a bounded number of polls and raises LBM_ERR_TIMEOUT.
 * After either error the model's state is undefined: restore a checkpoint
 * (lbm_load_state) or destroy the handle; the error word is cleared once
 * reported, so the handle itself stays usable.
 *
 * lbm_set_wait_limit: `polls` bounds every wait of the tick kernel (1 ..
 * 2^22, the default; a poll sleeps >= 128 ns).  `target_offset` is a test
 * knob: 1 raises the target of the fix-up items' wait above any count the
 * kernel can reach, so that wait runs into the limit; 0 in normal use.
 *
 * lbm_set_memory_limit: a process-wide cap on the device bytes any one handle
 * may hold (0, the default: no cap); an allocation beyond it fails with
 * LBM_ERR_OOM, as a failed cudaMalloc does. */
int lbm_set_wait_limit(lbm_handle* h, int64_t polls, int32_t target_offset);
int lbm_set_memory_limit(int64_t bytes);

/* Raw checkpoint of populations + particle FP64 state + tick/time. */
int lbm_save_state(lbm_handle* h, const char* path);
int lbm_load_state(lbm_handle* h, const char* path);

/* ---- batches of independent replicas -------------------------------------
 * Replicas of one velocity set, collision model and storage format, each with
 * its own grid, parameters and particles, advanced together: every tick runs
 * all replicas' bulk tiles, boundary fix-up blocks and particle updates as the
 * items of one work queue (tick.cuh), either as one persistent launch per
 * tick or as three queue launches in stream order.  The step loop is replayed
 * from CUDA graphs.  No counterpart in the reference, which steps one model
 * per call (parameter sweeps there are loops over modelInit/LBMpropagate!).
 * Every replica must take the vector bulk path: n[0] a multiple of 4, x-rows
 * of at most 256 nodes, no per-node force field, not FP64 storage. */
typedef struct lbm_batch lbm_batch;

typedef struct lbm_batch_tuning {
    int32_t schedule;     /* LBM_SCHEDULE_STREAM or LBM_SCHEDULE_PERSISTENT */
    int32_t ctas_per_sm;  /* resident CTAs per SM of the queue kernel (1..occupancy limit) */
    int32_t tile_order;   /* bulk tiles in the queue: 0 replica by replica, 1 interleaved across replicas */
    int32_t tile_cta;     /* STREAM only: 1 runs the bulk tiles one CTA each instead of through the queue */
    double ms_per_tick;   /* device time of one tick measured by lbm_batch_autotune (0 if not measured) */
} lbm_batch_tuning;

/* n replicas: cfgs[i] with nparticles[i] particles, taken in order from
 * `particles` (all replicas' particles back to back).  All on one device. */
int lbm_batch_create(int32_t n, const lbm_config* cfgs, const int32_t* nparticles,
                     const lbm_particle_params* particles, lbm_batch** out);
int32_t lbm_batch_size(const lbm_batch* b);
/* Replica i as a model handle, owned by the batch: every lbm_get_* call
 * works on it, and so does stepping it alone. */
lbm_handle* lbm_batch_replica(lbm_batch* b, int32_t i);
/* Advance every replica by nsteps ticks. */
int lbm_batch_step(lbm_batch* b, int64_t nsteps);
/* Time every candidate tuning (schedule x bulk kernel x CTAs per SM x tile order) over
 * `ticks` ticks each, with the state saved before and restored after, and
 * keep the fastest.  The measured candidates go to results[0..capacity),
 * their number to *count; the chosen one to *chosen (either may be null). */
int lbm_batch_autotune(lbm_batch* b, int32_t ticks, lbm_batch_tuning* results, int32_t capacity, int32_t* count,
                       lbm_batch_tuning* chosen);
int lbm_batch_set_tuning(lbm_batch* b, const lbm_batch_tuning* t);
int lbm_batch_get_tuning(const lbm_batch* b, lbm_batch_tuning* t);
/* level 0 off, 1 device time of each lbm_batch_step call (lbm_profile.total_ms) */
int lbm_batch_set_profiling(lbm_batch* b, int32_t level);
int lbm_batch_get_profile(const lbm_batch* b, lbm_profile* out);
/* Per-replica status: status[i] = LBM_ERR_NUMERIC for a replica whose density
 * sentinel fired in some lbm_batch_step (non-finite or negative density, see
 * "Failure detection" below), else LBM_OK; returns how many replicas
 * diverged.  A diverged replica does not stop the batch (a parameter sweep
 * runs on). */
int lbm_batch_status(const lbm_batch* b, int32_t* status);
const char* lbm_batch_last_error(const lbm_batch* b);
void lbm_batch_destroy(lbm_batch* b);

/* ---- gradients: discrete adjoint with binomial checkpointing --------------
 * Observable: the time average, over ticks window_begin..window_end (after
 * that many ticks, 1-based, inclusive), of the particle's velocity or of the
 * momentum-exchange force on it (spec.observable) along `direction` (zero
 * vector: its initial swimming direction), over a run of
 * `ticks` ticks from the handle's initial state (tick 0).  Returns its value
 * and its derivatives with respect to the particle's B1 and B2, the
 * relaxation time tau (tau+ with tau- following: dtau = dtau_plus +
 * tau_minus_slope * dtau_minus, the slope d tau-/d tau+ at fixed magic
 * parameter being given by the caller) and the three components of the
 * uniform body force.  The backward sweep runs a hand-written adjoint of the
 * tick (stream-collide, bounce-back and moving-boundary links, momentum
 * exchange) and of the particle update, recomputing forward segments from at
 * most `snapshots` stored states (binomial checkpointing).  The solid masks
 * are taken as the forward run computes them.  The handle is left in the
 * state it had on entry.  Walls (static or moving) are differentiated
 * through.  Requirements: one particle, the GPU module's particle rules, no
 * interactions, no per-node force field.  No counterpart in the reference (it
 * has no differentiation). */
typedef struct lbm_adjoint_spec {
    int64_t ticks;
    int64_t window_begin, window_end;
    double direction[3];
    double tau_minus_slope;
    int32_t snapshots;    /* stored states, including the initial one (>= 2) */
    int32_t observable;   /* LBM_OBSERVABLE_* */
} lbm_adjoint_spec;

/* Observables of lbm_adjoint, each averaged over the window along `direction`:
 *   VELOCITY  the particle's velocity (its swimming speed)
 *   FORCE     the momentum-exchange force of the tick (src/gpu/fluids.jl:191-205);
 *             for a held particle (coupleForces false, which the reference does
 *             not move) this is its drag: the force is accumulated for the
 *             observable only, never applied, and ordinary lbm_step calls keep
 *             reporting zero force for such a particle, as the reference does */
/* (lbm_record_force makes the same force visible in ordinary stepping) */
#define LBM_OBSERVABLE_VELOCITY 0
#define LBM_OBSERVABLE_FORCE 1

typedef struct lbm_adjoint_result {
    double value;         /* the observable */
    double dB1, dB2;
    double dtau, dtau_plus, dtau_minus;
    double dF[3];
    int64_t forward_ticks;   /* ticks run forward in total (sweep and recomputation) */
    int32_t snapshots_used;  /* most states held at once */
    int32_t reserved;
    double ms;               /* wall time of the call */
} lbm_adjoint_result;

int lbm_adjoint(lbm_handle* h, const lbm_adjoint_spec* spec, lbm_adjoint_result* out);

/* Allocation-free stepping.  No counterpart in the reference.
 *
 * Same ticks and results as lbm_step, for callers that must not allocate
 * device memory once their run has started: codes that reserve all device
 * memory up front (another library's memory pool, a fixed per-process budget)
 * and real-time or embedded hosts whose policy forbids allocation after
 * initialisation.  lbm_step instantiates CUDA graphs on its first call and
 * after every lbm_add_particle, which allocates; this entry point launches the
 * kernels directly and keeps the fix-up kernel's momentum-exchange partials in
 * a fixed device array compiled into the library (LBM_NOALLOC_SLOTS slots of
 * 8 doubles = 1 MiB, held by every device that loads the library until the
 * process exits) instead of the handle's buffer.  It calls no cudaMalloc,
 * cudaFree or other allocating routine.
 *
 * - The first call on a device looks up that array's device address
 *   (cudaGetSymbolAddress) with the device current; make that first call before
 *   any stream capture that the caller runs.
 * - Models whose particles need more than LBM_NOALLOC_SLOTS partial slots
 *   (one per particle and 64 near-box nodes) are rejected with
 *   LBM_ERR_UNSUPPORTED; the message names both sizes.
 * - All calls in the process share the array: calls that overlap on the GPU
 *   (two handles stepped concurrently on the same device) race and must be
 *   serialised by the caller.  The used slots are cleared at the start of
 *   every call; nothing else carries over between calls.
 * - The model itself (populations, particle records) is allocated earlier,
 *   by lbm_create and lbm_add_particle. */
#define LBM_NOALLOC_SLOTS 16384
int lbm_step_noalloc(lbm_handle* h, int64_t nsteps);

/* lbm_destroy waits for the handle's queued work and gives its device
 * buffers back.  The library keeps freed device blocks (up to 4 GiB in the
 * process) for later allocations of the same size, so a model built after
 * another does not pay cudaMalloc again; the kept blocks go back to the
 * driver when a cudaMalloc fails. */
const char* lbm_last_error(lbm_handle* h);
const char* lbm_last_global_error(void);
void lbm_destroy(lbm_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* LBM_B200_H */
