/*
 * efl.h — C ABI of the B200 Eulerian-fluid step library (libefl_b200.so).
 *
 * This boundary replaces the per-frame compute pass that the reference
 * plugin records in `EulerFluidNode::run` (src/euler_fluid/render_node.rs:193-476)
 * and the force read-back observer `forces_to_solid_readback`
 * (src/euler_fluid/fluid_to_solid.rs:180-209).  The plugin-level types stay
 * on the caller's side (FluidSettings, FluidSource, ForcesToFluid, the
 * rigid-body query); the caller copies them into the plain structs below.
 *
 * Conventions
 *  - Every function returns an efl_status; EFL_OK == 0.  On failure the
 *    message is available from efl_last_error(sim) (or efl_last_error(NULL)
 *    for errors raised before a handle exists).
 *  - Host arrays passed in are caller-owned and copied before the call
 *    returns.  Device memory is owned by the library.
 *  - Each efl_sim owns one CUDA stream.  Calls on one handle must be
 *    serialised by the caller; different handles are independent.
 *  - All fields are f32 row-major, x fastest.  Grid index (x, y) has y
 *    pointing down, as in the reference's textures.
 *  - u faces are (nx+1) x ny, v faces nx x (ny+1), cell fields nx x ny.
 *
 * Out-of-bounds texture reads in the reference are backend defined; this
 * library fixes them to "load returns 0, store is dropped" (robust-access
 * behaviour of DX12/Vulkan), which is what the examples' DX12 backend does.
 */
#ifndef EFL_H
#define EFL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define EFL_API __declspec(dllexport)
#else
#define EFL_API __attribute__((visibility("default")))
#endif

#define EFL_ABI_VERSION 1

/* Limits taken from the reference. */
#define EFL_MAX_SOLIDS 256        /* fluid_to_solid.rs:28 MAX_SOLIDS               */
#define EFL_MAX_FLUID_SOURCE 16   /* fluid_source_uniform.rs:19 MAX_FLUID_SOURCE   */

typedef enum efl_status {
    EFL_OK = 0,
    EFL_ERR_INVALID_ARGUMENT = 1, /* bad size, null pointer, bad enum       */
    EFL_ERR_CUDA = 2,             /* a CUDA runtime call failed             */
    EFL_ERR_OUT_OF_MEMORY = 3,
    EFL_NOT_CONVERGED = 4,        /* residual solve hit max_iterations      */
    EFL_ERR_TOO_MANY = 5,         /* > EFL_MAX_SOLIDS / EFL_MAX_FLUID_SOURCE */
    EFL_ERR_UNSUPPORTED_SHAPE = 6,/* obstacle shape id not 0/1/2/4           */
    EFL_ERR_STATE = 7,            /* call not valid in the current state     */
    EFL_ERR_NO_DEVICE = 8         /* no CUDA device / extension unusable     */
} efl_status;

/* ProjectionMethod (src/euler_fluid/projection.rs:44-52). */
typedef enum efl_projection_method {
    EFL_PROJECTION_JACOBI = 0,
    EFL_PROJECTION_GAUSS_SEIDEL = 1,
    EFL_PROJECTION_MULTIGRID = 2,
    /* Extension, no reference counterpart: conjugate gradients on the FP64
     * system preconditioned by one symmetric V-cycle of the reference's
     * multigrid structure (post-smoothing black then red); tolerance > 0
     * required, pressure_iterations counts CG iterations. */
    EFL_PROJECTION_MGPCG = 3
} efl_projection_method;

/* ReinitializeMethod (src/euler_fluid/reinitialize_levelset.rs:36-40). */
typedef enum efl_reinit_method {
    EFL_REINIT_JUMP_FLOODING = 0,
    EFL_REINIT_FAST_ITERATIVE = 1
} efl_reinit_method;

/*
 * Pressure projection settings.
 *  - gs_iterations / sor_weight: GaussSeidelConfig (gauss_seidel.rs:33-42,
 *    weight 1.9 at gauss_seidel.rs:72).
 *  - mg_pre/mg_post/mg_coarsest: MultiGridConfig (multi_grid.rs:56-71).
 *  - mg_levels: 0 = the reference rule max(1, floor(log2(min(nx,ny))) - 2)
 *    (multi_grid.rs:95-97); otherwise the explicit number of levels.
 *  - tolerance: 0 = the reference's fixed iteration count (one V-cycle for
 *    multigrid, gs_iterations red-black iterations for Gauss-Seidel).
 *    > 0 = iterate until ||b - A p||_2 / ||b||_2 <= tolerance (FP64 norms
 *    over cells with phi < 0 that are not fully solid), checking every
 *    check_interval RB iterations (Gauss-Seidel) or every V-cycle
 *    (multigrid), at most max_iterations iterations / V-cycles.
 */
typedef struct efl_projection {
    int32_t method;          /* efl_projection_method                        */
    uint32_t gs_iterations;  /* default 20                                    */
    float sor_weight;        /* default 1.9                                   */
    uint32_t mg_pre;         /* default 2                                     */
    uint32_t mg_post;        /* default 2                                     */
    uint32_t mg_coarsest;    /* default 3                                     */
    uint32_t mg_levels;      /* default 0 (reference rule)                    */
    float tolerance;         /* default 0 (fixed count)                       */
    uint32_t max_iterations; /* default 20000                                 */
    uint32_t check_interval; /* default 16 (Gauss-Seidel only)                */
} efl_projection;

typedef struct efl_reinit {
    int32_t method;          /* efl_reinit_method; default FAST_ITERATIVE      */
    uint32_t fim_iterations; /* FastIterativeMethodConfig, default 10          */
} efl_reinit;

/*
 * Creation parameters: FluidPlugin::new(length_unit) (euler_fluid.rs:47-53)
 * plus FluidSettings{rho, gravity, size} (settings.rs:110-114) plus the
 * fluid entity's Transform (setup_components.rs:100-103), column-major 4x4
 * as glam's Mat4.
 */
typedef struct efl_config {
    uint32_t nx, ny;         /* FluidSettings.size; multiples of 8, >= 16    */
    float length_unit;       /* dx = 1 / length_unit; must be > 0             */
    float rho;
    float gravity[2];        /* grid frame, y down: (0, +9.8) is downward     */
    float transform[16];     /* column-major fluid transform                  */
    efl_projection projection;
    efl_reinit reinit;
    int32_t device;          /* CUDA device ordinal                           */
} efl_config;

/* ShapeVariant ids (solid_obstacle.wgsl:4-7, parry2d ShapeType). */
enum {
    EFL_SHAPE_CIRCLE = 0,
    EFL_SHAPE_RECTANGLE = 1,
    EFL_SHAPE_CAPSULE = 2,
    EFL_SHAPE_TRIANGLE = 4
};

/*
 * SolidObstacle (obstacle.rs:24-32, solid_obstacle.wgsl:34-41).
 * values: circle {radius}; rectangle {half_x, half_y};
 * capsule {ax, ay, bx, by, radius}; triangle {ax, ay, bx, by, cx, cy}.
 * entity_id is the obstacle's index in the caller's body list; force bins
 * are keyed by it and obstacles[entity_id] gives the centre of mass
 * (sample_forces.wgsl:40-41), as in the reference.  176 bytes.
 */
typedef struct efl_solid_obstacle {
    uint32_t entity_id;
    uint32_t shape;
    float values[6];
    float transform[16];         /* column-major world transform            */
    float inverse_transform[16]; /* its inverse, as the reference uploads it */
    float linear_velocity[2];
    float angular_velocity;
    float _pad;
} efl_solid_obstacle;

/* ForceToFluid (apply_forces.rs:36-40): force in m/s^2 at a grid-pixel
 * position (y down).  The README's "LocalForces" is this type. */
typedef struct efl_force {
    float force[2];
    float position[2];
} efl_force;
typedef efl_force efl_local_force;

/* FluidSourceData (fluid_source_uniform.rs:48-55). */
enum { EFL_SOURCE_CIRCLE = 0, EFL_SOURCE_AABB = 1 };
enum { EFL_SOURCE_MODE_SOURCE = 0, EFL_SOURCE_MODE_SINK = 1 };
typedef struct efl_source {
    float center[2];   /* source Transform translation, grid-centred, y up  */
    float data[2];     /* circle {radius, 0}; aabb {half_x, half_y}          */
    float velocity[2]; /* FluidSourceVelocity (zero for one-shot sources)    */
    uint32_t shape;
    uint32_t mode;
} efl_source;

/* FluidToSolidForce (fluid_to_solid.rs:60-64): bins * 0.1. */
typedef struct efl_solid_force {
    float force[2];
    float torque;
    float _pad;
} efl_solid_force;

/* A rigid body integrated on the device at the end of every step, from the
 * step's FluidToSolidForce, moving the obstacle it drives for the next step
 * (extension: the reference hands the forces to avian2d on the host,
 * fluid_to_solid.rs:180-209, and reads them back a frame late).  World units
 * are grid cells, centred on the domain, y up.  Per step: force * dt /
 * grid_length with y flipped and the torque negated, semi-implicit Euler
 * under gravity (world units / s^2 along -y) in `substeps` equal substeps,
 * and a clamp keeping the centre `extent` + 1 inside the walls. */
typedef struct efl_rigid_body {
    double position[2];
    double rotation;         /* radians */
    double linear_velocity[2];
    double angular_velocity;
    double mass;
    double inertia;          /* 0: the rotation is not integrated */
    double extent;
    int32_t dynamic;         /* 0: left in place */
    int32_t obstacle;        /* index into the efl_set_obstacles list */
} efl_rigid_body;

typedef struct efl_step_stats {
    int32_t initialized_only;     /* 1: this call ran the init sequence only */
    uint32_t pressure_iterations; /* RB iterations (GS), V-cycles (MG), 50 (Jacobi) */
    int32_t converged;            /* 1 if tolerance met (or fixed-count mode) */
    int32_t _pad;
    double residual;              /* relative residual after the solve, -1 if not computed */
    double residual_initial;      /* relative residual before the solve, -1 if not computed */
} efl_step_stats;

/* Field ids for efl_get_field / efl_set_field / efl_field_shape. */
typedef enum efl_field {
    EFL_FIELD_U = 0,              /* u0: FluidTextures.u      (nx+1) x ny   */
    EFL_FIELD_V = 1,              /* v0: FluidTextures.v      nx x (ny+1)   */
    EFL_FIELD_U1 = 2,             /* advected/forced u                      */
    EFL_FIELD_V1 = 3,
    EFL_FIELD_U_SOLID = 4,        /* FluidTextures.u_solid                  */
    EFL_FIELD_V_SOLID = 5,        /* FluidTextures.v_solid                  */
    EFL_FIELD_LEVELSET_AIR = 6,   /* phi0: FluidTextures.levelset_air       */
    EFL_FIELD_LEVELSET_AIR1 = 7,  /* phi1                                   */
    EFL_FIELD_LEVELSET_SOLID = 8, /* FluidTextures.levelset_solid           */
    EFL_FIELD_SOLID_ID = 9,       /* i32                                    */
    EFL_FIELD_AREA_FRACTION = 10, /* 4 x f32 per cell (i-1/2, i+1/2, j-1/2, j+1/2) */
    EFL_FIELD_DIVERGENCE = 11,
    EFL_FIELD_PRESSURE = 12,      /* p0                                     */
    EFL_FIELD_GRAD_LEVELSET = 13, /* 2 x f32 per cell                        */
    EFL_FIELD_JFA_SEEDS = 14,     /* 2 x f32 per cell, final pass output     */
    EFL_FIELD_FIM_LABELS = 15,    /* u32                                     */
    EFL_FIELD_U_VALID = 16,       /* i32, extrapolation validity of u faces  */
    EFL_FIELD_V_VALID = 17,       /* i32                                     */
    EFL_FIELD_AREA_FRACTION_U = 18, /* x-face fractions (nx+1) x ny (device layout) */
    EFL_FIELD_AREA_FRACTION_V = 19, /* y-face fractions nx x (ny+1)          */
    EFL_FIELD_COUNT = 20
} efl_field;

/* Pipeline stages, in the order EulerFluidNode::run records them
 * (render_node.rs:290-463).  efl_run_stage runs one of them on the current
 * state; it exists for per-kernel parity tests and debugging. */
typedef enum efl_stage {
    EFL_STAGE_INIT = 0,               /* render_node.rs:219-277 */
    EFL_STAGE_UPDATE_SOLID = 1,       /* update_solid.wgsl      */
    EFL_STAGE_AREA_FRACTION = 2,      /* update_area_fraction.wgsl */
    EFL_STAGE_ADVECT_VELOCITY = 3,    /* advect_velocity.wgsl   */
    EFL_STAGE_APPLY_FORCES = 4,       /* apply_forces.wgsl      */
    EFL_STAGE_DIVERGENCE = 5,         /* divergence.wgsl        */
    EFL_STAGE_PROJECTION = 6,         /* projection.rs:89-164   */
    EFL_STAGE_SOLVE_VELOCITY = 7,     /* solve_velocity_{u,v}.wgsl */
    EFL_STAGE_EXTRAPOLATE = 8,        /* render_node.rs:540-608 */
    EFL_STAGE_ADVECT_LEVELSET = 9,    /* advect_levelset.wgsl   */
    EFL_STAGE_FLUID_SOURCE = 10,      /* update_fluid_source.wgsl */
    EFL_STAGE_REINITIALIZE = 11,      /* reinitialize_levelset.rs:162-243 */
    EFL_STAGE_LEVELSET_GRADIENT = 12, /* levelset_gradient.wgsl */
    EFL_STAGE_SOLID_FORCES = 13,      /* render_node.rs:610-641 */
    EFL_STAGE_COUNT = 14
} efl_stage;

typedef struct efl_sim efl_sim;

/* Library ABI version (EFL_ABI_VERSION). */
EFL_API int32_t efl_abi_version(void);

/* Fills *cfg with the reference defaults for an nx x ny grid:
 * length_unit 1, rho 1, gravity (0, 9.8), identity transform,
 * Gauss-Seidel 20 iterations at weight 1.9, FIM(10). */
EFL_API efl_status efl_default_config(uint32_t nx, uint32_t ny, efl_config* cfg);

/* Creates a simulation (watch_fluid_component, setup_components.rs:38-328).
 * The new simulation is in FluidStatus::Reset: the next efl_step runs the
 * init sequence. Errors: length_unit <= 0 (the reference panics,
 * euler_fluid.rs:49-51), nx/ny not multiples of 8 or < 16. Sizes that are
 * not multiples of 64 are accepted; as in the reference, the face kernels
 * then cover floor(n/64)*64 rows/columns only (pipeline.rs:180-186). */
EFL_API efl_status efl_create(const efl_config* cfg, efl_sim** out);
EFL_API efl_status efl_destroy(efl_sim* sim);

/* Message for the last error on this handle (NULL: the last error of a
 * call that had no handle, e.g. a failed efl_create). */
EFL_API const char* efl_last_error(const efl_sim* sim);

/* FluidStatus::Reset (fluid_status.rs:15-38): the next efl_step re-runs
 * the init sequence. */
EFL_API efl_status efl_reset(efl_sim* sim);

/* Runtime changes of the ProjectionMethod / ReinitializeMethod components. */
EFL_API efl_status efl_set_projection(efl_sim* sim, const efl_projection* p);
EFL_API efl_status efl_set_reinit(efl_sim* sim, const efl_reinit* r);
EFL_API efl_status efl_set_transform(efl_sim* sim, const float transform[16]);

/* construct_rigid_body_buffer_for_gpu (obstacle.rs:89-160): the full body
 * list, kept until replaced. n <= EFL_MAX_SOLIDS. */
EFL_API efl_status efl_set_obstacles(efl_sim* sim, const efl_solid_obstacle* obstacles, uint32_t n);

/* apply_forces_and_clear (apply_forces.rs:157-168): forces used by the next
 * step only, then cleared. */
EFL_API efl_status efl_set_local_forces(efl_sim* sim, const efl_force* forces, uint32_t n);

/* update_fluid_source_{init_,}buffer (fluid_source_uniform.rs:77-158).
 * oneshot != 0: the FluidSourceOneshot list, applied by the init sequence;
 * oneshot == 0: the continuous list, applied every step. n <= 16. */
EFL_API efl_status efl_set_sources(efl_sim* sim, const efl_source* sources, uint32_t n, int32_t oneshot);

/* One render-graph Update for this simulation: the init sequence if the
 * simulation is not initialised (stats->initialized_only = 1), else one
 * full step with time step dt (render_node.rs:278-466). Returns
 * EFL_NOT_CONVERGED (state still advanced) if a tolerance-driven pressure
 * solve hit max_iterations. stats may be NULL. */
EFL_API efl_status efl_step(efl_sim* sim, float dt, efl_step_stats* stats);

/* Runs one stage of the step on the current state (testing/debugging). */
EFL_API efl_status efl_run_stage(efl_sim* sim, int32_t stage, float dt, efl_step_stats* stats);

/* FluidToSolidForce[256] of the last step (fluid_to_solid.rs:180-209 reads
 * these); bins as raw fixed-point i32 (3 x 256: fx, fy, torque). */
EFL_API efl_status efl_read_solid_forces(efl_sim* sim, efl_solid_force out[EFL_MAX_SOLIDS]);
EFL_API efl_status efl_read_force_bins(efl_sim* sim, int32_t out[3 * EFL_MAX_SOLIDS]);

/* Field shape: width, height, channels and bytes per channel. */
EFL_API efl_status efl_field_shape(const efl_sim* sim, int32_t field, uint32_t* width,
                                   uint32_t* height, uint32_t* channels, uint32_t* elem_bytes);
/* Dense (unpitched) host copies of a field; bytes must equal
 * width*height*channels*elem_bytes. Synchronous. */
EFL_API efl_status efl_get_field(efl_sim* sim, int32_t field, void* host_dst, size_t bytes);
EFL_API efl_status efl_set_field(efl_sim* sim, int32_t field, const void* host_src, size_t bytes);
/* Device pointer and row pitch (bytes) of a field for zero-copy readers.
 * Not available for EFL_FIELD_AREA_FRACTION (stored as the two face
 * arrays EFL_FIELD_AREA_FRACTION_U / _V). */
EFL_API efl_status efl_field_device_ptr(efl_sim* sim, int32_t field, void** dptr, size_t* pitch_bytes);
/* The simulation's CUDA stream (cudaStream_t). */
EFL_API efl_status efl_stream(efl_sim* sim, void** stream);
EFL_API efl_status efl_synchronize(efl_sim* sim);

/* Relative residual ||b - A p||_2 / ||b||_2 of the current pressure against
 * the current divergence (operator of residual.wgsl:33-54), FP64 norms. */
EFL_API efl_status efl_residual(efl_sim* sim, double* relative, double* norm_r, double* norm_b);
/* efl_step replays each step segment whose kernel arguments repeat (the
 * whole step for fixed-count projections; the stages before and after the
 * projection for tolerance-driven ones) as a captured CUDA graph, from the
 * second time the same arguments occur.  enable = 0 runs every kernel as its
 * own launch (results are identical).  Default on.  No reference
 * counterpart (the reference records wgpu command buffers per frame). */
EFL_API efl_status efl_set_graph_capture(efl_sim* sim, int32_t enable);
/* Bounds of the device-side waits (extension, no reference counterpart).
 * barrier_polls: polls of the grid barrier inside the cooperative pressure
 * solves before a CTA gives up; every CTA then leaves the launch and the
 * step returns EFL_ERR_CUDA ("... a grid barrier timed out").
 * mbarrier_polls: polls of the TMA sweep's wait for a tile's copies; a CTA
 * that gives up waits (default bound) for its own copies still in flight and
 * leaves, and the next efl_synchronize / efl_read_solid_forces returns
 * EFL_ERR_CUDA ("TMA sweep: an mbarrier wait timed out").  0 restores the
 * defaults (2^25 and 2^24 polls, about a second).  A short limit turns a
 * stalled wait into an error status instead of a long spin, and lets a test
 * make a wait run out without any fault or hang. */
EFL_API efl_status efl_set_wait_limits(efl_sim* sim, uint64_t barrier_polls, uint64_t mbarrier_polls);
/* Device time of the last projection stage (efl_step or efl_run_stage), in
 * milliseconds; waits for it to finish.  No reference counterpart (the
 * reference has no per-stage timing). */
EFL_API efl_status efl_projection_ms(efl_sim* sim, float* ms);

/* Post-projection divergence: the operator of divergence.wgsl:16-42 applied
 * to the current velocity u0 / v0 (with the current face fractions and solid
 * velocities) at the cells the residual counts (levelset_air < 0, not fully
 * solid).  l2 = sqrt of the FP64 sum of squares, linf = the largest
 * magnitude (1/s).  Call it between EFL_STAGE_SOLVE_VELOCITY and the next
 * stage for the divergence the projection leaves (the reference evaluates
 * no such diagnostic; its volume diagnostic is efl_fluid_volume). */
EFL_API efl_status efl_divergence_norms(efl_sim* sim, double* l2, double* linf);
/* Number of cells with levelset_air < 0 (calculate_volume.wgsl:11-75). */
EFL_API efl_status efl_fluid_volume(efl_sim* sim, uint64_t* cells);
/* FluidMinVelocityMagnitude / FluidMaxVelocityMagnitude
 * (diagnostics/min_velocity.wgsl, max_velocity.wgsl): the cell-centred
 * speed |(u, v)| reduced by 16 x 16 workgroups (the minimum over fluid cells,
 * 1e30 elsewhere; the maximum over all cells), then by the reference's second
 * pass, which first ADDS the partials i, i + 512, i + 1024, ... from 0.0 per
 * lane before the min / max over 512 lanes -- so a grid of fewer than 512
 * workgroups reports a minimum of 0 and a grid of more than 512 can report a
 * maximum above the true one.  Both quirks are kept for parity; use them as
 * the reference's monitor, e.g. for a CFL time step. */
EFL_API efl_status efl_velocity_magnitude(efl_sim* sim, float* min_mag, float* max_mag);

/* Device-side coupling: after efl_set_rigid_bodies (n <= 256, each driving
 * one obstacle already set with efl_set_obstacles) every efl_step ends by
 * integrating the bodies and rewriting their obstacles' transforms and
 * velocities on the device -- no force read-back and no obstacle upload
 * per step.  n = 0 switches it off.  efl_get_rigid_bodies reads the state. */
EFL_API efl_status efl_set_rigid_bodies(efl_sim* sim, const efl_rigid_body* bodies, uint32_t n, double gravity,
                                        double grid_length, uint32_t substeps);
EFL_API efl_status efl_get_rigid_bodies(efl_sim* sim, efl_rigid_body* bodies, uint32_t n);

/* ---- Two-layer particle level set -------------------------------------- */

/* ParticleLevelsetTwoLayersPlugin (particle_levelset_two_layers/plugin.rs,
 * Enright et al. 2002; commented out of the reference's FluidPlugin at
 * euler_fluid.rs:81).  Positive particles (sign +1, layer 0) and negative
 * particles (sign -1, layer 1) seeded in the band |phi| < 3 around the
 * interface, at most 16 per cell and layer; capacity nx*ny*16 per layer
 * (plugin.rs:221-225).  When enabled, every efl_step / init sequence runs:
 *   init  : seed from levelset_air and its gradient (render_node.rs:250-258);
 *   step  : after the fluid sources, advect the particles (TVD RK3) and
 *           correct levelset_air1 with the escaped ones; after the
 *           reinitialisation, correct levelset_air0 again, update the radii,
 *           then reseed: delete far-off particles, keep at most 16 per band
 *           cell ranked by the per-cell heap, refill to 16
 *           (render_node.rs:389-441).
 * The particle order is fixed (cell order, then attempt order; a stable
 * counting sort by cell), one of the orders the reference's atomic appends
 * can produce, so results are reproducible run to run. */
typedef struct efl_particle {   /* particle.wgsl:5-11 (storage stride 24) */
    float position[2];          /* grid cells, cell (i, j) centre at (i, j) */
    float radius;
    float sign;                 /* +1 layer 0, -1 layer 1 */
    uint32_t escaped;           /* set by the last level-set correction */
    uint32_t _pad;
} efl_particle;
enum { EFL_PLS_POSITIVE = 0, EFL_PLS_NEGATIVE = 1 };
typedef enum efl_pls_phase {
    EFL_PLS_INITIALIZE = 0,     /* plugin.rs:131-158 (band mask + seeding)      */
    EFL_PLS_ADVECT = 1,         /* plugin.rs:160-182 (advect_particles.wgsl)     */
    EFL_PLS_CORRECT = 2,        /* levelset_correction.rs:96-155, levelset_air1  */
    EFL_PLS_CORRECT_SECOND = 3, /* levelset_correction.rs:157-236, levelset_air0 */
    EFL_PLS_RESEED = 4          /* reseed.rs:130-296                             */
} efl_pls_phase;
/* enable != 0 allocates the particle buffers (first time) and runs the
 * plugin in every following efl_step; 0 stops it (particles are kept).
 * Enabling an initialised simulation starts from no particles: the next
 * reseed fills the band. */
EFL_API efl_status efl_set_particle_levelset(efl_sim* sim, int32_t enable);
/* Live particles per layer; dropped = particles that did not fit the
 * capacity since creation (0 unless the capacity was exceeded). */
EFL_API efl_status efl_particle_counts(efl_sim* sim, uint32_t counts[2], uint32_t* dropped);
/* Copies min(count, capacity) particles of a layer; *n = the live count. */
EFL_API efl_status efl_read_particles(efl_sim* sim, int32_t layer, efl_particle* dst, uint32_t capacity,
                                      uint32_t* n);
/* Replaces a layer's particles (sign must match the layer; n <= nx*ny*16). */
EFL_API efl_status efl_write_particles(efl_sim* sim, int32_t layer, const efl_particle* src, uint32_t n);
/* Runs one phase on the current state (testing); dt is used by EFL_PLS_ADVECT. */
EFL_API efl_status efl_pls_run_phase(efl_sim* sim, int32_t phase, float dt);

/* ---- Batches of independent simulations ------------------------------ */

/* N independent simulations of possibly different sizes stepped together
 * (the reference steps each fluid entity with its own dispatches,
 * render_node.rs:205-217; examples/multiple.rs spawns several).  The
 * simulations share one CUDA stream.  Their tolerance-driven red-black
 * pressure solves run as ONE cooperative launch over a packed list of
 * (simulation, tile) items; each simulation's result and iteration count are
 * those of its own efl_step.  Simulations whose projection is not the
 * tolerance-driven Gauss-Seidel solve are projected one by one. */
typedef struct efl_batch efl_batch;
EFL_API efl_status efl_batch_create(const efl_config* configs, uint32_t n, efl_batch** out);
EFL_API efl_status efl_batch_destroy(efl_batch* batch);
EFL_API const char* efl_batch_last_error(const efl_batch* batch);
/* The handle of simulation i, for the per-simulation calls (sources,
 * obstacles, local forces, fields).  Owned by the batch: do not destroy it. */
EFL_API efl_status efl_batch_sim(efl_batch* batch, uint32_t i, efl_sim** sim);
/* One frame for every simulation (efl_step semantics); stats: n entries or NULL. */
EFL_API efl_status efl_batch_step(efl_batch* batch, float dt, efl_step_stats* stats);
/* Tile configurations of the batched solve (owned tile and red-black
 * iterations per streamed round): 0 = 64 x 32 x 2, 1 = 64 x 32 x 4,
 * 2 = 32 x 32 x 2, 3 = 64 x 32 x 8.  By default (config = -1) an autotuner
 * runs the first four batched solves with one configuration each, timing
 * device ns per
 * cell-iteration, and keeps the fastest; every configuration gives the same
 * iterates and iteration counts.  No reference counterpart. */
EFL_API efl_status efl_batch_set_tiles(efl_batch* batch, int32_t config);
/* The configuration in use (0, 0, 0 while tuning) and the measured cost of
 * each (ns_per_cell_iteration: 4 entries or NULL; 0 = not tried). */
EFL_API efl_status efl_batch_tiles(const efl_batch* batch, int32_t* tx, int32_t* ty, int32_t* k,
                                   double* ns_per_cell_iteration);
/* Grid-barrier poll limit of the batched solve (efl_set_wait_limits'
 * barrier_polls; 0 = the default).  A barrier that runs out makes
 * efl_batch_step return EFL_ERR_CUDA ("batched solver: a grid barrier timed
 * out"). */
EFL_API efl_status efl_batch_set_wait_limits(efl_batch* batch, uint64_t barrier_polls);
/* Device time of the last batched pressure solve (the cooperative launch), in
 * milliseconds; waits for it to finish. */
EFL_API efl_status efl_batch_projection_ms(efl_batch* batch, float* ms);

/* ---- Learned warm start ------------------------------------------------ */

/* Extension, no reference counterpart.  A small U-Net (BF16 weights and
 * activations, FP32 accumulation; 4 levels, 16/32/64/64 channels, 3x3
 * convolutions on the tensor cores) approximates the correction e = A^-1 r
 * that the previous step's pressure p_prev needs on the new system
 * (r = b - A p_prev); its prediction only warm-starts the tolerance-driven
 * solve (x = p_prev + prediction), which still iterates to the same
 * residual.  Features per cell, 16 channels (5 used): cdiv * r / sigma, the
 * u and v face fractions averaged to the centre, phi / ny clamped to
 * [-1, 1], 1 on the counted cells; sigma = RMS of cdiv * r over the counted
 * cells; output channel 0 = e / sigma.  The head starts at zero, so an
 * untrained network warm-starts from the previous pressure exactly. */
typedef struct efl_unet efl_unet;
enum { EFL_UNET_WARM_START = 1, EFL_UNET_RECORD = 2 };
EFL_API efl_status efl_unet_create(int32_t device, uint32_t max_nx, uint32_t max_ny, uint64_t seed, efl_unet** out);
EFL_API efl_status efl_unet_destroy(efl_unet* net);
EFL_API const char* efl_unet_last_error(const efl_unet* net);
EFL_API efl_status efl_unet_num_params(const efl_unet* net, uint64_t* n);
EFL_API efl_status efl_unet_get_params(efl_unet* net, float* params, uint64_t n);
EFL_API efl_status efl_unet_set_params(efl_unet* net, const float* params, uint64_t n);
/* Forward pass on host features [ny][nx][16]; pred [ny][nx] = output channel 0. */
EFL_API efl_status efl_unet_forward(efl_unet* net, uint32_t nx, uint32_t ny, const float* features, float* pred);
/* Forward + backward of the relative squared error against target [ny][nx]
 * over mask [ny][nx] != 0, sum (pred - t)^2 / sum t^2 (every sample weighs
 * the same whatever the size of its pressure change); loss and the
 * gradient of every parameter (efl_unet_num_params floats, the order of
 * get/set_params). */
EFL_API efl_status efl_unet_gradients(efl_unet* net, uint32_t nx, uint32_t ny, const float* features,
                                      const float* target, const uint8_t* mask, float* loss, float* grads);
/* Device time of one forward pass on the input already in the network (the
 * last recorded or uploaded one), averaged over reps passes, each replayed
 * from a CUDA graph of the pass (as a simulation step runs it). */
EFL_API efl_status efl_unet_time_forward(efl_unet* net, uint32_t nx, uint32_t ny, uint32_t reps, float* ms);
/* flags: EFL_UNET_WARM_START (warm-start sim's tolerance-driven solves),
 * EFL_UNET_RECORD (record each solve as a training sample); 0 detaches.
 * For the simulations of a batch use efl_batch_attach_unet. */
EFL_API efl_status efl_unet_attach(efl_sim* sim, efl_unet* net, uint32_t flags);
/* Runs the network on the grid coarsened by `factor` (1, 2, 4 or 8): the
 * features are averaged over factor x factor cells, the prediction is
 * interpolated back bilinearly, and recorded training targets are the block
 * means of the correction.  The sweeps remove the basin-scale error slowest,
 * and four levels of pooling on the coarse grid span it.  Attached grids must
 * be multiples of 8 x factor.  Default 1 (the network on the simulation's own
 * grid); a recorded sample of the other form is dropped. */
EFL_API efl_status efl_unet_set_coarsening(efl_unet* net, uint32_t factor);
/* Attaches the network to every simulation of a batch (flags:
 * EFL_UNET_WARM_START, or 0 to detach).  With a coarsening above 1 and every
 * simulation's coarse grid a multiple of 8 in both directions, the
 * simulations' coarse features are packed into one canvas (efl_canvas_pack)
 * and one forward pass over it serves them all; otherwise each simulation
 * gets a forward-only workspace of its own and the forwards run side by side.
 * Either way each simulation's warm start, iterates and iteration counts are
 * those of its own efl_step with the network attached.  Attach again after
 * efl_unet_set_coarsening. */
EFL_API efl_status efl_batch_attach_unet(efl_batch* batch, efl_unet* net, uint32_t flags);
/* The canvas of the batch's network forward (width and height in coarse
 * pixels), 0 x 0 when the simulations' forwards run one by one. */
EFL_API efl_status efl_batch_unet_canvas(const efl_batch* batch, int32_t* width, int32_t* height);
/* The canvas layout (host only, no device work): n images of wh[2 i] x
 * wh[2 i + 1] pixels (multiples of 8) on shelves of a canvas whose width is
 * the smallest multiple of 512 holding the widest, tallest first, 8-pixel
 * gaps; origins[2 i], origins[2 i + 1] = image i's top-left corner. */
EFL_API efl_status efl_canvas_pack(const int32_t* wh, uint32_t n, int32_t* origins, int32_t* width,
                                   int32_t* height);
/* One Adam step (lr; beta 0.9 / 0.999; gradient clipped to global norm 1)
 * on the last recorded sample. */
EFL_API efl_status efl_unet_train_step(efl_unet* net, float lr, float* loss);

/* ---- Diagnostics ------------------------------------------------------ */

/* Kernels this library has launched since it was loaded (all handles). */
EFL_API uint64_t efl_kernel_launches(void);

/* Runs exactly `iterations` red-black pressure iterations on the current
 * state, with the current dt and no residual checks, to time the sweep:
 * precision 32 = the reference's f32 sweep on the pressure field
 * (gauss_seidel.wgsl:12-88 at the configured SOR weight), 64 = the FP64
 * iterate of the tolerance-driven solve, in place. */
EFL_API efl_status efl_pressure_sweeps(efl_sim* sim, int32_t precision, uint32_t iterations);

/* ---- Row slabs of one domain across devices ---------------------------- */

/* One row slab of the tolerance-driven red-black Gauss-Seidel pressure solve
 * (the FP64-iterate form of EFL_PROJECTION_GAUSS_SEIDEL with tolerance > 0:
 * residual of residual.wgsl:33-54, update of gauss_seidel.wgsl:44-88 on an
 * f32 correction), for a domain split into horizontal slabs with one process
 * (and one device) per slab.  No counterpart in the reference, which runs
 * one domain on one device (render_node.rs:193-476).
 * The slab owns rows [row0, row0 + rows) of the nx x ny grid and holds one
 * halo row above and one below for the iterate x (f64), the correction d
 * (f32) and the level set (f32); the caller fills the halos from the
 * neighbouring slabs (efl_slab_halo) at the points the solve needs them:
 *   load own rows -> level-set halos -> efl_slab_prepare ->
 *   x halos -> efl_slab_residual -> [ per half-sweep (color 1, then 0):
 *   d halos -> efl_slab_sweep ] x check_interval -> efl_slab_apply ->
 *   x halos -> efl_slab_residual -> ...
 * and sums the per-row partials of all slabs in row order for the relative
 * residual sqrt(sum r^2) / sqrt(sum b^2) (bevy_eulerian_fluid_b200/slab.py
 * is that driver).  With the halos exchanged as above, the slabs together
 * compute the unsplit solve's iterates bit for bit.
 * Every call is synchronous on the slab's own stream.  Errors are reported
 * through efl_last_error(NULL). */
typedef struct efl_slab efl_slab;

typedef struct efl_slab_desc {
    int32_t device;
    uint32_t nx, ny;     /* the whole domain */
    uint32_t row0, rows; /* this slab: 1 <= rows, row0 + rows <= ny */
    float dx;            /* 1 / length_unit, as in the step */
    float dt, rho;
    float sor_weight;
} efl_slab_desc;

enum efl_slab_field {
    EFL_SLAB_X = 0,        /* FP64 iterate (double)          */
    EFL_SLAB_D = 1,        /* f32 correction (float)         */
    EFL_SLAB_LEVELSET = 2  /* levelset_air (float)           */
};

EFL_API efl_status efl_slab_create(const efl_slab_desc* desc, efl_slab** out);
EFL_API efl_status efl_slab_destroy(efl_slab* slab);
/* Own rows (rows x nx, row-major; area_fraction rows x nx x 4 in the order
 * of EFL_FIELD_AREA_FRACTION): levelset_air, face fractions, divergence and
 * the previous pressure (the start iterate, widened to f64).  Host or device
 * pointers (copied with cudaMemcpyDefault). */
EFL_API efl_status efl_slab_load(efl_slab* slab, const float* levelset_air, const float* area_fraction,
                                 const float* divergence, const float* pressure);
/* side 0: the top edge (own row 0, halo row above), 1: the bottom edge (own
 * row rows-1, halo row below).  write 0 copies the own edge row of `field`
 * into buf (nx elements), write 1 copies buf into the halo row on that side.
 * buf: host or device memory.  A halo row beyond the domain's edge is never
 * read; writing it returns EFL_ERR_INVALID_ARGUMENT. */
EFL_API efl_status efl_slab_halo(efl_slab* slab, int32_t field, int32_t side, int32_t write, void* buf);
/* Builds the stencil coefficients of the own rows (needs the level-set halos). */
EFL_API efl_status efl_slab_prepare(efl_slab* slab);
/* FP64 residual of the current iterate (needs the x halos), the next
 * correction's right-hand side, d = 0; row_partials (host, 2 x rows
 * doubles): per own row the sum of r^2 and of b^2 over the counted cells. */
EFL_API efl_status efl_slab_residual(efl_slab* slab, double* row_partials);
/* One half-sweep of the correction on the cells with (x + y) % 2 == color
 * (global coordinates; the solve runs color 1 first); needs the d halos. */
EFL_API efl_status efl_slab_sweep(efl_slab* slab, int32_t color);
/* x += d on updated cells, x = 0 on air, fully solid and singular cells. */
EFL_API efl_status efl_slab_apply(efl_slab* slab);
/* The own rows of the iterate (rows x nx doubles, host or device memory). */
EFL_API efl_status efl_slab_read(efl_slab* slab, double* x);

/* ---- Allocation-free entry point -------------------------------------- */

/* Relative residual ||b - A p||_2 / ||b||_2 (operator of residual.wgsl:33-54,
 * FP64 norms over cells with phi < 0 that are not fully solid) of fields held
 * in caller-owned device memory, for callers that cannot let a library
 * allocate device memory (an engine that owns all GPU buffers through its own
 * arena, a frame loop that forbids allocation once running).  It has no
 * counterpart in the reference.
 *  - Inputs: device planes sharing one row pitch (bytes, multiple of 4, at
 *    least (nx+1)*4): pressure, divergence and levelset_air (nx x ny),
 *    area_fraction_u ((nx+1) x ny) and area_fraction_v (nx x (ny+1)), the
 *    layout efl_field_device_ptr returns; dx = 1/length_unit, dt, rho as in
 *    the step.
 *  - Output: out_device[0..2] = relative residual, ||r||_2, ||b||_2 (device
 *    memory), written asynchronously on `stream` (NULL: the legacy stream).
 *  - Allocates nothing: the per-block partial sums live in a fixed 256 KiB
 *    device array inside the library, which every GPU that loads the library
 *    holds until exit.  Grids above 4096 x 4096 = 16,777,216 cells are
 *    rejected with EFL_ERR_INVALID_ARGUMENT.
 *  - The first call on a device looks up that array's device address (with
 *    that device current); make that first call before any stream capture.
 *    The address is kept for the life of the process, so a device reset
 *    (cudaDeviceReset, or tearing down and recreating the primary context)
 *    between calls is not supported.
 *  - All calls share the one array: calls whose work overlaps on the GPU
 *    (different streams, or different host threads, at the same time) race
 *    and may return wrong norms.  Each call overwrites every partial it
 *    reads, so nothing carries over from the previous call.
 * Errors are reported through efl_last_error(NULL). */
EFL_API efl_status efl_residual_norms_noalloc(const float* pressure, const float* divergence,
                                              const float* levelset_air, const float* area_fraction_u,
                                              const float* area_fraction_v, uint32_t nx, uint32_t ny,
                                              size_t pitch_bytes, float dx, float dt, float rho,
                                              double* out_device, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EFL_H */
