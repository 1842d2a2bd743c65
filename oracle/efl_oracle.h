/*
 * efl_oracle.h — TEST INFRASTRUCTURE, not product code.
 *
 * CPU restatement of the reference's per-step fluid pipeline
 * (narasan49/bevy_eulerian_fluid v0.4.0, WGSL kernels under
 * src/euler_fluid/), used only by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg as the parity checker.  The product library
 * (libefl_b200.so) never links or calls it.
 *
 * Parity is unpinned: the reference publishes no golden vectors or numeric
 * fixtures, and its WGSL/wgpu pipeline cannot run here (no graphics stack,
 * no Rust toolchain).  The oracle is pinned by its own known-answer tests
 * (tests/test_oracle_kat.py) and by committed fixtures it generated.
 *
 * The API mirrors include/efl.h one for one (eflo_* <-> efl_*), with the
 * same structs, so one test driver can run both backends.
 */
#ifndef EFL_ORACLE_H
#define EFL_ORACLE_H

#include "../include/efl.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct eflo_sim eflo_sim;

EFL_API efl_status eflo_create(const efl_config* cfg, eflo_sim** out);
EFL_API efl_status eflo_destroy(eflo_sim* sim);
EFL_API const char* eflo_last_error(const eflo_sim* sim);
EFL_API efl_status eflo_reset(eflo_sim* sim);
EFL_API efl_status eflo_set_projection(eflo_sim* sim, const efl_projection* p);
EFL_API efl_status eflo_set_reinit(eflo_sim* sim, const efl_reinit* r);
EFL_API efl_status eflo_set_transform(eflo_sim* sim, const float transform[16]);
EFL_API efl_status eflo_set_obstacles(eflo_sim* sim, const efl_solid_obstacle* obstacles, uint32_t n);
EFL_API efl_status eflo_set_local_forces(eflo_sim* sim, const efl_force* forces, uint32_t n);
EFL_API efl_status eflo_set_sources(eflo_sim* sim, const efl_source* sources, uint32_t n, int32_t oneshot);
EFL_API efl_status eflo_step(eflo_sim* sim, float dt, efl_step_stats* stats);
EFL_API efl_status eflo_run_stage(eflo_sim* sim, int32_t stage, float dt, efl_step_stats* stats);
EFL_API efl_status eflo_read_solid_forces(eflo_sim* sim, efl_solid_force out[EFL_MAX_SOLIDS]);
EFL_API efl_status eflo_read_force_bins(eflo_sim* sim, int32_t out[3 * EFL_MAX_SOLIDS]);
EFL_API efl_status eflo_field_shape(const eflo_sim* sim, int32_t field, uint32_t* width,
                                    uint32_t* height, uint32_t* channels, uint32_t* elem_bytes);
EFL_API efl_status eflo_get_field(eflo_sim* sim, int32_t field, void* host_dst, size_t bytes);
EFL_API efl_status eflo_set_field(eflo_sim* sim, int32_t field, const void* host_src, size_t bytes);
EFL_API efl_status eflo_residual(eflo_sim* sim, double* relative, double* norm_r, double* norm_b);
EFL_API efl_status eflo_fluid_volume(eflo_sim* sim, uint64_t* cells);
EFL_API efl_status eflo_velocity_magnitude(eflo_sim* sim, float* min_mag, float* max_mag);
EFL_API efl_status eflo_divergence_norms(eflo_sim* sim, double* l2, double* linf);

/* Two-layer particle level set (src/euler_fluid/particle_levelset_two_layers). */
EFL_API efl_status eflo_set_particle_levelset(eflo_sim* sim, int32_t enable);
EFL_API efl_status eflo_particle_counts(eflo_sim* sim, uint32_t counts[2], uint32_t* dropped);
EFL_API efl_status eflo_read_particles(eflo_sim* sim, int32_t layer, efl_particle* dst, uint32_t capacity,
                                       uint32_t* n);
EFL_API efl_status eflo_write_particles(eflo_sim* sim, int32_t layer, const efl_particle* src, uint32_t n);
EFL_API efl_status eflo_pls_run_phase(eflo_sim* sim, int32_t phase, float dt);

/* Number of OpenMP threads the oracle uses (0 = OpenMP default). */
EFL_API void eflo_set_threads(int32_t n);
EFL_API int32_t eflo_get_threads(void);

/* Literal single-thread raster-order execution of the reference's racy FIM
 * update kernel (update.wgsl:13-54), for the tolerance comparison against
 * the deterministic two-phase variant. 1 = use it, 0 = two-phase. */
EFL_API void eflo_set_fim_serial(eflo_sim* sim, int32_t on);

/* The shared exp restatement used by the Gaussian force splat. */
EFL_API float eflo_exp(float x);

#ifdef __cplusplus
}
#endif

#endif
