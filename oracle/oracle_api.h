/* oracle_api.h — C interface shared by the two CPU checkers.
 *
 * TEST INFRASTRUCTURE ONLY (see mpm_oracle.hpp). Two libraries export this
 * same set of functions under different prefixes:
 *
 *   orc_*  oracle/liboracle_mpm_f32.so and oracle/liboracle_mpm_f64.so —
 *          the restatement in mpm_oracle.hpp, instantiated in float / double;
 *   ref_*  oracle/_ref/libref_mpm.so — the reference's own MPMSolver,
 *          MPMRigidCouplerPIC and TimeIntegrator compiled from its headers by
 *          oracle/Makefile (never committed; rebuilt from the reference tree).
 *
 * All arrays are float at the boundary, particle data as SoA with 3 floats per
 * vector and 9 row-major floats per matrix. The collider matches bm_collider_t.
 */
#ifndef BM_ORACLE_API_H
#define BM_ORACLE_API_H
#include <stdint.h>

#ifndef ORACLE_PREFIX
#error "define ORACLE_PREFIX (orc or ref) before including oracle_api.h"
#endif
#define ORC_CAT2(a, b) a##_##b
#define ORC_CAT(a, b) ORC_CAT2(a, b)
#define ORC(name) ORC_CAT(ORACLE_PREFIX, name)
#define ORC_EXPORT extern "C" __attribute__((visibility("default")))

typedef struct orc_collider {
    float center[3];
    float orientation[4]; /* w, x, y, z */
    float half_extents[3];
    float linear_velocity[3];
    float angular_velocity[3];
    float friction;
    float mass;
    int32_t shape; /* 0 box, 1 cylinder */
} orc_collider_t;

ORC_EXPORT int ORC(precision_bytes)(void);
ORC_EXPORT void* ORC(create)(float dx);
ORC_EXPORT void ORC(destroy)(void* h);
ORC_EXPORT void ORC(set_material)(void* h, float E, float nu, float rho);
ORC_EXPORT void ORC(set_gravity)(void* h, float gx, float gy, float gz);
ORC_EXPORT void ORC(set_plastic_alpha)(void* h, float a);
ORC_EXPORT void ORC(set_floor_friction)(void* h, float mu);
ORC_EXPORT void ORC(add_particles)(void* h, int64_t n, const float* pos, const float* vel, const float* mass);
ORC_EXPORT int64_t ORC(num_particles)(void* h);
ORC_EXPORT void ORC(set_particle_state)(void* h, int64_t first, int64_t n, const float* pos, const float* vel,
                                       const float* F, const float* C);
ORC_EXPORT void ORC(get_particles)(void* h, float* pos, float* vel, float* F, float* C, float* mass, float* vol);
/* x, v (n x 3), F, C (n x 9, row-major) in the solver's own precision,
 * widened to double; NULL skips a field */
ORC_EXPORT void ORC(get_state_f64)(void* h, double* pos, double* vel, double* F, double* C);
/* set_particle_state from double arrays (rounded to the solver's precision) */
ORC_EXPORT void ORC(set_state_f64)(void* h, int64_t first, int64_t n, const double* pos, const double* vel,
                                   const double* F, const double* C);
ORC_EXPORT void ORC(step)(void* h, float dt, int n_steps);
ORC_EXPORT void ORC(p2g)(void* h, float dt);
ORC_EXPORT void ORC(grid_update)(void* h, float dt);
ORC_EXPORT void ORC(g2p)(void* h, float dt);
/* reaction: force[3], torque[3]; returns nodes_inside */
ORC_EXPORT int ORC(m1_apply)(void* h, const orc_collider_t* body, float dt, float* reaction6);
/* the M0 Dirichlet coupler (MPMRigidCoupler); same reaction layout */
ORC_EXPORT int ORC(m0_apply)(void* h, const orc_collider_t* body, float dt, float* reaction6);
/* the M4.5a two-pass sweep coupler; same reaction layout */
ORC_EXPORT int ORC(m45a_apply)(void* h, const orc_collider_t* body, float dt, float* reaction6);
/* M4.5b (+ friction tangent) and M4.5 (= M4_5c, + B-spline mass weight) */
ORC_EXPORT int ORC(m45b_apply)(void* h, const orc_collider_t* body, float dt, float* reaction6);
ORC_EXPORT int ORC(m45c_apply)(void* h, const orc_collider_t* body, float dt, float* reaction6);
ORC_EXPORT int64_t ORC(grid_num_nodes)(void* h);
/* every node of every allocated block; returns the count written (<= cap) */
ORC_EXPORT int64_t ORC(grid_get)(void* h, int32_t* ijk, float* vel, float* force, float* mass, uint8_t* active,
                                 int64_t cap);
ORC_EXPORT void ORC(grid_seed)(void* h, int64_t n, const int32_t* ijk, const float* vel, const float* mass);
/* The box_drop scene of the reference's research harness, method M1, grid
 * only: 720 steps; per step 10 floats: t, box x/y/z, box vy, p_body_y,
 * p_grid_y, p_sum_y, KE, nodes_inside. Returns the number of rows. */
ORC_EXPORT int ORC(box_drop_m1)(float* rows, int max_rows);
/* n coupled steps of a particle scene with one dynamic rigid body, in the
 * order of the research harness (bench_compare_all.cpp:96-116) around the
 * MPM phases: P2G, update_grid, weight m*g applied to the body, M1 coupler on
 * the body's current state, reaction added, TimeIntegrator step (zero
 * damping; body-space inverse inertia inv_inertia, row-major 3x3, applied to
 * the torque as the integrator does, or the identity the reference's bodies
 * start with when NULL), G2P. body is updated in place (center, orientation,
 * velocities). */
ORC_EXPORT void ORC(run_dynamic_body)(void* h, orc_collider_t* body, float gx, float gy, float gz, float dt,
                                      int n_steps, const float* inv_inertia);
/* Restatement only (orc_*): turns on (on != 0) or off the record of the run's
 * discontinuous decisions (SVD pair skip and sweep stop, M1 inside test) and
 * reads it: out = {svd hash, inside hash, rotations, sweeps, inside count},
 * each accumulated since the record was turned on. */
ORC_EXPORT void ORC(decisions_enable)(void* h, int on);
ORC_EXPORT void ORC(decisions_read)(void* h, uint64_t* out5);
/* Restatement only: a tape of those decisions. mode 1 records the solver's
 * decisions into the tape (cleared), 2 replays them from its start (the
 * solver takes the recorded decisions instead of its own comparisons), 0
 * detaches it. status: {SVD calls recorded, replayed; coupler calls
 * recorded, replayed + 2^40 if a replay ran past the record}. */
ORC_EXPORT void* ORC(tape_new)(void);
ORC_EXPORT void ORC(tape_free)(void* t);
ORC_EXPORT void ORC(solver_use_tape)(void* h, void* t, int mode);
ORC_EXPORT void ORC(tape_status)(void* t, int64_t* out4);
/* Restatement only: a tape's content as arrays (SVD codes; coupler inside sets
 * flattened, offsets of n_calls + 1; NULL arrays: sizes only, into sizes3 =
 * {SVD codes, coupler calls, keys}) and back, so that one checker's record can
 * be replayed by the other. */
ORC_EXPORT void ORC(tape_export)(void* t, uint16_t* svd, int64_t* keys, int64_t* offsets, int64_t* sizes3);
ORC_EXPORT void ORC(tape_import)(void* t, int64_t n_svd, const uint16_t* svd, int64_t n_calls, const int64_t* keys,
                                 const int64_t* offsets);
/* SVD of n row-major 3x3 matrices: U (n*9), sigma (n*3), V (n*9). */
ORC_EXPORT void ORC(svd)(int64_t n, const float* F, float* U, float* S, float* V);

#endif
