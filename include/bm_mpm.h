/* bm_mpm.h — C ABI of the B200-native MLS-MPM soil step.
 *
 * This is the drop-in boundary for the MPMSolver path of 2nugu/basements:
 * plain pointers and sizes, no C++ or CUDA types in the signatures, every
 * call returns a bm_status_t. One handle is driven by one host thread at a
 * time; each handle owns a CUDA stream and its device buffers on the device
 * that was current when it was created. Kernel work is enqueued on that
 * stream; calls that return host data synchronise it.
 *
 * Reference interfaces replaced (paths inside 2nugu/basements):
 *   MPMSolver               include/basements/physics/mpm/mpm_solver.h:15-95
 *   Particle                include/basements/physics/mpm/particle.h:9-23
 *   SPGridCPU / GridNode    include/basements/physics/mpm/spgrid_cpu.h:12-99
 *   RigidColliderState      include/basements/physics/coupling/mpm_rigid_coupler.h:72-84
 *   CouplingReaction        include/basements/physics/coupling/mpm_rigid_coupler.h:201-205
 *   MPMRigidCouplerPIC      include/basements/physics/coupling/mpm_rigid_coupler_pic.h:88-184
 *   ApplyFn (coupler table) research/mpm_rigid_coupling/bench_compare_all.cpp:50-51
 *   TimeIntegrator          include/basements/physics/dynamics/integrator.h:19-57
 *   plugin C-ABI idiom      include/basements/engine/plugins/plugin_capi.h:14-106
 */
#ifndef BM_MPM_H
#define BM_MPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define BM_API __declspec(dllexport)
#else
#define BM_API __attribute__((visibility("default")))
#endif

#define BM_API_VERSION 2

typedef enum bm_status {
    BM_OK = 0,
    BM_ERR_INVALID_ARGUMENT = 1, /* null handle, bad size, dx <= 0, ... */
    BM_ERR_OUT_OF_MEMORY = 2,    /* device allocation failed or budget exceeded */
    BM_ERR_CUDA = 3,             /* a CUDA runtime call failed */
    BM_ERR_DOMAIN_ESCAPE = 4,    /* a particle stencil left the dense grid box */
    BM_ERR_NON_FINITE = 5,       /* NaN or Inf found in particle state */
    BM_ERR_TIMEOUT = 6,          /* a bounded wait gave up */
    BM_ERR_NOT_FOUND = 7,        /* unknown request or scene id */
    BM_ERR_STATE = 8,            /* call out of order (e.g. g2p before p2g) */
    BM_ERR_NO_DEVICE = 9         /* no CUDA device or the library was built without sm_100a */
} bm_status_t;

/* Dense grid box in node indices (node i sits at x = i*dx for the particle
 * stencil; the floor test uses (j + 0.5)*dx like the reference). origin is
 * rounded down and origin+extent up to multiples of 4 (the reference's 4^3
 * block size, spgrid_cpu.h:38-40). */
typedef struct bm_domain {
    int32_t origin[3];
    int32_t extent[3];
} bm_domain_t;

typedef enum bm_shape { BM_SHAPE_BOX = 0, BM_SHAPE_CYLINDER = 1 } bm_shape_t;

/* Byte-for-byte the field meaning of RigidColliderState (mpm_rigid_coupler.h:72-84)
 * with unpadded float[3]/float[4] in place of the 16-byte Vec3 / Quaternion.
 * orientation is (w, x, y, z). CYLINDER: radius half_extents[0], half-length
 * half_extents[1] along local Y. */
typedef struct bm_collider {
    float center[3];
    float orientation[4];
    float half_extents[3];
    float linear_velocity[3];
    float angular_velocity[3];
    float friction;
    float mass;
    int32_t shape;
} bm_collider_t;

/* CouplingReaction (mpm_rigid_coupler.h:201-205). */
typedef struct bm_reaction {
    float force[3];
    float torque[3];
    int32_t nodes_inside;
} bm_reaction_t;

/* Host SoA view of the particle store, one row per particle in the order the
 * particles were added. Any pointer may be NULL to skip that field.
 * Vectors are 3 floats, matrices 9 floats row-major (Particle, particle.h:9-23). */
typedef struct bm_particles_view {
    float* position;
    float* velocity;
    float* F;
    float* C;
    float* mass;
    float* volume;
} bm_particles_view_t;

typedef struct bm_solver bm_solver_t;

/* ---- library ---------------------------------------------------------- */
BM_API int bm_get_version(void);
BM_API const char* bm_status_string(bm_status_t status);
/* Text of the last error raised on the calling thread (CUDA message, which argument). */
BM_API const char* bm_last_error(void);
/* Makes `device` current for the calling thread; handles created afterwards
 * live on it (one process per GPU uses this with its local rank). */
BM_API bm_status_t bm_set_device(int32_t device);

/* ---- MPMSolver (mpm_solver.h:15-95) ----------------------------------- */
/* MPMSolver() + initialize(dx) (:17-21). domain may be NULL: the box is then
 * sized at the first step from the particle bounds plus `margin` nodes. */
BM_API bm_status_t bm_solver_create(float dx, const bm_domain_t* domain, bm_solver_t** out);
BM_API bm_status_t bm_solver_destroy(bm_solver_t* s);
/* Sets the dense box explicitly (before the grid is first used). */
BM_API bm_status_t bm_solver_set_domain(bm_solver_t* s, const bm_domain_t* domain);
BM_API bm_status_t bm_solver_get_domain(bm_solver_t* s, bm_domain_t* out);
/* Margin (nodes per side, default 16) used when the box is auto-sized. */
BM_API bm_status_t bm_solver_set_auto_margin(bm_solver_t* s, int32_t margin_nodes);
/* Particles are reordered by stencil base node (grid order) every `steps`
 * steps (default 32; 1 = every step, 0 = only when particles are added or
 * overwritten), so that neighbouring threads share stencil nodes. The order
 * only changes speed and the order of the FP32 reductions. */
BM_API bm_status_t bm_solver_set_sort_interval(bm_solver_t* s, int32_t steps);
/* Arithmetic of the per-particle Jacobi SVD in the fused step: 0 (default)
 * IEEE division and square root like the reference; 1 takes the rotation
 * angle from the hardware approximations (about 1 ulp). Both meet the
 * accuracy bars against the reference (mode 1 drifts about 2.5x further over
 * 1000 steps) and mode 1 saves under 2% of the step on B200. */
BM_API bm_status_t bm_solver_set_math_mode(bm_solver_t* s, int32_t mode);
/* Launch shape of the fused G2P + P2G kernel, one of
 * bm_launch_variant_count(): threads per CTA x minimum CTAs per SM, and the
 * order of the particles over a CTA's lanes. The second half of the variants
 * repeat the shapes of the first half with interleaved lanes (a warp takes
 * every other particle of 64 consecutive ones; named "<shape>/i2"), which
 * pays at high particle counts per cell. Chosen by the autotuner of the
 * batched form or set here; the plain solver's default is 128x7. */
BM_API bm_status_t bm_solver_set_launch_variant(bm_solver_t* s, int32_t variant);
BM_API int32_t bm_launch_variant_count(void);
BM_API const char* bm_launch_variant_name(int32_t variant);
/* set_material (:42-51): rescales V0 of existing particles by rho_old / rho_new. */
BM_API bm_status_t bm_solver_set_material(bm_solver_t* s, float young_modulus, float poisson_ratio,
                                          float bulk_density);
BM_API bm_status_t bm_solver_set_gravity(bm_solver_t* s, const float gravity[3]);      /* :52 */
BM_API bm_status_t bm_solver_set_plastic_alpha(bm_solver_t* s, float alpha);           /* :53 */
BM_API bm_status_t bm_solver_set_floor_friction(bm_solver_t* s, float mu_floor);       /* :54 */
/* add_particle (:23-34) for n particles: V0 = m / rho, F = I, C = 0.
 * velocity NULL means zero, mass NULL means 1.0 (the reference default).
 * Returns when the arrays have been copied (through the process's pinned
 * chunk pair): the caller may reuse them at once. */
BM_API bm_status_t bm_solver_add_particles(bm_solver_t* s, int64_t n, const float* position,
                                           const float* velocity, const float* mass);
BM_API bm_status_t bm_solver_num_particles(bm_solver_t* s, int64_t* out);
/* get_particles (:89): device-to-host copy into the caller's SoA view
 * (rows of each field, add order), through the process's pinned chunk pair;
 * returns when the copies have landed. */
BM_API bm_status_t bm_solver_get_particles(bm_solver_t* s, const bm_particles_view_t* view);
/* get_particles_mutable (:59): overwrite fields of particles [first, first+n);
 * NULL fields are left as they are. mass/volume are ignored. */
BM_API bm_status_t bm_solver_set_particles(bm_solver_t* s, int64_t first, int64_t n,
                                           const bm_particles_view_t* view);
/* step(dt) (:62-87): clear, P2G, update_grid, G2P. Enqueued, returns at once. */
BM_API bm_status_t bm_solver_step(bm_solver_t* s, float dt);
/* n_steps plain steps, enqueued back to back. */
BM_API bm_status_t bm_solver_step_n(bm_solver_t* s, float dt, int32_t n_steps);

/* ---- split step + coupler plug-in (mpm_rigid_coupler.h:207-214) ------- */
/* grid.clear() + the P2G loop (:72-78). */
BM_API bm_status_t bm_solver_p2g(bm_solver_t* s, float dt);
/* update_grid (:250-291). */
BM_API bm_status_t bm_solver_grid_update(bm_solver_t* s, float dt);
/* MPMRigidCouplerPIC::apply (mpm_rigid_coupler_pic.h:88-184): call between
 * bm_solver_grid_update and bm_solver_g2p. dt <= 0 gives a zero reaction and
 * leaves the grid unchanged. `out` is written before the call returns. */
BM_API bm_status_t bm_coupler_m1_apply(bm_solver_t* s, const bm_collider_t* body, float dt,
                                       bm_reaction_t* out);
/* No counterpart in the reference. The M1 apply above for up to 64 bodies
 * that allocates nothing: its scratch is a fixed 256-byte-aligned device array
 * of about 15 KB in the library, not buffers grown with cudaMalloc. For hosts
 * that may not allocate device memory at the call site: a fixed-budget tick
 * (cudaMalloc/cudaFree can wait for the whole device), or a process whose HBM
 * a pool already holds. n_bodies > 64 gives BM_ERR_INVALID_ARGUMENT; calling it
 * before bm_solver_p2g + bm_solver_grid_update have built the grid gives
 * BM_ERR_STATE. The array is shared by all solvers on a device: calls that
 * overlap in time race on it, so serialise them. bm_solver_create looks up
 * the array's address and loads the M1 kernels on its device: under CUDA's
 * default lazy module loading that first use loads code and may allocate
 * device memory, which the create call is allowed to do and this one is not.
 * `out` (n_bodies entries) is written before the call returns. */
BM_API bm_status_t bm_coupler_m1_apply_noalloc(bm_solver_t* s, int32_t n_bodies, const bm_collider_t* bodies,
                                               float dt, bm_reaction_t* out);
/* The M4.5a two-pass sweep coupler (research/mpm_rigid_coupling/couplers/
 * m4_5_hybrid.h:104-212, rule M4_5a :242-257): pass 1 sums the overlap
 * fraction (mpm_rigid_coupler.h:139-164) of the nodes inside the shape over
 * the allocated blocks meeting its tight AABB (:167-200); pass 2 gives each
 * such node m_b = body mass * frac / sum and the mass-weighted average of node
 * and body velocity. Same call contract as bm_coupler_m1_apply. The sum is
 * taken in double on the device (the reference sums in float in hash-map
 * order), so node states and the reaction agree with the reference to
 * rounding rather than bit for bit. */
BM_API bm_status_t bm_coupler_m45a_apply(bm_solver_t* s, const bm_collider_t* body, float dt,
                                         bm_reaction_t* out);
/* The M0 Dirichlet coupler, MPMRigidCoupler::apply
 * (src/physics/coupling/mpm_rigid_coupler.cpp:58-143): over the allocated
 * blocks meeting the box-formula AABB, each node of mass > 1e-8 inside the
 * shape keeps its velocity along the closest face's outward normal
 * (shape_outward_normal_local, mpm_rigid_coupler.h:106-132) at least the
 * body's and blends its tangential velocity toward the body's by
 * min(1, friction); node masses are unchanged. The reaction is -dp/dt and its
 * moment. Same call contract as bm_coupler_m1_apply; the grid after the call
 * matches the reference bit for bit, the reaction to its summation order. */
BM_API bm_status_t bm_coupler_m0_apply(bm_solver_t* s, const bm_collider_t* body, float dt,
                                       bm_reaction_t* out);
/* The other two layers of the sweep (m4_5_hybrid.h): M4.5b, M4_5b::apply
 * (:259-275), adds to M4.5a the Coulomb tangent projection (the node's
 * tangential velocity about the closest face's normal blended toward the
 * body's by min(1, friction)); M4.5, M4_5c::apply (:282-305), also scales
 * each node's mass share by the quadratic B-spline weight of its offset from
 * the centre, which by design breaks sum m_b = M. Same contract and
 * precision as bm_coupler_m45a_apply. */
BM_API bm_status_t bm_coupler_m45b_apply(bm_solver_t* s, const bm_collider_t* body, float dt,
                                         bm_reaction_t* out);
BM_API bm_status_t bm_coupler_m45_apply(bm_solver_t* s, const bm_collider_t* body, float dt,
                                        bm_reaction_t* out);
/* Coupler that bm_solver_step_coupled applies to its bodies (each body in
 * order, the ApplyFn table of bench_compare_all.cpp:50-70): BM_COUPLER_M1
 * (default), BM_COUPLER_M45A, BM_COUPLER_M0, BM_COUPLER_M45B or
 * BM_COUPLER_M45. The batched and served forms and the tape use M1. */
#define BM_COUPLER_M1 0
#define BM_COUPLER_M45A 1
#define BM_COUPLER_M0 2
#define BM_COUPLER_M45B 3
#define BM_COUPLER_M45 4
BM_API bm_status_t bm_solver_set_coupler(bm_solver_t* s, int32_t coupler);
/* The G2P loop (:83-86). */
BM_API bm_status_t bm_solver_g2p(bm_solver_t* s, float dt);
/* P2G, grid update, M1 for each body in order, G2P, all on the handle's
 * stream. reactions (n_bodies entries) may be NULL: the reactions then stay on
 * the device until bm_solver_get_reactions. With a host pointer the call
 * waits for the step to finish. */
BM_API bm_status_t bm_solver_step_coupled(bm_solver_t* s, float dt, int32_t n_bodies,
                                          const bm_collider_t* bodies, bm_reaction_t* reactions);
BM_API bm_status_t bm_solver_get_reactions(bm_solver_t* s, int32_t n_bodies, bm_reaction_t* out);

/* ---- grid access (get_grid / get_grid_mutable, :90-95) ----------------- */
/* Number of nodes of the dense box (product of the rounded extents). */
BM_API bm_status_t bm_solver_grid_num_nodes(bm_solver_t* s, int64_t* out);
/* Dense copy in (i, j, k) order, k fastest, over the box of
 * bm_solver_get_domain. Any pointer may be NULL. velocity and mass hold what
 * the reference's GridNode holds at this point of the step (momentum after
 * P2G, velocity after update_grid and the couplers). force is the P2G force
 * after bm_solver_p2g; after bm_solver_step / _step_coupled the fused step
 * adds force*dt into the momentum during P2G, so force reads back as zero.
 * active is the reference's node.active (mass > 0: touched this step,
 * seeded, or claimed by a coupler). block_allocated (one byte per node)
 * reports whether the node's 4^3 block has ever been touched, the blocks the
 * reference's hash grid keeps (spgrid_cpu.h:78-91). */
BM_API bm_status_t bm_solver_get_grid(bm_solver_t* s, float* velocity, float* force, float* mass,
                                      uint8_t* active, uint8_t* block_allocated);
/* Seeds nodes like the reference tests and scenarios do through get_node()
 * (tests/test_mpm_rigid_coupler.cpp:30-34, scenario_box_drop.h:41-53): sets
 * velocity and mass, marks each node active and its block allocated. Nodes
 * outside the box are an error. */
BM_API bm_status_t bm_solver_seed_grid(bm_solver_t* s, int64_t n, const int32_t* ijk, const float* velocity,
                                       const float* mass);
/* Overwrites the velocity of every node of the box from a dense array as
 * returned by bm_solver_get_grid (mass is left as it is). */
BM_API bm_status_t bm_solver_set_grid_velocity(bm_solver_t* s, const float* velocity);

/* ---- status and diagnostics ------------------------------------------ */
/* Waits for the handle's stream and returns the first device-side error
 * seen since the last call (BM_ERR_DOMAIN_ESCAPE, BM_ERR_NON_FINITE), then
 * clears it. escaped (may be NULL) gets the number of stencil writes dropped
 * because they fell outside the box. */
BM_API bm_status_t bm_solver_sync(bm_solver_t* s, int64_t* escaped);
/* Nodes, counted since the handle was created, whose particle mass fell from
 * at least 1e-4 to (0, 1e-6] in one step. update_grid (mpm_solver.h:257)
 * keeps the momentum without force at nodes of mass <= 1e-6; the fused
 * kernel records the force of a light contribution except at nodes that held
 * at least 1e-4 in the previous step's grid, so only these nodes can miss a
 * record. 0 means every step so far kept the reference's rule exactly. No
 * counterpart in the reference. */
BM_API bm_status_t bm_solver_light_node_suspects(bm_solver_t* s, int64_t* out);
/* The CUDA stream (cudaStream_t) the handle enqueues on. */
BM_API bm_status_t bm_solver_stream(bm_solver_t* s, void** stream);
/* Per-kernel timing with CUDA events on the handle's stream (off by default).
 * bm_solver_profile_read returns up to `cap` entries: name (static string),
 * total milliseconds and launch count since the last reset. */
BM_API bm_status_t bm_solver_profile_enable(bm_solver_t* s, int32_t on);
BM_API bm_status_t bm_solver_profile_read(bm_solver_t* s, int32_t cap, const char** names, double* total_ms,
                                          int64_t* launches, int32_t* n_out);
BM_API bm_status_t bm_solver_profile_reset(bm_solver_t* s);
/* Stream-ordered wall timer: records a CUDA event on the handle's stream at
 * start; stop records a second one, waits for it and returns the elapsed
 * milliseconds between the two. */
BM_API bm_status_t bm_solver_timer_start(bm_solver_t* s);
BM_API bm_status_t bm_solver_timer_stop(bm_solver_t* s, double* ms);

/* ---- batched form: many scenes per launch -------------------------------
 * No reference counterpart (the reference steps one MPMSolver at a time,
 * mpm_solver.h:62-87). Scenes of uneven particle and grid counts are stepped
 * together: every phase of the step is one launch over a table of scenes,
 * each scene with its own dx, box, material, dt and optional rigid body
 * (coupled with M1 and integrated on the device like the reference's
 * TimeIntegrator, integrator.h:19-57), and chunks of steps replay as one CUDA
 * graph. */
typedef struct bm_scene_desc {
    float dx;
    int32_t has_domain;          /* 0: box from the particle bounds + 16 nodes */
    bm_domain_t domain;
    int64_t n_particles;
    const float* position;       /* n*3 */
    const float* velocity;       /* n*3 or NULL */
    const float* mass;           /* n or NULL (1.0) */
    float young_modulus, poisson_ratio, bulk_density, plastic_alpha, floor_friction;
    float gravity[3];
    float dt;
    int32_t has_body;
    bm_collider_t body;
    int32_t body_dynamic;        /* 0: kinematic (moved by its velocities only) */
    float body_inv_inertia[9];   /* body-space inverse inertia (integrator.h:33) */
    int32_t body_inv_inertia_given; /* 1: body_inv_inertia as given, all zero included
                                       (a body that cannot rotate); 0: all zero means
                                       the identity, the reference scenes' value */
} bm_scene_desc_t;

typedef struct bm_batch bm_batch_t;

typedef struct bm_tune_result {
    int32_t variant;        /* launch shape of the fused kernel */
    int32_t sort_interval;  /* steps between regroupings */
    int32_t bin_shift;      /* sort bins of 2^bin_shift cells per axis */
    float ms_per_step;      /* measured with the chosen setting */
} bm_tune_result_t;

BM_API bm_status_t bm_batch_create(int32_t n_scenes, const bm_scene_desc_t* scenes, bm_batch_t** out);
BM_API bm_status_t bm_batch_destroy(bm_batch_t* b);
BM_API bm_status_t bm_batch_num_scenes(bm_batch_t* b, int32_t* out);
BM_API bm_status_t bm_batch_num_particles(bm_batch_t* b, int32_t scene, int64_t* out);
/* Every scene advances n_steps steps of its own dt. Enqueued; graph chunks
 * replay once the launch setting is fixed. */
BM_API bm_status_t bm_batch_step(bm_batch_t* b, int32_t n_steps);
BM_API bm_status_t bm_batch_steps_done(bm_batch_t* b, int64_t* out);
BM_API bm_status_t bm_batch_get_particles(bm_batch_t* b, int32_t scene, const bm_particles_view_t* view);
BM_API bm_status_t bm_batch_get_body(bm_batch_t* b, int32_t scene, bm_collider_t* out);
/* Reaction of the last step's coupler on the scene's body. */
BM_API bm_status_t bm_batch_get_reaction(bm_batch_t* b, int32_t scene, bm_reaction_t* out);
/* Waits; returns the first device-side error of any scene (and which). */
BM_API bm_status_t bm_batch_sync(bm_batch_t* b, int32_t* bad_scene, int64_t* escaped);
/* bm_solver_light_node_suspects summed over the batch's scenes. */
BM_API bm_status_t bm_batch_light_node_suspects(bm_batch_t* b, int64_t* out);
BM_API bm_status_t bm_batch_set_graph(bm_batch_t* b, int32_t on);
/* Per-phase timing of the batch, as bm_solver_profile_*; while it is on the
 * steps run eagerly (no graph replay), so each launch can be timed. */
BM_API bm_status_t bm_batch_profile_enable(bm_batch_t* b, int32_t on);
BM_API bm_status_t bm_batch_profile_read(bm_batch_t* b, int32_t cap, const char** names, double* total_ms,
                                         int64_t* launches, int32_t* n_out);
BM_API bm_status_t bm_batch_profile_reset(bm_batch_t* b);
BM_API bm_status_t bm_batch_set_launch(bm_batch_t* b, int32_t variant, int32_t sort_interval, int32_t bin_shift);
/* Times each candidate launch setting for `trial_steps` steps on this batch
 * (the state is saved before and restored after every trial, so tuning does
 * not advance the scenes) and keeps the fastest. */
BM_API bm_status_t bm_batch_autotune(bm_batch_t* b, int32_t trial_steps, bm_tune_result_t* out);
BM_API bm_status_t bm_batch_timer_start(bm_batch_t* b);
BM_API bm_status_t bm_batch_timer_stop(bm_batch_t* b, double* ms);

/* ---- serving loop: continuous batching ---------------------------------
 * No reference counterpart. A server owns one GPU stream and a worker
 * thread. Requests (a scene and a number of steps) are queued by
 * bm_server_submit from any thread; at every step boundary the worker admits
 * queued requests in order while their estimated device footprint fits the
 * HBM budget, steps all co-resident scenes together (one launch per phase
 * for all of them, so their work overlaps on the device), and retires the
 * scenes that have done their steps, copying their particles and body back
 * to host memory. Waits are bounded (bm_server_wait returns BM_ERR_TIMEOUT). */
typedef struct bm_server bm_server_t;

typedef struct bm_server_config {
    double hbm_budget_bytes;  /* admission budget, default 150e9 */
    int32_t max_active;       /* most co-resident scenes, default 1024 */
    int32_t sort_interval;    /* steps between regroupings, default 32 */
    int32_t variant;          /* launch variant of the fused kernel (bm_solver_set_launch_variant),
                                 default 128x7/i2; negative: the default */
} bm_server_config_t;

typedef enum bm_request_state {
    BM_REQ_QUEUED = 0,
    BM_REQ_RUNNING = 1,
    BM_REQ_DONE = 2,
    BM_REQ_FAILED = 3,
    BM_REQ_CANCELLED = 4
} bm_request_state_t;

typedef struct bm_server_stats {
    int64_t submitted, completed, failed, cancelled, queued, active;
    int64_t iterations;        /* batched steps launched */
    double p50_latency_ms, p99_latency_ms, mean_latency_ms;  /* submit -> result ready */
    double particle_steps;     /* of completed requests */
    double busy_seconds;       /* wall time with scenes on the device */
    double peak_bytes;         /* largest admitted footprint */
    /* host time of the worker's phases: admitting requests (upload, grid,
     * bodies), enqueueing the batched steps, retiring finished requests
     * (read-back, release) */
    double admit_seconds, step_seconds, retire_seconds;
} bm_server_stats_t;

BM_API bm_status_t bm_server_create(const bm_server_config_t* config, bm_server_t** out);
/* Stops the worker; queued and running requests are cancelled. */
BM_API bm_status_t bm_server_destroy(bm_server_t* s);
/* Copies the scene's arrays; the caller may free them on return. */
BM_API bm_status_t bm_server_submit(bm_server_t* s, const bm_scene_desc_t* scene, int32_t n_steps,
                                    int64_t* request_id);
BM_API bm_status_t bm_server_poll(bm_server_t* s, int64_t request_id, int32_t* state);
/* Waits at most timeout_ms for the request to finish. */
BM_API bm_status_t bm_server_wait(bm_server_t* s, int64_t request_id, int32_t timeout_ms);
/* Final particles (add order) and body of a finished request; any pointer may be NULL. */
BM_API bm_status_t bm_server_result(bm_server_t* s, int64_t request_id, const bm_particles_view_t* view,
                                    bm_collider_t* body, double* latency_ms);
BM_API bm_status_t bm_server_release(bm_server_t* s, int64_t request_id);
BM_API bm_status_t bm_server_cancel(bm_server_t* s, int64_t request_id);
BM_API bm_status_t bm_server_stats(bm_server_t* s, bm_server_stats_t* out);
/* Device bytes the admission policy charges for a scene. */
BM_API bm_status_t bm_server_estimate_bytes(const bm_scene_desc_t* scene, double* bytes);

/* ---- differentiable run --------------------------------------------------
 * The reference declares AutodiffTape (mpm_autodiff_tape.h:37-92) and passes
 * it to MPMSolver::step(dt, tape*) (mpm_solver.h:71-87), but the tape records
 * nothing: there is no reference gradient. These calls give the split step
 * (bm_solver_p2g, _grid_update, bm_coupler_m1_apply, _g2p) a reverse pass with
 * hand-written adjoint kernels and checkpoints every K steps.
 * Particle arrays are in add order, rows of 3 floats (9 for F and C). */
typedef struct bm_tape bm_tape_t;
/* A tape on solver s; checkpoint_every = K >= 1. The tape keeps
 * ceil(n_steps/K)+1 checkpoints and K step states of 96 B per particle. */
BM_API bm_status_t bm_tape_create(bm_solver_t* s, int32_t checkpoint_every, bm_tape_t** out);
/* Frees the tape's buffers; valid before or after its solver is destroyed. */
BM_API bm_status_t bm_tape_destroy(bm_tape_t* t);
/* n_steps split steps from the solver's current particle state. With a
 * body, its centre follows the piecewise-linear path through n_waypoints
 * points (xyz each) spread evenly over n_steps*dt, its linear velocity is the
 * slope of the current segment, everything else stays as in *body; body NULL:
 * no coupler. The solver ends in the final state. */
BM_API bm_status_t bm_tape_forward(bm_tape_t* t, float dt, int32_t n_steps, const bm_collider_t* body,
                                   int32_t n_waypoints, const float* waypoints);
/* Reverse pass of the last bm_tape_forward. dL_dx (required) and dL_dv (or
 * NULL) are the loss gradient at the final state; outputs, each may be NULL:
 * dL_dwaypoints (n_waypoints x 3), dL_dx0 and dL_dv0 (gradient at the initial
 * state). The solver is left in the final state. */
BM_API bm_status_t bm_adjoint_backward(bm_tape_t* t, const float* dL_dx, const float* dL_dv,
                                       float* dL_dwaypoints, float* dL_dx0, float* dL_dv0);
/* The same reverse pass for the whole particle state: dL_dfinal holds the
 * loss gradient at the final state (position/velocity n x 3, F/C n x 9; NULL
 * fields are zero, mass/volume ignored); dL_dinitial (or NULL) receives the
 * gradient at the initial state in the fields it points to. */
BM_API bm_status_t bm_adjoint_backward_state(bm_tape_t* t, const bm_particles_view_t* dL_dfinal,
                                             float* dL_dwaypoints, const bm_particles_view_t* dL_dinitial);
/* dL/d(body linear velocity) and dL/d(body angular velocity) of every step
 * of the last backward pass: n_steps x 6 doubles. */
BM_API bm_status_t bm_tape_body_grad(bm_tape_t* t, int32_t n_steps, double* out);

/* ---- test support ----------------------------------------------------- */
/* SVD::compute (include/basements/core/math/svd.h:18-108) as the step kernels
 * run it on the device, for n row-major 3x3 matrices F (host arrays): U, V
 * (n x 9) and the unsorted singular values S (n x 3). fast_math selects the
 * fast-intrinsic arithmetic of bm_solver_set_math_mode. Synchronous; it
 * allocates device memory for the call. */
BM_API bm_status_t bm_debug_svd3(int64_t n, const float* F, float* U, float* S, float* V, int32_t fast_math);

#ifdef __cplusplus
}
#endif
#endif /* BM_MPM_H */
