// ref_harness.cpp — C interface over the reference's OWN solver code.
//
// TEST INFRASTRUCTURE ONLY. oracle/Makefile compiles this file against the
// reference's header tree (include/ and research/mpm_rigid_coupling/ of
// 2nugu/basements) with the reference's flags (-O2 -std=c++17 -mavx2) into
// oracle/_ref/libref_mpm.so, exporting the ref_* names of oracle_api.h. No
// reference source is copied here: every computation below is a call into
// the reference's MPMSolver (include/basements/physics/mpm/mpm_solver.h),
// SVD (include/basements/core/math/svd.h), MPMRigidCouplerPIC
// (include/basements/physics/coupling/mpm_rigid_coupler_pic.h), the M0
// Dirichlet coupler MPMRigidCoupler (src/physics/coupling/mpm_rigid_coupler.cpp,
// compiled where it lies by oracle/Makefile), the M4.5a
// sweep coupler (research/mpm_rigid_coupling/couplers/m4_5_hybrid.h) and
// TimeIntegrator (include/basements/physics/dynamics/integrator.h).
//
// The split phases (grid.clear / p2g_single / update_grid / g2p_single) are
// private members of MPMSolver; they are reached by compiling the header
// with `private` redefined as `public`, which changes no generated code.
#include <algorithm>
#include <cmath>
#include <unordered_map>
#include <vector>
#define private public
#include "basements/physics/mpm/mpm_solver.h"
#undef private
#include "basements/physics/coupling/mpm_rigid_coupler_pic.h"
#include "basements/physics/dynamics/integrator.h"
#include "basements/physics/rigid_body.h"
#include "scenarios/scenario_box_drop.h"
#include "couplers/m4_5_hybrid.h"

#define ORACLE_PREFIX ref
#include "oracle_api.h"

using namespace basements;
using math::Matrix3;
using math::Vec3;
using mpm::MPMSolver;
namespace cp = basements::physics::coupling;

static MPMSolver* sv(void* h) { return static_cast<MPMSolver*>(h); }

static cp::RigidColliderState to_state(const orc_collider_t* b) {
    cp::RigidColliderState s;
    s.center = Vec3(b->center[0], b->center[1], b->center[2]);
    s.orientation = math::Quaternion(b->orientation[0], b->orientation[1], b->orientation[2], b->orientation[3]);
    s.half_extents = Vec3(b->half_extents[0], b->half_extents[1], b->half_extents[2]);
    s.linear_velocity = Vec3(b->linear_velocity[0], b->linear_velocity[1], b->linear_velocity[2]);
    s.angular_velocity = Vec3(b->angular_velocity[0], b->angular_velocity[1], b->angular_velocity[2]);
    s.friction = b->friction;
    s.mass = b->mass;
    s.shape = b->shape == 1 ? cp::ShapeKind::CYLINDER : cp::ShapeKind::BOX;
    return s;
}

ORC_EXPORT int ref_precision_bytes(void) { return 4; }
ORC_EXPORT void* ref_create(float dx) {
    MPMSolver* s = new MPMSolver();
    s->initialize(dx);
    return s;
}
ORC_EXPORT void ref_destroy(void* h) { delete sv(h); }
ORC_EXPORT void ref_set_material(void* h, float E, float nu, float rho) { sv(h)->set_material(E, nu, rho); }
ORC_EXPORT void ref_set_gravity(void* h, float gx, float gy, float gz) { sv(h)->set_gravity(Vec3(gx, gy, gz)); }
ORC_EXPORT void ref_set_plastic_alpha(void* h, float a) { sv(h)->set_plastic_alpha(a); }
ORC_EXPORT void ref_set_floor_friction(void* h, float mu) { sv(h)->set_floor_friction(mu); }

ORC_EXPORT void ref_add_particles(void* h, int64_t n, const float* pos, const float* vel, const float* mass) {
    for (int64_t p = 0; p < n; ++p) {
        Vec3 v = vel ? Vec3(vel[3 * p], vel[3 * p + 1], vel[3 * p + 2]) : Vec3(0, 0, 0);
        sv(h)->add_particle(Vec3(pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]), v, mass ? mass[p] : 1.0f);
    }
}
ORC_EXPORT int64_t ref_num_particles(void* h) { return (int64_t)sv(h)->get_particles().size(); }

ORC_EXPORT void ref_set_particle_state(void* h, int64_t first, int64_t n, const float* pos, const float* vel,
                                       const float* F, const float* C) {
    auto& ps = sv(h)->get_particles_mutable();
    for (int64_t q = 0; q < n; ++q) {
        mpm::Particle& p = ps[first + q];
        if (pos) p.position = Vec3(pos[3 * q], pos[3 * q + 1], pos[3 * q + 2]);
        if (vel) p.velocity = Vec3(vel[3 * q], vel[3 * q + 1], vel[3 * q + 2]);
        for (int a = 0; a < 9; ++a) {
            if (F) p.F.m[a / 3][a % 3] = F[9 * q + a];
            if (C) p.C.m[a / 3][a % 3] = C[9 * q + a];
        }
    }
}

ORC_EXPORT void ref_set_state_f64(void* h, int64_t first, int64_t n, const double* pos, const double* vel,
                                  const double* F, const double* C) {
    auto& ps = sv(h)->get_particles_mutable();
    for (int64_t q = 0; q < n; ++q) {
        mpm::Particle& p = ps[first + q];
        if (pos) p.position = Vec3((float)pos[3 * q], (float)pos[3 * q + 1], (float)pos[3 * q + 2]);
        if (vel) p.velocity = Vec3((float)vel[3 * q], (float)vel[3 * q + 1], (float)vel[3 * q + 2]);
        for (int a = 0; a < 9; ++a) {
            if (F) p.F.m[a / 3][a % 3] = (float)F[9 * q + a];
            if (C) p.C.m[a / 3][a % 3] = (float)C[9 * q + a];
        }
    }
}

ORC_EXPORT void ref_get_state_f64(void* h, double* pos, double* vel, double* F, double* C) {
    int64_t q = 0;
    for (const auto& p : sv(h)->get_particles()) {
        const float x[3] = {p.position.x, p.position.y, p.position.z};
        const float v[3] = {p.velocity.x, p.velocity.y, p.velocity.z};
        for (int a = 0; a < 3; ++a) {
            if (pos) pos[3 * q + a] = x[a];
            if (vel) vel[3 * q + a] = v[a];
        }
        for (int a = 0; a < 9; ++a) {
            if (F) F[9 * q + a] = p.F.m[a / 3][a % 3];
            if (C) C[9 * q + a] = p.C.m[a / 3][a % 3];
        }
        ++q;
    }
}

ORC_EXPORT void ref_get_particles(void* h, float* pos, float* vel, float* F, float* C, float* mass, float* vol) {
    int64_t q = 0;
    for (const auto& p : sv(h)->get_particles()) {
        if (pos) { pos[3 * q] = p.position.x; pos[3 * q + 1] = p.position.y; pos[3 * q + 2] = p.position.z; }
        if (vel) { vel[3 * q] = p.velocity.x; vel[3 * q + 1] = p.velocity.y; vel[3 * q + 2] = p.velocity.z; }
        for (int a = 0; a < 9; ++a) {
            if (F) F[9 * q + a] = p.F.m[a / 3][a % 3];
            if (C) C[9 * q + a] = p.C.m[a / 3][a % 3];
        }
        if (mass) mass[q] = p.mass;
        if (vol) vol[q] = p.volume;
        ++q;
    }
}

ORC_EXPORT void ref_step(void* h, float dt, int n_steps) {
    for (int i = 0; i < n_steps; ++i) sv(h)->step(dt);
}
ORC_EXPORT void ref_p2g(void* h, float dt) {
    MPMSolver* s = sv(h);
    s->grid.clear();
    for (auto& p : s->particles) s->p2g_single(p, dt);
}
ORC_EXPORT void ref_grid_update(void* h, float dt) { sv(h)->update_grid(dt); }
ORC_EXPORT void ref_g2p(void* h, float dt) {
    MPMSolver* s = sv(h);
    for (auto& p : s->particles) s->g2p_single(p, dt);
}

ORC_EXPORT int ref_m1_apply(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    cp::CouplingReaction r = cp::MPMRigidCouplerPIC::apply(sv(h)->get_grid_mutable(), to_state(body), dt);
    reaction6[0] = r.force.x; reaction6[1] = r.force.y; reaction6[2] = r.force.z;
    reaction6[3] = r.torque.x; reaction6[4] = r.torque.y; reaction6[5] = r.torque.z;
    return r.nodes_inside;
}

ORC_EXPORT int ref_m0_apply(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    cp::CouplingReaction r = cp::MPMRigidCoupler::apply(sv(h)->get_grid_mutable(), to_state(body), dt);
    reaction6[0] = r.force.x; reaction6[1] = r.force.y; reaction6[2] = r.force.z;
    reaction6[3] = r.torque.x; reaction6[4] = r.torque.y; reaction6[5] = r.torque.z;
    return r.nodes_inside;
}

template <class Coupler>
static int coupler_export(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    cp::CouplingReaction r = Coupler::apply(sv(h)->get_grid_mutable(), to_state(body), dt);
    reaction6[0] = r.force.x; reaction6[1] = r.force.y; reaction6[2] = r.force.z;
    reaction6[3] = r.torque.x; reaction6[4] = r.torque.y; reaction6[5] = r.torque.z;
    return r.nodes_inside;
}
ORC_EXPORT int ref_m45b_apply(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    return coupler_export<research::mpm_rigid::M4_5b>(h, body, dt, reaction6);
}
ORC_EXPORT int ref_m45c_apply(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    return coupler_export<research::mpm_rigid::M4_5c>(h, body, dt, reaction6);
}

ORC_EXPORT int ref_m45a_apply(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    cp::CouplingReaction r = research::mpm_rigid::M4_5a::apply(sv(h)->get_grid_mutable(), to_state(body), dt);
    reaction6[0] = r.force.x; reaction6[1] = r.force.y; reaction6[2] = r.force.z;
    reaction6[3] = r.torque.x; reaction6[4] = r.torque.y; reaction6[5] = r.torque.z;
    return r.nodes_inside;
}

ORC_EXPORT int64_t ref_grid_num_nodes(void* h) { return (int64_t)sv(h)->get_grid().get_blocks().size() * 64; }

ORC_EXPORT int64_t ref_grid_get(void* h, int32_t* ijk, float* vel, float* force, float* mass, uint8_t* active,
                                int64_t cap) {
    int64_t q = 0;
    for (const auto& kv : sv(h)->get_grid().get_blocks()) {
        const mpm::GridBlock& b = kv.second;
        for (int i = 0; i < 64 && q < cap; ++i, ++q) {
            const mpm::GridNode& n = b.nodes[i];
            if (ijk) { ijk[3 * q] = b.origin_x + (i >> 4); ijk[3 * q + 1] = b.origin_y + ((i >> 2) & 3); ijk[3 * q + 2] = b.origin_z + (i & 3); }
            if (vel) { vel[3 * q] = n.velocity.x; vel[3 * q + 1] = n.velocity.y; vel[3 * q + 2] = n.velocity.z; }
            if (force) { force[3 * q] = n.force.x; force[3 * q + 1] = n.force.y; force[3 * q + 2] = n.force.z; }
            if (mass) mass[q] = n.mass;
            if (active) active[q] = n.active ? 1 : 0;
        }
    }
    return q;
}

ORC_EXPORT void ref_grid_seed(void* h, int64_t n, const int32_t* ijk, const float* vel, const float* mass) {
    for (int64_t q = 0; q < n; ++q) {
        mpm::GridNode* nd = sv(h)->get_grid_mutable().get_node(ijk[3 * q], ijk[3 * q + 1], ijk[3 * q + 2]);
        nd->active = true;
        nd->mass = mass[q];
        nd->velocity = Vec3(vel[3 * q], vel[3 * q + 1], vel[3 * q + 2]);
    }
}

// Runs the reference's box_drop scene objects (ScenarioBoxDrop, seed_sand,
// make_box) through MPMRigidCouplerPIC and TimeIntegrator in the order of the
// research harness loop, recording the columns of box_drop_M1.csv.
ORC_EXPORT int ref_box_drop_m1(float* rows, int max_rows) {
    namespace rm = research::mpm_rigid;
    rm::ScenarioBoxDrop S;
    mpm::SPGridCPU grid(S.dx);
    rm::seed_sand(grid, S);
    physics::RigidBody box = rm::make_box(S);
    const int N = S.num_steps();
    int r_out = 0;
    for (int i = 0; i < N; ++i) {
        box.apply_force(Vec3(0.0f, -S.gravity_g * box.mass, 0.0f));
        cp::RigidColliderState col;
        col.center = box.position;
        col.orientation = box.orientation;
        col.half_extents = S.box_half_extents;
        col.linear_velocity = box.linear_velocity;
        col.angular_velocity = box.angular_velocity;
        col.friction = 0.5f;
        col.mass = box.mass;
        cp::CouplingReaction r = cp::MPMRigidCouplerPIC::apply(grid, col, S.dt);
        box.force += r.force;
        box.torque += r.torque;
        dynamics::TimeIntegrator::integrate(&box, 1, S.dt);
        for (auto& kv : grid.get_blocks_mutable())
            for (auto& nn : kv.second.nodes) {
                if (!nn.active || nn.mass <= 0.0f) continue;
                nn.velocity.y += -S.gravity_g * S.dt;
                if (nn.velocity.y < 0.0f) nn.velocity.y = 0.0f;
            }
        Vec3 pg = Vec3::zero();
        for (const auto& kv : grid.get_blocks())
            for (const auto& nn : kv.second.nodes)
                if (nn.active) pg += nn.velocity * nn.mass;
        const Vec3 pb = box.linear_velocity * box.mass;
        if (r_out < max_rows) {
            float* row = rows + 10 * r_out;
            row[0] = (i + 1) * S.dt;
            row[1] = box.position.x; row[2] = box.position.y; row[3] = box.position.z;
            row[4] = box.linear_velocity.y; row[5] = pb.y; row[6] = pg.y; row[7] = (pb + pg).y;
            row[8] = 0.5f * box.mass * box.linear_velocity.length_squared();
            row[9] = (float)r.nodes_inside;
            ++r_out;
        }
    }
    return r_out;
}

ORC_EXPORT void ref_run_dynamic_body(void* h, orc_collider_t* body, float gx, float gy, float gz, float dt,
                                     int n_steps, const float* inv_inertia) {
    MPMSolver* s = sv(h);
    physics::RigidBody rb;
    rb.make_dynamic(body->mass);
    if (inv_inertia)
        rb.inv_inertia_tensor = math::Matrix3(inv_inertia[0], inv_inertia[1], inv_inertia[2], inv_inertia[3],
                                              inv_inertia[4], inv_inertia[5], inv_inertia[6], inv_inertia[7],
                                              inv_inertia[8]);
    rb.position = Vec3(body->center[0], body->center[1], body->center[2]);
    rb.orientation = math::Quaternion(body->orientation[0], body->orientation[1], body->orientation[2],
                                      body->orientation[3]);
    rb.linear_velocity = Vec3(body->linear_velocity[0], body->linear_velocity[1], body->linear_velocity[2]);
    rb.angular_velocity = Vec3(body->angular_velocity[0], body->angular_velocity[1], body->angular_velocity[2]);
    rb.linear_damping = 0.0f;
    rb.angular_damping = 0.0f;
    for (int i = 0; i < n_steps; ++i) {
        s->grid.clear();
        for (auto& p : s->particles) s->p2g_single(p, dt);
        s->update_grid(dt);
        rb.apply_force(Vec3(gx * rb.mass, gy * rb.mass, gz * rb.mass));
        orc_collider_t c = *body;
        c.center[0] = rb.position.x; c.center[1] = rb.position.y; c.center[2] = rb.position.z;
        c.orientation[0] = rb.orientation.w; c.orientation[1] = rb.orientation.x;
        c.orientation[2] = rb.orientation.y; c.orientation[3] = rb.orientation.z;
        c.linear_velocity[0] = rb.linear_velocity.x; c.linear_velocity[1] = rb.linear_velocity.y;
        c.linear_velocity[2] = rb.linear_velocity.z;
        c.angular_velocity[0] = rb.angular_velocity.x; c.angular_velocity[1] = rb.angular_velocity.y;
        c.angular_velocity[2] = rb.angular_velocity.z;
        cp::CouplingReaction r = cp::MPMRigidCouplerPIC::apply(s->grid, to_state(&c), dt);
        rb.force += r.force;
        rb.torque += r.torque;
        dynamics::TimeIntegrator::integrate(&rb, 1, dt);
        for (auto& p : s->particles) s->g2p_single(p, dt);
    }
    body->center[0] = rb.position.x; body->center[1] = rb.position.y; body->center[2] = rb.position.z;
    body->orientation[0] = rb.orientation.w; body->orientation[1] = rb.orientation.x;
    body->orientation[2] = rb.orientation.y; body->orientation[3] = rb.orientation.z;
    body->linear_velocity[0] = rb.linear_velocity.x; body->linear_velocity[1] = rb.linear_velocity.y;
    body->linear_velocity[2] = rb.linear_velocity.z;
    body->angular_velocity[0] = rb.angular_velocity.x; body->angular_velocity[1] = rb.angular_velocity.y;
    body->angular_velocity[2] = rb.angular_velocity.z;
}

ORC_EXPORT void ref_svd(int64_t n, const float* F, float* U, float* Sg, float* V) {
    for (int64_t q = 0; q < n; ++q) {
        Matrix3 f, u, v;
        Vec3 s;
        for (int a = 0; a < 9; ++a) f.m[a / 3][a % 3] = F[9 * q + a];
        math::SVD::compute(f, u, s, v);
        for (int a = 0; a < 9; ++a) {
            U[9 * q + a] = u.m[a / 3][a % 3];
            V[9 * q + a] = v.m[a / 3][a % 3];
        }
        Sg[3 * q] = s.x; Sg[3 * q + 1] = s.y; Sg[3 * q + 2] = s.z;
    }
}
