// oracle_capi.cpp — C interface over the restatement in mpm_oracle.hpp.
//
// TEST INFRASTRUCTURE ONLY: built twice by oracle/Makefile, with
// -DORACLE_REAL=float (liboracle_mpm_f32.so) and -DORACLE_REAL=double
// (liboracle_mpm_f64.so), both exporting the orc_* names of oracle_api.h.
// The box_drop loop restates the reference research harness
// (research/mpm_rigid_coupling/bench_compare_all.cpp:72-208 with
// scenarios/scenario_box_drop.h:14-80) and the rigid update
// (include/basements/physics/dynamics/integrator.h:19-57).
#define ORACLE_PREFIX orc
#include "oracle_api.h"
#include "mpm_oracle.hpp"

#include <cstring>

#ifndef ORACLE_REAL
#define ORACLE_REAL float
#endif

using R = ORACLE_REAL;
using namespace bm_oracle;
using S = Solver<R>;

static S* sv(void* h) { return static_cast<S*>(h); }

static ColliderF to_collider(const orc_collider_t* b) {
    ColliderF c;
    for (int i = 0; i < 3; ++i) {
        c.center[i] = b->center[i];
        c.half_extents[i] = b->half_extents[i];
        c.linear_velocity[i] = b->linear_velocity[i];
        c.angular_velocity[i] = b->angular_velocity[i];
    }
    for (int i = 0; i < 4; ++i) c.orientation[i] = b->orientation[i];
    c.friction = b->friction;
    c.mass = b->mass;
    c.shape = b->shape;
    return c;
}

ORC_EXPORT int orc_precision_bytes(void) { return (int)sizeof(R); }
ORC_EXPORT void* orc_create(float dx) {
    S* s = new S();
    s->initialize((R)dx);
    return s;
}
ORC_EXPORT void orc_destroy(void* h) { delete sv(h); }
ORC_EXPORT void orc_set_material(void* h, float E, float nu, float rho) { sv(h)->set_material(E, nu, rho); }
ORC_EXPORT void orc_set_gravity(void* h, float gx, float gy, float gz) { sv(h)->gravity = V3<R>(gx, gy, gz); }
ORC_EXPORT void orc_set_plastic_alpha(void* h, float a) { sv(h)->alpha = a; }
ORC_EXPORT void orc_set_floor_friction(void* h, float mu) { sv(h)->floor_friction = mu; }

ORC_EXPORT void orc_add_particles(void* h, int64_t n, const float* pos, const float* vel, const float* mass) {
    S* s = sv(h);
    for (int64_t p = 0; p < n; ++p) {
        V3<R> x(pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]);
        V3<R> v = vel ? V3<R>(vel[3 * p], vel[3 * p + 1], vel[3 * p + 2]) : V3<R>(0, 0, 0);
        s->add_particle(x, v, mass ? (R)mass[p] : R(1));
    }
}
ORC_EXPORT int64_t orc_num_particles(void* h) { return (int64_t)sv(h)->particles.size(); }

ORC_EXPORT void orc_set_particle_state(void* h, int64_t first, int64_t n, const float* pos, const float* vel,
                                       const float* F, const float* C) {
    S* s = sv(h);
    for (int64_t q = 0; q < n; ++q) {
        Particle<R>& p = s->particles[first + q];
        if (pos) p.x = V3<R>(pos[3 * q], pos[3 * q + 1], pos[3 * q + 2]);
        if (vel) p.v = V3<R>(vel[3 * q], vel[3 * q + 1], vel[3 * q + 2]);
        for (int a = 0; a < 9; ++a) {
            if (F) p.F.m[a / 3][a % 3] = F[9 * q + a];
            if (C) p.C.m[a / 3][a % 3] = C[9 * q + a];
        }
    }
}

ORC_EXPORT void orc_set_state_f64(void* h, int64_t first, int64_t n, const double* pos, const double* vel,
                                  const double* F, const double* C) {
    S* s = sv(h);
    for (int64_t q = 0; q < n; ++q) {
        Particle<R>& p = s->particles[first + q];
        if (pos) p.x = V3<R>((R)pos[3 * q], (R)pos[3 * q + 1], (R)pos[3 * q + 2]);
        if (vel) p.v = V3<R>((R)vel[3 * q], (R)vel[3 * q + 1], (R)vel[3 * q + 2]);
        for (int a = 0; a < 9; ++a) {
            if (F) p.F.m[a / 3][a % 3] = (R)F[9 * q + a];
            if (C) p.C.m[a / 3][a % 3] = (R)C[9 * q + a];
        }
    }
}

ORC_EXPORT void orc_get_particles(void* h, float* pos, float* vel, float* F, float* C, float* mass, float* vol) {
    S* s = sv(h);
    int64_t q = 0;
    for (const auto& p : s->particles) {
        if (pos) { pos[3 * q] = (float)p.x.x; pos[3 * q + 1] = (float)p.x.y; pos[3 * q + 2] = (float)p.x.z; }
        if (vel) { vel[3 * q] = (float)p.v.x; vel[3 * q + 1] = (float)p.v.y; vel[3 * q + 2] = (float)p.v.z; }
        for (int a = 0; a < 9; ++a) {
            if (F) F[9 * q + a] = (float)p.F.m[a / 3][a % 3];
            if (C) C[9 * q + a] = (float)p.C.m[a / 3][a % 3];
        }
        if (mass) mass[q] = (float)p.mass;
        if (vol) vol[q] = (float)p.volume;
        ++q;
    }
}

ORC_EXPORT void orc_get_state_f64(void* h, double* pos, double* vel, double* F, double* C) {
    int64_t q = 0;
    for (const auto& p : sv(h)->particles) {
        const double x[3] = {(double)p.x.x, (double)p.x.y, (double)p.x.z};
        const double v[3] = {(double)p.v.x, (double)p.v.y, (double)p.v.z};
        for (int a = 0; a < 3; ++a) {
            if (pos) pos[3 * q + a] = x[a];
            if (vel) vel[3 * q + a] = v[a];
        }
        for (int a = 0; a < 9; ++a) {
            if (F) F[9 * q + a] = (double)p.F.m[a / 3][a % 3];
            if (C) C[9 * q + a] = (double)p.C.m[a / 3][a % 3];
        }
        ++q;
    }
}

ORC_EXPORT void orc_step(void* h, float dt, int n_steps) {
    for (int i = 0; i < n_steps; ++i) sv(h)->step(dt);
}
ORC_EXPORT void orc_p2g(void* h, float dt) { sv(h)->p2g(dt); }
ORC_EXPORT void orc_grid_update(void* h, float dt) { sv(h)->update_grid(dt); }
ORC_EXPORT void orc_g2p(void* h, float dt) { sv(h)->g2p(dt); }

ORC_EXPORT void orc_decisions_enable(void* h, int on) {
    S* s = sv(h);
    DecisionTape* keep = s->log_store.tape;
    s->log_store = DecisionLog();
    s->log_store.tape = keep;
    s->log = (on || keep) ? &s->log_store : nullptr;
}

ORC_EXPORT void* orc_tape_new(void) { return new DecisionTape(); }
ORC_EXPORT void orc_tape_free(void* t) { delete static_cast<DecisionTape*>(t); }
ORC_EXPORT void orc_solver_use_tape(void* h, void* t, int mode) {
    S* s = sv(h);
    DecisionTape* T = static_cast<DecisionTape*>(t);
    if (!T || mode == 0) {
        s->log_store.tape = nullptr;
        return;
    }
    T->replay = mode == 2;
    T->svd_pos = T->inside_pos = 0;
    T->overrun = false;
    if (mode == 1) {
        T->svd.clear();
        T->inside.clear();
    }
    s->log_store.tape = T;
    s->log = &s->log_store;
}
// Copies of a tape's content, so that a tape recorded by one checker (the
// float restatement) can be replayed by another (the double one): the SVD
// codes, the inside sets flattened with their offsets (inside.size() + 1).
// Pass NULL arrays to read the sizes first.
ORC_EXPORT void orc_tape_export(void* t, uint16_t* svd, int64_t* keys, int64_t* offsets, int64_t* sizes3) {
    const DecisionTape* T = static_cast<const DecisionTape*>(t);
    int64_t nk = 0;
    for (const auto& v : T->inside) nk += (int64_t)v.size();
    sizes3[0] = (int64_t)T->svd.size();
    sizes3[1] = (int64_t)T->inside.size();
    sizes3[2] = nk;
    if (svd) std::memcpy(svd, T->svd.data(), sizeof(uint16_t) * T->svd.size());
    if (keys && offsets) {
        int64_t o = 0;
        for (size_t c = 0; c < T->inside.size(); ++c) {
            offsets[c] = o;
            for (int64_t k : T->inside[c]) keys[o++] = k;
        }
        offsets[T->inside.size()] = o;
    }
}
ORC_EXPORT void orc_tape_import(void* t, int64_t n_svd, const uint16_t* svd, int64_t n_calls, const int64_t* keys,
                                const int64_t* offsets) {
    DecisionTape* T = static_cast<DecisionTape*>(t);
    T->svd.assign(svd, svd + n_svd);
    T->inside.assign((size_t)n_calls, {});
    for (int64_t c = 0; c < n_calls; ++c) T->inside[c].assign(keys + offsets[c], keys + offsets[c + 1]);
    T->svd_pos = T->inside_pos = 0;
    T->overrun = false;
}

ORC_EXPORT void orc_tape_status(void* t, int64_t* out4) {
    const DecisionTape* T = static_cast<const DecisionTape*>(t);
    out4[0] = (int64_t)T->svd.size();
    out4[1] = (int64_t)T->svd_pos;
    out4[2] = (int64_t)T->inside.size();
    out4[3] = (int64_t)T->inside_pos + (T->overrun ? (int64_t(1) << 40) : 0);
}

ORC_EXPORT void orc_decisions_read(void* h, uint64_t* out5) {
    const DecisionLog& L = sv(h)->log_store;
    out5[0] = L.svd_hash;
    out5[1] = L.inside_hash;
    out5[2] = (uint64_t)L.rotations;
    out5[3] = (uint64_t)L.sweeps;
    out5[4] = (uint64_t)L.inside;
}

ORC_EXPORT int orc_m1_apply(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    Reaction<R> r = m1_apply<R>(sv(h)->grid, to_collider(body), (R)dt, sv(h)->log);
    reaction6[0] = (float)r.force.x; reaction6[1] = (float)r.force.y; reaction6[2] = (float)r.force.z;
    reaction6[3] = (float)r.torque.x; reaction6[4] = (float)r.torque.y; reaction6[5] = (float)r.torque.z;
    return r.nodes_inside;
}

ORC_EXPORT int orc_m0_apply(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    Reaction<R> r = m0_apply<R>(sv(h)->grid, to_collider(body), (R)dt);
    reaction6[0] = (float)r.force.x; reaction6[1] = (float)r.force.y; reaction6[2] = (float)r.force.z;
    reaction6[3] = (float)r.torque.x; reaction6[4] = (float)r.torque.y; reaction6[5] = (float)r.torque.z;
    return r.nodes_inside;
}

static int m45_export(void* h, const orc_collider_t* body, float dt, float* reaction6, int layer) {
    Reaction<R> r = m45_apply<R>(sv(h)->grid, to_collider(body), (R)dt, layer);
    reaction6[0] = (float)r.force.x; reaction6[1] = (float)r.force.y; reaction6[2] = (float)r.force.z;
    reaction6[3] = (float)r.torque.x; reaction6[4] = (float)r.torque.y; reaction6[5] = (float)r.torque.z;
    return r.nodes_inside;
}
ORC_EXPORT int orc_m45b_apply(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    return m45_export(h, body, dt, reaction6, 1);
}
ORC_EXPORT int orc_m45c_apply(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    return m45_export(h, body, dt, reaction6, 2);
}

ORC_EXPORT int orc_m45a_apply(void* h, const orc_collider_t* body, float dt, float* reaction6) {
    Reaction<R> r = m45a_apply<R>(sv(h)->grid, to_collider(body), (R)dt);
    reaction6[0] = (float)r.force.x; reaction6[1] = (float)r.force.y; reaction6[2] = (float)r.force.z;
    reaction6[3] = (float)r.torque.x; reaction6[4] = (float)r.torque.y; reaction6[5] = (float)r.torque.z;
    return r.nodes_inside;
}

ORC_EXPORT int64_t orc_grid_num_nodes(void* h) { return (int64_t)sv(h)->grid.blocks.size() * 64; }

ORC_EXPORT int64_t orc_grid_get(void* h, int32_t* ijk, float* vel, float* force, float* mass, uint8_t* active,
                                int64_t cap) {
    int64_t q = 0;
    for (const auto& kv : sv(h)->grid.blocks) {
        const Block<R>& b = kv.second;
        for (int i = 0; i < 64 && q < cap; ++i, ++q) {
            const Node<R>& n = b.n[i];
            if (ijk) { ijk[3 * q] = b.ox + (i >> 4); ijk[3 * q + 1] = b.oy + ((i >> 2) & 3); ijk[3 * q + 2] = b.oz + (i & 3); }
            if (vel) { vel[3 * q] = (float)n.v.x; vel[3 * q + 1] = (float)n.v.y; vel[3 * q + 2] = (float)n.v.z; }
            if (force) { force[3 * q] = (float)n.f.x; force[3 * q + 1] = (float)n.f.y; force[3 * q + 2] = (float)n.f.z; }
            if (mass) mass[q] = (float)n.m;
            if (active) active[q] = n.active ? 1 : 0;
        }
    }
    return q;
}

ORC_EXPORT void orc_grid_seed(void* h, int64_t n, const int32_t* ijk, const float* vel, const float* mass) {
    S* s = sv(h);
    for (int64_t q = 0; q < n; ++q) {
        Node<R>* nd = s->grid.node(ijk[3 * q], ijk[3 * q + 1], ijk[3 * q + 2]);
        nd->active = true;
        nd->m = mass[q];
        nd->v = V3<R>(vel[3 * q], vel[3 * q + 1], vel[3 * q + 2]);
    }
}

// Quaternion helpers for the rigid update (quaternion.h: Hamilton product,
// normalized() = q * (1/|q|) unless |q| < 1e-6).
struct Q4 { R w, x, y, z; };
static Q4 qmul(const Q4& a, const Q4& b) {
    return Q4{((a.w * b.w - a.x * b.x) - a.y * b.y) - a.z * b.z,
              ((a.w * b.x + a.x * b.w) + a.y * b.z) - a.z * b.y,
              ((a.w * b.y - a.x * b.z) + a.y * b.w) + a.z * b.x,
              ((a.w * b.z + a.x * b.y) - a.y * b.x) + a.z * b.w};
}
static Q4 qnormalize(const Q4& q) {
    const R n = std::sqrt(((q.w * q.w + q.x * q.x) + q.y * q.y) + q.z * q.z);
    if (n < R(1e-6f)) return Q4{1, 0, 0, 0};
    const R inv = R(1) / n;
    return Q4{q.w * inv, q.x * inv, q.y * inv, q.z * inv};
}

ORC_EXPORT int orc_box_drop_m1(float* rows, int max_rows) {
    const R dx = R(0.1f), dt = R(1.0f / 240.0f), g = R(9.81f), mass = R(1.0f);
    const int n_steps = (int)(3.0f / (1.0f / 240.0f) + 0.5f);
    Grid<R> grid(dx);
    for (int i = -3; i <= 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = -3; k <= 3; ++k) {
                Node<R>* n = grid.node(i, j, k);
                n->active = true; n->m = R(0.01f); n->v = V3<R>(0, 0, 0);
            }
    V3<R> pos(0, R(0.55f), 0), vel(0, 0, 0), omg(0, 0, 0), force(0, 0, 0), torque(0, 0, 0);
    Q4 q{1, 0, 0, 0};
    const R inv_mass = R(1) / mass;
    int r_out = 0;
    for (int i = 0; i < n_steps; ++i) {
        force += V3<R>(R(0), -g * mass, R(0));
        ColliderF col;
        col.center[0] = (float)pos.x; col.center[1] = (float)pos.y; col.center[2] = (float)pos.z;
        col.orientation[0] = (float)q.w; col.orientation[1] = (float)q.x;
        col.orientation[2] = (float)q.y; col.orientation[3] = (float)q.z;
        col.half_extents[0] = col.half_extents[1] = col.half_extents[2] = 0.2f;
        col.linear_velocity[0] = (float)vel.x; col.linear_velocity[1] = (float)vel.y; col.linear_velocity[2] = (float)vel.z;
        col.angular_velocity[0] = (float)omg.x; col.angular_velocity[1] = (float)omg.y; col.angular_velocity[2] = (float)omg.z;
        col.friction = 0.5f; col.mass = (float)mass; col.shape = 0;
        Reaction<R> r = m1_apply<R>(grid, col, dt);
        force += r.force;
        torque += r.torque;
        // integrator.h:19-57 with zero damping and identity body-space inverse inertia.
        vel += force * inv_mass * dt;
        omg += (M3<R>::identity() * torque) * dt;
        vel = vel * (R(1) - R(0) * dt);
        omg = omg * (R(1) - R(0) * dt);
        pos += vel * dt;
        Q4 qv{0, omg.x, omg.y, omg.z};
        Q4 dq = qmul(qv, q);
        const R h = R(0.5f) * dt;
        q = Q4{q.w + dq.w * h, q.x + dq.x * h, q.y + dq.y * h, q.z + dq.z * h};
        q = qnormalize(q);
        force = V3<R>(0, 0, 0);
        torque = V3<R>(0, 0, 0);
        // Harness grid step: gravity on the grid and clamp v_y >= 0.
        for (auto& kv : grid.blocks)
            for (auto& n : kv.second.n) {
                if (!n.active || n.m <= R(0)) continue;
                n.v.y += -g * dt;
                if (n.v.y < R(0)) n.v.y = 0;
            }
        V3<R> pg(0, 0, 0);
        for (auto& kv : grid.blocks)
            for (auto& n : kv.second.n)
                if (n.active) pg += n.v * n.m;
        const V3<R> pb = vel * mass;
        if (r_out < max_rows) {
            float* row = rows + 10 * r_out;
            row[0] = (float)((R)(i + 1) * dt);
            row[1] = (float)pos.x; row[2] = (float)pos.y; row[3] = (float)pos.z;
            row[4] = (float)vel.y; row[5] = (float)pb.y; row[6] = (float)pg.y;
            row[7] = (float)(pb + pg).y;
            row[8] = (float)(R(0.5f) * mass * vel.dot(vel));
            row[9] = (float)r.nodes_inside;
            ++r_out;
        }
    }
    return r_out;
}

ORC_EXPORT void orc_run_dynamic_body(void* h, orc_collider_t* body, float gx, float gy, float gz, float dt,
                                     int n_steps, const float* inv_inertia) {
    S* s = sv(h);
    // integrator.h:34 applies the body-space inverse inertia to the torque as
    // it is (rigid_body.h:121-122: the identity unless set)
    M3<R> inv_i = M3<R>::identity();
    if (inv_inertia)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) inv_i.m[i][j] = (R)inv_inertia[3 * i + j];
    V3<R> pos(body->center[0], body->center[1], body->center[2]);
    V3<R> vel(body->linear_velocity[0], body->linear_velocity[1], body->linear_velocity[2]);
    V3<R> omg(body->angular_velocity[0], body->angular_velocity[1], body->angular_velocity[2]);
    Q4 q{body->orientation[0], body->orientation[1], body->orientation[2], body->orientation[3]};
    const R mass = body->mass, inv_mass = mass > R(0) ? R(1) / mass : R(0);
    for (int i = 0; i < n_steps; ++i) {
        s->p2g((R)dt);
        s->update_grid((R)dt);
        V3<R> force = V3<R>(0, 0, 0) + V3<R>((R)gx * mass, (R)gy * mass, (R)gz * mass);
        ColliderF c = to_collider(body);
        c.center[0] = (float)pos.x; c.center[1] = (float)pos.y; c.center[2] = (float)pos.z;
        c.orientation[0] = (float)q.w; c.orientation[1] = (float)q.x; c.orientation[2] = (float)q.y;
        c.orientation[3] = (float)q.z;
        c.linear_velocity[0] = (float)vel.x; c.linear_velocity[1] = (float)vel.y; c.linear_velocity[2] = (float)vel.z;
        c.angular_velocity[0] = (float)omg.x; c.angular_velocity[1] = (float)omg.y; c.angular_velocity[2] = (float)omg.z;
        Reaction<R> r = m1_apply<R>(s->grid, c, (R)dt);
        force += r.force;
        V3<R> torque = V3<R>(0, 0, 0) + r.torque;
        vel += force * inv_mass * (R)dt;
        omg += (inv_i * torque) * (R)dt;
        pos += vel * (R)dt;
        Q4 qv{0, omg.x, omg.y, omg.z};
        Q4 dq = qmul(qv, q);
        const R hh = R(0.5f) * (R)dt;
        q = qnormalize(Q4{q.w + dq.w * hh, q.x + dq.x * hh, q.y + dq.y * hh, q.z + dq.z * hh});
        s->g2p((R)dt);
    }
    body->center[0] = (float)pos.x; body->center[1] = (float)pos.y; body->center[2] = (float)pos.z;
    body->orientation[0] = (float)q.w; body->orientation[1] = (float)q.x; body->orientation[2] = (float)q.y;
    body->orientation[3] = (float)q.z;
    body->linear_velocity[0] = (float)vel.x; body->linear_velocity[1] = (float)vel.y;
    body->linear_velocity[2] = (float)vel.z;
    body->angular_velocity[0] = (float)omg.x; body->angular_velocity[1] = (float)omg.y;
    body->angular_velocity[2] = (float)omg.z;
}

ORC_EXPORT void orc_svd(int64_t n, const float* F, float* U, float* Sg, float* V) {
    for (int64_t q = 0; q < n; ++q) {
        M3<R> f, u, v;
        V3<R> s;
        for (int a = 0; a < 9; ++a) f.m[a / 3][a % 3] = F[9 * q + a];
        svd3(f, u, s, v);
        for (int a = 0; a < 9; ++a) {
            U[9 * q + a] = (float)u.m[a / 3][a % 3];
            V[9 * q + a] = (float)v.m[a / 3][a % 3];
        }
        Sg[3 * q] = (float)s.x; Sg[3 * q + 1] = (float)s.y; Sg[3 * q + 2] = (float)s.z;
    }
}
