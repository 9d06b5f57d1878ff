// mpm_oracle.hpp — CPU restatement of the reference MLS-MPM soil step.
//
// TEST INFRASTRUCTURE ONLY. This header is the checker for the CUDA product
// in basements_b200/: only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load it (through oracle/liboracle_mpm_f32.so and
// oracle/liboracle_mpm_f64.so). The product never calls, links or falls back
// to it.
//
// It restates, templated on the arithmetic type R (float or double), the
// reference's algorithm in the same order of operations, so that R=float
// reproduces the reference bit for bit when built with the reference's flags
// (g++ -O2 -mavx2, no FMA contraction), and R=double is the FP64 run.
// Citations are file:line inside 2nugu/basements:
//
//   include/basements/physics/mpm/mpm_solver.h
//       :19-34    initialize / add_particle (V0 = m / rho)
//       :42-54    set_material (V0 rescale), setters
//       :62-87    step = clear, P2G loop, update_grid, G2P loop
//       :100-112  defaults and Lame parameters
//       :114-166  apply_plasticity (Drucker-Prager return map)
//       :168-248  p2g_single (quadratic B-spline, Hencky-Kirchhoff stress)
//       :250-291  update_grid (gravity, floor BC with Coulomb friction)
//       :293-348  g2p_single (APIC gather, advection, plasticity, floor clamp)
//   include/basements/physics/mpm/spgrid_cpu.h:40-125  sparse 4^3-block grid
//   include/basements/core/math/svd.h:18-108          Jacobi SVD on F^T F
//   include/basements/core/math/vec3.h:41-101,162-182  Vec3 ops (AVX branch)
//   include/basements/core/math/matrix3.h:177-251,405-447  Matrix3 ops
//   include/basements/physics/coupling/mpm_rigid_coupler.h:90-103  shape_inside
//   include/basements/physics/coupling/mpm_rigid_coupler_pic.h:88-184  M1
//   include/basements/physics/coupling/mpm_rigid_coupler.h:139-200  overlap
//       fraction and tight world AABB of a shape
//   research/mpm_rigid_coupling/couplers/m4_5_hybrid.h:104-305  M4.5a/b/c
//   include/basements/physics/coupling/mpm_rigid_coupler.h:106-132  outward normal
//   src/physics/coupling/mpm_rigid_coupler.cpp:58-143  M0 (Dirichlet)
//   include/basements/physics/dynamics/integrator.h:19-57  rigid update
//
// Thresholds are the reference's float literals, converted to R, so both
// instantiations branch on the same values.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

namespace bm_oracle {

template <class R> struct V3 {
    R x = 0, y = 0, z = 0;
    V3() = default;
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    explicit V3(R s) : x(s), y(s), z(s) {}
    V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
    V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
    V3 operator*(R s) const { return V3(x * s, y * s, z * s); }
    // vec3.h:80-101, AVX branch: true per-component division, zero below 1e-6.
    V3 operator/(R s) const {
        if (std::abs(s) < R(1e-6f)) return V3(R(0));
        return V3(x / s, y / s, z / s);
    }
    V3& operator+=(const V3& o) { *this = *this + o; return *this; }
    R dot(const V3& o) const { return (x * o.x + y * o.y) + z * o.z; }
    V3 cross(const V3& o) const {
        return V3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x);
    }
    R length() const { return std::sqrt(dot(*this)); }
};

template <class R> struct M3 {
    R m[3][3];
    static M3 identity() { M3 a; a.set(1, 0, 0, 0, 1, 0, 0, 0, 1); return a; }
    static M3 zero() { M3 a; a.set(0, 0, 0, 0, 0, 0, 0, 0, 0); return a; }
    static M3 diag(const V3<R>& s) { M3 a; a.set(s.x, 0, 0, 0, s.y, 0, 0, 0, s.z); return a; }
    void set(R a, R b, R c, R d, R e, R f, R g, R h, R i) {
        m[0][0] = a; m[0][1] = b; m[0][2] = c;
        m[1][0] = d; m[1][1] = e; m[1][2] = f;
        m[2][0] = g; m[2][1] = h; m[2][2] = i;
    }
    M3 operator+(const M3& o) const {
        M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = m[i][j] + o.m[i][j];
        return r;
    }
    M3 operator*(R s) const {
        M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = m[i][j] * s;
        return r;
    }
    M3 operator*(const M3& o) const {
        M3 r;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                r.m[i][j] = (m[i][0] * o.m[0][j] + m[i][1] * o.m[1][j]) + m[i][2] * o.m[2][j];
        return r;
    }
    V3<R> operator*(const V3<R>& v) const {
        return V3<R>((m[0][0] * v.x + m[0][1] * v.y) + m[0][2] * v.z,
                     (m[1][0] * v.x + m[1][1] * v.y) + m[1][2] * v.z,
                     (m[2][0] * v.x + m[2][1] * v.y) + m[2][2] * v.z);
    }
    M3 T() const {
        M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = m[j][i];
        return r;
    }
    static M3 outer(const V3<R>& a, const V3<R>& b) {
        M3 r;
        r.set(a.x * b.x, a.x * b.y, a.x * b.z,
              a.y * b.x, a.y * b.y, a.y * b.z,
              a.z * b.x, a.z * b.y, a.z * b.z);
        return r;
    }
    // matrix3.h:432-447, quaternion (w, x, y, z) to rotation matrix.
    static M3 from_quat(R w, R x, R y, R z) {
        const R xx = x * x, yy = y * y, zz = z * z;
        const R xy = x * y, xz = x * z, yz = y * z;
        const R wx = w * x, wy = w * y, wz = w * z;
        M3 r;
        r.set(R(1) - R(2) * (yy + zz), R(2) * (xy - wz), R(2) * (xz + wy),
              R(2) * (xy + wz), R(1) - R(2) * (xx + zz), R(2) * (yz - wx),
              R(2) * (xz - wy), R(2) * (yz + wx), R(1) - R(2) * (xx + yy));
        return r;
    }
};

// Record of the discontinuous decisions of a run, for the finite-difference
// checks of the adjoint: a central difference is only a derivative of the
// run if its two sides take the same decisions. Covered: the SVD's pair skip
// (|a_ij| < 1e-6) and sweep stop (below 1e-5), and the coupler's inside test
// per node; each is folded into a hash in the order the run makes them (FNV-1a
// steps), with counts beside.
// A DecisionTape holds the decisions themselves, so that a run can record
// them and another run replay them: the two sides of a central difference
// then follow the same branch, and their difference is a derivative of that
// branch. One 16-bit code per SVD call (the skip bit of each pair in the
// order visited; the number of sweeps in bits 12-14, or bit 15 for all five
// sweeps with the 15 skip bits below), and per coupler call the sorted keys of
// the nodes inside.
struct DecisionTape {
    std::vector<uint16_t> svd;
    std::vector<std::vector<int64_t>> inside;
    size_t svd_pos = 0, inside_pos = 0;
    bool replay = false;
    bool overrun = false;  // a replay asked for more decisions than recorded
};

struct DecisionLog {
    uint64_t svd_hash = 14695981039346656037ull, inside_hash = 14695981039346656037ull;
    int64_t rotations = 0, sweeps = 0, inside = 0;
    DecisionTape* tape = nullptr;
    static void mix(uint64_t& h, uint64_t v) { h = (h ^ v) * 1099511628211ull; }
};

// svd.h:18-108. Cyclic Jacobi eigen-solve of A = F^T F: at most 5 sweeps over
// the pairs (0,1),(0,2),(1,2); a pair is skipped when |a_ij| < 1e-6; the sweep
// loop stops once the largest off-diagonal seen in a sweep is below 1e-5.
// sigma_k = sqrt(max(0, A_kk)), U_k = (F V)_k / sigma_k or the unit axis when
// sigma_k <= 1e-6. Singular values are left unsorted, no determinant fix.
template <class R>
void svd3(const M3<R>& F, M3<R>& U, V3<R>& S, M3<R>& V, DecisionLog* L = nullptr) {
    M3<R> A = F.T() * F;
    V = M3<R>::identity();
    DecisionTape* T = L ? L->tape : nullptr;
    uint16_t code = 0;
    int rep_sweeps = 0;
    if (T && T->replay) {
        if (T->svd_pos < T->svd.size()) code = T->svd[T->svd_pos++];
        else T->overrun = true;
        rep_sweeps = (code & 0x8000u) ? 5 : ((code >> 12) & 7);
    }
    int bit = 0, done = 0;
    for (int sweep = 0; sweep < 5; ++sweep) {
        R max_off = 0;
        for (int i = 0; i < 2; ++i) {
            for (int j = i + 1; j < 3; ++j) {
                const R a_ij = A.m[i][j], a_ii = A.m[i][i], a_jj = A.m[j][j];
                max_off = std::max(max_off, std::abs(a_ij));
                const bool skip = (T && T->replay) ? ((code >> bit) & 1u) != 0 : std::abs(a_ij) < R(1e-6f);
                if (T && !T->replay && skip) code |= (uint16_t)(1u << bit);
                ++bit;
                if (L) {
                    DecisionLog::mix(L->svd_hash, skip ? 1u : 2u);
                    L->rotations += skip ? 0 : 1;
                }
                if (skip) continue;
                const R tau = (a_jj - a_ii) / (R(2) * a_ij);
                R t;
                if (tau >= R(0)) t = R(1) / (tau + std::sqrt(R(1) + tau * tau));
                else             t = R(-1) / (-tau + std::sqrt(R(1) + tau * tau));
                const R c = R(1) / std::sqrt(R(1) + t * t);
                const R s = c * t;
                const R n_ii = (c * c * a_ii - R(2) * s * c * a_ij) + s * s * a_jj;
                const R n_jj = (s * s * a_ii + R(2) * s * c * a_ij) + c * c * a_jj;
                A.m[i][i] = n_ii; A.m[j][j] = n_jj;
                A.m[i][j] = 0; A.m[j][i] = 0;
                for (int k = 0; k < 3; ++k) {
                    if (k == i || k == j) continue;
                    const R aik = A.m[i][k], ajk = A.m[j][k];
                    A.m[i][k] = c * aik - s * ajk; A.m[k][i] = A.m[i][k];
                    A.m[j][k] = s * aik + c * ajk; A.m[k][j] = A.m[j][k];
                }
                for (int k = 0; k < 3; ++k) {
                    const R vki = V.m[k][i], vkj = V.m[k][j];
                    V.m[k][i] = c * vki - s * vkj;
                    V.m[k][j] = s * vki + c * vkj;
                }
            }
        }
        const bool stop = (T && T->replay) ? sweep + 1 == rep_sweeps : max_off < R(1e-5f);
        if (L) {
            DecisionLog::mix(L->svd_hash, stop ? 3u : 4u);
            L->sweeps += 1;
        }
        done = sweep + 1;
        if (stop) break;
    }
    if (T && !T->replay) {
        if (done == 5) code |= 0x8000u;
        else code |= (uint16_t)(done << 12);
        T->svd.push_back(code);
    }
    const R s0 = std::sqrt(std::max(R(0), A.m[0][0]));
    const R s1 = std::sqrt(std::max(R(0), A.m[1][1]));
    const R s2 = std::sqrt(std::max(R(0), A.m[2][2]));
    S = V3<R>(s0, s1, s2);
    const M3<R> FV = F * V;
    const R sig[3] = {s0, s1, s2};
    for (int c = 0; c < 3; ++c) {
        V3<R> col(FV.m[0][c], FV.m[1][c], FV.m[2][c]);
        V3<R> u;
        if (sig[c] > R(1e-6f)) u = col / sig[c];
        else u = V3<R>(R(c == 0), R(c == 1), R(c == 2));
        U.m[0][c] = u.x; U.m[1][c] = u.y; U.m[2][c] = u.z;
    }
}

template <class R> struct Particle {
    V3<R> x, v;
    M3<R> F = M3<R>::identity();
    M3<R> C = M3<R>::zero();
    R mass = 1, volume = 1;
};

template <class R> struct Node {
    V3<R> v, f;
    R m = 0;
    bool active = false;
};

// Sparse grid of 4^3-node blocks, created on first touch and never freed
// (spgrid_cpu.h:40-125). The block key packs (b + 100000) & 0x1FFFFF per axis
// at bit offsets 0/21/42 like the reference, so that iteration over blocks
// visits them in the same order and float sums come out bit-identical.
template <class R> struct Block {
    Node<R> n[64];
    int ox = 0, oy = 0, oz = 0;
    void clear() { for (auto& q : n) q = Node<R>(); }
};

template <class R> class Grid {
public:
    explicit Grid(R dx_) : dx(dx_), inv_dx(R(1) / dx_) {}
    R dx, inv_dx;
    std::unordered_map<uint64_t, Block<R>> blocks;

    static uint64_t key(int bi, int bj, int bk) {
        return ((uint64_t)(bi + 100000) & 0x1FFFFF) |
               (((uint64_t)(bj + 100000) & 0x1FFFFF) << 21) |
               (((uint64_t)(bk + 100000) & 0x1FFFFF) << 42);
    }
    void clear() { for (auto& kv : blocks) kv.second.clear(); }
    Node<R>* node(int i, int j, int k) {
        const int bi = i >> 2, bj = j >> 2, bk = k >> 2;
        const uint64_t kk = key(bi, bj, bk);
        auto it = blocks.find(kk);
        Block<R>* b;
        if (it != blocks.end()) {
            b = &it->second;
        } else {
            b = &blocks[kk];
            b->ox = bi * 4; b->oy = bj * 4; b->oz = bk * 4;
            b->clear();
        }
        return &b->n[((i & 3) * 16) + ((j & 3) * 4) + (k & 3)];
    }
};

struct ColliderF {  // field meaning of RigidColliderState (mpm_rigid_coupler.h:72-84)
    float center[3], orientation[4], half_extents[3];
    float linear_velocity[3], angular_velocity[3];
    float friction, mass;
    int shape;  // 0 box, 1 cylinder
};

template <class R> struct Reaction {
    V3<R> force, torque;
    int nodes_inside = 0;
};

template <class R> class Solver {
public:
    std::vector<Particle<R>> particles;
    Grid<R> grid{R(0.1f)};
    V3<R> gravity{R(0), R(-9.81f), R(0)};
    R alpha = R(0.40f), E = R(1.0e5f), nu = R(0.3f), density = R(1500.0f);
    R floor_friction = R(0.4f);
    DecisionLog* log = nullptr;  // records the SVD decisions of the steps when set
    DecisionLog log_store;

    void initialize(R dx) { grid = Grid<R>(dx); }
    R mu_lame() const { return E / (R(2) * (R(1) + nu)); }
    R lambda_lame() const { return E * nu / ((R(1) + nu) * (R(1) - R(2) * nu)); }

    void add_particle(const V3<R>& x, const V3<R>& v, R mass) {
        Particle<R> p;
        p.x = x; p.v = v; p.mass = mass;
        p.volume = (density > R(1e-12f)) ? (mass / density) : R(1);
        particles.push_back(p);
    }
    void set_material(R e, R n, R rho) {
        E = e; nu = n;
        if (rho > R(1e-12f) && density > R(1e-12f) && rho != density && !particles.empty()) {
            const R rescale = density / rho;
            for (auto& p : particles) p.volume *= rescale;
        }
        density = rho;
    }

    void step(R dt) {
        p2g(dt);
        update_grid(dt);
        g2p(dt);
    }
    void p2g(R dt) {
        grid.clear();
        for (auto& p : particles) p2g_single(p, dt);
    }
    void g2p(R dt) {
        for (auto& p : particles) g2p_single(p, dt);
    }

    static void weights(R f, R w[3]) {
        w[0] = R(0.5f) * (R(1) - f) * (R(1) - f);
        w[1] = R(0.75f) - (f - R(0.5f)) * (f - R(0.5f));
        w[2] = R(0.5f) * f * f;
    }

    void apply_plasticity(Particle<R>& p, R dt) {
        const M3<R> Ft = (M3<R>::identity() + p.C * dt) * p.F;
        M3<R> U, V;
        V3<R> sig;
        svd3(Ft, U, sig, V, log);
        sig.x = std::max(sig.x, R(1e-6f));
        sig.y = std::max(sig.y, R(1e-6f));
        sig.z = std::max(sig.z, R(1e-6f));
        V3<R> eps(std::log(sig.x), std::log(sig.y), std::log(sig.z));
        const R tr = (eps.x + eps.y) + eps.z;
        V3<R> eh = eps - V3<R>(tr / R(3));
        const R ehn = eh.length();
        if (tr > R(0)) {
            sig = V3<R>(R(1), R(1), R(1));
        } else {
            const R mu = mu_lame(), la = lambda_lame();
            const R koh = (R(3) * la + R(2) * mu) / (R(2) * mu);
            const R limit = -alpha * koh * tr;
            if (ehn > limit) {
                const R scale = limit / ehn;
                eh = eh * scale;
                eps = eh + V3<R>(tr / R(3));
                sig.x = std::exp(eps.x);
                sig.y = std::exp(eps.y);
                sig.z = std::exp(eps.z);
            }
        }
        p.F = (U * M3<R>::diag(sig)) * V.T();
    }

    void p2g_single(Particle<R>& p, R dt) {
        (void)dt;
        const R inv_dx = grid.inv_dx;
        const R fx = p.x.x * inv_dx - R(0.5f), fy = p.x.y * inv_dx - R(0.5f), fz = p.x.z * inv_dx - R(0.5f);
        const int bx = (int)std::floor(fx), by = (int)std::floor(fy), bz = (int)std::floor(fz);
        R wx[3], wy[3], wz[3];
        weights(fx - bx, wx); weights(fy - by, wy); weights(fz - bz, wz);

        M3<R> U, V;
        V3<R> sg;
        svd3(p.F, U, sg, V, log);
        sg.x = std::max(sg.x, R(1e-6f));
        sg.y = std::max(sg.y, R(1e-6f));
        sg.z = std::max(sg.z, R(1e-6f));
        const R lx = std::log(sg.x), ly = std::log(sg.y), lz = std::log(sg.z);
        const R tr = (lx + ly) + lz;
        const R mu = mu_lame(), la = lambda_lame();
        const V3<R> td(R(2) * mu * lx + la * tr, R(2) * mu * ly + la * tr, R(2) * mu * lz + la * tr);
        const M3<R> tau = (U * M3<R>::diag(td)) * U.T();
        const R ff = R(-4.0f) * inv_dx * inv_dx * p.volume;
        const M3<R> sk = tau * ff;

        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    const R w = wx[i] * wy[j] * wz[k];
                    if (w == R(0)) continue;
                    const int ni = bx + i, nj = by + j, nk = bz + k;
                    const V3<R> d(((R)ni - fx - R(0.5f)) * grid.dx,
                                  ((R)nj - fy - R(0.5f)) * grid.dx,
                                  ((R)nk - fz - R(0.5f)) * grid.dx);
                    const V3<R> aff = p.C * d;
                    Node<R>* n = grid.node(ni, nj, nk);
                    const R mc = w * p.mass;
                    n->m += mc;
                    n->v += (p.v + aff) * mc;
                    n->f += (sk * d) * w;
                    n->active = true;
                }
    }

    void update_grid(R dt) {
        const R dx = grid.dx;
        for (auto& kv : grid.blocks) {
            Block<R>& b = kv.second;
            for (int i = 0; i < 64; ++i) {
                Node<R>& n = b.n[i];
                if (!n.active || n.m <= R(1e-6f)) continue;
                n.v = (n.v + n.f * dt) / n.m;
                n.v += gravity * dt;
                const int ny = b.oy + ((i >> 2) & 3);
                const R node_y = ((R)ny + R(0.5f)) * dx;
                if (node_y < dx && n.v.y < R(0)) {
                    const R vn = -n.v.y;
                    n.v.y = 0;
                    const R tx = n.v.x, tz = n.v.z;
                    const R mag = std::sqrt(tx * tx + tz * tz);
                    const R budget = floor_friction * vn;
                    if (mag > R(1e-12f)) {
                        const R sc = std::max(R(0), (mag - budget) / mag);
                        n.v.x = tx * sc;
                        n.v.z = tz * sc;
                    }
                }
            }
        }
    }

    void g2p_single(Particle<R>& p, R dt) {
        const R inv_dx = grid.inv_dx;
        const R fx = p.x.x * inv_dx - R(0.5f), fy = p.x.y * inv_dx - R(0.5f), fz = p.x.z * inv_dx - R(0.5f);
        const int bx = (int)std::floor(fx), by = (int)std::floor(fy), bz = (int)std::floor(fz);
        R wx[3], wy[3], wz[3];
        weights(fx - bx, wx); weights(fy - by, wy); weights(fz - bz, wz);
        p.v = V3<R>(0, 0, 0);
        p.C = M3<R>::zero();
        const R cscale = R(4.0f) * inv_dx * inv_dx;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    const R w = wx[i] * wy[j] * wz[k];
                    if (w == R(0)) continue;
                    const int ni = bx + i, nj = by + j, nk = bz + k;
                    Node<R>* n = grid.node(ni, nj, nk);
                    const V3<R> d(((R)ni - fx - R(0.5f)) * grid.dx,
                                  ((R)nj - fy - R(0.5f)) * grid.dx,
                                  ((R)nk - fz - R(0.5f)) * grid.dx);
                    const V3<R> wv = n->v * w;
                    p.v += wv;
                    p.C = p.C + M3<R>::outer(wv, d) * cscale;
                }
        p.x += p.v * dt;
        apply_plasticity(p, dt);
        if (p.x.y < R(0)) { p.x.y = 0; p.v.y = 0; }
    }
};

template <class R> bool shape_inside(const ColliderF& b, const V3<R>& l) {
    if (b.shape == 1) {
        const R Rr = (R)b.half_extents[0], L = (R)b.half_extents[1];
        const R r2 = l.x * l.x + l.z * l.z;
        return std::abs(l.y) <= L && r2 <= Rr * Rr;
    }
    return std::abs(l.x) <= (R)b.half_extents[0] && std::abs(l.y) <= (R)b.half_extents[1] &&
           std::abs(l.z) <= (R)b.half_extents[2];
}

// mpm_rigid_coupler_pic.h:88-184 (M1 PIC-rigid). Visits the allocated blocks
// whose node-centre span overlaps the box-formula AABB; nodes inside the shape
// take the mass-weighted average of node and body velocity and gain m_b; the
// reaction sums m_b (v_after - v_body) / dt and its moment about the centre.
template <class R> Reaction<R> m1_apply(Grid<R>& grid, const ColliderF& b, R dt, DecisionLog* L = nullptr) {
    Reaction<R> out;
    if (dt <= R(0)) return out;
    const R dx = grid.dx;
    const M3<R> Rl2w = M3<R>::from_quat(b.orientation[0], b.orientation[1], b.orientation[2], b.orientation[3]);
    const M3<R> Rw2l = Rl2w.T();
    const R hx = b.half_extents[0], hy = b.half_extents[1], hz = b.half_extents[2];
    const R vol = R(8.0f) * hx * hy * hz;
    const int approx = std::max(1, (int)std::round(vol / (dx * dx * dx)));
    const R mb = (R)b.mass / (R)approx;
    const V3<R> ah(std::abs(Rl2w.m[0][0]) * hx + std::abs(Rl2w.m[0][1]) * hy + std::abs(Rl2w.m[0][2]) * hz,
                   std::abs(Rl2w.m[1][0]) * hx + std::abs(Rl2w.m[1][1]) * hy + std::abs(Rl2w.m[1][2]) * hz,
                   std::abs(Rl2w.m[2][0]) * hx + std::abs(Rl2w.m[2][1]) * hy + std::abs(Rl2w.m[2][2]) * hz);
    const V3<R> c(b.center[0], b.center[1], b.center[2]);
    const V3<R> lo = c - ah, hi = c + ah;
    const V3<R> vl(b.linear_velocity[0], b.linear_velocity[1], b.linear_velocity[2]);
    const V3<R> w(b.angular_velocity[0], b.angular_velocity[1], b.angular_velocity[2]);
    // decision tape: the nodes found inside (recording) or to treat as inside
    // (replay) in this call
    std::vector<int64_t> rec_in;
    static const std::vector<int64_t> kNone;
    const std::vector<int64_t>* rep_in = &kNone;
    if (L && L->tape && L->tape->replay) {
        if (L->tape->inside_pos < L->tape->inside.size()) rep_in = &L->tape->inside[L->tape->inside_pos++];
        else L->tape->overrun = true;
    }
    V3<R> fsum, tsum;
    for (auto& kv : grid.blocks) {
        Block<R>& blk = kv.second;
        const V3<R> blo(((R)blk.ox + R(0.5f)) * dx, ((R)blk.oy + R(0.5f)) * dx, ((R)blk.oz + R(0.5f)) * dx);
        const V3<R> bhi(((R)(blk.ox + 3) + R(0.5f)) * dx, ((R)(blk.oy + 3) + R(0.5f)) * dx,
                        ((R)(blk.oz + 3) + R(0.5f)) * dx);
        if (bhi.x < lo.x || blo.x > hi.x) continue;
        if (bhi.y < lo.y || blo.y > hi.y) continue;
        if (bhi.z < lo.z || blo.z > hi.z) continue;
        for (int li = 0; li < 4; ++li)
            for (int lj = 0; lj < 4; ++lj)
                for (int lk = 0; lk < 4; ++lk) {
                    Node<R>& n = blk.n[li * 16 + lj * 4 + lk];
                    const V3<R> xn(((R)(blk.ox + li) + R(0.5f)) * dx, ((R)(blk.oy + lj) + R(0.5f)) * dx,
                                   ((R)(blk.oz + lk) + R(0.5f)) * dx);
                    const V3<R> local = Rw2l * (xn - c);
                    bool in = shape_inside<R>(b, local);
                    if (L && L->tape) {
                        const int64_t key = ((int64_t)(blk.ox + li + (1 << 20)) << 42) |
                                            ((int64_t)(blk.oy + lj + (1 << 20)) << 21) |
                                            (int64_t)(blk.oz + lk + (1 << 20));
                        if (L->tape->replay) in = std::binary_search(rep_in->begin(), rep_in->end(), key);
                        else if (in) rec_in.push_back(key);
                    }
                    if (L) {
                        DecisionLog::mix(L->inside_hash, in ? 5u : 6u);
                        L->inside += in ? 1 : 0;
                    }
                    if (!in) continue;
                    const V3<R> r = xn - c;
                    const V3<R> vb = vl + w.cross(r);
                    V3<R> va;
                    if (!n.active || n.m < R(1e-9f)) {
                        n.active = true; n.m = mb; n.v = vb; va = vb;
                    } else {
                        const V3<R> pold = n.v * n.m;
                        const V3<R> padd = vb * mb;
                        const R mn = n.m + mb;
                        va = (pold + padd) / mn;
                        n.v = va; n.m = mn;
                    }
                    const V3<R> dF = (va - vb) * (mb / dt);
                    fsum += dF;
                    tsum += r.cross(dF);
                    ++out.nodes_inside;
                }
    }
    if (L && L->tape && !L->tape->replay) {
        std::sort(rec_in.begin(), rec_in.end());
        L->tape->inside.push_back(std::move(rec_in));
    }
    out.force = fsum;
    out.torque = tsum;
    return out;
}

// mpm_rigid_coupler.h:106-132: outward normal of the closest face in the
// body frame. Cylinder: the cap (0, +-1, 0) when the axial distance is the
// smaller, else radial (x/r, 0, z/r), or (1, 0, 0) on the axis. Box: the
// axis of the smallest face distance, x before y before z on ties.
template <class R> V3<R> outward_normal_local(const ColliderF& b, const V3<R>& l) {
    if (b.shape == 1) {
        const R Rr = (R)b.half_extents[0], L = (R)b.half_extents[1];
        const R r = std::sqrt(l.x * l.x + l.z * l.z);
        const R axial = L - std::abs(l.y);
        const R radial = Rr - r;
        if (axial < radial) return V3<R>(R(0), l.y >= R(0) ? R(1) : R(-1), R(0));
        if (r > R(1e-9f)) return V3<R>(l.x / r, R(0), l.z / r);
        return V3<R>(R(1), R(0), R(0));
    }
    const R dx = (R)b.half_extents[0] - std::abs(l.x);
    const R dy = (R)b.half_extents[1] - std::abs(l.y);
    const R dz = (R)b.half_extents[2] - std::abs(l.z);
    if (dx <= dy && dx <= dz) return V3<R>(l.x >= R(0) ? R(1) : R(-1), R(0), R(0));
    if (dy <= dz) return V3<R>(R(0), l.y >= R(0) ? R(1) : R(-1), R(0));
    return V3<R>(R(0), R(0), l.z >= R(0) ? R(1) : R(-1));
}

// mpm_rigid_coupler.h:139-164: 1 at the centre, 0 at the surface; box
// (1-|x|/hx)(1-|y|/hy)(1-|z|/hz), cylinder (1-|y|/L)(1-r/R), each clamped to [0,1].
template <class R> R overlap_fraction(const ColliderF& b, const V3<R>& l) {
    auto clamp01 = [](R v) { return v < R(0) ? R(0) : (v > R(1) ? R(1) : v); };
    if (b.shape == 1) {
        const R Rr = (R)b.half_extents[0], L = (R)b.half_extents[1];
        const R r = std::sqrt(l.x * l.x + l.z * l.z);
        const R axial = R(1) - std::abs(l.y) / std::max(L, R(1e-9f));
        const R radial = R(1) - r / std::max(Rr, R(1e-9f));
        return clamp01(axial) * clamp01(radial);
    }
    const R ux = clamp01(R(1) - std::abs(l.x) / std::max((R)b.half_extents[0], R(1e-9f)));
    const R uy = clamp01(R(1) - std::abs(l.y) / std::max((R)b.half_extents[1], R(1e-9f)));
    const R uz = clamp01(R(1) - std::abs(l.z) / std::max((R)b.half_extents[2], R(1e-9f)));
    return ux * uy * uz;
}

// mpm_rigid_coupler.h:167-200: box |R| he per row; cylinder |a_i| L +
// sqrt(max(0, 1 - a_i^2)) R with a the body's y axis in world coordinates.
template <class R> V3<R> world_aabb_half(const ColliderF& b, const M3<R>& Rl2w) {
    if (b.shape == 1) {
        const R Rr = (R)b.half_extents[0], L = (R)b.half_extents[1];
        auto perp = [](R a) { const R s = R(1) - a * a; return s > R(0) ? std::sqrt(s) : R(0); };
        const R ax = Rl2w.m[0][1], ay = Rl2w.m[1][1], az = Rl2w.m[2][1];
        return V3<R>(std::abs(ax) * L + perp(ax) * Rr, std::abs(ay) * L + perp(ay) * Rr,
                     std::abs(az) * L + perp(az) * Rr);
    }
    const R hx = b.half_extents[0], hy = b.half_extents[1], hz = b.half_extents[2];
    return V3<R>(std::abs(Rl2w.m[0][0]) * hx + std::abs(Rl2w.m[0][1]) * hy + std::abs(Rl2w.m[0][2]) * hz,
                 std::abs(Rl2w.m[1][0]) * hx + std::abs(Rl2w.m[1][1]) * hy + std::abs(Rl2w.m[1][2]) * hz,
                 std::abs(Rl2w.m[2][0]) * hx + std::abs(Rl2w.m[2][1]) * hy + std::abs(Rl2w.m[2][2]) * hz);
}

// m4_5_hybrid.h:104-212, the two-pass sweep, with the per-node rule of layer
// 0 = M4_5a (:242-257), 1 = M4_5b (:259-275), 2 = M4_5c (:282-305): pass 1
// sums the overlap fraction of the nodes inside the shape over the allocated
// blocks whose node-centre span meets the shape's tight AABB; pass 2 gives
// each such node m_b = M frac / sum (skipped when m_b <= 0). Layer c scales
// m_b by the quadratic B-spline weight of (x_node - centre) / dx (below 1e-6
// the node takes the body velocity and no mass); every layer takes the
// mass-weighted average of node and body velocity (an empty node, mass <
// 1e-9, takes the body's); layers b and c then blend its tangential part
// toward the body's by min(1, friction) about the closest face's normal. The
// reaction sums m_b (v_after - v_body) / dt and its moment.
template <class R> R bspline1d(R xi) {
    const R a = std::abs(xi);
    if (a < R(0.5f)) return R(0.75f) - a * a;
    if (a < R(1.5f)) { const R t = R(1.5f) - a; return R(0.5f) * t * t; }
    return R(0);
}

template <class R> V3<R> friction_tangent(const V3<R>& v, const V3<R>& vb, const V3<R>& n, R friction) {
    const R vn = v.dot(n);
    const V3<R> vt = v - n * vn;
    const V3<R> vtb = vb - n * vb.dot(n);
    const V3<R> vtn = vt + (vtb - vt) * std::min(R(1), friction);
    return n * vn + vtn;
}

template <class R> Reaction<R> m45_apply(Grid<R>& grid, const ColliderF& b, R dt, int layer) {
    Reaction<R> out;
    if (dt <= R(0)) return out;
    const R dx = grid.dx;
    const M3<R> Rl2w = M3<R>::from_quat(b.orientation[0], b.orientation[1], b.orientation[2], b.orientation[3]);
    const M3<R> Rw2l = Rl2w.T();
    const V3<R> ah = world_aabb_half<R>(b, Rl2w);
    const V3<R> c(b.center[0], b.center[1], b.center[2]);
    const V3<R> lo = c - ah, hi = c + ah;
    auto visit = [&](auto&& fn) {
        for (auto& kv : grid.blocks) {
            Block<R>& blk = kv.second;
            const V3<R> blo(((R)blk.ox + R(0.5f)) * dx, ((R)blk.oy + R(0.5f)) * dx, ((R)blk.oz + R(0.5f)) * dx);
            const V3<R> bhi(((R)(blk.ox + 3) + R(0.5f)) * dx, ((R)(blk.oy + 3) + R(0.5f)) * dx,
                            ((R)(blk.oz + 3) + R(0.5f)) * dx);
            if (bhi.x < lo.x || blo.x > hi.x) continue;
            if (bhi.y < lo.y || blo.y > hi.y) continue;
            if (bhi.z < lo.z || blo.z > hi.z) continue;
            for (int li = 0; li < 4; ++li)
                for (int lj = 0; lj < 4; ++lj)
                    for (int lk = 0; lk < 4; ++lk) {
                        const V3<R> xn(((R)(blk.ox + li) + R(0.5f)) * dx, ((R)(blk.oy + lj) + R(0.5f)) * dx,
                                       ((R)(blk.oz + lk) + R(0.5f)) * dx);
                        const V3<R> local = Rw2l * (xn - c);
                        if (!shape_inside<R>(b, local)) continue;
                        fn(blk.n[li * 16 + lj * 4 + lk], xn, local);
                    }
        }
    };
    R frac_sum = 0;
    visit([&](Node<R>&, const V3<R>&, const V3<R>& local) { frac_sum += overlap_fraction<R>(b, local); });
    if (frac_sum < R(1e-9f)) return out;
    const R per_frac = (R)b.mass / frac_sum;
    const V3<R> vl(b.linear_velocity[0], b.linear_velocity[1], b.linear_velocity[2]);
    const V3<R> w(b.angular_velocity[0], b.angular_velocity[1], b.angular_velocity[2]);
    V3<R> fsum, tsum;
    visit([&](Node<R>& n, const V3<R>& xn, const V3<R>& local) {
        R mb = per_frac * overlap_fraction<R>(b, local);
        if (mb <= R(0)) return;
        const V3<R> r = xn - c;
        const V3<R> vb = vl + w.cross(r);
        const bool was_active = n.active && n.m >= R(1e-9f);
        const R old_m = was_active ? n.m : R(0);
        const V3<R> old_v = was_active ? n.v : V3<R>(R(0));
        V3<R> va = vb;
        bool rule = true;
        if (layer == 2) {
            const R k = bspline1d<R>((xn.x - c.x) / dx) * bspline1d<R>((xn.y - c.y) / dx) *
                        bspline1d<R>((xn.z - c.z) / dx);
            if (k < R(1e-6f)) {
                mb = R(0);
                rule = false;
            } else {
                mb = mb * k;
            }
        }
        if (rule) {
            if (was_active) va = (old_v * old_m + vb * mb) / (old_m + mb);
            if (layer >= 1) {
                const V3<R> nw0 = Rl2w * outward_normal_local<R>(b, local);
                const R len = nw0.length();
                const V3<R> nw = len < R(1e-6f) ? V3<R>(R(0)) : nw0 / len;
                va = friction_tangent<R>(va, vb, nw, (R)b.friction);
            }
        }
        n.active = true;
        n.m = old_m + mb;
        n.v = va;
        const V3<R> dF = (va - vb) * (mb / dt);
        fsum += dF;
        tsum += r.cross(dF);
        ++out.nodes_inside;
    });
    out.force = fsum;
    out.torque = tsum;
    return out;
}

template <class R> Reaction<R> m45a_apply(Grid<R>& grid, const ColliderF& b, R dt) {
    return m45_apply<R>(grid, b, dt, 0);
}

// mpm_rigid_coupler.cpp:58-143 (M0, Dirichlet): over the allocated blocks
// meeting the box-formula AABB, every node with mass > 1e-8 inside the shape
// keeps its normal velocity no slower outward than the body's (n = the
// closest face's normal in world, normalised) and blends its tangential
// velocity toward the body's by min(1, friction); its mass is unchanged. The
// reaction is minus the momentum change over dt, and its moment.
template <class R> Reaction<R> m0_apply(Grid<R>& grid, const ColliderF& b, R dt) {
    Reaction<R> out;
    if (dt <= R(0)) return out;
    const R dx = grid.dx;
    const M3<R> Rl2w = M3<R>::from_quat(b.orientation[0], b.orientation[1], b.orientation[2], b.orientation[3]);
    const M3<R> Rw2l = Rl2w.T();
    const R hx = b.half_extents[0], hy = b.half_extents[1], hz = b.half_extents[2];
    const V3<R> ah(std::abs(Rl2w.m[0][0]) * hx + std::abs(Rl2w.m[0][1]) * hy + std::abs(Rl2w.m[0][2]) * hz,
                   std::abs(Rl2w.m[1][0]) * hx + std::abs(Rl2w.m[1][1]) * hy + std::abs(Rl2w.m[1][2]) * hz,
                   std::abs(Rl2w.m[2][0]) * hx + std::abs(Rl2w.m[2][1]) * hy + std::abs(Rl2w.m[2][2]) * hz);
    const V3<R> c(b.center[0], b.center[1], b.center[2]);
    const V3<R> lo = c - ah, hi = c + ah;
    const V3<R> vl(b.linear_velocity[0], b.linear_velocity[1], b.linear_velocity[2]);
    const V3<R> w(b.angular_velocity[0], b.angular_velocity[1], b.angular_velocity[2]);
    const R fr = std::min(R(1), (R)b.friction);
    V3<R> fsum, tsum;
    for (auto& kv : grid.blocks) {
        Block<R>& blk = kv.second;
        const V3<R> blo(((R)blk.ox + R(0.5f)) * dx, ((R)blk.oy + R(0.5f)) * dx, ((R)blk.oz + R(0.5f)) * dx);
        const V3<R> bhi(((R)(blk.ox + 3) + R(0.5f)) * dx, ((R)(blk.oy + 3) + R(0.5f)) * dx,
                        ((R)(blk.oz + 3) + R(0.5f)) * dx);
        if (bhi.x < lo.x || blo.x > hi.x) continue;
        if (bhi.y < lo.y || blo.y > hi.y) continue;
        if (bhi.z < lo.z || blo.z > hi.z) continue;
        for (int li = 0; li < 4; ++li)
            for (int lj = 0; lj < 4; ++lj)
                for (int lk = 0; lk < 4; ++lk) {
                    Node<R>& n = blk.n[li * 16 + lj * 4 + lk];
                    if (!n.active || n.m <= R(1e-8f)) continue;
                    const V3<R> xn(((R)(blk.ox + li) + R(0.5f)) * dx, ((R)(blk.oy + lj) + R(0.5f)) * dx,
                                   ((R)(blk.oz + lk) + R(0.5f)) * dx);
                    const V3<R> local = Rw2l * (xn - c);
                    if (!shape_inside<R>(b, local)) continue;
                    const V3<R> r = xn - c;
                    const V3<R> vb = vl + w.cross(r);
                    const V3<R> vn_ = n.v;
                    const V3<R> nw0 = Rl2w * outward_normal_local<R>(b, local);
                    const R len = nw0.length();
                    const V3<R> nw = len < R(1e-6f) ? V3<R>(R(0)) : nw0 / len;
                    const R vn_node = vn_.dot(nw);
                    const R vn_body = vb.dot(nw);
                    const R vn_clamped = std::max(vn_node, vn_body);
                    const V3<R> vt_node = vn_ - nw * vn_node;
                    const V3<R> vt_body = vb - nw * vn_body;
                    const V3<R> vt_new = vt_node + (vt_body - vt_node) * fr;
                    const V3<R> va = nw * vn_clamped + vt_new;
                    const V3<R> dp = (va - vn_) * n.m;
                    n.v = va;
                    fsum = fsum - dp / dt;
                    tsum = tsum - r.cross(dp) / dt;
                    ++out.nodes_inside;
                }
    }
    out.force = fsum;
    out.torque = tsum;
    return out;
}

}  // namespace bm_oracle
