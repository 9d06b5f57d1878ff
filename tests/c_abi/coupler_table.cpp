// A C++ caller of the C ABI in the style of the reference's research harness
// (research/mpm_rigid_coupling/bench_compare_all.cpp:50-70): a table of
// coupler entry points with one signature, each applied between
// bm_solver_grid_update and bm_solver_g2p of a small sand bed with a box
// pressed into it. Built against include/bm_mpm.h and libbm_mpm.so only (no
// Python); exits 0 when every call succeeds, every coupler finds nodes inside
// the box and, for every coupler that conserves the body's mass (all but
// M4.5), the sand pushes the box up.
#include <cmath>
#include <cstdio>
#include <vector>

#include "bm_mpm.h"

using BmApplyFn = bm_status_t (*)(bm_solver_t*, const bm_collider_t*, float, bm_reaction_t*);
static const struct {
    const char* name;
    BmApplyFn fn;
} kMethods[] = {
    {"M0", &bm_coupler_m0_apply},      {"M1", &bm_coupler_m1_apply},     {"M4.5a", &bm_coupler_m45a_apply},
    {"M4.5b", &bm_coupler_m45b_apply}, {"M4.5", &bm_coupler_m45_apply},
};

#define CHECK(call)                                                                                 \
    do {                                                                                            \
        const bm_status_t st_ = (call);                                                             \
        if (st_ != BM_OK) {                                                                         \
            std::fprintf(stderr, "%s failed: %s (%s)\n", #call, bm_status_string(st_), bm_last_error()); \
            return 1;                                                                               \
        }                                                                                           \
    } while (0)

int main() {
    const float dx = 1.0f / 32.0f, dt = 1e-4f;
    // 16 x 6 x 16 cells of sand, 4 particles per cell on a regular sub-lattice
    std::vector<float> pos;
    for (int i = 0; i < 16; ++i)
        for (int j = 0; j < 6; ++j)
            for (int k = 0; k < 16; ++k)
                for (int q = 0; q < 4; ++q) {
                    pos.push_back((8 + i + 0.25f + 0.5f * (q & 1)) * dx);
                    pos.push_back((j + 0.25f + 0.5f * ((q >> 1) & 1)) * dx);
                    pos.push_back((8 + k + 0.5f) * dx);
                }
    const int64_t n = (int64_t)pos.size() / 3;
    std::vector<float> mass(n, 1600.0f * dx * dx * dx / 4.0f);
    bm_domain_t dom = {{0, -4, 0}, {32, 24, 32}};
    bm_collider_t box = {};
    box.center[0] = box.center[2] = 16 * dx;
    box.center[1] = 6 * dx;  // sunk half a box deep into the bed
    box.orientation[0] = 1.0f;
    box.half_extents[0] = box.half_extents[1] = box.half_extents[2] = 2 * dx;
    box.linear_velocity[1] = -0.2f;
    box.friction = 0.5f;
    box.mass = 1.0f;
    box.shape = BM_SHAPE_BOX;
    for (const auto& m : kMethods) {
        bm_solver_t* s = nullptr;
        CHECK(bm_solver_create(dx, &dom, &s));
        CHECK(bm_solver_set_material(s, 3.5e5f, 0.3f, 1600.0f));
        CHECK(bm_solver_add_particles(s, n, pos.data(), nullptr, mass.data()));
        bm_reaction_t r = {};
        for (int step = 0; step < 5; ++step) {
            CHECK(bm_solver_p2g(s, dt));
            CHECK(bm_solver_grid_update(s, dt));
            CHECK(m.fn(s, &box, dt, &r));
            CHECK(bm_solver_g2p(s, dt));
        }
        int64_t escaped = 0;
        CHECK(bm_solver_sync(s, &escaped));
        std::printf("%-6s force (%+.4e, %+.4e, %+.4e) N, %d nodes inside\n", m.name, r.force[0], r.force[1],
                    r.force[2], r.nodes_inside);
        CHECK(bm_solver_destroy(s));
        // M4.5 weighs each node's mass share by a B-spline of its offset and
        // gives nodes beyond 1.5 dx the body velocity with no mass, so its net
        // reaction need not oppose the motion; the others must push back up
        const bool conserving = m.fn != &bm_coupler_m45_apply;
        if (r.nodes_inside <= 0 || !std::isfinite(r.force[1]) || (conserving && !(r.force[1] > 0.0f))) {
            std::fprintf(stderr, "%s: expected nodes inside and an upward reaction\n", m.name);
            return 1;
        }
    }
    return 0;
}
