// bm_solver.cu — the bm_solver_* C ABI: the plain single-scene MPM solver.
//
// Mirrors the reference MPMSolver (include/basements/physics/mpm/mpm_solver.h:15-95):
// same parameter defaults (:100-109), the same V0 = m / rho rule and its
// rescale on set_material (:28-51), the same step order (:71-87). The solver
// is a World (bm_world.h) of one scene: device-resident FP32 SoA particles
// and a dense grid box fixed at its first use.
//
// bm_solver_step runs the fused path: P2G(n) is precomputed by the previous
// step's fused kernel (or computed when missing), then the grid update, the
// couplers, and G2P(n) fused with P2G(n+1). The split calls (p2g,
// grid_update, m1_apply, g2p) run the same phases one by one.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "bm_solver_impl.h"

namespace bm {
const char* last_error_text();
}
using namespace bm;

namespace bm {
namespace sol {

bm_status_t ensure_reactions(bm_solver* s, int n) {
    if (n <= s->react_cap) return BM_OK;
    cudaFree(s->d_acc);
    cudaFree(s->d_react);
    cudaFree(s->d_params);
    cudaFree(s->d_frac_sum);
    s->d_acc = nullptr;
    s->d_react = nullptr;
    s->d_params = nullptr;
    s->d_frac_sum = nullptr;
    BM_CHECK_CUDA(cudaMalloc((void**)&s->d_acc, sizeof(double) * 7 * n));
    // the reaction sums start at zero; each finalize zeroes the sums it read
    BM_CHECK_CUDA(cudaMemset(s->d_acc, 0, sizeof(double) * 7 * n));
    BM_CHECK_CUDA(cudaMalloc((void**)&s->d_react, sizeof(bm_reaction_t) * n));
    BM_CHECK_CUDA(cudaMalloc((void**)&s->d_params, sizeof(M1Params) * n));
    BM_CHECK_CUDA(cudaMalloc((void**)&s->d_frac_sum, sizeof(double) * n));
    s->react_cap = n;
    return BM_OK;
}

// Sets the scene's dt (read by the kernels from the scene table).
void set_dt(bm_solver* s, float dt) {
    if (s->sc().dev.dt != dt) {
        s->sc().dev.dt = dt;
        s->w.dirty = true;
    }
}

bm_status_t prepare(bm_solver* s) {
    bm_status_t st = s->w.ensure_grid(s->sc());
    if (st == BM_OK) st = s->w.sync_table();
    return st;
}

bm_status_t do_p2g(bm_solver* s) {
    bm_status_t st = prepare(s);
    if (st != BM_OK) return st;
    st = s->w.clear_and_p2g();
    s->acc_valid = true;
    s->folded[s->w.cur] = false;
    s->view = s->w.cur;
    return st;
}

bm_status_t do_grid_update(bm_solver* s, float dt) {
    if (!s->sc().grid_ready || !s->acc_valid) {
        set_last_error("grid_update needs the P2G of the current particle state (call p2g first)");
        return BM_ERR_STATE;
    }
    // the precomputed P2G folded another dt into the momentum: redo it unfolded
    if (s->folded[s->w.cur] && dt != s->fold_dt[s->w.cur]) {
        bm_status_t st = do_p2g(s);
        if (st != BM_OK) return st;
    }
    set_dt(s, dt);
    bm_status_t st = prepare(s);
    if (st != BM_OK) return st;
    st = s->w.update(s->folded[s->w.cur]);
    s->view = s->w.cur;
    return st;
}

bm_status_t do_m1(bm_solver* s, int n_bodies, const bm_collider_t* bodies, float dt) {
    bm_status_t st = ensure_reactions(s, std::max(1, n_bodies));
    if (st != BM_OK) return st;
    s->h_params.resize(n_bodies);
    std::vector<M1Params>& hp = s->h_params;
    bool any_active = false;
    for (int b = 0; b < n_bodies; ++b) {
        m1_prepare(s->sc().dev.g, bodies[b], dt, 0, &hp[b]);
        any_active = any_active || hp[b].active;
    }
    // (the FP64 sums in d_acc are zero: the last finalize zeroed them)
    if (any_active && n_bodies == 1) {
        // one launch: the M1 kernel's last CTA writes the reaction
        bool launched = false;
        s->w.timed("m1_coupler", [&] {
            launched = launch_m1_one(s->w.table(), hp[0], s->w.cur, s->d_acc, s->d_react, s->w.d_repair + 3,
                                     s->w.stream);
        });
        if (!launched) launch_reaction_finalize(s->d_acc, n_bodies, s->d_react, s->w.stream);
        s->view = s->w.cur;
        return launch_status("m1");
    } else if (any_active) {
        BM_CHECK_CUDA(cudaMemcpyAsync(s->d_params, hp.data(), sizeof(M1Params) * n_bodies, cudaMemcpyHostToDevice,
                                      s->w.stream));
        // The reference applies its couplers one after another, each on the
        // grid its predecessor left. Bodies whose candidate blocks are
        // disjoint touch disjoint nodes and share one launch; a body that
        // overlaps an earlier body of the current launch starts the next one.
        s->w.timed("m1_coupler", [&] {
            int first = 0;
            while (first < n_bodies) {
                int last = first;
                int64_t cand = 0;
                for (; last < n_bodies; ++last) {
                    const M1Params& P = hp[last];
                    if (!P.active) continue;
                    bool clash = false;
                    for (int q = first; q < last && !clash; ++q) clash = hp[q].active && m1_blocks_overlap(hp[q], P);
                    if (clash) break;
                    cand = std::max<int64_t>(cand, (int64_t)P.nbi * P.nbj * P.nbk);
                }
                if (cand > 0)
                    launch_m1(s->w.table(), s->d_params + first, last - first, cand, s->w.cur, s->d_acc + 7 * first,
                              s->w.stream);
                first = last;
            }
        });
    }
    launch_reaction_finalize(s->d_acc, n_bodies, s->d_react, s->w.stream);
    s->view = s->w.cur;
    return launch_status("m1");
}

bm_status_t do_m0(bm_solver* s, int n_bodies, const bm_collider_t* bodies, float dt) {
    bm_status_t st = ensure_reactions(s, std::max(1, n_bodies));
    if (st != BM_OK) return st;
    s->h_params.resize(n_bodies);
    std::vector<M1Params>& hp = s->h_params;
    for (int b = 0; b < n_bodies; ++b) m1_prepare(s->sc().dev.g, bodies[b], dt, 0, &hp[b]);
    BM_CHECK_CUDA(cudaMemsetAsync(s->d_acc, 0, sizeof(double) * 7 * n_bodies, s->w.stream));
    if (n_bodies > 0)
        BM_CHECK_CUDA(cudaMemcpyAsync(s->d_params, hp.data(), sizeof(M1Params) * n_bodies, cudaMemcpyHostToDevice,
                                      s->w.stream));
    s->w.timed("m0_coupler", [&] {
        for (int b = 0; b < n_bodies; ++b) {
            const M1Params& P = hp[b];
            if (!P.active) continue;
            launch_m0(s->w.table(), s->d_params + b, (int64_t)P.nbi * P.nbj * P.nbk, s->w.cur, dt, s->d_acc + 7 * b,
                      s->w.stream);
        }
    });
    launch_reaction_finalize(s->d_acc, n_bodies, s->d_react, s->w.stream);
    s->view = s->w.cur;
    return launch_status("m0");
}

// The reference applies a coupler to one body at a time (ApplyFn,
// bench_compare_all.cpp:50-51); each body's two passes run in order.
bm_status_t do_m45(bm_solver* s, int n_bodies, const bm_collider_t* bodies, float dt, int layer) {
    bm_status_t st = ensure_reactions(s, std::max(1, n_bodies));
    if (st != BM_OK) return st;
    s->h_params.resize(n_bodies);
    std::vector<M1Params>& hp = s->h_params;
    for (int b = 0; b < n_bodies; ++b) m45a_prepare(s->sc().dev.g, bodies[b], dt, &hp[b]);
    BM_CHECK_CUDA(cudaMemsetAsync(s->d_acc, 0, sizeof(double) * 7 * n_bodies, s->w.stream));
    BM_CHECK_CUDA(cudaMemsetAsync(s->d_frac_sum, 0, sizeof(double) * n_bodies, s->w.stream));
    if (n_bodies > 0)
        BM_CHECK_CUDA(cudaMemcpyAsync(s->d_params, hp.data(), sizeof(M1Params) * n_bodies, cudaMemcpyHostToDevice,
                                      s->w.stream));
    s->w.timed("m45_coupler", [&] {
        for (int b = 0; b < n_bodies; ++b) {
            const M1Params& P = hp[b];
            if (!P.active) continue;
            launch_m45(s->w.table(), s->d_params + b, (int64_t)P.nbi * P.nbj * P.nbk, s->w.cur, dt,
                       s->d_frac_sum + b, s->d_acc + 7 * b, layer, s->w.stream);
        }
    });
    launch_reaction_finalize(s->d_acc, n_bodies, s->d_react, s->w.stream);
    s->view = s->w.cur;
    return launch_status("m45");
}

bm_status_t do_g2p(bm_solver* s, float dt) {
    if (!s->sc().grid_ready || !s->acc_valid) {
        set_last_error("g2p needs a grid from p2g / grid_update");
        return BM_ERR_STATE;
    }
    set_dt(s, dt);
    bm_status_t st = prepare(s);
    if (st == BM_OK) st = s->w.g2p();
    s->acc_valid = false;
    s->view = s->w.cur;
    return st;
}

// G2P of this step fused with the P2G of the next one; regroups the
// particles by stencil base node first when due.
bm_status_t do_g2p2g(bm_solver* s, float dt) {
    set_dt(s, dt);
    bm_status_t st = prepare(s);
    if (st != BM_OK) return st;
    if (s->sc().n() > 0 && (!s->sorted || (s->sort_interval > 0 && s->steps_since_sort >= s->sort_interval))) {
        st = s->w.sort_particles();
        if (st != BM_OK) return st;
        s->sorted = true;
        s->steps_since_sort = 0;
    }
    const int before = s->w.cur;
    st = s->w.g2p2g(s->fast_math, s->variant);
    s->view = before;
    s->folded[s->w.cur] = true;
    s->fold_dt[s->w.cur] = dt;
    s->acc_valid = true;
    s->steps_since_sort += 1;
    return st;
}

bm_status_t do_step(bm_solver* s, float dt, int32_t n_bodies, const bm_collider_t* bodies) {
    bm_status_t st = prepare(s);
    if (st == BM_OK && s->acc_valid && s->folded[s->w.cur] && dt != s->fold_dt[s->w.cur]) s->acc_valid = false;
    if (st == BM_OK && !s->acc_valid) st = do_p2g(s);
    if (st == BM_OK) st = do_grid_update(s, dt);
    if (st == BM_OK && n_bodies > 0)
        st = s->coupler == BM_COUPLER_M45A   ? do_m45(s, n_bodies, bodies, dt, 0)
             : s->coupler == BM_COUPLER_M45B ? do_m45(s, n_bodies, bodies, dt, 1)
             : s->coupler == BM_COUPLER_M45  ? do_m45(s, n_bodies, bodies, dt, 2)
             : s->coupler == BM_COUPLER_M0   ? do_m0(s, n_bodies, bodies, dt)
                                             : do_m1(s, n_bodies, bodies, dt);
    if (st == BM_OK) st = do_g2p2g(s, dt);
    return st;
}

void invalidate_state(bm_solver* s) {
    s->acc_valid = false;
    s->sorted = false;
}

bm_status_t noalloc_setup(int dev);  // defined with the no-alloc coupler below

}  // namespace sol
}  // namespace bm

using namespace bm::sol;

extern "C" {

BM_API int bm_get_version(void) { return BM_API_VERSION; }

BM_API const char* bm_status_string(bm_status_t st) {
    switch (st) {
        case BM_OK: return "ok";
        case BM_ERR_INVALID_ARGUMENT: return "invalid argument";
        case BM_ERR_OUT_OF_MEMORY: return "out of device memory";
        case BM_ERR_CUDA: return "CUDA error";
        case BM_ERR_DOMAIN_ESCAPE: return "particle left the grid box";
        case BM_ERR_NON_FINITE: return "non-finite particle state";
        case BM_ERR_TIMEOUT: return "timeout";
        case BM_ERR_NOT_FOUND: return "not found";
        case BM_ERR_STATE: return "call out of order";
        case BM_ERR_NO_DEVICE: return "no usable CUDA device";
    }
    return "unknown status";
}

BM_API const char* bm_last_error(void) { return last_error_text(); }

BM_API bm_status_t bm_set_device(int32_t device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_last_error("no CUDA device");
        return BM_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return invalid_arg("device index out of range");
    BM_CHECK_CUDA(cudaSetDevice(device));
    return BM_OK;
}

BM_API bm_status_t bm_solver_create(float dx, const bm_domain_t* domain, bm_solver_t** out) {
    if (!out) return invalid_arg("out is NULL");
    *out = nullptr;
    if (!(dx > 0.0f) || !std::isfinite(dx)) return invalid_arg("dx must be a positive finite number");
    if (domain)
        for (int a = 0; a < 3; ++a)
            if (domain->extent[a] <= 0) return invalid_arg("domain extent must be positive");
    bm_solver* s = new bm_solver();
    bm_status_t st = s->w.init();
    if (st != BM_OK) {
        delete s;
        return st;
    }
    s->w.add_scene();
    SceneHost& h = s->sc();
    h.dev.g.dx = dx;
    h.dev.g.inv_dx = 1.0f / dx;
    if (domain) {
        h.domain = *domain;
        h.domain_set = true;
    }
    st = ensure_reactions(s, 4);
    if (st == BM_OK) st = noalloc_setup(s->w.device);
    if (st != BM_OK) {
        bm_solver_destroy(s);
        return st;
    }
    *out = s;
    return BM_OK;
}

BM_API bm_status_t bm_solver_destroy(bm_solver_t* s) {
    if (!s) return invalid_arg("NULL handle");
    DeviceGuard dg(s->w.device);
    s->w.release();
    cudaFree(s->d_acc);
    cudaFree(s->d_react);
    cudaFree(s->d_params);
    cudaFree(s->d_frac_sum);
    delete s;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_domain(bm_solver_t* s, const bm_domain_t* d) {
    if (!s || !d) return invalid_arg("NULL argument");
    if (s->sc().grid_ready) {
        set_last_error("the grid box is fixed once the grid has been used");
        return BM_ERR_STATE;
    }
    for (int a = 0; a < 3; ++a)
        if (d->extent[a] <= 0) return invalid_arg("domain extent must be positive");
    s->sc().domain = *d;
    s->sc().domain_set = true;
    return BM_OK;
}

BM_API bm_status_t bm_solver_get_domain(bm_solver_t* s, bm_domain_t* out) {
    if (!s || !out) return invalid_arg("NULL argument");
    DeviceGuard dg(s->w.device);
    bm_status_t st = s->w.ensure_grid(s->sc());
    if (st != BM_OK) return st;
    const GridDesc& g = s->sc().dev.g;
    out->origin[0] = g.ox; out->origin[1] = g.oy; out->origin[2] = g.oz;
    out->extent[0] = g.ex(); out->extent[1] = g.ey(); out->extent[2] = g.ez();
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_auto_margin(bm_solver_t* s, int32_t margin) {
    if (!s || margin < 0) return invalid_arg("bad margin");
    s->sc().margin = margin;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_sort_interval(bm_solver_t* s, int32_t steps) {
    if (!s || steps < 0) return invalid_arg("bad sort interval");
    s->sort_interval = steps;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_math_mode(bm_solver_t* s, int32_t mode) {
    if (!s || mode < 0 || mode > 1) return invalid_arg("math mode must be 0 (IEEE) or 1 (fast)");
    s->fast_math = mode == 1;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_material(bm_solver_t* s, float E, float nu, float rho) {
    if (!s) return invalid_arg("NULL handle");
    if (!std::isfinite(E) || !std::isfinite(nu) || !std::isfinite(rho)) return invalid_arg("non-finite material");
    DeviceGuard dg(s->w.device);
    SceneHost& h = s->sc();
    h.E = E;
    h.nu = nu;
    if (rho > 1e-12f && h.density > 1e-12f && rho != h.density && h.n() > 0) {
        // V0 *= rho_old / rho_new for every particle (mpm_solver.h:45-49).
        const float rescale = h.density / rho;
        ParticleSoA& ps = h.dev.store[s->w.sel];
        std::vector<float> v0(h.n());
        BM_CHECK_CUDA(cudaMemcpyAsync(v0.data(), ps.plane(P_V0), sizeof(float) * h.n(), cudaMemcpyDeviceToHost,
                                      s->w.stream));
        BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
        for (auto& x : v0) x *= rescale;
        BM_CHECK_CUDA(cudaMemcpyAsync(ps.plane(P_V0), v0.data(), sizeof(float) * h.n(), cudaMemcpyHostToDevice,
                                      s->w.stream));
        BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
    }
    h.density = rho;
    s->w.dirty = true;
    s->acc_valid = false;  // the precomputed P2G used the old stress
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_gravity(bm_solver_t* s, const float g[3]) {
    if (!s || !g) return invalid_arg("NULL argument");
    for (int a = 0; a < 3; ++a) s->sc().gravity[a] = g[a];
    s->w.dirty = true;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_plastic_alpha(bm_solver_t* s, float a) {
    if (!s) return invalid_arg("NULL handle");
    s->sc().alpha = a;
    s->w.dirty = true;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_floor_friction(bm_solver_t* s, float mu) {
    if (!s) return invalid_arg("NULL handle");
    s->sc().floor_friction = mu;
    s->w.dirty = true;
    return BM_OK;
}

BM_API bm_status_t bm_solver_add_particles(bm_solver_t* s, int64_t n, const float* pos, const float* vel,
                                           const float* mass) {
    if (!s) return invalid_arg("NULL handle");
    if (n < 0) return invalid_arg("n < 0");
    if (n == 0) return BM_OK;
    if (!pos) return invalid_arg("position is NULL");
    DeviceGuard dg(s->w.device);
    bm_status_t st = s->w.append_particles(s->sc(), n, pos, vel, mass);
    invalidate_state(s);
    return st;
}

BM_API bm_status_t bm_solver_num_particles(bm_solver_t* s, int64_t* out) {
    if (!s || !out) return invalid_arg("NULL argument");
    *out = s->sc().n();
    return BM_OK;
}

BM_API bm_status_t bm_solver_get_particles(bm_solver_t* s, const bm_particles_view_t* v) {
    if (!s || !v) return invalid_arg("NULL argument");
    DeviceGuard dg(s->w.device);
    const World::ReadField fields[] = {{v->position, P_X, 3}, {v->velocity, P_V, 3}, {v->F, P_F, 9},
                                       {v->C, P_C, 9},        {v->mass, P_M, 1},     {v->volume, P_V0, 1}};
    return s->w.read_fields(s->sc(), fields, 6);
}

BM_API bm_status_t bm_solver_set_particles(bm_solver_t* s, int64_t first, int64_t n, const bm_particles_view_t* v) {
    if (!s || !v) return invalid_arg("NULL argument");
    if (first < 0 || n < 0 || first + n > s->sc().n()) return invalid_arg("particle range out of bounds");
    if (n == 0) return BM_OK;
    DeviceGuard dg(s->w.device);
    SceneHost& h = s->sc();
    const ParticleSoA& ps = h.dev.store[s->w.sel];
    struct Field { const float* src; int plane; int width; };
    const Field fields[] = {{v->position, P_X, 3}, {v->velocity, P_V, 3}, {v->F, P_F, 9}, {v->C, P_C, 9}};
    float* tmp = nullptr;
    BM_CHECK_CUDA(cudaMallocAsync((void**)&tmp, sizeof(float) * 9 * n, s->w.stream));
    launch_inverse_pid(ps, h.d_inv, s->w.stream);
    for (const Field& f : fields) {
        if (!f.src) continue;
        cudaMemcpyAsync(tmp, f.src, sizeof(float) * f.width * n, cudaMemcpyHostToDevice, s->w.stream);
        launch_scatter_rows(ps, f.plane, f.width, tmp, first, n, h.d_inv, s->w.stream);
    }
    cudaFreeAsync(tmp, s->w.stream);
    BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
    if (v->position) s->w.update_bbox(h, n, v->position);
    invalidate_state(s);
    return launch_status("set_particles");
}

BM_API bm_status_t bm_solver_step(bm_solver_t* s, float dt) {
    if (!s) return invalid_arg("NULL handle");
    if (!std::isfinite(dt)) return invalid_arg("dt is not finite");
    DeviceGuard dg(s->w.device);
    return do_step(s, dt, 0, nullptr);
}

BM_API bm_status_t bm_solver_step_n(bm_solver_t* s, float dt, int32_t n_steps) {
    if (!s) return invalid_arg("NULL handle");
    if (n_steps < 0) return invalid_arg("n_steps < 0");
    for (int32_t i = 0; i < n_steps; ++i) {
        bm_status_t st = bm_solver_step(s, dt);
        if (st != BM_OK) return st;
    }
    return BM_OK;
}

BM_API bm_status_t bm_solver_p2g(bm_solver_t* s, float dt) {
    if (!s) return invalid_arg("NULL handle");
    (void)dt;  // P2G does not depend on dt (mpm_solver.h:168)
    DeviceGuard dg(s->w.device);
    return do_p2g(s);
}

BM_API bm_status_t bm_solver_grid_update(bm_solver_t* s, float dt) {
    if (!s) return invalid_arg("NULL handle");
    if (!std::isfinite(dt)) return invalid_arg("dt is not finite");
    DeviceGuard dg(s->w.device);
    return do_grid_update(s, dt);
}

BM_API bm_status_t bm_solver_g2p(bm_solver_t* s, float dt) {
    if (!s) return invalid_arg("NULL handle");
    if (!std::isfinite(dt)) return invalid_arg("dt is not finite");
    DeviceGuard dg(s->w.device);
    return do_g2p(s, dt);
}

BM_API bm_status_t bm_coupler_m1_apply(bm_solver_t* s, const bm_collider_t* body, float dt, bm_reaction_t* out) {
    if (!s || !body || !out) return invalid_arg("NULL argument");
    DeviceGuard dg(s->w.device);
    std::memset(out, 0, sizeof(*out));
    bm_status_t st = prepare(s);
    if (st != BM_OK) return st;
    if (!s->acc_valid && s->sc().n() > 0) {
        set_last_error("the coupler needs a grid from p2g / grid_update");
        return BM_ERR_STATE;
    }
    st = do_m1(s, 1, body, dt);
    if (st != BM_OK) return st;
    BM_CHECK_CUDA(cudaMemcpyAsync(out, s->d_react, sizeof(bm_reaction_t), cudaMemcpyDeviceToHost, s->w.stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
    return BM_OK;
}

namespace {
// One coupler call of the split API: checks, the coupler, the reaction read back.
bm_status_t coupler_call(bm_solver_t* s, const bm_collider_t* body, float dt, bm_reaction_t* out,
                         bm_status_t (*coupler)(bm_solver*, int, const bm_collider_t*, float)) {
    if (!s || !body || !out) return invalid_arg("NULL argument");
    DeviceGuard dg(s->w.device);
    std::memset(out, 0, sizeof(*out));
    bm_status_t st = prepare(s);
    if (st != BM_OK) return st;
    if (!s->acc_valid && s->sc().n() > 0) {
        set_last_error("the coupler needs a grid from p2g / grid_update");
        return BM_ERR_STATE;
    }
    st = coupler(s, 1, body, dt);
    if (st != BM_OK) return st;
    BM_CHECK_CUDA(cudaMemcpyAsync(out, s->d_react, sizeof(bm_reaction_t), cudaMemcpyDeviceToHost, s->w.stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
    return BM_OK;
}
}  // namespace

BM_API bm_status_t bm_coupler_m0_apply(bm_solver_t* s, const bm_collider_t* body, float dt, bm_reaction_t* out) {
    return coupler_call(s, body, dt, out, &do_m0);
}

bm_status_t do_m45a(bm_solver* s, int n, const bm_collider_t* b, float dt) { return do_m45(s, n, b, dt, 0); }
bm_status_t do_m45b(bm_solver* s, int n, const bm_collider_t* b, float dt) { return do_m45(s, n, b, dt, 1); }
bm_status_t do_m45c(bm_solver* s, int n, const bm_collider_t* b, float dt) { return do_m45(s, n, b, dt, 2); }

BM_API bm_status_t bm_coupler_m45a_apply(bm_solver_t* s, const bm_collider_t* body, float dt, bm_reaction_t* out) {
    return coupler_call(s, body, dt, out, &do_m45a);
}

BM_API bm_status_t bm_coupler_m45b_apply(bm_solver_t* s, const bm_collider_t* body, float dt, bm_reaction_t* out) {
    return coupler_call(s, body, dt, out, &do_m45b);
}

BM_API bm_status_t bm_coupler_m45_apply(bm_solver_t* s, const bm_collider_t* body, float dt, bm_reaction_t* out) {
    return coupler_call(s, body, dt, out, &do_m45c);
}

BM_API bm_status_t bm_solver_set_coupler(bm_solver_t* s, int32_t coupler) {
    if (!s) return invalid_arg("NULL handle");
    if (coupler < BM_COUPLER_M1 || coupler > BM_COUPLER_M45) return invalid_arg("unknown coupler");
    s->coupler = coupler;
    return BM_OK;
}

BM_API bm_status_t bm_solver_step_coupled(bm_solver_t* s, float dt, int32_t n_bodies, const bm_collider_t* bodies,
                                          bm_reaction_t* reactions) {
    if (!s) return invalid_arg("NULL handle");
    if (n_bodies < 0 || (n_bodies > 0 && !bodies)) return invalid_arg("bad bodies");
    if (!std::isfinite(dt)) return invalid_arg("dt is not finite");
    DeviceGuard dg(s->w.device);
    bm_status_t st = do_step(s, dt, n_bodies, bodies);
    if (st == BM_OK && reactions && n_bodies > 0) {
        BM_CHECK_CUDA(cudaMemcpyAsync(reactions, s->d_react, sizeof(bm_reaction_t) * n_bodies,
                                      cudaMemcpyDeviceToHost, s->w.stream));
        BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
    }
    return st;
}

BM_API bm_status_t bm_solver_get_reactions(bm_solver_t* s, int32_t n, bm_reaction_t* out) {
    if (!s || !out || n < 0 || n > s->react_cap) return invalid_arg("bad arguments");
    DeviceGuard dg(s->w.device);
    if (n == 0) return BM_OK;
    BM_CHECK_CUDA(cudaMemcpyAsync(out, s->d_react, sizeof(bm_reaction_t) * n, cudaMemcpyDeviceToHost, s->w.stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
    return BM_OK;
}

BM_API bm_status_t bm_solver_grid_num_nodes(bm_solver_t* s, int64_t* out) {
    if (!s || !out) return invalid_arg("NULL argument");
    DeviceGuard dg(s->w.device);
    bm_status_t st = s->w.ensure_grid(s->sc());
    if (st != BM_OK) return st;
    *out = s->sc().dev.g.num_nodes();
    return BM_OK;
}

BM_API bm_status_t bm_solver_get_grid(bm_solver_t* s, float* vel, float* force, float* mass, uint8_t* active,
                                      uint8_t* balloc) {
    if (!s) return invalid_arg("NULL handle");
    DeviceGuard dg(s->w.device);
    bm_status_t st = s->w.ensure_grid(s->sc());
    if (st != BM_OK) return st;
    SceneHost& h = s->sc();
    const int64_t nn = h.dev.g.num_nodes();
    if (force && s->folded[s->view]) {
        // after a fused step the force is folded into the momentum (see header)
        std::memset(force, 0, sizeof(float) * 3 * nn);
        force = nullptr;
    }
    cudaStream_t stream = s->w.stream;
    float *dv = nullptr, *df = nullptr, *dm = nullptr;
    uint8_t *da = nullptr, *db = nullptr;
    if (vel) BM_CHECK_CUDA(cudaMallocAsync((void**)&dv, sizeof(float) * 3 * nn, stream));
    if (force) BM_CHECK_CUDA(cudaMallocAsync((void**)&df, sizeof(float) * 3 * nn, stream));
    if (mass) BM_CHECK_CUDA(cudaMallocAsync((void**)&dm, sizeof(float) * nn, stream));
    if (active) BM_CHECK_CUDA(cudaMallocAsync((void**)&da, (size_t)nn, stream));
    if (balloc) BM_CHECK_CUDA(cudaMallocAsync((void**)&db, (size_t)nn, stream));
    launch_grid_to_dense(h.dev.g, h.dev.acc[s->view], h.dev.alloc, dv, df, dm, da, db, stream);
    st = launch_status("grid_to_dense");
    if (vel) cudaMemcpyAsync(vel, dv, sizeof(float) * 3 * nn, cudaMemcpyDeviceToHost, stream);
    if (force) cudaMemcpyAsync(force, df, sizeof(float) * 3 * nn, cudaMemcpyDeviceToHost, stream);
    if (mass) cudaMemcpyAsync(mass, dm, sizeof(float) * nn, cudaMemcpyDeviceToHost, stream);
    if (active) cudaMemcpyAsync(active, da, (size_t)nn, cudaMemcpyDeviceToHost, stream);
    if (balloc) cudaMemcpyAsync(balloc, db, (size_t)nn, cudaMemcpyDeviceToHost, stream);
    for (void* p : {(void*)dv, (void*)df, (void*)dm, (void*)da, (void*)db})
        if (p) cudaFreeAsync(p, stream);
    BM_CHECK_CUDA(cudaStreamSynchronize(stream));
    return st;
}

BM_API bm_status_t bm_solver_seed_grid(bm_solver_t* s, int64_t n, const int32_t* ijk, const float* vel,
                                       const float* mass) {
    if (!s) return invalid_arg("NULL handle");
    if (n < 0 || (n > 0 && (!ijk || !vel || !mass))) return invalid_arg("bad seed arrays");
    DeviceGuard dg(s->w.device);
    SceneHost& h = s->sc();
    bm_status_t st = s->w.ensure_grid(h);
    if (st != BM_OK) return st;
    if (n == 0) return BM_OK;
    for (int64_t q = 0; q < n; ++q)
        if (h.dev.g.node(ijk[3 * q], ijk[3 * q + 1], ijk[3 * q + 2]) < 0)
            return invalid_arg("seed node outside the box");
    cudaStream_t stream = s->w.stream;
    int32_t* di = nullptr;
    float *dv = nullptr, *dm = nullptr;
    BM_CHECK_CUDA(cudaMallocAsync((void**)&di, sizeof(int32_t) * 3 * n, stream));
    BM_CHECK_CUDA(cudaMallocAsync((void**)&dv, sizeof(float) * 3 * n, stream));
    BM_CHECK_CUDA(cudaMallocAsync((void**)&dm, sizeof(float) * n, stream));
    cudaMemcpyAsync(di, ijk, sizeof(int32_t) * 3 * n, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(dv, vel, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(dm, mass, sizeof(float) * n, cudaMemcpyHostToDevice, stream);
    launch_seed_grid(h.dev.g, h.dev.acc[s->w.cur], h.dev.alloc, n, di, dv, dm, h.dev.status, stream);
    st = launch_status("seed_grid");
    cudaFreeAsync(di, stream);
    cudaFreeAsync(dv, stream);
    cudaFreeAsync(dm, stream);
    BM_CHECK_CUDA(cudaStreamSynchronize(stream));
    s->acc_valid = true;  // the seeded grid stands for this step's grid
    s->folded[s->w.cur] = false;
    s->view = s->w.cur;
    return st;
}

BM_API bm_status_t bm_solver_set_grid_velocity(bm_solver_t* s, const float* vel) {
    if (!s || !vel) return invalid_arg("NULL argument");
    DeviceGuard dg(s->w.device);
    SceneHost& h = s->sc();
    bm_status_t st = s->w.ensure_grid(h);
    if (st != BM_OK) return st;
    const int64_t nn = h.dev.g.num_nodes();
    float* dv = nullptr;
    BM_CHECK_CUDA(cudaMallocAsync((void**)&dv, sizeof(float) * 3 * nn, s->w.stream));
    cudaMemcpyAsync(dv, vel, sizeof(float) * 3 * nn, cudaMemcpyHostToDevice, s->w.stream);
    launch_dense_velocity_to_grid(h.dev.g, h.dev.acc[s->view], dv, s->w.stream);
    st = launch_status("set_grid_velocity");
    cudaFreeAsync(dv, s->w.stream);
    BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
    return st;
}

BM_API bm_status_t bm_solver_light_node_suspects(bm_solver_t* s, int64_t* out) {
    if (!s || !out) return invalid_arg("NULL argument");
    DeviceGuard dg(s->w.device);
    unsigned long long n = 0;
    BM_CHECK_CUDA(cudaMemcpyAsync(&n, s->sc().dev.escaped + 1, sizeof(n), cudaMemcpyDeviceToHost, s->w.stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
    *out = (int64_t)n;
    return BM_OK;
}

BM_API bm_status_t bm_solver_sync(bm_solver_t* s, int64_t* escaped) {
    if (!s) return invalid_arg("NULL handle");
    DeviceGuard dg(s->w.device);
    SceneHost& h = s->sc();
    uint32_t status = 0;
    unsigned long long esc = 0;
    BM_CHECK_CUDA(cudaMemcpyAsync(&status, h.dev.status, sizeof(status), cudaMemcpyDeviceToHost, s->w.stream));
    BM_CHECK_CUDA(cudaMemcpyAsync(&esc, h.dev.escaped, sizeof(esc), cudaMemcpyDeviceToHost, s->w.stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
    BM_CHECK_CUDA(cudaMemsetAsync(h.dev.status, 0, sizeof(uint32_t), s->w.stream));
    BM_CHECK_CUDA(cudaMemsetAsync(h.dev.escaped, 0, sizeof(unsigned long long), s->w.stream));
    if (escaped) *escaped = (int64_t)esc;
    if (status & ERR_NONFINITE) {
        set_last_error("non-finite particle position or F after G2P");
        return BM_ERR_NON_FINITE;
    }
    if (status & ERR_ESCAPE) {
        set_last_error("particle stencil outside the grid box (" + std::to_string(esc) + " node writes dropped)");
        return BM_ERR_DOMAIN_ESCAPE;
    }
    return BM_OK;
}

BM_API bm_status_t bm_solver_stream(bm_solver_t* s, void** stream) {
    if (!s || !stream) return invalid_arg("NULL argument");
    *stream = (void*)s->w.stream;
    return BM_OK;
}

BM_API bm_status_t bm_solver_profile_enable(bm_solver_t* s, int32_t on) {
    if (!s) return invalid_arg("NULL handle");
    s->w.profiling = on != 0;
    return BM_OK;
}

BM_API bm_status_t bm_solver_profile_read(bm_solver_t* s, int32_t cap, const char** names, double* total_ms,
                                          int64_t* launches, int32_t* n_out) {
    if (!s || !n_out) return invalid_arg("NULL argument");
    DeviceGuard dg(s->w.device);
    BM_CHECK_CUDA(cudaStreamSynchronize(s->w.stream));
    s->w.fold_pending();
    int32_t n = 0;
    for (const auto& sl : s->w.slots) {
        if (n >= cap) break;
        if (names) names[n] = sl.name;
        if (total_ms) total_ms[n] = sl.total_ms;
        if (launches) launches[n] = sl.launches;
        ++n;
    }
    *n_out = n;
    return BM_OK;
}

BM_API bm_status_t bm_solver_profile_reset(bm_solver_t* s) {
    if (!s) return invalid_arg("NULL handle");
    DeviceGuard dg(s->w.device);
    cudaStreamSynchronize(s->w.stream);
    s->w.fold_pending();
    for (auto& sl : s->w.slots) {
        sl.total_ms = 0;
        sl.launches = 0;
    }
    return BM_OK;
}

BM_API bm_status_t bm_solver_timer_start(bm_solver_t* s) {
    if (!s) return invalid_arg("NULL handle");
    DeviceGuard dg(s->w.device);
    if (!s->w.t0) BM_CHECK_CUDA(cudaEventCreate(&s->w.t0));
    if (!s->w.t1) BM_CHECK_CUDA(cudaEventCreate(&s->w.t1));
    BM_CHECK_CUDA(cudaEventRecord(s->w.t0, s->w.stream));
    return BM_OK;
}

BM_API bm_status_t bm_solver_timer_stop(bm_solver_t* s, double* ms) {
    if (!s || !ms) return invalid_arg("NULL argument");
    if (!s->w.t0) return invalid_arg("timer not started");
    DeviceGuard dg(s->w.device);
    BM_CHECK_CUDA(cudaEventRecord(s->w.t1, s->w.stream));
    BM_CHECK_CUDA(cudaEventSynchronize(s->w.t1));
    float f = 0;
    BM_CHECK_CUDA(cudaEventElapsedTime(&f, s->w.t0, s->w.t1));
    *ms = f;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_launch_variant(bm_solver_t* s, int32_t variant) {
    if (!s || variant < 0 || variant >= fused_variant_count()) return invalid_arg("unknown launch variant");
    s->variant = variant;
    return BM_OK;
}

BM_API int32_t bm_launch_variant_count(void) { return fused_variant_count(); }

BM_API const char* bm_launch_variant_name(int32_t variant) { return fused_variant_name(variant); }

}  // extern "C"

// ---- M1 coupler without allocation ----------------------------------------
//
// bm_coupler_m1_apply_noalloc runs the M1 kernels of bm_coupler_m1_apply, but
// its scratch comes from one fixed array in this file, not from the
// per-solver buffers that the other coupler calls grow with cudaMalloc on first
// use. The scratch holds the per-body FP64 reaction sums, the per-body
// parameter blocks and the finished reactions, for at most kNoAllocMaxBodies
// bodies. Some hosts call the coupler where a device allocation is not
// allowed. One is a fixed-budget simulation tick: cudaMalloc and cudaFree can
// wait for the whole device. Another is a process whose HBM is already held
// by a memory pool, where even a small cudaMalloc fails. Such hosts call this
// entry point instead.
//
// The array is shared by every solver on a device. Two calls that overlap in
// time (from two host threads, on any streams) race on it and give wrong
// reactions; callers must serialise them. Its device address is looked up
// (cudaGetSymbolAddress) and the M1 kernels are loaded once per device by
// bm_solver_create, a call that allocates anyway: under CUDA's default lazy
// module loading, the first lookup of the array or launch of a kernel loads
// code and may allocate device memory, so leaving them to the first no-alloc
// call would allocate in the one call that must not.

namespace {

constexpr int kNoAllocMaxBodies = 64;
constexpr int kNoAllocMaxDevices = 64;

constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kNoAllocAccOff = 0;  // double[7] per body: force, torque, nodes_inside
constexpr size_t kNoAllocParamOff = kNoAllocAccOff + align256(sizeof(double) * 7 * kNoAllocMaxBodies);
constexpr size_t kNoAllocReactOff = kNoAllocParamOff + align256(sizeof(M1Params) * kNoAllocMaxBodies);
constexpr size_t kNoAllocBytes = kNoAllocReactOff + align256(sizeof(bm_reaction_t) * kNoAllocMaxBodies);
static_assert(alignof(M1Params) <= 256 && alignof(bm_reaction_t) <= 256, "scratch regions start on 256 B");
static_assert(kNoAllocBytes <= 32 * 1024, "the fixed scratch stays modest");

}  // namespace

static __device__ __align__(256) unsigned char g_m1_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on `dev` (the current device), looked up
// once per device.
bm_status_t noalloc_scratch(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) return invalid_arg("device index beyond the no-alloc scratch table");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_m1_noalloc_scratch);
        if (e == cudaSuccess && !p) e = cudaErrorInvalidSymbol;
        if (e == cudaSuccess) e = load_m1_kernels();
        if (e != cudaSuccess) {
            set_last_error(std::string("no-alloc M1 set-up (scratch address, kernel load): ") + cudaGetErrorString(e));
            return BM_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return BM_OK;
}

}  // namespace

namespace bm {
namespace sol {
// Set-up of bm_coupler_m1_apply_noalloc on the current device, from
// bm_solver_create.
bm_status_t noalloc_setup(int dev) {
    unsigned char* p = nullptr;
    return noalloc_scratch(dev, &p);
}
}  // namespace sol
}  // namespace bm

BM_API bm_status_t bm_coupler_m1_apply_noalloc(bm_solver_t* s, int32_t n_bodies, const bm_collider_t* bodies,
                                               float dt, bm_reaction_t* out) {
    if (!s) return invalid_arg("NULL handle");
    if (n_bodies < 0 || (n_bodies > 0 && (!bodies || !out))) return invalid_arg("bad bodies or reactions");
    if (n_bodies > kNoAllocMaxBodies)
        return invalid_arg("bm_coupler_m1_apply_noalloc takes at most 64 bodies per call (fixed scratch)");
    DeviceGuard dg(s->w.device);
    if (n_bodies > 0) std::memset(out, 0, sizeof(bm_reaction_t) * n_bodies);
    // The grid and the scene table must already exist: building them allocates.
    if (!s->sc().grid_ready || s->w.dirty || (!s->acc_valid && s->sc().n() > 0)) {
        set_last_error("bm_coupler_m1_apply_noalloc needs the grid of bm_solver_p2g and bm_solver_grid_update");
        return BM_ERR_STATE;
    }
    if (n_bodies == 0) return BM_OK;
    unsigned char* base = nullptr;
    bm_status_t st = noalloc_scratch(s->w.device, &base);
    if (st != BM_OK) return st;
    double* acc = reinterpret_cast<double*>(base + kNoAllocAccOff);
    M1Params* params = reinterpret_cast<M1Params*>(base + kNoAllocParamOff);
    bm_reaction_t* react = reinterpret_cast<bm_reaction_t*>(base + kNoAllocReactOff);

    M1Params hp[kNoAllocMaxBodies];
    for (int b = 0; b < n_bodies; ++b) m1_prepare(s->sc().dev.g, bodies[b], dt, 0, &hp[b]);
    cudaStream_t stream = s->w.stream;
    // the reaction sums start at zero on every call
    BM_CHECK_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 7 * n_bodies, stream));
    BM_CHECK_CUDA(cudaMemcpyAsync(params, hp, sizeof(M1Params) * n_bodies, cudaMemcpyHostToDevice, stream));
    // one launch per body, in order: a body sees the grid its predecessors
    // projected, as the reference's couplers applied one after another do
    for (int b = 0; b < n_bodies; ++b)
        if (hp[b].active)
            launch_m1(s->w.table(), params + b, 1, (int64_t)hp[b].nbi * hp[b].nbj * hp[b].nbk, s->w.cur,
                      acc + 7 * b, stream);
    launch_reaction_finalize(acc, n_bodies, react, stream);
    s->view = s->w.cur;
    st = launch_status("m1 (no-alloc)");
    if (st != BM_OK) return st;
    BM_CHECK_CUDA(cudaMemcpyAsync(out, react, sizeof(bm_reaction_t) * n_bodies, cudaMemcpyDeviceToHost, stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(stream));
    return BM_OK;
}
