// bm_solver.cu — the bm_solver_* C ABI: particle store, dense grid, stream.
//
// Mirrors the reference MPMSolver (include/basements/physics/mpm/mpm_solver.h:15-95):
// same parameter defaults (:100-109), the same V0 = m / rho rule and its
// rescale on set_material (:28-51), the same step order (:71-87). The store
// is device-resident FP32 SoA; the grid is a dense box of 4^3-node blocks
// sized once (explicitly, or from the particle bounds at the first step).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "bm_internal.h"

namespace bm {

static thread_local std::string g_last_error;
void set_last_error(const std::string& s) { g_last_error = s; }

}  // namespace bm

using namespace bm;

namespace {

struct ProfileSlot {
    const char* name;
    double total_ms = 0;
    int64_t launches = 0;
};

struct PendingEvent {
    int slot;
    cudaEvent_t a, b;
};

}  // namespace

struct bm_solver {
    int device = 0;
    cudaStream_t stream = nullptr;
    float dx = 0.1f;
    // Material (mpm_solver.h:100-109 defaults).
    float alpha = 0.40f, E = 1.0e5f, nu = 0.3f, density = 1500.0f, floor_friction = 0.4f;
    float gravity[3] = {0.0f, -9.81f, 0.0f};
    // Particles (two stores: the bin sort permutes from one into the other).
    ParticleSoA ps{nullptr, nullptr, 0, 0};
    ParticleSoA ps_alt{nullptr, nullptr, 0, 0};
    int32_t* d_inv = nullptr;  // add order -> stored slot (scratch for set_particles)
    double bbox_lo[3] = {1e300, 1e300, 1e300}, bbox_hi[3] = {-1e300, -1e300, -1e300};
    // Grid.
    bool domain_set = false;
    bm_domain_t domain{};
    int32_t margin = 16;
    bool grid_ready = false;
    GridDesc g{};
    GridAcc acc[2]{};
    uint8_t* alloc = nullptr;
    int cur = 0;           // accumulation buffer of the current step
    int view = 0;          // buffer that holds the grid a caller sees after the last call
    bool acc_valid = false;  // acc[cur] holds P2G of the current particle state
    bool folded[2] = {false, false};  // acc[b].mv holds momentum + force * fold_dt[b]
    float fold_dt[2] = {0.0f, 0.0f};
    // Binned order.
    BinBuffers bins{};
    bool bins_valid = false;
    int32_t sort_interval = 16;
    int64_t steps_since_sort = 0;
    int num_sms = 148;
    bool fast_math = false;
    // Status.
    uint32_t* d_status = nullptr;
    unsigned long long* d_escaped = nullptr;
    // Coupler accumulators and reactions.
    double* d_acc = nullptr;
    bm_reaction_t* d_react = nullptr;
    int react_cap = 0;
    // Profiling.
    bool profiling = false;
    std::vector<ProfileSlot> slots;
    std::vector<PendingEvent> pending;
    std::vector<cudaEvent_t> event_pool;
    cudaEvent_t t0 = nullptr, t1 = nullptr;

    GridBuffers gbuf(int idx) const { return GridBuffers{acc[idx], alloc}; }
};

namespace {

#define BM_CHECK_CUDA(expr)                                                                       \
    do {                                                                                          \
        cudaError_t e__ = (expr);                                                                 \
        if (e__ != cudaSuccess) {                                                                 \
            set_last_error(std::string(#expr) + ": " + cudaGetErrorString(e__));                  \
            return e__ == cudaErrorMemoryAllocation ? BM_ERR_OUT_OF_MEMORY : BM_ERR_CUDA;         \
        }                                                                                         \
    } while (0)

bm_status_t invalid(const char* what) {
    set_last_error(what);
    return BM_ERR_INVALID_ARGUMENT;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

Material material_of(const bm_solver* s) {
    Material m;
    m.mu = s->E / (2.0f * (1.0f + s->nu));
    m.lambda = s->E * s->nu / ((1.0f + s->nu) * (1.0f - 2.0f * s->nu));
    const float koh = (3.0f * m.lambda + 2.0f * m.mu) / (2.0f * m.mu);
    m.neg_alpha_koh = -s->alpha * koh;
    m.floor_friction = s->floor_friction;
    m.gx = s->gravity[0];
    m.gy = s->gravity[1];
    m.gz = s->gravity[2];
    return m;
}

int floor_div4(int v) { return (v >= 0) ? (v / 4) : -((-v + 3) / 4); }

GridDesc desc_from_domain(const bm_domain_t& d, float dx) {
    GridDesc g{};
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = floor_div4(d.origin[a]) * 4;
        hi[a] = (floor_div4(d.origin[a] + d.extent[a] + 3)) * 4;
    }
    g.ox = lo[0]; g.oy = lo[1]; g.oz = lo[2];
    g.nbx = (hi[0] - lo[0]) / 4; g.nby = (hi[1] - lo[1]) / 4; g.nbz = (hi[2] - lo[2]) / 4;
    g.dx = dx;
    g.inv_dx = 1.0f / dx;
    return g;
}

// Time a launch with CUDA events on the handle's stream when profiling is on.
template <class Fn>
void timed(bm_solver* s, const char* name, Fn&& fn) {
    if (!s->profiling) {
        fn();
        return;
    }
    int slot = -1;
    for (size_t i = 0; i < s->slots.size(); ++i)
        if (std::strcmp(s->slots[i].name, name) == 0) slot = (int)i;
    if (slot < 0) {
        s->slots.push_back(ProfileSlot{name});
        slot = (int)s->slots.size() - 1;
    }
    auto get_event = [&]() {
        cudaEvent_t e;
        if (!s->event_pool.empty()) {
            e = s->event_pool.back();
            s->event_pool.pop_back();
        } else {
            cudaEventCreate(&e);
        }
        return e;
    };
    PendingEvent pe{slot, get_event(), get_event()};
    cudaEventRecord(pe.a, s->stream);
    fn();
    cudaEventRecord(pe.b, s->stream);
    s->pending.push_back(pe);
    if (s->pending.size() > 4096) {  // fold finished timings to bound the pool
        cudaEventSynchronize(s->pending.back().b);
        for (auto& p : s->pending) {
            float ms = 0;
            cudaEventElapsedTime(&ms, p.a, p.b);
            s->slots[p.slot].total_ms += ms;
            s->slots[p.slot].launches += 1;
            s->event_pool.push_back(p.a);
            s->event_pool.push_back(p.b);
        }
        s->pending.clear();
    }
}

bm_status_t alloc_store(bm_solver* s, ParticleSoA* ps, int64_t cap) {
    BM_CHECK_CUDA(cudaMallocAsync((void**)&ps->base, sizeof(float) * N_PLANES * cap, s->stream));
    BM_CHECK_CUDA(cudaMallocAsync((void**)&ps->pid, sizeof(int32_t) * cap, s->stream));
    ps->cap = cap;
    return BM_OK;
}

void free_store(bm_solver* s, ParticleSoA* ps) {
    if (ps->base) cudaFreeAsync(ps->base, s->stream);
    if (ps->pid) cudaFreeAsync(ps->pid, s->stream);
    ps->base = nullptr;
    ps->pid = nullptr;
    ps->cap = 0;
}

bm_status_t ensure_particle_capacity(bm_solver* s, int64_t need) {
    if (need <= s->ps.cap) return BM_OK;
    if (need > INT32_MAX) return invalid("more than 2^31-1 particles");
    int64_t cap = std::max<int64_t>(need, std::max<int64_t>(1024, s->ps.cap * 3 / 2));
    cap = (cap + 31) / 32 * 32;
    ParticleSoA nb{nullptr, nullptr, 0, s->ps.n};
    bm_status_t st = alloc_store(s, &nb, cap);
    if (st != BM_OK) return st;
    if (s->ps.base && s->ps.n > 0) {
        for (int p = 0; p < N_PLANES; ++p)
            BM_CHECK_CUDA(cudaMemcpyAsync(nb.plane(p), s->ps.plane(p), sizeof(float) * s->ps.n,
                                          cudaMemcpyDeviceToDevice, s->stream));
        BM_CHECK_CUDA(cudaMemcpyAsync(nb.pid, s->ps.pid, sizeof(int32_t) * s->ps.n, cudaMemcpyDeviceToDevice,
                                      s->stream));
    }
    free_store(s, &s->ps);
    free_store(s, &s->ps_alt);
    if (s->d_inv) cudaFreeAsync(s->d_inv, s->stream);
    s->d_inv = nullptr;
    s->ps = nb;
    ParticleSoA alt{nullptr, nullptr, 0, s->ps.n};
    st = alloc_store(s, &alt, cap);
    if (st != BM_OK) return st;
    s->ps_alt = alt;
    BM_CHECK_CUDA(cudaMallocAsync((void**)&s->d_inv, sizeof(int32_t) * cap, s->stream));
    return BM_OK;
}

bm_status_t ensure_grid(bm_solver* s) {
    if (s->grid_ready) return BM_OK;
    if (!s->domain_set) {
        if (s->ps.n == 0) return invalid("grid box unknown: no particles and no bm_solver_set_domain");
        bm_domain_t d;
        for (int a = 0; a < 3; ++a) {
            const int lo = (int)std::floor(s->bbox_lo[a] / s->dx - 0.5) - s->margin;
            const int hi = (int)std::floor(s->bbox_hi[a] / s->dx - 0.5) + 3 + s->margin;
            d.origin[a] = lo;
            d.extent[a] = hi - lo;
        }
        s->domain = d;
        s->domain_set = true;
    }
    s->g = desc_from_domain(s->domain, s->dx);
    const int64_t nn = s->g.num_nodes(), nb = s->g.num_blocks();
    if (nb > INT32_MAX / 64) return invalid("grid box too large");
    for (int b = 0; b < 2; ++b) {
        GridAcc& a = s->acc[b];
        BM_CHECK_CUDA(cudaMallocAsync((void**)&a.mv, sizeof(float4) * nn, s->stream));
        BM_CHECK_CUDA(cudaMallocAsync((void**)&a.f, sizeof(float4) * nn, s->stream));
        BM_CHECK_CUDA(cudaMallocAsync((void**)&a.touched, sizeof(uint32_t) * nb, s->stream));
        BM_CHECK_CUDA(cudaMallocAsync((void**)&a.list, sizeof(int32_t) * nb, s->stream));
        BM_CHECK_CUDA(cudaMallocAsync((void**)&a.count, sizeof(int32_t), s->stream));
        BM_CHECK_CUDA(cudaMemsetAsync(a.mv, 0, sizeof(float4) * nn, s->stream));
        BM_CHECK_CUDA(cudaMemsetAsync(a.f, 0, sizeof(float4) * nn, s->stream));
        BM_CHECK_CUDA(cudaMemsetAsync(a.touched, 0, sizeof(uint32_t) * nb, s->stream));
        BM_CHECK_CUDA(cudaMemsetAsync(a.count, 0, sizeof(int32_t), s->stream));
    }
    BM_CHECK_CUDA(cudaMallocAsync((void**)&s->alloc, (size_t)nb, s->stream));
    BM_CHECK_CUDA(cudaMemsetAsync(s->alloc, 0, (size_t)nb, s->stream));
    BinBuffers& bb = s->bins;
    bb.nkeys = nn;
    BM_CHECK_CUDA(cudaMallocAsync((void**)&bb.count, sizeof(int32_t) * (nn + 1), s->stream));
    BM_CHECK_CUDA(cudaMallocAsync((void**)&bb.start, sizeof(int32_t) * (nn + 2), s->stream));
    BM_CHECK_CUDA(cudaMallocAsync((void**)&bb.tile_sum, sizeof(int64_t) * scan_tiles(nn), s->stream));
    s->grid_ready = true;
    return BM_OK;
}

bm_status_t ensure_bin_keys(bm_solver* s) {
    if (s->bins.key && s->bins.key_cap >= s->ps.cap) return BM_OK;
    if (s->bins.key) cudaFreeAsync(s->bins.key, s->stream);
    if (s->bins.rank) cudaFreeAsync(s->bins.rank, s->stream);
    BM_CHECK_CUDA(cudaMallocAsync((void**)&s->bins.key, sizeof(int32_t) * std::max<int64_t>(1, s->ps.cap), s->stream));
    BM_CHECK_CUDA(cudaMallocAsync((void**)&s->bins.rank, sizeof(int32_t) * std::max<int64_t>(1, s->ps.cap), s->stream));
    s->bins.key_cap = s->ps.cap;
    return BM_OK;
}

bm_status_t ensure_reactions(bm_solver* s, int n) {
    if (n <= s->react_cap) return BM_OK;
    if (s->d_acc) cudaFreeAsync(s->d_acc, s->stream);
    if (s->d_react) cudaFreeAsync(s->d_react, s->stream);
    s->d_acc = nullptr;
    s->d_react = nullptr;
    BM_CHECK_CUDA(cudaMallocAsync((void**)&s->d_acc, sizeof(double) * 7 * n, s->stream));
    BM_CHECK_CUDA(cudaMallocAsync((void**)&s->d_react, sizeof(bm_reaction_t) * n, s->stream));
    s->react_cap = n;
    return BM_OK;
}

bm_status_t launch_error(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string(where) + ": " + cudaGetErrorString(e));
        return BM_ERR_CUDA;
    }
    return BM_OK;
}

// Standalone P2G of the current particle state into acc[cur] (grid.clear()
// + the P2G loop).
bm_status_t do_p2g(bm_solver* s) {
    bm_status_t st = ensure_grid(s);
    if (st != BM_OK) return st;
    const int64_t nn = s->g.num_nodes(), nb = s->g.num_blocks();
    GridAcc& a = s->acc[s->cur];
    timed(s, "grid_clear", [&] {
        cudaMemsetAsync(a.mv, 0, sizeof(float4) * nn, s->stream);
        cudaMemsetAsync(a.f, 0, sizeof(float4) * nn, s->stream);
        cudaMemsetAsync(a.touched, 0, sizeof(uint32_t) * nb, s->stream);
        cudaMemsetAsync(a.count, 0, sizeof(int32_t), s->stream);
    });
    const Material m = material_of(s);
    timed(s, "p2g", [&] { launch_p2g(s->ps, s->g, s->gbuf(s->cur), m, s->d_status, s->d_escaped, s->stream); });
    s->acc_valid = true;
    s->folded[s->cur] = false;
    s->view = s->cur;
    return launch_error("p2g");
}

bm_status_t do_grid_update(bm_solver* s, float dt) {
    if (!s->grid_ready || !s->acc_valid) {
        set_last_error("grid_update needs the P2G of the current particle state (call p2g first)");
        return BM_ERR_STATE;
    }
    const Material m = material_of(s);
    GridAcc& other = s->acc[1 - s->cur];
    if (s->folded[s->cur] && dt != s->fold_dt[s->cur]) {
        set_last_error("grid_update dt differs from the dt folded into the precomputed P2G");
        return BM_ERR_STATE;
    }
    timed(s, "grid_update", [&] {
        launch_grid_update(s->g, s->acc[s->cur], other, m, dt, s->folded[s->cur], s->g.num_blocks(), s->stream);
        cudaMemsetAsync(other.count, 0, sizeof(int32_t), s->stream);
    });
    s->view = s->cur;
    return launch_error("grid_update");
}

// G2P alone (split API): the particles advance, acc[cur] keeps this step's grid.
bm_status_t do_g2p(bm_solver* s, float dt) {
    if (!s->grid_ready || !s->acc_valid) {
        set_last_error("g2p needs a grid from p2g / grid_update");
        return BM_ERR_STATE;
    }
    const Material m = material_of(s);
    timed(s, "g2p", [&] {
        launch_g2p(s->ps, s->g, s->gbuf(s->cur), m, dt, s->d_status, s->d_escaped, s->stream);
    });
    s->acc_valid = false;
    s->view = s->cur;
    return launch_error("g2p");
}

bm_status_t do_m1(bm_solver* s, const bm_collider_t* body, float dt, int slot) {
    M1Params P;
    const bool any = m1_prepare(s->g, *body, dt, &P);
    BM_CHECK_CUDA(cudaMemsetAsync(s->d_acc + 7 * slot, 0, sizeof(double) * 7, s->stream));
    if (any) timed(s, "m1_coupler", [&] { launch_m1(s->g, s->gbuf(s->cur), P, s->d_acc + 7 * slot, s->stream); });
    return launch_error("m1");
}

// G2P of this step fused with the P2G of the next one (into the other
// buffer); re-bins the particles first when due.
bm_status_t do_g2p2g(bm_solver* s, float dt) {
    if (s->ps.n > 0) {
        bm_status_t st = ensure_bin_keys(s);
        if (st != BM_OK) return st;
        if (!s->bins_valid || (s->sort_interval > 0 && s->steps_since_sort >= s->sort_interval)) {
            timed(s, "bin_sort", [&] {
                ParticleSoA dst = s->ps_alt;
                dst.n = s->ps.n;
                launch_bin_sort(s->ps, dst, s->g, s->bins, s->stream);
            });
            std::swap(s->ps, s->ps_alt);
            s->ps.n = s->ps_alt.n;
            s->bins_valid = true;
            s->steps_since_sort = 0;
            st = launch_error("bin_sort");
            if (st != BM_OK) return st;
        }
    }
    const Material m = material_of(s);
    const int next = 1 - s->cur;
    timed(s, "g2p2g", [&] {
        launch_g2p2g(s->ps, s->g, s->acc[s->cur], s->acc[next], s->alloc, m, dt, dt, s->fast_math, s->d_status,
                     s->d_escaped, s->stream);
    });
    s->folded[next] = true;
    s->fold_dt[next] = dt;
    s->view = s->cur;
    s->cur = next;
    s->acc_valid = true;
    s->steps_since_sort += 1;
    return launch_error("g2p2g");
}

// One step on the fused path: [P2G if not precomputed], update, couplers, G2P+P2G.
bm_status_t do_step(bm_solver* s, float dt, int32_t n_bodies, const bm_collider_t* bodies) {
    bm_status_t st = ensure_grid(s);
    // the precomputed P2G folded the previous dt into the momentum: redo it
    // (unfolded) when this step uses another dt
    if (st == BM_OK && s->acc_valid && s->folded[s->cur] && dt != s->fold_dt[s->cur]) s->acc_valid = false;
    if (st == BM_OK && !s->acc_valid) st = do_p2g(s);
    if (st == BM_OK) st = do_grid_update(s, dt);
    for (int32_t b = 0; st == BM_OK && b < n_bodies; ++b) st = do_m1(s, bodies + b, dt, b);
    if (st == BM_OK && n_bodies > 0) launch_reaction_finalize(s->d_acc, n_bodies, s->d_react, s->stream);
    if (st == BM_OK) st = do_g2p2g(s, dt);
    return st;
}

void invalidate_state(bm_solver* s) {
    s->acc_valid = false;
    s->bins_valid = false;
}

void update_bbox(bm_solver* s, int64_t n, const float* pos) {
    for (int64_t p = 0; p < n; ++p)
        for (int a = 0; a < 3; ++a) {
            const double v = pos[3 * p + a];
            if (!std::isfinite(v)) continue;
            s->bbox_lo[a] = std::min(s->bbox_lo[a], v);
            s->bbox_hi[a] = std::max(s->bbox_hi[a], v);
        }
}

}  // namespace

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

BM_API const char* bm_last_error(void) { return g_last_error.c_str(); }

BM_API bm_status_t bm_set_device(int32_t device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_last_error("no CUDA device");
        return BM_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return invalid("device index out of range");
    BM_CHECK_CUDA(cudaSetDevice(device));
    return BM_OK;
}

BM_API bm_status_t bm_solver_create(float dx, const bm_domain_t* domain, bm_solver_t** out) {
    if (!out) return invalid("out is NULL");
    *out = nullptr;
    if (!(dx > 0.0f) || !std::isfinite(dx)) return invalid("dx must be a positive finite number");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_last_error("no CUDA device");
        return BM_ERR_NO_DEVICE;
    }
    bm_solver* s = new bm_solver();
    cudaGetDevice(&s->device);
    cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device);
    s->dx = dx;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_last_error("cudaStreamCreate failed");
        delete s;
        return BM_ERR_CUDA;
    }
    cudaError_t e1 = cudaMalloc((void**)&s->d_status, sizeof(uint32_t));
    cudaError_t e2 = cudaMalloc((void**)&s->d_escaped, sizeof(unsigned long long));
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        set_last_error("status allocation failed");
        bm_solver_destroy(s);
        return BM_ERR_OUT_OF_MEMORY;
    }
    cudaMemsetAsync(s->d_status, 0, sizeof(uint32_t), s->stream);
    cudaMemsetAsync(s->d_escaped, 0, sizeof(unsigned long long), s->stream);
    if (domain) {
        for (int a = 0; a < 3; ++a)
            if (domain->extent[a] <= 0) {
                bm_solver_destroy(s);
                return invalid("domain extent must be positive");
            }
        s->domain = *domain;
        s->domain_set = true;
    }
    if (ensure_reactions(s, 4) != BM_OK) {
        bm_solver_destroy(s);
        return BM_ERR_OUT_OF_MEMORY;
    }
    *out = s;
    return BM_OK;
}

BM_API bm_status_t bm_solver_destroy(bm_solver_t* s) {
    if (!s) return invalid("NULL handle");
    DeviceGuard dg(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& p : s->pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : s->event_pool) cudaEventDestroy(e);
    if (s->t0) cudaEventDestroy(s->t0);
    if (s->t1) cudaEventDestroy(s->t1);
    for (ParticleSoA* p : {&s->ps, &s->ps_alt}) {
        cudaFree(p->base);
        cudaFree(p->pid);
    }
    cudaFree(s->d_inv);
    for (GridAcc& a : s->acc) {
        cudaFree(a.mv);
        cudaFree(a.f);
        cudaFree(a.touched);
        cudaFree(a.list);
        cudaFree(a.count);
    }
    cudaFree(s->alloc);
    for (void* p : {(void*)s->bins.key, (void*)s->bins.rank, (void*)s->bins.count, (void*)s->bins.start,
                    (void*)s->bins.tile_sum})
        cudaFree(p);
    cudaFree(s->d_status);
    cudaFree(s->d_escaped);
    cudaFree(s->d_acc);
    cudaFree(s->d_react);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_domain(bm_solver_t* s, const bm_domain_t* d) {
    if (!s || !d) return invalid("NULL argument");
    if (s->grid_ready) {
        set_last_error("the grid box is fixed once the grid has been used");
        return BM_ERR_STATE;
    }
    for (int a = 0; a < 3; ++a)
        if (d->extent[a] <= 0) return invalid("domain extent must be positive");
    s->domain = *d;
    s->domain_set = true;
    return BM_OK;
}

BM_API bm_status_t bm_solver_get_domain(bm_solver_t* s, bm_domain_t* out) {
    if (!s || !out) return invalid("NULL argument");
    DeviceGuard dg(s->device);
    bm_status_t st = ensure_grid(s);
    if (st != BM_OK) return st;
    out->origin[0] = s->g.ox; out->origin[1] = s->g.oy; out->origin[2] = s->g.oz;
    out->extent[0] = s->g.nbx * 4; out->extent[1] = s->g.nby * 4; out->extent[2] = s->g.nbz * 4;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_auto_margin(bm_solver_t* s, int32_t margin) {
    if (!s || margin < 0) return invalid("bad margin");
    s->margin = margin;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_sort_interval(bm_solver_t* s, int32_t steps) {
    if (!s || steps < 0) return invalid("bad sort interval");
    s->sort_interval = steps;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_math_mode(bm_solver_t* s, int32_t mode) {
    if (!s || mode < 0 || mode > 1) return invalid("math mode must be 0 (IEEE) or 1 (fast)");
    s->fast_math = mode == 1;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_material(bm_solver_t* s, float E, float nu, float rho) {
    if (!s) return invalid("NULL handle");
    if (!std::isfinite(E) || !std::isfinite(nu) || !std::isfinite(rho)) return invalid("non-finite material");
    DeviceGuard dg(s->device);
    s->E = E;
    s->nu = nu;
    if (rho > 1e-12f && s->density > 1e-12f && rho != s->density && s->ps.n > 0) {
        // V0 *= rho_old / rho_new for every particle (mpm_solver.h:45-49).
        const float rescale = s->density / rho;
        std::vector<float> v0(s->ps.n);
        BM_CHECK_CUDA(cudaMemcpyAsync(v0.data(), s->ps.plane(P_V0), sizeof(float) * s->ps.n, cudaMemcpyDeviceToHost,
                                      s->stream));
        BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
        for (auto& x : v0) x *= rescale;
        BM_CHECK_CUDA(cudaMemcpyAsync(s->ps.plane(P_V0), v0.data(), sizeof(float) * s->ps.n, cudaMemcpyHostToDevice,
                                      s->stream));
        BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    }
    s->density = rho;
    s->acc_valid = false;  // the precomputed P2G used the old stress
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_gravity(bm_solver_t* s, const float g[3]) {
    if (!s || !g) return invalid("NULL argument");
    for (int a = 0; a < 3; ++a) s->gravity[a] = g[a];
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_plastic_alpha(bm_solver_t* s, float a) {
    if (!s) return invalid("NULL handle");
    s->alpha = a;
    return BM_OK;
}

BM_API bm_status_t bm_solver_set_floor_friction(bm_solver_t* s, float mu) {
    if (!s) return invalid("NULL handle");
    s->floor_friction = mu;
    return BM_OK;
}

BM_API bm_status_t bm_solver_add_particles(bm_solver_t* s, int64_t n, const float* pos, const float* vel,
                                           const float* mass) {
    if (!s) return invalid("NULL handle");
    if (n < 0) return invalid("n < 0");
    if (n == 0) return BM_OK;
    if (!pos) return invalid("position is NULL");
    DeviceGuard dg(s->device);
    const int64_t n0 = s->ps.n;
    bm_status_t st = ensure_particle_capacity(s, n0 + n);
    if (st != BM_OK) return st;
    // Host staging of the new rows, plane by plane (SoA), appended in add order.
    std::vector<float> buf((size_t)n * N_PLANES);
    std::vector<int32_t> pid((size_t)n);
    auto col = [&](int p) { return buf.data() + (size_t)p * n; };
    for (int64_t q = 0; q < n; ++q) {
        for (int a = 0; a < 3; ++a) {
            col(P_X + a)[q] = pos[3 * q + a];
            col(P_V + a)[q] = vel ? vel[3 * q + a] : 0.0f;
        }
        for (int a = 0; a < 9; ++a) {
            col(P_F + a)[q] = (a % 4 == 0) ? 1.0f : 0.0f;
            col(P_C + a)[q] = 0.0f;
        }
        const float m = mass ? mass[q] : 1.0f;
        col(P_M)[q] = m;
        col(P_V0)[q] = (s->density > 1e-12f) ? (m / s->density) : 1.0f;
        pid[q] = (int32_t)(n0 + q);
    }
    for (int p = 0; p < N_PLANES; ++p)
        BM_CHECK_CUDA(cudaMemcpyAsync(s->ps.plane(p) + n0, col(p), sizeof(float) * n, cudaMemcpyHostToDevice,
                                      s->stream));
    BM_CHECK_CUDA(cudaMemcpyAsync(s->ps.pid + n0, pid.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice,
                                  s->stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    s->ps.n = n0 + n;
    s->ps_alt.n = s->ps.n;
    update_bbox(s, n, pos);
    invalidate_state(s);
    return BM_OK;
}

BM_API bm_status_t bm_solver_num_particles(bm_solver_t* s, int64_t* out) {
    if (!s || !out) return invalid("NULL argument");
    *out = s->ps.n;
    return BM_OK;
}

BM_API bm_status_t bm_solver_get_particles(bm_solver_t* s, const bm_particles_view_t* v) {
    if (!s || !v) return invalid("NULL argument");
    DeviceGuard dg(s->device);
    const int64_t n = s->ps.n;
    if (n == 0) return BM_OK;
    struct Field { float* dst; int plane; int width; };
    const Field fields[] = {{v->position, P_X, 3}, {v->velocity, P_V, 3}, {v->F, P_F, 9},
                            {v->C, P_C, 9},        {v->mass, P_M, 1},     {v->volume, P_V0, 1}};
    float* tmp = nullptr;
    BM_CHECK_CUDA(cudaMallocAsync((void**)&tmp, sizeof(float) * 9 * n, s->stream));
    bm_status_t st = BM_OK;
    for (const Field& f : fields) {
        if (!f.dst) continue;
        launch_gather_rows(s->ps, f.plane, f.width, tmp, s->stream);
        if (cudaMemcpyAsync(f.dst, tmp, sizeof(float) * f.width * n, cudaMemcpyDeviceToHost, s->stream) !=
            cudaSuccess)
            st = BM_ERR_CUDA;
    }
    cudaFreeAsync(tmp, s->stream);
    BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    if (st != BM_OK) set_last_error("device-to-host copy of particles failed");
    return st;
}

BM_API bm_status_t bm_solver_set_particles(bm_solver_t* s, int64_t first, int64_t n, const bm_particles_view_t* v) {
    if (!s || !v) return invalid("NULL argument");
    if (first < 0 || n < 0 || first + n > s->ps.n) return invalid("particle range out of bounds");
    if (n == 0) return BM_OK;
    DeviceGuard dg(s->device);
    struct Field { const float* src; int plane; int width; };
    const Field fields[] = {{v->position, P_X, 3}, {v->velocity, P_V, 3}, {v->F, P_F, 9}, {v->C, P_C, 9}};
    float* tmp = nullptr;
    BM_CHECK_CUDA(cudaMallocAsync((void**)&tmp, sizeof(float) * 9 * n, s->stream));
    launch_inverse_pid(s->ps, s->d_inv, s->stream);
    for (const Field& f : fields) {
        if (!f.src) continue;
        cudaMemcpyAsync(tmp, f.src, sizeof(float) * f.width * n, cudaMemcpyHostToDevice, s->stream);
        launch_scatter_rows(s->ps, f.plane, f.width, tmp, first, n, s->d_inv, s->stream);
    }
    cudaFreeAsync(tmp, s->stream);
    BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    if (v->position) update_bbox(s, n, v->position);
    invalidate_state(s);
    return launch_error("set_particles");
}

BM_API bm_status_t bm_solver_step(bm_solver_t* s, float dt) {
    if (!s) return invalid("NULL handle");
    if (!std::isfinite(dt)) return invalid("dt is not finite");
    DeviceGuard dg(s->device);
    return do_step(s, dt, 0, nullptr);
}

BM_API bm_status_t bm_solver_step_n(bm_solver_t* s, float dt, int32_t n_steps) {
    if (!s) return invalid("NULL handle");
    if (n_steps < 0) return invalid("n_steps < 0");
    for (int32_t i = 0; i < n_steps; ++i) {
        bm_status_t st = bm_solver_step(s, dt);
        if (st != BM_OK) return st;
    }
    return BM_OK;
}

BM_API bm_status_t bm_solver_p2g(bm_solver_t* s, float dt) {
    if (!s) return invalid("NULL handle");
    (void)dt;  // P2G does not depend on dt (mpm_solver.h:168)
    DeviceGuard dg(s->device);
    return do_p2g(s);
}

BM_API bm_status_t bm_solver_grid_update(bm_solver_t* s, float dt) {
    if (!s) return invalid("NULL handle");
    DeviceGuard dg(s->device);
    return do_grid_update(s, dt);
}

BM_API bm_status_t bm_solver_g2p(bm_solver_t* s, float dt) {
    if (!s) return invalid("NULL handle");
    DeviceGuard dg(s->device);
    return do_g2p(s, dt);
}

BM_API bm_status_t bm_coupler_m1_apply(bm_solver_t* s, const bm_collider_t* body, float dt, bm_reaction_t* out) {
    if (!s || !body || !out) return invalid("NULL argument");
    DeviceGuard dg(s->device);
    std::memset(out, 0, sizeof(*out));
    bm_status_t st = ensure_grid(s);
    if (st != BM_OK) return st;
    if (!s->acc_valid && s->ps.n > 0) {
        set_last_error("the coupler needs a grid from p2g / grid_update");
        return BM_ERR_STATE;
    }
    st = do_m1(s, body, dt, 0);
    if (st != BM_OK) return st;
    launch_reaction_finalize(s->d_acc, 1, s->d_react, s->stream);
    BM_CHECK_CUDA(cudaMemcpyAsync(out, s->d_react, sizeof(bm_reaction_t), cudaMemcpyDeviceToHost, s->stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    return BM_OK;
}

BM_API bm_status_t bm_solver_step_coupled(bm_solver_t* s, float dt, int32_t n_bodies, const bm_collider_t* bodies,
                                          bm_reaction_t* reactions) {
    if (!s) return invalid("NULL handle");
    if (n_bodies < 0 || (n_bodies > 0 && !bodies)) return invalid("bad bodies");
    if (!std::isfinite(dt)) return invalid("dt is not finite");
    DeviceGuard dg(s->device);
    bm_status_t st = ensure_reactions(s, std::max(1, n_bodies));
    if (st == BM_OK) st = do_step(s, dt, n_bodies, bodies);
    if (st == BM_OK && reactions && n_bodies > 0) {
        BM_CHECK_CUDA(cudaMemcpyAsync(reactions, s->d_react, sizeof(bm_reaction_t) * n_bodies,
                                      cudaMemcpyDeviceToHost, s->stream));
        BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    }
    return st;
}

BM_API bm_status_t bm_solver_get_reactions(bm_solver_t* s, int32_t n, bm_reaction_t* out) {
    if (!s || !out || n < 0 || n > s->react_cap) return invalid("bad arguments");
    DeviceGuard dg(s->device);
    if (n == 0) return BM_OK;
    BM_CHECK_CUDA(cudaMemcpyAsync(out, s->d_react, sizeof(bm_reaction_t) * n, cudaMemcpyDeviceToHost, s->stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    return BM_OK;
}

BM_API bm_status_t bm_solver_grid_num_nodes(bm_solver_t* s, int64_t* out) {
    if (!s || !out) return invalid("NULL argument");
    DeviceGuard dg(s->device);
    bm_status_t st = ensure_grid(s);
    if (st != BM_OK) return st;
    *out = s->g.num_nodes();
    return BM_OK;
}

BM_API bm_status_t bm_solver_get_grid(bm_solver_t* s, float* vel, float* force, float* mass, uint8_t* active,
                                      uint8_t* balloc) {
    if (!s) return invalid("NULL handle");
    DeviceGuard dg(s->device);
    bm_status_t st = ensure_grid(s);
    if (st != BM_OK) return st;
    const int64_t nn = s->g.num_nodes();
    if (force && s->folded[s->view]) {
        // after a fused step the force is folded into the momentum (see header)
        std::memset(force, 0, sizeof(float) * 3 * nn);
        force = nullptr;
    }
    float *dv = nullptr, *df = nullptr, *dm = nullptr;
    uint8_t *da = nullptr, *db = nullptr;
    if (vel) BM_CHECK_CUDA(cudaMallocAsync((void**)&dv, sizeof(float) * 3 * nn, s->stream));
    if (force) BM_CHECK_CUDA(cudaMallocAsync((void**)&df, sizeof(float) * 3 * nn, s->stream));
    if (mass) BM_CHECK_CUDA(cudaMallocAsync((void**)&dm, sizeof(float) * nn, s->stream));
    if (active) BM_CHECK_CUDA(cudaMallocAsync((void**)&da, (size_t)nn, s->stream));
    if (balloc) BM_CHECK_CUDA(cudaMallocAsync((void**)&db, (size_t)nn, s->stream));
    launch_grid_to_dense(s->g, s->gbuf(s->view), dv, df, dm, da, db, s->stream);
    st = launch_error("grid_to_dense");
    if (vel) cudaMemcpyAsync(vel, dv, sizeof(float) * 3 * nn, cudaMemcpyDeviceToHost, s->stream);
    if (force) cudaMemcpyAsync(force, df, sizeof(float) * 3 * nn, cudaMemcpyDeviceToHost, s->stream);
    if (mass) cudaMemcpyAsync(mass, dm, sizeof(float) * nn, cudaMemcpyDeviceToHost, s->stream);
    if (active) cudaMemcpyAsync(active, da, (size_t)nn, cudaMemcpyDeviceToHost, s->stream);
    if (balloc) cudaMemcpyAsync(balloc, db, (size_t)nn, cudaMemcpyDeviceToHost, s->stream);
    for (void* p : {(void*)dv, (void*)df, (void*)dm, (void*)da, (void*)db})
        if (p) cudaFreeAsync(p, s->stream);
    BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    return st;
}

BM_API bm_status_t bm_solver_seed_grid(bm_solver_t* s, int64_t n, const int32_t* ijk, const float* vel,
                                       const float* mass) {
    if (!s) return invalid("NULL handle");
    if (n < 0 || (n > 0 && (!ijk || !vel || !mass))) return invalid("bad seed arrays");
    DeviceGuard dg(s->device);
    bm_status_t st = ensure_grid(s);
    if (st != BM_OK) return st;
    if (n == 0) return BM_OK;
    for (int64_t q = 0; q < n; ++q)
        if (s->g.node(ijk[3 * q], ijk[3 * q + 1], ijk[3 * q + 2]) < 0) return invalid("seed node outside the box");
    int32_t* di = nullptr;
    float *dv = nullptr, *dm = nullptr;
    BM_CHECK_CUDA(cudaMallocAsync((void**)&di, sizeof(int32_t) * 3 * n, s->stream));
    BM_CHECK_CUDA(cudaMallocAsync((void**)&dv, sizeof(float) * 3 * n, s->stream));
    BM_CHECK_CUDA(cudaMallocAsync((void**)&dm, sizeof(float) * n, s->stream));
    cudaMemcpyAsync(di, ijk, sizeof(int32_t) * 3 * n, cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(dv, vel, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(dm, mass, sizeof(float) * n, cudaMemcpyHostToDevice, s->stream);
    launch_seed_grid(s->g, s->gbuf(s->cur), n, di, dv, dm, s->d_status, s->stream);
    st = launch_error("seed_grid");
    s->acc_valid = true;  // the seeded grid stands for this step's grid
    s->folded[s->cur] = false;
    s->view = s->cur;
    cudaFreeAsync(di, s->stream);
    cudaFreeAsync(dv, s->stream);
    cudaFreeAsync(dm, s->stream);
    BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    return st;
}

BM_API bm_status_t bm_solver_set_grid_velocity(bm_solver_t* s, const float* vel) {
    if (!s || !vel) return invalid("NULL argument");
    DeviceGuard dg(s->device);
    bm_status_t st = ensure_grid(s);
    if (st != BM_OK) return st;
    const int64_t nn = s->g.num_nodes();
    float* dv = nullptr;
    BM_CHECK_CUDA(cudaMallocAsync((void**)&dv, sizeof(float) * 3 * nn, s->stream));
    cudaMemcpyAsync(dv, vel, sizeof(float) * 3 * nn, cudaMemcpyHostToDevice, s->stream);
    launch_dense_velocity_to_grid(s->g, s->gbuf(s->cur), dv, s->stream);
    st = launch_error("set_grid_velocity");
    cudaFreeAsync(dv, s->stream);
    BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    return st;
}

BM_API bm_status_t bm_solver_sync(bm_solver_t* s, int64_t* escaped) {
    if (!s) return invalid("NULL handle");
    DeviceGuard dg(s->device);
    uint32_t status = 0;
    unsigned long long esc = 0;
    BM_CHECK_CUDA(cudaMemcpyAsync(&status, s->d_status, sizeof(status), cudaMemcpyDeviceToHost, s->stream));
    BM_CHECK_CUDA(cudaMemcpyAsync(&esc, s->d_escaped, sizeof(esc), cudaMemcpyDeviceToHost, s->stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    BM_CHECK_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(uint32_t), s->stream));
    BM_CHECK_CUDA(cudaMemsetAsync(s->d_escaped, 0, sizeof(unsigned long long), s->stream));
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
    if (!s || !stream) return invalid("NULL argument");
    *stream = (void*)s->stream;
    return BM_OK;
}

BM_API bm_status_t bm_solver_profile_enable(bm_solver_t* s, int32_t on) {
    if (!s) return invalid("NULL handle");
    s->profiling = on != 0;
    return BM_OK;
}

BM_API bm_status_t bm_solver_profile_read(bm_solver_t* s, int32_t cap, const char** names, double* total_ms,
                                          int64_t* launches, int32_t* n_out) {
    if (!s || !n_out) return invalid("NULL argument");
    DeviceGuard dg(s->device);
    BM_CHECK_CUDA(cudaStreamSynchronize(s->stream));
    for (auto& p : s->pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        s->slots[p.slot].total_ms += ms;
        s->slots[p.slot].launches += 1;
        s->event_pool.push_back(p.a);
        s->event_pool.push_back(p.b);
    }
    s->pending.clear();
    int32_t n = 0;
    for (const auto& sl : s->slots) {
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
    if (!s) return invalid("NULL handle");
    int32_t n = 0;
    bm_solver_profile_read(s, 0, nullptr, nullptr, nullptr, &n);
    for (auto& sl : s->slots) {
        sl.total_ms = 0;
        sl.launches = 0;
    }
    return BM_OK;
}

BM_API bm_status_t bm_solver_timer_start(bm_solver_t* s) {
    if (!s) return invalid("NULL handle");
    DeviceGuard dg(s->device);
    if (!s->t0) BM_CHECK_CUDA(cudaEventCreate(&s->t0));
    if (!s->t1) BM_CHECK_CUDA(cudaEventCreate(&s->t1));
    BM_CHECK_CUDA(cudaEventRecord(s->t0, s->stream));
    return BM_OK;
}

BM_API bm_status_t bm_solver_timer_stop(bm_solver_t* s, double* ms) {
    if (!s || !ms) return invalid("NULL argument");
    if (!s->t0) return invalid("timer not started");
    DeviceGuard dg(s->device);
    BM_CHECK_CUDA(cudaEventRecord(s->t1, s->stream));
    BM_CHECK_CUDA(cudaEventSynchronize(s->t1));
    float f = 0;
    BM_CHECK_CUDA(cudaEventElapsedTime(&f, s->t0, s->t1));
    *ms = f;
    return BM_OK;
}

}  // extern "C"
