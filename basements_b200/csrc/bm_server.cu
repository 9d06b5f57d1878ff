// bm_server.cu — serving loop with continuous batching.
//
// One worker thread owns a World (bm_world.h) of the co-resident scenes and
// the GPU stream. Each iteration: admit queued requests in order while their
// estimated footprint fits the HBM budget (new scenes get their first P2G
// while the running ones keep their precomputed one), step every co-resident
// scene together (grid update, M1 + rigid update of every body, regrouping
// when due, fused G2P + next P2G: one launch per phase for all scenes), and
// retire the scenes that have done their steps. Latency is measured from
// submit to the moment the result is on the host.
//
// The worker never waits for the GPU while scenes are running: uploads go
// on the World's upload stream, the scene table and the body arrays are
// rebuilt in stream order (the bodies stay on the device and are remapped by
// a kernel when the scene set changes), and a retired scene's particles and
// body are read back into pinned memory behind an event; the request is
// completed when its event has fired.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bm_world.h"

using namespace bm;
using Clock = std::chrono::steady_clock;

namespace {

struct Request {
    int64_t id = 0;
    bm_scene_desc_t desc{};
    std::vector<float> pos, vel, mass;
    int32_t n_steps = 0;
    double bytes = 0;
    int32_t state = BM_REQ_QUEUED;
    bm_status_t error = BM_OK;
    bool cancel = false;
    Clock::time_point t_submit, t_done;
    // read-back in flight: pinned block (x, v, F, C rows, status, body) and
    // the event after its copies
    void* pinned = nullptr;
    size_t pinned_cap = 0;
    cudaEvent_t ready = nullptr;
    // results
    std::vector<float> out_pos, out_vel, out_F, out_C;
    bm_collider_t out_body{};
};

struct Active {
    std::shared_ptr<Request> req;
    int32_t steps_left = 0;
    int body = -1;  // index in the device body arrays
};

double estimate_bytes(const bm_scene_desc_t& d) {
    // particles: two stores of 26 floats + id, and the sort key/rank + the
    // scratch inverse map
    const double per_particle = 2.0 * (N_PLANES * 4 + 4) + 3 * 4;
    double nodes = 0;
    if (d.has_domain) {
        nodes = 1;
        for (int a = 0; a < 3; ++a) nodes *= (double)(d.domain.extent[a] + 8);
    } else if (d.n_particles > 0) {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int64_t p = 0; p < d.n_particles; ++p)
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], (double)d.position[3 * p + a]);
                hi[a] = std::max(hi[a], (double)d.position[3 * p + a]);
            }
        nodes = 1;
        for (int a = 0; a < 3; ++a) nodes *= std::floor((hi[a] - lo[a]) / d.dx) + 3 + 2 * 16 + 8;
    }
    // two accumulators (2 float4 each), per-block flags and lists, sort keys
    const double per_node = 2 * 32 + 8 + 17.0 / 64;
    return per_particle * (double)d.n_particles + per_node * nodes + (1 << 16);
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)std::floor(pos);
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

size_t up16(size_t b) { return (b + 15) & ~size_t(15); }

// Byte layout of a read-back block for n particles.
struct Layout {
    size_t rows, status, body, total;
    explicit Layout(int64_t n) {
        rows = 0;
        status = up16(sizeof(float) * 24 * (size_t)n);
        body = status + 16;
        total = up16(body + sizeof(bm_collider_t));
    }
};

}  // namespace

struct bm_server {
    bm_server_config_t cfg{};
    int device = 0;
    World w;
    std::vector<Active> active;  // same order as w.scenes
    // device bodies of the active scenes (pool memory, rebuilt in stream
    // order when the scene set changes)
    BodyDev* d_bodies = nullptr;
    M1Params* d_params = nullptr;
    double* d_acc = nullptr;
    bm_reaction_t* d_react = nullptr;
    int64_t* d_cand_prefix = nullptr;  // body b owns M1 CTAs [prefix[b], prefix[b+1])
    int n_bodies = 0;
    int64_t total_cand = 0;
    double used_bytes = 0;
    // pinned read-back blocks and events, reused
    std::multimap<size_t, void*> pinned_free;
    std::vector<void*> pinned_all;
    std::vector<cudaEvent_t> events_free;
    std::vector<std::shared_ptr<Request>> draining;
    // shared state
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::unordered_map<int64_t, std::shared_ptr<Request>> all;
    int64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    // stats (under mu)
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, iterations = 0, n_active = 0;
    std::vector<double> latencies;
    double particle_steps = 0, busy = 0, peak_bytes = 0;
    double t_admit = 0, t_step = 0, t_retire = 0;
};

namespace {

template <class T>
bm_status_t pool_alloc(bm_server* s, T** p, size_t count) {
    *p = nullptr;
    BM_CHECK_CUDA(cudaMallocFromPoolAsync((void**)p, sizeof(T) * std::max<size_t>(count, 1), s->w.pool, s->w.stream));
    return BM_OK;
}

void pool_free(bm_server* s, void* p) {
    if (p) cudaFreeAsync(p, s->w.stream);
}

// Rebuilds the device body arrays for the current active scenes. old_body[i]
// is the index, in the arrays being replaced, of active scene i's body (-1:
// a new scene, whose body starts from its request). Everything is enqueued
// on the stream: no wait for the GPU.
bm_status_t rebuild_bodies(bm_server* s, const std::vector<int>& old_body) {
    World& w = s->w;
    std::vector<BodyDev> staged;
    std::vector<int32_t> src;
    std::vector<int64_t> prefix(1, 0);
    for (size_t i = 0; i < s->active.size(); ++i) {
        Active& a = s->active[i];
        const Request& r = *a.req;
        a.body = -1;
        if (!r.desc.has_body) continue;
        BodyDev B{};
        B.state = r.desc.body;
        B.inv_mass = r.desc.body.mass > 0.0f ? 1.0f / r.desc.body.mass : 0.0f;
        bool zero = true;
        for (int q = 0; q < 9; ++q) zero = zero && r.desc.body_inv_inertia[q] == 0.0f && !r.desc.body_inv_inertia_given;
        for (int q = 0; q < 9; ++q)
            B.inv_inertia[q] = zero ? ((q % 4 == 0) ? 1.0f : 0.0f) : r.desc.body_inv_inertia[q];
        for (int c = 0; c < 3; ++c) B.gravity[c] = r.desc.gravity[c];
        B.dt = r.desc.dt;
        B.dynamic = r.desc.body_dynamic;
        B.scene = (int32_t)i;
        a.body = (int)staged.size();
        src.push_back(i < old_body.size() ? old_body[i] : -1);
        staged.push_back(B);
        prefix.push_back(prefix.back() + m1_max_candidates(w.scenes[i].dev.g, r.desc.body.half_extents));
    }
    const int nb = (int)staged.size();
    BodyDev* bodies = nullptr;
    M1Params* params = nullptr;
    double* acc = nullptr;
    bm_reaction_t* react = nullptr;
    int64_t* cand = nullptr;
    bm_status_t st = BM_OK;
    if (nb > 0) {
        if ((st = pool_alloc(s, &bodies, nb)) != BM_OK) return st;
        if ((st = pool_alloc(s, &params, nb)) != BM_OK) return st;
        if ((st = pool_alloc(s, &acc, 7 * (size_t)nb)) != BM_OK) return st;
        if ((st = pool_alloc(s, &react, nb)) != BM_OK) return st;
        if ((st = pool_alloc(s, &cand, nb + 1)) != BM_OK) return st;
        BodyDev* d_staged = nullptr;
        int32_t* d_src = nullptr;
        if ((st = pool_alloc(s, &d_staged, nb)) != BM_OK) return st;
        if ((st = pool_alloc(s, &d_src, nb)) != BM_OK) return st;
        const size_t b0 = up16(sizeof(BodyDev) * nb), b1 = up16(sizeof(int32_t) * nb), b2 = sizeof(int64_t) * (nb + 1);
        void* buf = nullptr;
        if ((st = w.stage_begin(b0 + b1 + b2, &buf)) != BM_OK) return st;
        char* h = static_cast<char*>(buf);
        std::memcpy(h, staged.data(), sizeof(BodyDev) * nb);
        std::memcpy(h + b0, src.data(), sizeof(int32_t) * nb);
        std::memcpy(h + b0 + b1, prefix.data(), b2);
        BM_CHECK_CUDA(cudaMemcpyAsync(d_staged, h, sizeof(BodyDev) * nb, cudaMemcpyHostToDevice, w.stream));
        BM_CHECK_CUDA(cudaMemcpyAsync(d_src, h + b0, sizeof(int32_t) * nb, cudaMemcpyHostToDevice, w.stream));
        BM_CHECK_CUDA(cudaMemcpyAsync(cand, h + b0 + b1, b2, cudaMemcpyHostToDevice, w.stream));
        w.stage_done();
        launch_body_remap(s->d_bodies, bodies, d_staged, d_src, nb, w.stream);
        pool_free(s, d_staged);
        pool_free(s, d_src);
    }
    pool_free(s, s->d_bodies);
    pool_free(s, s->d_params);
    pool_free(s, s->d_acc);
    pool_free(s, s->d_react);
    pool_free(s, s->d_cand_prefix);
    s->d_bodies = bodies;
    s->d_params = params;
    s->d_acc = acc;
    s->d_react = react;
    s->d_cand_prefix = cand;
    s->n_bodies = nb;
    s->total_cand = prefix.back();
    return launch_status("server bodies");
}

bm_status_t admit(bm_server* s, std::shared_ptr<Request> r) {
    World& w = s->w;
    const bm_scene_desc_t& d = r->desc;
    w.add_scene();
    SceneHost& h = w.scenes.back();
    h.dev.g.dx = d.dx;
    h.dev.g.inv_dx = 1.0f / d.dx;
    h.dev.dt = d.dt;
    h.dev.fresh = 1;
    h.E = d.young_modulus;
    h.nu = d.poisson_ratio;
    h.density = d.bulk_density;
    h.alpha = d.plastic_alpha;
    h.floor_friction = d.floor_friction;
    for (int a = 0; a < 3; ++a) h.gravity[a] = d.gravity[a];
    if (d.has_domain) {
        h.domain = d.domain;
        h.domain_set = true;
    }
    bm_status_t st = BM_OK;
    if (!r->pos.empty())
        st = w.append_particles(h, (int64_t)r->mass.size(), r->pos.data(), r->vel.empty() ? nullptr : r->vel.data(),
                                r->mass.data());
    if (st == BM_OK) st = w.ensure_grid(h);
    if (st != BM_OK) {
        w.remove_scene((int)w.scenes.size() - 1);
        return st;
    }
    r->out_body = d.body;
    Active a;
    a.req = r;
    a.steps_left = r->n_steps;
    s->active.push_back(a);
    s->used_bytes += r->bytes;
    return BM_OK;
}

bm_status_t pinned_acquire(bm_server* s, size_t bytes, void** out, size_t* cap) {
    auto it = s->pinned_free.lower_bound(bytes);
    if (it != s->pinned_free.end()) {
        *cap = it->first;
        *out = it->second;
        s->pinned_free.erase(it);
        return BM_OK;
    }
    size_t c = 1 << 16;
    while (c < bytes) c <<= 1;
    BM_CHECK_CUDA(cudaMallocHost(out, c));
    s->pinned_all.push_back(*out);
    *cap = c;
    return BM_OK;
}

// Enqueues the read-back of active scene i (particles in add order, status
// word, body) into a pinned block behind an event; the scene's device
// memory may be freed right after (stream order).
bm_status_t enqueue_collect(bm_server* s, int i) {
    World& w = s->w;
    SceneHost& h = w.scenes[i];
    Active& a = s->active[i];
    Request& r = *a.req;
    const int64_t n = h.n();
    const Layout L(n);
    bm_status_t st = pinned_acquire(s, L.total, &r.pinned, &r.pinned_cap);
    if (st != BM_OK) return st;
    char* base = static_cast<char*>(r.pinned);
    if (n > 0) {
        float* tmp = nullptr;
        if ((st = pool_alloc(s, &tmp, 24 * (size_t)n)) != BM_OK) return st;
        const ParticleSoA& ps = h.dev.store[w.sel];
        const int planes[4] = {P_X, P_V, P_F, P_C}, widths[4] = {3, 3, 9, 9};
        size_t off = 0;
        for (int f = 0; f < 4; ++f) {
            launch_gather_rows(ps, planes[f], widths[f], tmp + off, w.stream);
            off += (size_t)widths[f] * n;
        }
        BM_CHECK_CUDA(cudaMemcpyAsync(base + L.rows, tmp, sizeof(float) * 24 * n, cudaMemcpyDeviceToHost, w.stream));
        pool_free(s, tmp);
    }
    BM_CHECK_CUDA(cudaMemcpyAsync(base + L.status, h.dev.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, w.stream));
    if (a.body >= 0)
        BM_CHECK_CUDA(cudaMemcpyAsync(base + L.body, &s->d_bodies[a.body].state, sizeof(bm_collider_t),
                                      cudaMemcpyDeviceToHost, w.stream));
    else
        std::memcpy(base + L.body, &r.out_body, sizeof(bm_collider_t));
    if (s->events_free.empty()) {
        cudaEvent_t e;
        BM_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        s->events_free.push_back(e);
    }
    r.ready = s->events_free.back();
    s->events_free.pop_back();
    BM_CHECK_CUDA(cudaEventRecord(r.ready, w.stream));
    return BM_OK;
}

// Completes the requests whose read-back has arrived (all of them, waiting,
// when `block`).
void drain(bm_server* s, bool block) {
    for (size_t k = 0; k < s->draining.size();) {
        auto r = s->draining[k];
        if (block) cudaEventSynchronize(r->ready);
        else if (cudaEventQuery(r->ready) != cudaSuccess) {
            ++k;
            continue;
        }
        const int64_t n = (int64_t)r->mass.size();
        const Layout L(n);
        const char* base = static_cast<const char*>(r->pinned);
        r->out_pos.resize(3 * n);
        r->out_vel.resize(3 * n);
        r->out_F.resize(9 * n);
        r->out_C.resize(9 * n);
        const float* rows = reinterpret_cast<const float*>(base + L.rows);
        std::memcpy(r->out_pos.data(), rows, sizeof(float) * 3 * n);
        std::memcpy(r->out_vel.data(), rows + 3 * n, sizeof(float) * 3 * n);
        std::memcpy(r->out_F.data(), rows + 6 * n, sizeof(float) * 9 * n);
        std::memcpy(r->out_C.data(), rows + 15 * n, sizeof(float) * 9 * n);
        uint32_t status;
        std::memcpy(&status, base + L.status, sizeof(status));
        std::memcpy(&r->out_body, base + L.body, sizeof(bm_collider_t));
        s->pinned_free.insert({r->pinned_cap, r->pinned});
        r->pinned = nullptr;
        s->events_free.push_back(r->ready);
        r->ready = nullptr;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->error = (status & ERR_NONFINITE) ? BM_ERR_NON_FINITE
                       : (status & ERR_ESCAPE)  ? BM_ERR_DOMAIN_ESCAPE
                                                : BM_OK;
            r->t_done = Clock::now();
            r->state = BM_REQ_DONE;
            ++s->completed;
            s->particle_steps += (double)n * r->n_steps;
            s->latencies.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
            r->pos.clear();
            r->vel.clear();
        }
        s->draining.erase(s->draining.begin() + k);
        s->cv_done.notify_all();
    }
}

bm_status_t step_all(bm_server* s, bool admitted) {
    World& w = s->w;
    bm_status_t st = w.sync_table();
    if (st != BM_OK) return st;
    bool any_fresh = false;
    for (auto& h : w.scenes) any_fresh = any_fresh || h.dev.fresh;
    if (any_fresh) st = w.p2g_fresh();
    if (st == BM_OK) st = w.update(true);
    if (st == BM_OK && s->n_bodies > 0) {
        const int nb = s->n_bodies;
        BM_CHECK_CUDA(cudaMemsetAsync(s->d_acc, 0, sizeof(double) * 7 * nb, w.stream));
        launch_body_prepare(w.table(), s->d_bodies, nb, s->d_params, w.stream);
        launch_m1_flat(w.table(), s->d_params, nb, s->d_cand_prefix, s->total_cand, w.cur, s->d_acc, w.stream);
        launch_body_integrate(s->d_bodies, nb, s->d_acc, w.stream);
        st = launch_status("server coupler");
    }
    const int K = std::max(1, s->cfg.sort_interval);
    if (st == BM_OK && (admitted || s->iterations % K == 0)) st = w.sort_particles();
    if (st == BM_OK) st = w.g2p2g(false, s->cfg.variant);
    for (auto& h : w.scenes)
        if (h.dev.fresh) {
            h.dev.fresh = 0;
            w.dirty = true;
        }
    return st;
}

void fail_request(bm_server* s, const std::shared_ptr<Request>& r, bm_status_t st) {
    std::lock_guard<std::mutex> lk(s->mu);
    r->t_done = Clock::now();
    if (r->cancel && st == BM_OK) {
        r->state = BM_REQ_CANCELLED;
        ++s->cancelled;
    } else {
        r->state = BM_REQ_FAILED;
        r->error = st != BM_OK ? st : BM_ERR_CUDA;
        ++s->failed;
    }
    r->pos.clear();
    r->vel.clear();
    s->cv_done.notify_all();
}

void worker_main(bm_server* s) {
    cudaSetDevice(s->device);
    World& w = s->w;
    for (;;) {
        std::vector<std::shared_ptr<Request>> to_admit;
        if (s->active.empty() && !s->draining.empty()) drain(s, true);
        {
            std::unique_lock<std::mutex> lk(s->mu);
            while (!s->stop && s->queue.empty() && s->active.empty())
                s->cv_work.wait_for(lk, std::chrono::milliseconds(100));
            if (s->stop) break;
            // admit in arrival order while the footprint fits
            double used = s->used_bytes;
            int n_active = (int)s->active.size();
            while (!s->queue.empty()) {
                auto r = s->queue.front();
                if (r->cancel) {
                    s->queue.pop_front();
                    r->state = BM_REQ_CANCELLED;
                    ++s->cancelled;
                    s->cv_done.notify_all();
                    continue;
                }
                if (n_active >= s->cfg.max_active) break;
                if (used + r->bytes > s->cfg.hbm_budget_bytes && n_active > 0) break;
                s->queue.pop_front();
                r->state = BM_REQ_RUNNING;
                used += r->bytes;
                ++n_active;
                to_admit.push_back(r);
            }
        }
        const auto t0 = Clock::now();
        auto since = [](Clock::time_point a) { return std::chrono::duration<double>(Clock::now() - a).count(); };
        double dt_admit = 0, dt_step = 0, dt_retire = 0;
        bool changed = false;
        if (!to_admit.empty()) {
            std::vector<int> old_body;
            for (const Active& a : s->active) old_body.push_back(a.body);
            for (auto& r : to_admit) {
                const bm_status_t st = admit(s, r);
                if (st != BM_OK) fail_request(s, r, st);
                else old_body.push_back(-1);
            }
            changed = true;
            s->peak_bytes = std::max(s->peak_bytes, s->used_bytes);
            const bm_status_t st = rebuild_bodies(s, old_body);
            if (st != BM_OK) {
                for (auto& a : s->active) a.steps_left = 0;  // retire everything below as failed
            }
            dt_admit = since(t0);
        }
        if (s->active.empty()) {
            std::lock_guard<std::mutex> lk(s->mu);
            s->t_admit += dt_admit;
            continue;
        }
        const auto t1 = Clock::now();
        bm_status_t st = step_all(s, changed);
        dt_step = since(t1);
        const auto t2 = Clock::now();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            ++s->iterations;
        }
        // retire finished, cancelled or failed scenes
        std::vector<int> done;
        for (int i = 0; i < (int)s->active.size(); ++i) {
            Active& a = s->active[i];
            a.steps_left -= 1;
            if (st != BM_OK || a.steps_left <= 0 || a.req->cancel) done.push_back(i);
        }
        if (!done.empty()) {
            for (int k = (int)done.size() - 1; k >= 0; --k) {
                const int i = done[k];
                auto r = s->active[i].req;
                bm_status_t cst = st;
                if (cst == BM_OK && !r->cancel) cst = enqueue_collect(s, i);
                if (cst == BM_OK && !r->cancel) s->draining.push_back(r);
                else fail_request(s, r, cst);
                s->used_bytes -= r->bytes;
                w.remove_scene(i);
                s->active.erase(s->active.begin() + i);
            }
            std::vector<int> old_body;
            for (const Active& a : s->active) old_body.push_back(a.body);
            rebuild_bodies(s, old_body);
        }
        drain(s, false);
        dt_retire = since(t2);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->busy += std::chrono::duration<double>(Clock::now() - t0).count();
            s->t_admit += dt_admit;
            s->t_step += dt_step;
            s->t_retire += dt_retire;
            s->n_active = (int64_t)s->active.size();
        }
    }
    // shutdown: finish the read-backs in flight, cancel what is left
    drain(s, true);
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto& r : s->queue) r->state = BM_REQ_CANCELLED;
    for (auto& a : s->active) a.req->state = BM_REQ_CANCELLED;
    s->queue.clear();
    s->cv_done.notify_all();
}

}  // namespace

extern "C" {

BM_API bm_status_t bm_server_estimate_bytes(const bm_scene_desc_t* scene, double* bytes) {
    if (!scene || !bytes) return invalid_arg("NULL argument");
    *bytes = estimate_bytes(*scene);
    return BM_OK;
}

BM_API bm_status_t bm_server_create(const bm_server_config_t* config, bm_server_t** out) {
    if (!out) return invalid_arg("out is NULL");
    *out = nullptr;
    bm_server* s = new bm_server();
    s->cfg.hbm_budget_bytes = 150e9;
    s->cfg.max_active = 1024;
    s->cfg.sort_interval = 32;  // measured 3 % faster than 16 on the served request mix
    s->cfg.variant = fused_variant_index(128, 7, 1);  // as the batched form's default
    if (config) {
        if (config->hbm_budget_bytes > 0) s->cfg.hbm_budget_bytes = config->hbm_budget_bytes;
        if (config->max_active > 0) s->cfg.max_active = config->max_active;
        if (config->sort_interval > 0) s->cfg.sort_interval = config->sort_interval;
        if (config->variant >= 0 && config->variant < fused_variant_count()) s->cfg.variant = config->variant;
    }
    bm_status_t st = s->w.init();
    if (st != BM_OK) {
        delete s;
        return st;
    }
    s->device = s->w.device;
    s->worker = std::thread(worker_main, s);
    *out = s;
    return BM_OK;
}

BM_API bm_status_t bm_server_destroy(bm_server_t* s) {
    if (!s) return invalid_arg("NULL handle");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->device);
    pool_free(s, s->d_bodies);
    pool_free(s, s->d_params);
    pool_free(s, s->d_acc);
    pool_free(s, s->d_react);
    pool_free(s, s->d_cand_prefix);
    s->w.release();
    for (void* p : s->pinned_all) cudaFreeHost(p);
    for (cudaEvent_t e : s->events_free) cudaEventDestroy(e);
    delete s;
    return BM_OK;
}

BM_API bm_status_t bm_server_submit(bm_server_t* s, const bm_scene_desc_t* scene, int32_t n_steps,
                                    int64_t* request_id) {
    if (!s || !scene || !request_id) return invalid_arg("NULL argument");
    if (n_steps <= 0) return invalid_arg("n_steps must be positive");
    const bm_scene_desc_t& d = *scene;
    if (!(d.dx > 0.0f) || !(d.dt > 0.0f)) return invalid_arg("scene dx and dt must be positive");
    if (d.n_particles < 0 || (d.n_particles > 0 && !d.position)) return invalid_arg("bad particle arrays");
    if (!d.has_domain && d.n_particles == 0) return invalid_arg("a scene without particles needs a domain");
    auto r = std::make_shared<Request>();
    r->desc = d;
    r->n_steps = n_steps;
    const size_t n = (size_t)d.n_particles;
    r->pos.assign(d.position, d.position + 3 * n);
    if (d.velocity) r->vel.assign(d.velocity, d.velocity + 3 * n);
    r->mass.resize(n);
    for (size_t q = 0; q < n; ++q) r->mass[q] = d.mass ? d.mass[q] : 1.0f;
    r->bytes = estimate_bytes(d);
    r->desc.position = nullptr;
    r->desc.velocity = nullptr;
    r->desc.mass = nullptr;
    if (r->bytes > s->cfg.hbm_budget_bytes) {
        set_last_error("scene footprint exceeds the server's HBM budget");
        return BM_ERR_OUT_OF_MEMORY;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        r->t_submit = Clock::now();
        s->all[r->id] = r;
        s->queue.push_back(r);
        ++s->submitted;
    }
    s->cv_work.notify_all();
    *request_id = r->id;
    return BM_OK;
}

BM_API bm_status_t bm_server_poll(bm_server_t* s, int64_t id, int32_t* state) {
    if (!s || !state) return invalid_arg("NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return BM_ERR_NOT_FOUND;
    *state = it->second->state;
    return BM_OK;
}

BM_API bm_status_t bm_server_wait(bm_server_t* s, int64_t id, int32_t timeout_ms) {
    if (!s) return invalid_arg("NULL handle");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return BM_ERR_NOT_FOUND;
    auto r = it->second;
    const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(std::max(0, timeout_ms)), [&] {
        return r->state == BM_REQ_DONE || r->state == BM_REQ_FAILED || r->state == BM_REQ_CANCELLED;
    });
    if (!ok) {
        set_last_error("request not finished within the timeout");
        return BM_ERR_TIMEOUT;
    }
    if (r->state == BM_REQ_FAILED) return r->error != BM_OK ? r->error : BM_ERR_CUDA;
    if (r->state == BM_REQ_CANCELLED) return BM_ERR_STATE;
    return r->error;
}

BM_API bm_status_t bm_server_result(bm_server_t* s, int64_t id, const bm_particles_view_t* v, bm_collider_t* body,
                                    double* latency_ms) {
    if (!s) return invalid_arg("NULL handle");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return BM_ERR_NOT_FOUND;
    Request& r = *it->second;
    if (r.state != BM_REQ_DONE) {
        set_last_error("request has no result");
        return BM_ERR_STATE;
    }
    const size_t n = r.mass.size();
    if (v && n > 0) {
        if (v->position) std::memcpy(v->position, r.out_pos.data(), sizeof(float) * 3 * n);
        if (v->velocity) std::memcpy(v->velocity, r.out_vel.data(), sizeof(float) * 3 * n);
        if (v->F) std::memcpy(v->F, r.out_F.data(), sizeof(float) * 9 * n);
        if (v->C) std::memcpy(v->C, r.out_C.data(), sizeof(float) * 9 * n);
        if (v->mass) std::memcpy(v->mass, r.mass.data(), sizeof(float) * n);
    }
    if (body) *body = r.out_body;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count();
    return BM_OK;
}

BM_API bm_status_t bm_server_release(bm_server_t* s, int64_t id) {
    if (!s) return invalid_arg("NULL handle");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return BM_ERR_NOT_FOUND;
    if (it->second->state == BM_REQ_QUEUED || it->second->state == BM_REQ_RUNNING) return BM_ERR_STATE;
    s->all.erase(it);
    return BM_OK;
}

BM_API bm_status_t bm_server_cancel(bm_server_t* s, int64_t id) {
    if (!s) return invalid_arg("NULL handle");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return BM_ERR_NOT_FOUND;
    it->second->cancel = true;
    s->cv_work.notify_all();
    return BM_OK;
}

BM_API bm_status_t bm_server_stats(bm_server_t* s, bm_server_stats_t* out) {
    if (!s || !out) return invalid_arg("NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    bm_server_stats_t r{};
    r.submitted = s->submitted;
    r.completed = s->completed;
    r.failed = s->failed;
    r.cancelled = s->cancelled;
    r.queued = (int64_t)s->queue.size();
    r.active = s->n_active;
    r.iterations = s->iterations;
    r.p50_latency_ms = percentile(s->latencies, 0.50);
    r.p99_latency_ms = percentile(s->latencies, 0.99);
    double sum = 0;
    for (double x : s->latencies) sum += x;
    r.mean_latency_ms = s->latencies.empty() ? 0.0 : sum / (double)s->latencies.size();
    r.particle_steps = s->particle_steps;
    r.busy_seconds = s->busy;
    r.peak_bytes = s->peak_bytes;
    r.admit_seconds = s->t_admit;
    r.step_seconds = s->t_step;
    r.retire_seconds = s->t_retire;
    *out = r;
    return BM_OK;
}

}  // extern "C"
