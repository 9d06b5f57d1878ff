// bm_batch.cu — the batched form: many scenes of uneven particle and grid
// counts stepped together, CUDA-graph replay and the launch autotuner.
//
// A batch is a World (bm_world.h) of many scenes. One step is, for all
// scenes at once: the grid update (one grid row per scene), the M1 coupler of
// every scene's rigid body with its parameters computed on the device from
// the body state, the rigid update of every body (integrator.h:19-57), every
// K steps the regrouping of particles by sort bin, and the fused
// G2P + next P2G over the scene table. Nothing in a step reads back to the
// host, so a chunk of 2K steps (after which the buffer parities return to
// their start) is captured once as a CUDA graph and replayed.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bm_world.h"

using namespace bm;

struct bm_batch {
    World w;
    std::vector<int> body_of_scene;  // body index or -1
    std::vector<BodyDev> h_bodies;
    BodyDev* d_bodies = nullptr;
    M1Params* d_params = nullptr;
    double* d_acc = nullptr;
    bm_reaction_t* d_react = nullptr;
    int n_bodies = 0;
    std::vector<int64_t> h_cand_prefix{0};  // body b owns M1 CTAs [prefix[b], prefix[b+1])
    int64_t* d_cand_prefix = nullptr;
    int64_t steps_done = 0;
    bool started = false;  // P2G of the first step done
    int32_t sort_interval = 16;
    // 128 threads x 7 CTAs per SM with interleaved lanes: the autotuner's
    // usual pick for scenes at 8 particles per cell
    int variant = fused_variant_index(128, 7, 1);
    bool fast_math = false;
    bool use_graph = true;
    cudaGraphExec_t graph = nullptr;
    int64_t graph_chunk = 0;
};

namespace {

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

void drop_graph(bm_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_chunk = 0;
}

// One step of every scene, enqueued on the batch stream.
bm_status_t eager_step(bm_batch* b) {
    World& w = b->w;
    bm_status_t st = BM_OK;
    if (!b->started) {
        st = w.clear_and_p2g();
        if (st != BM_OK) return st;
        b->started = true;
        st = w.update(false);
    } else {
        st = w.update(true);
    }
    if (st != BM_OK) return st;
    if (b->n_bodies > 0) {
        BM_CHECK_CUDA(cudaMemsetAsync(b->d_acc, 0, sizeof(double) * 7 * b->n_bodies, w.stream));
        w.timed("m1_coupler", [&] {
            launch_body_prepare(w.table(), b->d_bodies, b->n_bodies, b->d_params, w.stream);
            launch_m1_flat(w.table(), b->d_params, b->n_bodies, b->d_cand_prefix, b->h_cand_prefix.back(), w.cur,
                           b->d_acc, w.stream);
            launch_body_integrate(b->d_bodies, b->n_bodies, b->d_acc, w.stream);
            launch_reaction_finalize(b->d_acc, b->n_bodies, b->d_react, w.stream);
        });
        st = launch_status("coupler");
        if (st != BM_OK) return st;
    }
    const int64_t K = b->sort_interval;
    if ((K > 0 && b->steps_done % K == 0) || (K == 0 && b->steps_done == 0)) {
        st = w.sort_particles();
        if (st != BM_OK) return st;
    }
    st = w.g2p2g(b->fast_math, b->variant);
    b->steps_done += 1;
    return st;
}

// Length of a replayable chunk: cur flips every step, sel every K steps.
int64_t chunk_len(const bm_batch* b) { return b->sort_interval > 0 ? 2 * (int64_t)b->sort_interval : 2; }

bool chunk_aligned(const bm_batch* b) {
    if (!b->started || b->steps_done == 0) return false;
    const int64_t K = b->sort_interval;
    return K > 0 ? (b->steps_done % K == 0) : true;
}

bm_status_t capture_chunk(bm_batch* b) {
    World& w = b->w;
    drop_graph(b);
    const bool prof = w.profiling;
    w.profiling = false;
    const int64_t C = chunk_len(b);
    const int64_t steps0 = b->steps_done;
    const int cur0 = w.cur, sel0 = w.sel;
    cudaGraph_t g = nullptr;
    BM_CHECK_CUDA(cudaStreamBeginCapture(w.stream, cudaStreamCaptureModeThreadLocal));
    bm_status_t st = BM_OK;
    for (int64_t i = 0; i < C && st == BM_OK; ++i) st = eager_step(b);
    cudaError_t e = cudaStreamEndCapture(w.stream, &g);
    w.profiling = prof;
    // the capture only recorded the work: rewind the host-side step state
    b->steps_done = steps0;
    w.cur = cur0;
    w.sel = sel0;
    if (st != BM_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("graph capture: ") + cudaGetErrorString(e));
        return BM_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->graph = nullptr;
        set_last_error(std::string("graph instantiate: ") + cudaGetErrorString(e));
        return BM_ERR_CUDA;
    }
    b->graph_chunk = C;
    return BM_OK;
}

bm_status_t run_steps(bm_batch* b, int64_t n) {
    World& w = b->w;
    bm_status_t st = w.sync_table();
    if (st != BM_OK) return st;
    while (n > 0) {
        const int64_t C = chunk_len(b);
        if (b->use_graph && !w.profiling && chunk_aligned(b) && n >= C) {
            if (!b->graph) {
                st = capture_chunk(b);
                if (st != BM_OK) return st;
            }
            BM_CHECK_CUDA(cudaGraphLaunch(b->graph, w.stream));
            b->steps_done += C;
            n -= C;
            // parities after C steps equal those at the start (C even, C/K even)
            continue;
        }
        st = eager_step(b);
        if (st != BM_OK) return st;
        n -= 1;
    }
    return BM_OK;
}

// ---- snapshot / restore for the autotuner ------------------------------------------

struct Snapshot {
    std::vector<float*> planes;    // per scene: N_PLANES * n floats
    std::vector<int32_t*> pids;
    std::vector<uint8_t*> allocs;
    BodyDev* bodies = nullptr;
    int64_t steps_done = 0;
};

bm_status_t take_snapshot(bm_batch* b, Snapshot& s) {
    World& w = b->w;
    s.steps_done = b->steps_done;
    for (auto& h : w.scenes) {
        const int64_t n = h.n(), nb = h.dev.g.num_blocks();
        float* p = nullptr;
        int32_t* q = nullptr;
        uint8_t* a = nullptr;
        BM_CHECK_CUDA(cudaMalloc((void**)&p, sizeof(float) * N_PLANES * std::max<int64_t>(1, n)));
        BM_CHECK_CUDA(cudaMalloc((void**)&q, sizeof(int32_t) * std::max<int64_t>(1, n)));
        BM_CHECK_CUDA(cudaMalloc((void**)&a, (size_t)std::max<int64_t>(1, nb)));
        const ParticleSoA& src = h.dev.store[w.sel];
        for (int c = 0; c < N_PLANES; ++c)
            BM_CHECK_CUDA(cudaMemcpyAsync(p + (int64_t)c * n, src.plane(c), sizeof(float) * n, cudaMemcpyDeviceToDevice,
                                          w.stream));
        BM_CHECK_CUDA(cudaMemcpyAsync(q, src.pid, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, w.stream));
        BM_CHECK_CUDA(cudaMemcpyAsync(a, h.dev.alloc, (size_t)nb, cudaMemcpyDeviceToDevice, w.stream));
        s.planes.push_back(p);
        s.pids.push_back(q);
        s.allocs.push_back(a);
    }
    if (b->n_bodies > 0) {
        BM_CHECK_CUDA(cudaMalloc((void**)&s.bodies, sizeof(BodyDev) * b->n_bodies));
        BM_CHECK_CUDA(cudaMemcpyAsync(s.bodies, b->d_bodies, sizeof(BodyDev) * b->n_bodies, cudaMemcpyDeviceToDevice,
                                      w.stream));
    }
    return BM_OK;
}

// Puts the saved particles, blocks and bodies back and clears both grid
// accumulators; the next step recomputes P2G from the particles.
bm_status_t restore_snapshot(bm_batch* b, const Snapshot& s) {
    World& w = b->w;
    for (size_t i = 0; i < w.scenes.size(); ++i) {
        SceneHost& h = w.scenes[i];
        const int64_t n = h.n(), nn = h.dev.g.num_nodes(), nb = h.dev.g.num_blocks();
        const ParticleSoA& dst = h.dev.store[w.sel];
        for (int c = 0; c < N_PLANES; ++c)
            BM_CHECK_CUDA(cudaMemcpyAsync(dst.plane(c), s.planes[i] + (int64_t)c * n, sizeof(float) * n,
                                          cudaMemcpyDeviceToDevice, w.stream));
        BM_CHECK_CUDA(cudaMemcpyAsync(dst.pid, s.pids[i], sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, w.stream));
        BM_CHECK_CUDA(cudaMemcpyAsync(h.dev.alloc, s.allocs[i], (size_t)nb, cudaMemcpyDeviceToDevice, w.stream));
        for (auto& a : h.dev.acc) {
            BM_CHECK_CUDA(cudaMemsetAsync(a.mv, 0, sizeof(float4) * nn, w.stream));
            BM_CHECK_CUDA(cudaMemsetAsync(a.f, 0, sizeof(float4) * nn, w.stream));
            BM_CHECK_CUDA(cudaMemsetAsync(a.touched, 0, sizeof(uint32_t) * nb, w.stream));
            BM_CHECK_CUDA(cudaMemsetAsync(a.count, 0, sizeof(int32_t), w.stream));
        }
    }
    if (b->n_bodies > 0)
        BM_CHECK_CUDA(cudaMemcpyAsync(b->d_bodies, s.bodies, sizeof(BodyDev) * b->n_bodies, cudaMemcpyDeviceToDevice,
                                      w.stream));
    b->steps_done = s.steps_done;
    b->started = false;
    BM_CHECK_CUDA(cudaStreamSynchronize(w.stream));
    return BM_OK;
}

void free_snapshot(Snapshot& s) {
    for (auto p : s.planes) cudaFree(p);
    for (auto p : s.pids) cudaFree(p);
    for (auto p : s.allocs) cudaFree(p);
    cudaFree(s.bodies);
    s = Snapshot{};
}

bm_status_t set_bin_shift(bm_batch* b, int shift) {
    for (auto& h : b->w.scenes) h.dev.bin_shift = shift;
    b->w.dirty = true;
    drop_graph(b);
    return b->w.sync_table();
}

bm_status_t time_steps(bm_batch* b, int64_t n, float* ms) {
    World& w = b->w;
    if (!w.t0) BM_CHECK_CUDA(cudaEventCreate(&w.t0));
    if (!w.t1) BM_CHECK_CUDA(cudaEventCreate(&w.t1));
    BM_CHECK_CUDA(cudaEventRecord(w.t0, w.stream));
    bm_status_t st = run_steps(b, n);
    if (st != BM_OK) return st;
    BM_CHECK_CUDA(cudaEventRecord(w.t1, w.stream));
    BM_CHECK_CUDA(cudaEventSynchronize(w.t1));
    BM_CHECK_CUDA(cudaEventElapsedTime(ms, w.t0, w.t1));
    return BM_OK;
}

}  // namespace

extern "C" {

BM_API bm_status_t bm_batch_create(int32_t n_scenes, const bm_scene_desc_t* scenes, bm_batch_t** out) {
    if (!out) return invalid_arg("out is NULL");
    *out = nullptr;
    if (n_scenes <= 0 || !scenes) return invalid_arg("need at least one scene");
    for (int32_t i = 0; i < n_scenes; ++i) {
        const bm_scene_desc_t& d = scenes[i];
        if (!(d.dx > 0.0f) || !std::isfinite(d.dx)) return invalid_arg("scene dx must be positive");
        if (!(d.dt > 0.0f) || !std::isfinite(d.dt)) return invalid_arg("scene dt must be positive");
        if (d.n_particles < 0 || (d.n_particles > 0 && !d.position)) return invalid_arg("bad particle arrays");
        if (!d.has_domain && d.n_particles == 0) return invalid_arg("a scene without particles needs a domain");
    }
    bm_batch* b = new bm_batch();
    bm_status_t st = b->w.init();
    if (st != BM_OK) {
        delete b;
        return st;
    }
    World& w = b->w;
    for (int32_t i = 0; i < n_scenes && st == BM_OK; ++i) {
        const bm_scene_desc_t& d = scenes[i];
        w.add_scene();
        SceneHost& h = w.scenes.back();
        h.dev.g.dx = d.dx;
        h.dev.g.inv_dx = 1.0f / d.dx;
        h.dev.dt = d.dt;
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
        if (d.n_particles > 0) st = w.append_particles(h, d.n_particles, d.position, d.velocity, d.mass);
        if (st == BM_OK) st = w.ensure_grid(h);
        int body = -1;
        if (st == BM_OK && d.has_body) {
            BodyDev B{};
            B.state = d.body;
            B.inv_mass = d.body.mass > 0.0f ? 1.0f / d.body.mass : 0.0f;
            bool zero = true;
            for (int q = 0; q < 9; ++q) zero = zero && d.body_inv_inertia[q] == 0.0f && !d.body_inv_inertia_given;
            for (int q = 0; q < 9; ++q) B.inv_inertia[q] = zero ? ((q % 4 == 0) ? 1.0f : 0.0f) : d.body_inv_inertia[q];
            for (int a = 0; a < 3; ++a) B.gravity[a] = d.gravity[a];
            B.dt = d.dt;
            B.dynamic = d.body_dynamic;
            B.scene = i;
            body = (int)b->h_bodies.size();
            b->h_bodies.push_back(B);
            b->h_cand_prefix.push_back(b->h_cand_prefix.back() + m1_max_candidates(h.dev.g, d.body.half_extents));
        }
        b->body_of_scene.push_back(body);
    }
    b->n_bodies = (int)b->h_bodies.size();
    if (st == BM_OK) {
        const int nb = std::max(1, b->n_bodies);
        if (cudaMalloc((void**)&b->d_bodies, sizeof(BodyDev) * nb) != cudaSuccess ||
            cudaMalloc((void**)&b->d_params, sizeof(M1Params) * nb) != cudaSuccess ||
            cudaMalloc((void**)&b->d_acc, sizeof(double) * 7 * nb) != cudaSuccess ||
            cudaMalloc((void**)&b->d_react, sizeof(bm_reaction_t) * nb) != cudaSuccess ||
            cudaMalloc((void**)&b->d_cand_prefix, sizeof(int64_t) * (nb + 1)) != cudaSuccess) {
            set_last_error("batch body buffers");
            st = BM_ERR_OUT_OF_MEMORY;
        }
    }
    if (st == BM_OK && b->n_bodies > 0) {
        if (cudaMemcpy(b->d_bodies, b->h_bodies.data(), sizeof(BodyDev) * b->n_bodies, cudaMemcpyHostToDevice) !=
            cudaSuccess)
            st = BM_ERR_CUDA;
        cudaMemset(b->d_react, 0, sizeof(bm_reaction_t) * b->n_bodies);
        if (cudaMemcpy(b->d_cand_prefix, b->h_cand_prefix.data(), sizeof(int64_t) * b->h_cand_prefix.size(),
                       cudaMemcpyHostToDevice) != cudaSuccess)
            st = BM_ERR_CUDA;
    }
    if (st == BM_OK) st = w.sync_table();
    if (st == BM_OK && cudaStreamSynchronize(w.stream) != cudaSuccess) st = BM_ERR_CUDA;
    if (st != BM_OK) {
        bm_batch_destroy(b);
        return st;
    }
    *out = b;
    return BM_OK;
}

BM_API bm_status_t bm_batch_destroy(bm_batch_t* b) {
    if (!b) return invalid_arg("NULL handle");
    DeviceGuard dg(b->w.device);
    drop_graph(b);
    b->w.release();
    cudaFree(b->d_bodies);
    cudaFree(b->d_params);
    cudaFree(b->d_acc);
    cudaFree(b->d_react);
    cudaFree(b->d_cand_prefix);
    delete b;
    return BM_OK;
}

BM_API bm_status_t bm_batch_num_scenes(bm_batch_t* b, int32_t* out) {
    if (!b || !out) return invalid_arg("NULL argument");
    *out = (int32_t)b->w.scenes.size();
    return BM_OK;
}

BM_API bm_status_t bm_batch_num_particles(bm_batch_t* b, int32_t scene, int64_t* out) {
    if (!b || !out) return invalid_arg("NULL argument");
    if (scene < 0 || scene >= (int32_t)b->w.scenes.size()) return BM_ERR_NOT_FOUND;
    *out = b->w.scenes[scene].n();
    return BM_OK;
}

BM_API bm_status_t bm_batch_step(bm_batch_t* b, int32_t n_steps) {
    if (!b) return invalid_arg("NULL handle");
    if (n_steps < 0) return invalid_arg("n_steps < 0");
    DeviceGuard dg(b->w.device);
    return run_steps(b, n_steps);
}

BM_API bm_status_t bm_batch_steps_done(bm_batch_t* b, int64_t* out) {
    if (!b || !out) return invalid_arg("NULL argument");
    *out = b->steps_done;
    return BM_OK;
}

BM_API bm_status_t bm_batch_get_particles(bm_batch_t* b, int32_t scene, const bm_particles_view_t* v) {
    if (!b || !v) return invalid_arg("NULL argument");
    if (scene < 0 || scene >= (int32_t)b->w.scenes.size()) return BM_ERR_NOT_FOUND;
    DeviceGuard dg(b->w.device);
    const World::ReadField fields[] = {{v->position, P_X, 3}, {v->velocity, P_V, 3}, {v->F, P_F, 9},
                                       {v->C, P_C, 9},        {v->mass, P_M, 1},     {v->volume, P_V0, 1}};
    return b->w.read_fields(b->w.scenes[scene], fields, 6);
}

BM_API bm_status_t bm_batch_get_body(bm_batch_t* b, int32_t scene, bm_collider_t* out) {
    if (!b || !out) return invalid_arg("NULL argument");
    if (scene < 0 || scene >= (int32_t)b->w.scenes.size() || b->body_of_scene[scene] < 0) return BM_ERR_NOT_FOUND;
    DeviceGuard dg(b->w.device);
    BodyDev B;
    BM_CHECK_CUDA(cudaMemcpyAsync(&B, b->d_bodies + b->body_of_scene[scene], sizeof(BodyDev), cudaMemcpyDeviceToHost,
                                  b->w.stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(b->w.stream));
    *out = B.state;
    return BM_OK;
}

BM_API bm_status_t bm_batch_get_reaction(bm_batch_t* b, int32_t scene, bm_reaction_t* out) {
    if (!b || !out) return invalid_arg("NULL argument");
    if (scene < 0 || scene >= (int32_t)b->w.scenes.size() || b->body_of_scene[scene] < 0) return BM_ERR_NOT_FOUND;
    DeviceGuard dg(b->w.device);
    BM_CHECK_CUDA(cudaMemcpyAsync(out, b->d_react + b->body_of_scene[scene], sizeof(bm_reaction_t),
                                  cudaMemcpyDeviceToHost, b->w.stream));
    BM_CHECK_CUDA(cudaStreamSynchronize(b->w.stream));
    return BM_OK;
}

BM_API bm_status_t bm_batch_light_node_suspects(bm_batch_t* b, int64_t* out) {
    if (!b || !out) return invalid_arg("NULL argument");
    DeviceGuard dg(b->w.device);
    BM_CHECK_CUDA(cudaStreamSynchronize(b->w.stream));
    int64_t total = 0;
    for (SceneHost& h : b->w.scenes) {
        unsigned long long n = 0;
        BM_CHECK_CUDA(cudaMemcpy(&n, h.dev.escaped + 1, sizeof(n), cudaMemcpyDeviceToHost));
        total += (int64_t)n;
    }
    *out = total;
    return BM_OK;
}

BM_API bm_status_t bm_batch_sync(bm_batch_t* b, int32_t* bad_scene, int64_t* escaped) {
    if (!b) return invalid_arg("NULL handle");
    DeviceGuard dg(b->w.device);
    BM_CHECK_CUDA(cudaStreamSynchronize(b->w.stream));
    if (bad_scene) *bad_scene = -1;
    if (escaped) *escaped = 0;
    bm_status_t result = BM_OK;
    for (size_t i = 0; i < b->w.scenes.size(); ++i) {
        SceneHost& h = b->w.scenes[i];
        uint32_t status = 0;
        unsigned long long esc = 0;
        BM_CHECK_CUDA(cudaMemcpy(&status, h.dev.status, sizeof(status), cudaMemcpyDeviceToHost));
        BM_CHECK_CUDA(cudaMemcpy(&esc, h.dev.escaped, sizeof(esc), cudaMemcpyDeviceToHost));
        if (escaped) *escaped += (int64_t)esc;
        if (status && result == BM_OK) {
            result = (status & ERR_NONFINITE) ? BM_ERR_NON_FINITE : BM_ERR_DOMAIN_ESCAPE;
            if (bad_scene) *bad_scene = (int32_t)i;
            set_last_error("scene " + std::to_string(i) +
                           ((status & ERR_NONFINITE) ? ": non-finite particle state" : ": particle left the grid box"));
        }
        cudaMemset(h.dev.status, 0, sizeof(uint32_t));
        cudaMemset(h.dev.escaped, 0, sizeof(unsigned long long));
    }
    return result;
}

BM_API bm_status_t bm_batch_profile_enable(bm_batch_t* b, int32_t on) {
    if (!b) return invalid_arg("NULL handle");
    b->w.profiling = on != 0;
    return BM_OK;
}

BM_API bm_status_t bm_batch_profile_read(bm_batch_t* b, int32_t cap, const char** names, double* total_ms,
                                         int64_t* launches, int32_t* n_out) {
    if (!b || !n_out) return invalid_arg("NULL argument");
    DeviceGuard dg(b->w.device);
    BM_CHECK_CUDA(cudaStreamSynchronize(b->w.stream));
    b->w.fold_pending();
    int32_t n = 0;
    for (const auto& sl : b->w.slots) {
        if (n >= cap) break;
        if (names) names[n] = sl.name;
        if (total_ms) total_ms[n] = sl.total_ms;
        if (launches) launches[n] = sl.launches;
        ++n;
    }
    *n_out = n;
    return BM_OK;
}

BM_API bm_status_t bm_batch_profile_reset(bm_batch_t* b) {
    if (!b) return invalid_arg("NULL handle");
    DeviceGuard dg(b->w.device);
    cudaStreamSynchronize(b->w.stream);
    b->w.fold_pending();
    for (auto& sl : b->w.slots) {
        sl.total_ms = 0;
        sl.launches = 0;
    }
    return BM_OK;
}

BM_API bm_status_t bm_batch_set_graph(bm_batch_t* b, int32_t on) {
    if (!b) return invalid_arg("NULL handle");
    b->use_graph = on != 0;
    if (!b->use_graph) drop_graph(b);
    return BM_OK;
}

BM_API bm_status_t bm_batch_set_launch(bm_batch_t* b, int32_t variant, int32_t sort_interval, int32_t bin_shift) {
    if (!b) return invalid_arg("NULL handle");
    if (variant < 0 || variant >= fused_variant_count()) return invalid_arg("unknown launch variant");
    if (sort_interval < 0 || bin_shift < 0 || bin_shift > 3) return invalid_arg("bad sort interval or bin size");
    DeviceGuard dg(b->w.device);
    // the regrouping schedule is keyed on the step count: realign it
    if (sort_interval != b->sort_interval || variant != b->variant) drop_graph(b);
    b->variant = variant;
    b->sort_interval = sort_interval;
    if (b->w.scenes[0].dev.bin_shift != bin_shift) return set_bin_shift(b, bin_shift);
    return BM_OK;
}

BM_API bm_status_t bm_batch_autotune(bm_batch_t* b, int32_t trial_steps, bm_tune_result_t* out) {
    if (!b) return invalid_arg("NULL handle");
    if (trial_steps <= 0) return invalid_arg("trial_steps must be positive");
    DeviceGuard dg(b->w.device);
    Snapshot snap;
    bm_status_t st = take_snapshot(b, snap);
    if (st != BM_OK) {
        free_snapshot(snap);
        return st;
    }
    const int nv = fused_variant_count();
    const int32_t intervals[] = {8, 16, 32};

    const int32_t shifts[] = {0, 1};
    int32_t best_v = b->variant, best_k = b->sort_interval, best_s = b->w.scenes[0].dev.bin_shift;
    float best_ms = 1e30f;
    // One trial: restore, one eager step (first P2G), eager steps up to the
    // next chunk boundary, one chunk (captures the graph), then the timed
    // chunks only.
    auto trial = [&](int v, int32_t k, int32_t sh, float* ms) -> bm_status_t {
        bm_status_t r = bm_batch_set_launch(b, v, k, sh);
        if (r == BM_OK) r = restore_snapshot(b, snap);
        if (r == BM_OK) r = run_steps(b, 1);
        const int64_t C = chunk_len(b);
        const int64_t K = std::max<int32_t>(1, k);
        if (r == BM_OK) r = run_steps(b, (K - b->steps_done % K) % K + C);
        const int64_t T = C * std::max<int64_t>(1, (trial_steps + C - 1) / C);
        if (r == BM_OK) r = time_steps(b, T, ms);
        if (r == BM_OK) *ms /= (float)T;
        return r;
    };
    // launch variant first (every shape in both lane orders) at interval 16,
    // then the three fastest once more, each keeping the lower of its two
    // times (one trial's noise, about 1 %, is as large as their differences),
    // then bin size and interval with the best of those, each timed twice
    std::vector<std::pair<float, int>> vt;
    for (int v = 0; v < nv && st == BM_OK; ++v) {
        float ms = 0;
        st = trial(v, 16, best_s, &ms);
        if (st == BM_OK) vt.emplace_back(ms, v);
    }
    std::sort(vt.begin(), vt.end());
    for (size_t q = 0; q < vt.size() && q < 3 && st == BM_OK; ++q) {
        float ms = 0;
        st = trial(vt[q].second, 16, best_s, &ms);
        if (st == BM_OK) vt[q].first = std::min(vt[q].first, ms);
    }
    for (size_t q = 0; q < vt.size() && q < 3; ++q)
        if (vt[q].first < best_ms) {
            best_ms = vt[q].first;
            best_v = vt[q].second;
            best_k = 16;
        }
    for (int32_t sh : shifts)
        for (int32_t k : intervals) {
            float ms = 1e30f;
            for (int rep = 0; rep < 2 && st == BM_OK; ++rep) {
                float t = 0;
                st = trial(best_v, k, sh, &t);
                if (st == BM_OK) ms = std::min(ms, t);
            }
            if (st != BM_OK) break;
            if (ms < best_ms) {
                best_ms = ms;
                best_k = k;
                best_s = sh;
            }
        }
    if (st == BM_OK) st = bm_batch_set_launch(b, best_v, best_k, best_s);
    bm_status_t rs = restore_snapshot(b, snap);
    free_snapshot(snap);
    if (st == BM_OK) st = rs;
    if (st == BM_OK && out) {
        out->variant = best_v;
        out->sort_interval = best_k;
        out->bin_shift = best_s;
        out->ms_per_step = best_ms;
    }
    return st;
}

BM_API bm_status_t bm_batch_timer_start(bm_batch_t* b) {
    if (!b) return invalid_arg("NULL handle");
    DeviceGuard dg(b->w.device);
    if (!b->w.t0) BM_CHECK_CUDA(cudaEventCreate(&b->w.t0));
    if (!b->w.t1) BM_CHECK_CUDA(cudaEventCreate(&b->w.t1));
    BM_CHECK_CUDA(cudaEventRecord(b->w.t0, b->w.stream));
    return BM_OK;
}

BM_API bm_status_t bm_batch_timer_stop(bm_batch_t* b, double* ms) {
    if (!b || !ms) return invalid_arg("NULL argument");
    if (!b->w.t0) return invalid_arg("timer not started");
    DeviceGuard dg(b->w.device);
    BM_CHECK_CUDA(cudaEventRecord(b->w.t1, b->w.stream));
    BM_CHECK_CUDA(cudaEventSynchronize(b->w.t1));
    float f = 0;
    BM_CHECK_CUDA(cudaEventElapsedTime(&f, b->w.t0, b->w.t1));
    *ms = f;
    return BM_OK;
}

}  // extern "C"
