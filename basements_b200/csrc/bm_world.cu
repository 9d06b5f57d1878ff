// bm_world.cu — host core shared by the plain solver, the batch and the server.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <system_error>
#include <thread>
#include <utility>
#include <vector>

#include "bm_world.h"

namespace bm {

namespace {

// Bytes per pinned read-back chunk.
constexpr size_t kReadChunk = size_t(8) << 20;

// The pinned chunk pair of read_fields and upload_bytes, shared by every
// World of the process and kept until it exits: pinning 16 MB takes
// milliseconds, more than a read of millions of particles, and a solver is
// often created for one job. Pinned memory serves every device of the
// process; callers take turns.
struct ReadBack {
    std::mutex mu;
    void* buf[2] = {nullptr, nullptr};
};

ReadBack& read_back() {
    static ReadBack* r = new ReadBack;  // never destroyed: no teardown-order question
    return *r;
}

// Waits, on every exit of a holder of the ReadBack lock, for the copies that
// still use the pinned pair (error paths included), so that the next holder
// never refills a buffer a copy is reading or writing. Declared after the
// lock, it runs before the unlock.
struct DrainPinned {
    cudaEvent_t* done;
    bool in_flight[2] = {false, false};
    ~DrainPinned() {
        for (int q = 0; q < 2; ++q)
            if (in_flight[q]) cudaEventSynchronize(done[q]);
    }
};

// Pinned staging blocks of released Worlds, handed to the next World of the
// process: pinning host memory costs about a millisecond per call, as much as
// a short job's table uploads. At most kKeptStageBlocks are kept.
constexpr size_t kKeptStageBlocks = 16;

struct StagePool {
    std::mutex mu;
    std::vector<std::pair<size_t, void*>> blocks;  // (capacity, pointer)
};

StagePool& stage_pool() {
    static StagePool* p = new StagePool;  // never destroyed: no teardown-order question
    return *p;
}

// A kept block of at least `bytes` (the smallest such), or none.
bool take_stage_block(size_t bytes, void** buf, size_t* cap) {
    StagePool& sp = stage_pool();
    std::lock_guard<std::mutex> lk(sp.mu);
    int best = -1;
    for (int i = 0; i < (int)sp.blocks.size(); ++i)
        if (sp.blocks[i].first >= bytes && (best < 0 || sp.blocks[i].first < sp.blocks[best].first)) best = i;
    if (best < 0) return false;
    *cap = sp.blocks[best].first;
    *buf = sp.blocks[best].second;
    sp.blocks.erase(sp.blocks.begin() + best);
    return true;
}

// Keeps a block for a later World, or unpins it when enough are kept. The
// caller guarantees that no copy still reads it.
void give_stage_block(void* buf, size_t cap) {
    if (!buf) return;
    StagePool& sp = stage_pool();
    {
        std::lock_guard<std::mutex> lk(sp.mu);
        if (sp.blocks.size() < kKeptStageBlocks) {
            sp.blocks.emplace_back(cap, buf);
            return;
        }
    }
    cudaFreeHost(buf);
}

// memcpy between pinned and pageable memory, in parts of at least 2 MB on up
// to four threads. A fresh pageable destination (a new numpy array) takes a
// page fault per page on first touch, and those dominate such a copy.
void host_copy(void* dst, const void* src, size_t bytes) {
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>(std::min<size_t>(4, hw), std::max<size_t>(1, bytes >> 21));
    const size_t part = (bytes / nt + 63) & ~size_t(63);
    // piece t is [part t, part (t+1)), the last one ending at `bytes`
    auto piece = [=](size_t t) {
        const size_t o = std::min(bytes, part * t);
        const size_t e = t + 1 == nt ? bytes : std::min(bytes, part * (t + 1));
        if (e > o) std::memcpy(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o, e - o);
    };
    std::vector<std::thread> threads;
    size_t t = 1;
    for (; t < nt; ++t) {
        try {
            threads.emplace_back(piece, t);
        } catch (const std::system_error&) {
            break;
        }
    }
    for (size_t r = t; r < nt; ++r) piece(r);  // the pieces no thread took
    piece(0);
    for (auto& th : threads) th.join();
}

}  // namespace

static thread_local std::string g_last_error;
void set_last_error(const std::string& s) { g_last_error = s; }
const char* last_error_text() { return g_last_error.c_str(); }

bm_status_t invalid_arg(const char* what) {
    set_last_error(what);
    return BM_ERR_INVALID_ARGUMENT;
}

bm_status_t launch_status(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string(where) + ": " + cudaGetErrorString(e));
        return BM_ERR_CUDA;
    }
    return BM_OK;
}

namespace {

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

// Stream-ordered allocation from the World's pool (freed with cudaFreeAsync).
template <class T>
bm_status_t dmalloc(T** p, size_t n, cudaStream_t st, cudaMemPool_t pool) {
    *p = nullptr;
    if (n == 0) n = 1;
    BM_CHECK_CUDA(cudaMallocFromPoolAsync((void**)p, sizeof(T) * n, pool, st));
    return BM_OK;
}

}  // namespace

bm_status_t World::init() {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_last_error("no CUDA device");
        return BM_ERR_NO_DEVICE;
    }
    BM_CHECK_CUDA(cudaGetDevice(&device));
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
    BM_CHECK_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    // Scene buffers come from a pool of this World that keeps freed memory
    // for the next scene: the served form admits and retires scenes all the
    // time, and returning the memory to the driver at every synchronisation
    // (the default pool's behaviour) made each admission map hundreds of MB
    // afresh.
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    BM_CHECK_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = UINT64_MAX;
    BM_CHECK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    BM_CHECK_CUDA(cudaStreamCreateWithFlags(&upload, cudaStreamNonBlocking));
    BM_CHECK_CUDA(cudaEventCreateWithFlags(&upload_done, cudaEventDisableTiming));
    BM_CHECK_CUDA(cudaMalloc((void**)&d_repair, kWorldWords * sizeof(uint32_t)));
    BM_CHECK_CUDA(cudaMemsetAsync(d_repair, 0, kWorldWords * sizeof(uint32_t), stream));
    return BM_OK;
}

bm_status_t World::stage_begin(size_t bytes, void** out) {
    // a slot whose copies have run (an event never recorded counts as done),
    // searched from the one after the last handed out
    const int n = (int)stage.size();
    int k = -1;
    for (int q = 0; q < n && k < 0; ++q) {
        const int c = (stage_next + q) % n;
        const cudaError_t e = cudaEventQuery(stage[c].used);
        if (e == cudaSuccess) k = c;
        else if (e != cudaErrorNotReady) BM_CHECK_CUDA(e);
    }
    if (k < 0 && n < kMaxStageSlots) {
        StageSlot slot;
        BM_CHECK_CUDA(cudaEventCreateWithFlags(&slot.used, cudaEventDisableTiming));
        stage.push_back(slot);
        k = n;
    }
    if (k < 0) {  // every slot in flight: wait for the next in turn
        k = stage_next % n;
        BM_CHECK_CUDA(cudaEventSynchronize(stage[k].used));
    }
    StageSlot& sl = stage[k];
    if (sl.cap < bytes) {
        give_stage_block(sl.buf, sl.cap);
        sl.buf = nullptr;
        sl.cap = 0;
        if (!take_stage_block(bytes, &sl.buf, &sl.cap)) {
            const size_t cap = std::max<size_t>(bytes * 2, 1 << 16);
            BM_CHECK_CUDA(cudaMallocHost(&sl.buf, cap));
            sl.cap = cap;
        }
    }
    stage_cur = k;
    *out = sl.buf;
    return BM_OK;
}

void World::stage_done() {
    if (stage_cur < 0) return;
    cudaEventRecord(stage[stage_cur].used, stream);
    stage_next = (stage_cur + 1) % (int)stage.size();
    stage_cur = -1;
}

void World::free_scene(SceneHost& h) {
    SceneDev& d = h.dev;
    auto drop = [&](void* p) {
        if (p) cudaFreeAsync(p, stream);
    };
    for (auto& s : d.store) {
        drop(s.base);
        drop(s.pid);
        s = ParticleSoA{nullptr, nullptr, 0, 0};
    }
    for (auto& a : d.acc) {
        drop(a.mv);
        drop(a.f);
        drop(a.touched);
        drop(a.list);
        drop(a.count);
        a = GridAcc{};
    }
    drop(d.alloc);
    drop(d.key);
    drop(d.rank);
    drop(d.status);
    drop(d.escaped);
    drop(h.d_inv);
    d.alloc = nullptr;
    d.key = d.rank = nullptr;
    d.status = nullptr;
    d.escaped = nullptr;
    h.d_inv = nullptr;
}

void World::release() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& h : scenes) free_scene(h);
    scenes.clear();
    cudaFree(d_scenes);
    cudaFree(d_prefix);
    cudaFree(sort.count);
    cudaFree(sort.start);
    cudaFree(sort.tile_sum);
    d_scenes = nullptr;
    d_prefix = nullptr;
    sort = SortBuffers{};
    for (auto& p : pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    pending.clear();
    for (auto e : event_pool) cudaEventDestroy(e);
    event_pool.clear();
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    t0 = t1 = nullptr;
    if (stream) cudaStreamSynchronize(stream);
    if (upload) cudaStreamSynchronize(upload);
    for (auto& sl : stage) {
        give_stage_block(sl.buf, sl.cap);  // the streams are idle: no copy reads it
        if (sl.used) cudaEventDestroy(sl.used);
    }
    stage.clear();
    stage_next = 0;
    stage_cur = -1;
    for (int k = 0; k < 2; ++k) {
        if (read_done[k]) cudaEventDestroy(read_done[k]);
        read_done[k] = nullptr;
    }
    if (upload_done) cudaEventDestroy(upload_done);
    upload_done = nullptr;
    cudaFree(d_repair);
    d_repair = nullptr;
    if (upload) cudaStreamDestroy(upload);
    upload = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    if (pool) cudaMemPoolDestroy(pool);
    pool = nullptr;
}

void World::remove_scene(int index) {
    if (index < 0 || index >= (int)scenes.size()) return;
    free_scene(scenes[index]);  // stream-ordered: after the work already queued
    scenes.erase(scenes.begin() + index);
    dirty = true;
}

bm_status_t World::p2g_fresh() {
    timed("p2g", [&] { launch_p2g(table(), n_ctas(), cur, sel, stream, true); });
    return launch_status("p2g_fresh");
}

int World::add_scene() {
    scenes.emplace_back();
    SceneHost& h = scenes.back();
    if (dmalloc(&h.dev.status, 1, stream, pool) == BM_OK && dmalloc(&h.dev.escaped, 3, stream, pool) == BM_OK) {
        cudaMemsetAsync(h.dev.status, 0, sizeof(uint32_t), stream);
        cudaMemsetAsync(h.dev.escaped, 0, 3 * sizeof(unsigned long long), stream);
    }
    dirty = true;
    return (int)scenes.size() - 1;
}

Material World::material(const SceneHost& h) const {
    Material m;
    m.mu = h.E / (2.0f * (1.0f + h.nu));
    m.lambda = h.E * h.nu / ((1.0f + h.nu) * (1.0f - 2.0f * h.nu));
    const float koh = (3.0f * m.lambda + 2.0f * m.mu) / (2.0f * m.mu);
    m.neg_alpha_koh = -h.alpha * koh;
    m.floor_friction = h.floor_friction;
    m.gx = h.gravity[0];
    m.gy = h.gravity[1];
    m.gz = h.gravity[2];
    return m;
}

bm_status_t World::ensure_particle_capacity(SceneHost& h, int64_t need) {
    if (need <= h.cap()) return BM_OK;
    if (need > INT32_MAX) return invalid_arg("more than 2^31-1 particles in one scene");
    int64_t cap = std::max<int64_t>(need, std::max<int64_t>(1024, h.cap() * 3 / 2));
    cap = (cap + 31) / 32 * 32;
    const int64_t n = h.n();
    ParticleSoA fresh[2];
    for (int s = 0; s < 2; ++s) {
        fresh[s] = ParticleSoA{nullptr, nullptr, cap, n};
        bm_status_t st = dmalloc(&fresh[s].base, (size_t)N_PLANES * cap, stream, pool);
        if (st == BM_OK) st = dmalloc(&fresh[s].pid, (size_t)cap, stream, pool);
        if (st != BM_OK) return st;
    }
    const ParticleSoA& old = h.dev.store[sel];
    if (old.base && n > 0) {
        for (int p = 0; p < N_PLANES; ++p)
            BM_CHECK_CUDA(cudaMemcpyAsync(fresh[sel].plane(p), old.plane(p), sizeof(float) * n,
                                          cudaMemcpyDeviceToDevice, stream));
        BM_CHECK_CUDA(cudaMemcpyAsync(fresh[sel].pid, old.pid, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, stream));
    }
    for (auto& s : h.dev.store) {
        if (s.base) cudaFreeAsync(s.base, stream);
        if (s.pid) cudaFreeAsync(s.pid, stream);
    }
    h.dev.store[0] = fresh[0];
    h.dev.store[1] = fresh[1];
    for (int32_t** p : {&h.dev.key, &h.dev.rank, &h.d_inv}) {
        if (*p) cudaFreeAsync(*p, stream);
        bm_status_t st = dmalloc(p, (size_t)cap, stream, pool);
        if (st != BM_OK) return st;
    }
    dirty = true;
    return BM_OK;
}

void World::update_bbox(SceneHost& h, int64_t n, const float* pos) {
    if (h.domain_set || h.grid_ready) return;  // the box is fixed: the bounds are never read
    // finite coordinates only; min/max in float convert exactly to double
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    bool any[3] = {false, false, false};
    for (int64_t p = 0; p < n; ++p)
        for (int a = 0; a < 3; ++a) {
            const float v = pos[3 * p + a];
            const bool ok = std::fabs(v) <= FLT_MAX;  // false for NaN and infinities
            lo[a] = ok && v < lo[a] ? v : lo[a];
            hi[a] = ok && v > hi[a] ? v : hi[a];
            any[a] = any[a] || ok;
        }
    for (int a = 0; a < 3; ++a)
        if (any[a]) {
            h.bbox_lo[a] = std::min(h.bbox_lo[a], (double)lo[a]);
            h.bbox_hi[a] = std::max(h.bbox_hi[a], (double)hi[a]);
        }
}

bm_status_t World::upload_bytes(void* d_dst, const void* h_src, size_t bytes) {
    ReadBack& rb = read_back();
    std::lock_guard<std::mutex> lk(rb.mu);
    for (int k = 0; k < 2; ++k) {
        if (!rb.buf[k]) BM_CHECK_CUDA(cudaMallocHost(&rb.buf[k], kReadChunk));
        if (!read_done[k]) BM_CHECK_CUDA(cudaEventCreateWithFlags(&read_done[k], cudaEventDisableTiming));
    }
    DrainPinned drain{read_done};
    const char* src = static_cast<const char*>(h_src);
    char* dst = static_cast<char*>(d_dst);
    // chunk i is copied into a pinned buffer while the DMA of chunk i-1 runs;
    // a buffer is refilled only after the DMA that read it finished
    size_t off = 0;
    int k = 0;
    while (off < bytes) {
        const size_t len = std::min(kReadChunk, bytes - off);
        if (drain.in_flight[k]) BM_CHECK_CUDA(cudaEventSynchronize(read_done[k]));
        host_copy(rb.buf[k], src + off, len);
        drain.in_flight[k] = true;  // from here a failed enqueue may still have left a copy running
        BM_CHECK_CUDA(cudaMemcpyAsync(dst + off, rb.buf[k], len, cudaMemcpyHostToDevice, upload));
        BM_CHECK_CUDA(cudaEventRecord(read_done[k], upload));
        k ^= 1;
        off += len;
    }
    // the pinned pair is shared: its DMAs end before another caller may refill it
    for (int q = 0; q < 2; ++q)
        if (drain.in_flight[q]) BM_CHECK_CUDA(cudaEventSynchronize(read_done[q]));
    return BM_OK;
}

bm_status_t World::read_fields(SceneHost& h, const ReadField* fields, int n_fields) {
    const int64_t n = h.n();
    if (n == 0) return BM_OK;
    const ParticleSoA& ps = h.dev.store[sel];
    // the sort's destination store is scratch between steps (N_PLANES >= 9
    // floats per particle)
    float* rows = h.dev.store[sel ^ 1].base;
    ReadBack& rb = read_back();
    std::lock_guard<std::mutex> lk(rb.mu);
    void* const* read_buf = rb.buf;
    for (int k = 0; k < 2; ++k) {
        if (!rb.buf[k]) BM_CHECK_CUDA(cudaMallocHost(&rb.buf[k], kReadChunk));
        if (!read_done[k]) BM_CHECK_CUDA(cudaEventCreateWithFlags(&read_done[k], cudaEventDisableTiming));
    }
    DrainPinned drain{read_done};
    for (int f = 0; f < n_fields; ++f) {
        if (!fields[f].dst) continue;
        launch_gather_rows(ps, fields[f].plane, fields[f].width, rows, stream);
        char* dst = reinterpret_cast<char*>(fields[f].dst);
        const char* src = reinterpret_cast<const char*>(rows);
        const size_t bytes = sizeof(float) * (size_t)fields[f].width * (size_t)n;
        // the DMA of chunk i overlaps the host copy of chunk i-1 (a buffer is
        // refilled only after its host copy returned)
        size_t off = 0, prev_off = 0, prev_len = 0;
        int k = 0;
        while (off < bytes) {
            const size_t len = std::min(kReadChunk, bytes - off);
            drain.in_flight[k] = true;
            BM_CHECK_CUDA(cudaMemcpyAsync(read_buf[k], src + off, len, cudaMemcpyDeviceToHost, stream));
            BM_CHECK_CUDA(cudaEventRecord(read_done[k], stream));
            if (prev_len) {
                BM_CHECK_CUDA(cudaEventSynchronize(read_done[k ^ 1]));
                host_copy(dst + prev_off, read_buf[k ^ 1], prev_len);
            }
            prev_off = off;
            prev_len = len;
            k ^= 1;
            off += len;
        }
        if (prev_len) {
            BM_CHECK_CUDA(cudaEventSynchronize(read_done[k ^ 1]));
            host_copy(dst + prev_off, read_buf[k ^ 1], prev_len);
        }
    }
    return launch_status("read particles");
}

bm_status_t World::append_particles(SceneHost& h, int64_t n, const float* pos, const float* vel, const float* mass) {
    const int64_t n0 = h.n();
    bm_status_t st = ensure_particle_capacity(h, n0 + n);
    if (st != BM_OK) return st;
    // only the caller's rows cross PCIe (28 B per particle); a kernel fills
    // the remaining planes
    float* rows = nullptr;
    const size_t nf = (size_t)n * (vel ? 7 : 4);
    st = dmalloc(&rows, nf, upload, pool);
    if (st != BM_OK) return st;
    float* d_pos = rows;
    float* d_mass = rows + 3 * (size_t)n;
    float* d_vel = vel ? rows + 4 * (size_t)n : nullptr;
    st = upload_bytes(d_pos, pos, sizeof(float) * 3 * n);
    if (st == BM_OK && mass) st = upload_bytes(d_mass, mass, sizeof(float) * n);
    if (st == BM_OK && vel) st = upload_bytes(d_vel, vel, sizeof(float) * 3 * n);
    if (st != BM_OK) return st;
    BM_CHECK_CUDA(cudaEventRecord(upload_done, upload));
    BM_CHECK_CUDA(cudaStreamWaitEvent(stream, upload_done, 0));
    launch_fill_particles(h.dev.store[sel], n0, n, d_pos, d_vel, mass ? d_mass : nullptr, h.density, stream);
    cudaFreeAsync(rows, stream);
    st = launch_status("append_particles");
    if (st != BM_OK) return st;
    // the caller may reuse its arrays when this returns, pinned ones too:
    // wait for the copies only (not for the compute stream)
    BM_CHECK_CUDA(cudaStreamSynchronize(upload));
    h.dev.store[0].n = h.dev.store[1].n = n0 + n;
    update_bbox(h, n, pos);
    dirty = true;
    return BM_OK;
}

bm_status_t World::ensure_grid(SceneHost& h) {
    if (h.grid_ready) return BM_OK;
    if (!h.domain_set) {
        if (h.n() == 0) return invalid_arg("grid box unknown: no particles and no domain");
        const float dx = h.dev.g.dx;
        bm_domain_t d;
        for (int a = 0; a < 3; ++a) {
            const int lo = (int)std::floor(h.bbox_lo[a] / dx - 0.5) - h.margin;
            const int hi = (int)std::floor(h.bbox_hi[a] / dx - 0.5) + 3 + h.margin;
            d.origin[a] = lo;
            d.extent[a] = hi - lo;
        }
        h.domain = d;
        h.domain_set = true;
    }
    const float dx = h.dev.g.dx;
    GridDesc g = desc_from_domain(h.domain, dx);
    const int64_t nn = g.num_nodes(), nb = g.num_blocks();
    if (nn <= 0 || nn > (int64_t)INT32_MAX / 2) return invalid_arg("grid box too large or empty");
    h.dev.g = g;
    for (auto& a : h.dev.acc) {
        bm_status_t st = dmalloc(&a.mv, (size_t)nn, stream, pool);
        if (st == BM_OK) st = dmalloc(&a.f, (size_t)nn, stream, pool);
        if (st == BM_OK) st = dmalloc(&a.touched, (size_t)nb, stream, pool);
        if (st == BM_OK) st = dmalloc(&a.list, (size_t)nb, stream, pool);
        if (st == BM_OK) st = dmalloc(&a.count, 1, stream, pool);
        if (st != BM_OK) return st;
        BM_CHECK_CUDA(cudaMemsetAsync(a.mv, 0, sizeof(float4) * nn, stream));
        BM_CHECK_CUDA(cudaMemsetAsync(a.f, 0, sizeof(float4) * nn, stream));
        BM_CHECK_CUDA(cudaMemsetAsync(a.touched, 0, sizeof(uint32_t) * nb, stream));
        BM_CHECK_CUDA(cudaMemsetAsync(a.count, 0, sizeof(int32_t), stream));
    }
    bm_status_t st = dmalloc(&h.dev.alloc, (size_t)nb, stream, pool);
    if (st != BM_OK) return st;
    BM_CHECK_CUDA(cudaMemsetAsync(h.dev.alloc, 0, (size_t)nb, stream));
    h.grid_ready = true;
    dirty = true;
    return BM_OK;
}

int64_t World::max_blocks() const {
    int64_t m = 0;
    for (const auto& h : scenes) m = std::max<int64_t>(m, h.dev.g.num_blocks());
    return m;
}

bm_status_t World::sync_table() {
    if (!dirty) return BM_OK;
    const int ns = (int)scenes.size();
    prefix.assign(ns + 1, 0);
    int64_t keys = 0;
    std::vector<SceneDev> host(ns);
    for (int s = 0; s < ns; ++s) {
        SceneHost& h = scenes[s];
        h.dev.mat = material(h);
        h.dev.key_base = keys;
        if (h.grid_ready) keys += sort_keys_of(h.dev.g, h.dev.bin_shift);
        prefix[s + 1] = prefix[s] + (h.n() + kParticleCTA - 1) / kParticleCTA;
        host[s] = h.dev;
    }
    if (keys >= (int64_t)INT32_MAX) return invalid_arg("too many grid nodes in one table");
    if ((size_t)ns > table_cap) {
        cudaFree(d_scenes);
        cudaFree(d_prefix);
        d_scenes = nullptr;
        d_prefix = nullptr;
        const size_t cap = std::max<size_t>(ns, table_cap * 2);
        BM_CHECK_CUDA(cudaMalloc((void**)&d_scenes, sizeof(SceneDev) * cap));
        BM_CHECK_CUDA(cudaMalloc((void**)&d_prefix, sizeof(int64_t) * (cap + 1)));
        table_cap = cap;
    }
    if (keys > sort_cap) {
        cudaFree(sort.count);
        cudaFree(sort.start);
        cudaFree(sort.tile_sum);
        const int64_t cap = std::max<int64_t>(keys, sort_cap * 3 / 2);
        BM_CHECK_CUDA(cudaMalloc((void**)&sort.count, sizeof(int32_t) * cap));
        BM_CHECK_CUDA(cudaMalloc((void**)&sort.start, sizeof(int32_t) * (cap + 1)));
        BM_CHECK_CUDA(cudaMalloc((void**)&sort.tile_sum, sizeof(int64_t) * std::max<int64_t>(1, scan_tiles(cap))));
        sort_cap = cap;
    }
    sort.nkeys = keys;
    for (int c = 0; c < 2; ++c)
        for (int p = 0; p < 2; ++p) {
            h_views[c][p].resize(ns);
            for (int q = 0; q < ns; ++q) h_views[c][p][q] = fused_view(host[q], c, p);
        }
    if (ns > 0) {
        // one pinned staging buffer: the scene table, the prefix
        auto up16 = [](size_t b) { return (b + 15) & ~size_t(15); };
        const size_t sb = up16(sizeof(SceneDev) * ns), pb = sizeof(int64_t) * (ns + 1);
        void* buf = nullptr;
        bm_status_t st = stage_begin(sb + pb, &buf);
        if (st != BM_OK) return st;
        char* b = static_cast<char*>(buf);
        std::memcpy(b, host.data(), sizeof(SceneDev) * ns);
        std::memcpy(b + sb, prefix.data(), pb);
        BM_CHECK_CUDA(cudaMemcpyAsync(d_scenes, b, sizeof(SceneDev) * ns, cudaMemcpyHostToDevice, stream));
        BM_CHECK_CUDA(cudaMemcpyAsync(d_prefix, b + sb, pb, cudaMemcpyHostToDevice, stream));
        stage_done();
    }
    dirty = false;
    return BM_OK;
}

bm_status_t World::clear_and_p2g() {
    timed("grid_clear", [&] {
        for (auto& h : scenes) {
            if (!h.grid_ready) continue;
            const GridAcc& a = h.dev.acc[cur];
            const int64_t nn = h.dev.g.num_nodes(), nb = h.dev.g.num_blocks();
            cudaMemsetAsync(a.mv, 0, sizeof(float4) * nn, stream);
            cudaMemsetAsync(a.f, 0, sizeof(float4) * nn, stream);
            cudaMemsetAsync(a.touched, 0, sizeof(uint32_t) * nb, stream);
            cudaMemsetAsync(a.count, 0, sizeof(int32_t), stream);
        }
    });
    timed("p2g", [&] { launch_p2g(table(), n_ctas(), cur, sel, stream); });
    return launch_status("p2g");
}

bm_status_t World::update(bool folded) {
    const LightRepair repair{d_repair, n_ctas(), sel, num_sms};
    timed("grid_update", [&] { launch_grid_update(table(), max_blocks(), cur, folded, stream, &repair); });
    return launch_status("grid_update");
}

bm_status_t World::g2p() {
    timed("g2p", [&] { launch_g2p(table(), n_ctas(), cur, sel, stream); });
    return launch_status("g2p");
}

bm_status_t World::g2p2g(bool fast_math, int variant) {
    timed("g2p2g", [&] {
        if (scenes.size() == 1) {
            SceneDev d = scenes[0].dev;
            d.mat = material(scenes[0]);
            launch_g2p2g_one(fused_view(d, cur, sel), fast_math, variant, cur == 1, stream);
        } else {
            launch_g2p2g_many(h_views[cur][sel].data(), prefix.data(), (int)scenes.size(), fast_math, variant,
                              cur == 1, stream);
        }
    });
    cur = 1 - cur;
    return launch_status("g2p2g");
}

bm_status_t World::sort_particles() {
    timed("bin_sort", [&] { launch_sort(table(), n_ctas(), sel, sort, stream); });
    sel = 1 - sel;
    return launch_status("bin_sort");
}

void World::fold_pending() {
    if (pending.empty()) return;
    cudaEventSynchronize(pending.back().b);
    for (auto& p : pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        slots[p.slot].total_ms += ms;
        slots[p.slot].launches += 1;
        event_pool.push_back(p.a);
        event_pool.push_back(p.b);
    }
    pending.clear();
}

}  // namespace bm
