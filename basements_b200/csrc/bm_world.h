// bm_world.h — host core: a set of scenes on one device and one stream.
//
// The plain solver (bm_solver.cu) owns a World of one scene; the batched form
// (bm_batch.cu) and the serving loop own Worlds of many scenes. A World keeps
// each scene's device buffers, the device scene table the kernels read, and
// the shared counting-sort arrays, and launches each phase of the step for
// all its scenes at once.
#pragma once
#include <cstring>
#include <string>
#include <vector>

#include "bm_internal.h"

namespace bm {

#define BM_CHECK_CUDA(expr)                                                                       \
    do {                                                                                          \
        cudaError_t e__ = (expr);                                                                 \
        if (e__ != cudaSuccess) {                                                                 \
            set_last_error(std::string(#expr) + ": " + cudaGetErrorString(e__));                  \
            return e__ == cudaErrorMemoryAllocation ? BM_ERR_OUT_OF_MEMORY : BM_ERR_CUDA;         \
        }                                                                                         \
    } while (0)

bm_status_t invalid_arg(const char* what);
bm_status_t launch_status(const char* where);

// Host side of one scene.
struct SceneHost {
    SceneDev dev{};  // host copy of the device descriptor
    // MPMSolver parameters (mpm_solver.h:100-109 defaults)
    float E = 1.0e5f, nu = 0.3f, density = 1500.0f, alpha = 0.40f, floor_friction = 0.4f;
    float gravity[3] = {0.0f, -9.81f, 0.0f};
    // particle bounds seen so far (for the automatic box)
    double bbox_lo[3] = {1e300, 1e300, 1e300}, bbox_hi[3] = {-1e300, -1e300, -1e300};
    bool domain_set = false;
    bm_domain_t domain{};
    int32_t margin = 16;
    bool grid_ready = false;
    int32_t* d_inv = nullptr;  // add order -> stored slot (scratch of set_particles)
    int64_t n() const { return dev.store[0].n; }
    int64_t cap() const { return dev.store[0].cap; }
};

struct ProfileSlot {
    const char* name;
    double total_ms = 0;
    int64_t launches = 0;
};

class World {
public:
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;  // scene buffers (kept for reuse when freed)
    // Host-to-device copies from pageable memory block their stream until all
    // earlier work on it has run; particle uploads therefore go on their own
    // stream, ordered before the compute stream's next kernel by an event.
    cudaStream_t upload = nullptr;
    cudaEvent_t upload_done = nullptr;
    // Pinned staging for small uploads on `stream` (the scene table, the
    // served form's body arrays): a ring of slots, each rewritten only after
    // the copies that read it ran. Those copies wait on the stream behind the
    // work already enqueued, so a slot stays busy for as long as the GPU lags
    // the host; the ring takes any slot whose copies have landed and grows
    // (up to kMaxStageSlots) instead of waiting for one.
    struct StageSlot {
        void* buf = nullptr;
        size_t cap = 0;
        cudaEvent_t used = nullptr;
    };
    static constexpr int kMaxStageSlots = 32;
    std::vector<StageSlot> stage;
    int stage_next = 0;  // where the search for a free slot starts
    int stage_cur = -1;  // slot handed out by the last stage_begin
    // Events of the pinned chunk pair through which read_fields brings
    // particle rows back into pageable host arrays and upload_bytes sends
    // them up.
    cudaEvent_t read_done[2] = {nullptr, nullptr};
    // Device words of the grid update, the light-node repair and the
    // single-body M1 launch (kWorldWords, LightRepair::word), zero between
    // launches.
    uint32_t* d_repair = nullptr;
    std::vector<SceneHost> scenes;
    int cur = 0;  // accumulation buffer of the current step
    int sel = 0;  // current particle store

    // Device table (rebuilt by sync_table when `dirty`).
    SceneDev* d_scenes = nullptr;
    int64_t* d_prefix = nullptr;
    size_t table_cap = 0;
    std::vector<int64_t> prefix;
    bool dirty = true;
    SortBuffers sort{};
    int64_t sort_cap = 0;
    // The fused kernel's view of every scene for each (cur, sel), on the host:
    // the many-scene kernel takes them as a kernel parameter.
    std::vector<FusedScene> h_views[2][2];

    // Profiling with CUDA events on the stream.
    bool profiling = false;
    std::vector<ProfileSlot> slots;
    struct Pending { int slot; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    cudaEvent_t t0 = nullptr, t1 = nullptr;

    bm_status_t init();
    void release();

    // Scenes.
    int add_scene();
    Material material(const SceneHost& h) const;
    bm_status_t ensure_particle_capacity(SceneHost& h, int64_t need);
    bm_status_t ensure_grid(SceneHost& h);
    bm_status_t append_particles(SceneHost& h, int64_t n, const float* pos, const float* vel, const float* mass);
    void update_bbox(SceneHost& h, int64_t n, const float* pos);
    // Copies fields of a scene's particles (AoS rows, add order) into host
    // arrays: rows gathered into the idle particle store, brought back
    // through the pinned chunk pair. Waits for the copies.
    struct ReadField { float* dst; int plane; int width; };
    bm_status_t read_fields(SceneHost& h, const ReadField* fields, int n_fields);
    // Host-to-device copy on the upload stream through the same pinned pair;
    // returns when the copy has landed.
    bm_status_t upload_bytes(void* d_dst, const void* h_src, size_t bytes);
    void free_scene(SceneHost& h);
    void remove_scene(int index);
    // P2G into acc[cur] of the scenes flagged `fresh` (their accumulators
    // are still zero), leaving the other scenes' precomputed P2G alone.
    bm_status_t p2g_fresh();

    // A pinned buffer of at least `bytes` for copies enqueued on `stream`;
    // stage_done() after enqueueing the copies that read it.
    bm_status_t stage_begin(size_t bytes, void** out);
    void stage_done();

    // Device table.
    bm_status_t sync_table();
    SceneTable table() const { return SceneTable{d_scenes, d_prefix, (int)scenes.size()}; }
    int64_t n_ctas() const { return prefix.empty() ? 0 : prefix.back(); }
    int64_t max_blocks() const;

    // Phases, for every scene of the table.
    bm_status_t clear_and_p2g();  // grid.clear() + P2G into acc[cur]
    bm_status_t update(bool folded);
    bm_status_t g2p();
    bm_status_t g2p2g(bool fast_math, int variant);  // flips cur
    bm_status_t sort_particles();                      // flips sel

    // Profiling.
    template <class Fn>
    void timed(const char* name, Fn&& fn);
    void fold_pending();
};

template <class Fn>
void World::timed(const char* name, Fn&& fn) {
    if (!profiling) {
        fn();
        return;
    }
    int slot = -1;
    for (size_t i = 0; i < slots.size(); ++i)
        if (std::strcmp(slots[i].name, name) == 0) slot = (int)i;
    if (slot < 0) {
        slots.push_back(ProfileSlot{name});
        slot = (int)slots.size() - 1;
    }
    auto get_event = [&]() {
        cudaEvent_t e;
        if (!event_pool.empty()) {
            e = event_pool.back();
            event_pool.pop_back();
        } else {
            cudaEventCreate(&e);
        }
        return e;
    };
    Pending pe{slot, get_event(), get_event()};
    cudaEventRecord(pe.a, stream);
    fn();
    cudaEventRecord(pe.b, stream);
    pending.push_back(pe);
    if (pending.size() > 4096) fold_pending();
}

}  // namespace bm
