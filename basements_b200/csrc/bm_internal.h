// bm_internal.h — shared host/device definitions of the B200 MPM library.
//
// Every kernel works on a table of scenes (SceneTable): the plain solver is a
// table of one scene, the batched and served forms hold many scenes of uneven
// particle and grid counts, stepped together by the same launches.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/bm_mpm.h"

namespace bm {

// Device-side error bits, OR-ed into a scene's status word.
enum : uint32_t { ERR_ESCAPE = 1u, ERR_NONFINITE = 2u };

// Node mass (particle contributions only) from which a node counts as heavy
// for the light-contribution rule of the fused kernel: 100x the reference's
// 1e-6 threshold of update_grid (mpm_solver.h:257).
constexpr float kHeavyNodeMass = 1e-4f;

// Total mass of a node after the couplers of this step: the coupler keeps the
// particle mass in mv.w and writes the node's new total into f.w (0 until a
// coupler touches the node).
__host__ __device__ __forceinline__ float node_total_mass(const float4& mv, const float4& f) {
    return f.w != 0.0f ? f.w : mv.w;
}

// Threads per CTA of every per-particle kernel except the fused one (the
// CTA -> scene prefix table is built for this size; the fused kernel's
// variants use multiples of it).
constexpr int kParticleCTA = 128;

// Particle planes of the SoA store (each plane holds `cap` floats).
enum Plane : int {
    P_X = 0,   // position x, y, z       (3)
    P_V = 3,   // velocity               (3)
    P_F = 6,   // deformation gradient   (9, row-major)
    P_C = 15,  // APIC affine matrix     (9, row-major)
    P_M = 24,  // mass                   (1)
    P_V0 = 25, // reference volume V0    (1)
    N_PLANES = 26
};

// Dense grid box: nodes stored x-major with k fastest (node (i,j,k) at
// ((i-ox)*EY + (j-oy))*EZ + (k-oz)), so the 27 stencil nodes of a particle
// sit at constant offsets from its base node. The box is a whole number of
// 4^3-node blocks aligned to absolute node indices (the reference's block
// grid, spgrid_cpu.h:93-105); per-block flags (allocated, touched) use block
// (bi,bj,bk) = ((i-ox)>>2, (j-oy)>>2, (k-oz)>>2), local slot li*16+lj*4+lk.
struct GridDesc {
    int ox, oy, oz;       // origin node, multiple of 4
    int nbx, nby, nbz;    // blocks per axis
    float dx, inv_dx;
    __host__ __device__ int ex() const { return nbx * 4; }
    __host__ __device__ int ey() const { return nby * 4; }
    __host__ __device__ int ez() const { return nbz * 4; }
    __host__ __device__ int64_t num_blocks() const { return (int64_t)nbx * nby * nbz; }
    __host__ __device__ int64_t num_nodes() const { return num_blocks() * 64; }
    __host__ __device__ __forceinline__ int64_t block_of(int bi, int bj, int bk) const {
        return ((int64_t)bi * nby + bj) * nbz + bk;
    }
    // Node index from box-relative coordinates (no check).
    __host__ __device__ __forceinline__ int64_t node_rel(int ri, int rj, int rk) const {
        return ((int64_t)ri * (nby * 4) + rj) * (nbz * 4) + rk;
    }
    // Linear node index, or -1 outside the box.
    __host__ __device__ __forceinline__ int64_t node(int i, int j, int k) const {
        const int ri = i - ox, rj = j - oy, rk = k - oz;
        if ((unsigned)ri >= (unsigned)(nbx * 4) || (unsigned)rj >= (unsigned)(nby * 4) ||
            (unsigned)rk >= (unsigned)(nbz * 4))
            return -1;
        return node_rel(ri, rj, rk);
    }
    // Block coordinates of block b (unsigned 32-bit division: a box holds
    // fewer than 2^31 nodes, so fewer than 2^25 blocks; 64-bit division would
    // cost several times the instructions in the per-node kernels).
    __host__ __device__ __forceinline__ void block_coords(int64_t b, int& bi, int& bj, int& bk) const {
        const unsigned ub = (unsigned)b, nz = (unsigned)nbz, ny = (unsigned)nby;
        const unsigned q = ub / nz, r = q / ny;
        bk = (int)(ub - q * nz);
        bj = (int)(q - r * ny);
        bi = (int)r;
    }
    // Node of block b at local slot t = li*16 + lj*4 + lk.
    __host__ __device__ __forceinline__ int64_t node_of_block(int64_t b, int t) const {
        int bi, bj, bk;
        block_coords(b, bi, bj, bk);
        return node_rel(4 * bi + (t >> 4), 4 * bj + ((t >> 2) & 3), 4 * bk + (t & 3));
    }
    // Block of a linear node index.
    __host__ __device__ __forceinline__ int64_t block_of_node(int64_t id) const {
        const int64_t ez_ = nbz * 4, ey_ = nby * 4;
        const int rk = (int)(id % ez_), rj = (int)((id / ez_) % ey_), ri = (int)(id / (ez_ * ey_));
        return block_of(ri >> 2, rj >> 2, rk >> 2);
    }
};

// Material and integration constants, derived on the host in float exactly
// like mpm_solver.h:111-112 and :149-151.
struct Material {
    float mu, lambda;
    float neg_alpha_koh;  // (-alpha) * (3 lambda + 2 mu) / (2 mu)
    float floor_friction;
    float gx, gy, gz;
};

struct ParticleSoA {
    float* base;   // N_PLANES planes of `cap` floats
    int32_t* pid;  // add-order index of each stored particle
    int64_t cap;
    int64_t n;
    __host__ __device__ __forceinline__ float* plane(int p) const { return base + (int64_t)p * cap; }
};

// One accumulation buffer of the grid: (momentum -> velocity, mass) and
// (force, 0) per node, plus the list of blocks that hold non-zero data.
struct GridAcc {
    float4* mv;
    float4* f;
    uint32_t* touched;  // per block: listed in `list`
    int32_t* list;      // touched block ids
    int32_t* count;     // number of entries in `list`
};

// Device descriptor of one scene. Two particle stores (the sort permutes
// from one into the other) and two grid accumulators (step n's grid and the
// next step's P2G); which ones are current is a launch parameter.
struct SceneDev {
    ParticleSoA store[2];
    GridDesc g;
    GridAcc acc[2];
    uint8_t* alloc;        // per block: ever touched (the reference's allocated blocks)
    Material mat;
    float dt;              // this scene's step
    int32_t* key;          // per particle: sort key (local)
    int32_t* rank;         // per particle: slot among equal keys
    int64_t key_base;      // first key of this scene in the shared counting-sort arrays
    int32_t bin_shift;     // sort bins are 2^bin_shift nodes per axis (0: one cell)
    int32_t fresh;         // 1: acc[cur] holds a standalone (unfolded) P2G this step
    uint32_t* status;      // error bits
    // [0] dropped stencil writes, [1] light-node suspects (k_grid_update),
    // [2] nonzero while this step's grid is being repaired (the suspects' step)
    unsigned long long* escaped;
};

struct SceneTable {
    const SceneDev* scenes;     // device array, n_scenes entries
    const int64_t* cta_prefix;  // n_scenes + 1: per-particle CTAs before each scene
    int n_scenes;
};

// Scene of particle CTA `cta` (binary search of the prefix table).
__device__ __forceinline__ int scene_of_cta(const SceneTable& t, int64_t cta) {
    int lo = 0, hi = t.n_scenes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t.cta_prefix[mid] <= cta) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// True in the last CTA of the launch to reach this call (every CTA must
// reach it): each CTA, after its own work, fences its writes and counts itself
// on *counter; the CTA that completes the count sees the others' writes and
// resets the counter for the next launch. Nothing waits.
__device__ __forceinline__ bool last_cta(uint32_t* counter) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned total = gridDim.x * gridDim.y * gridDim.z;
        last = atomicAdd(counter, 1u) == total - 1;
        if (last) *counter = 0u;
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// Marks block b as holding data in `a` (appends it to the list once).
__device__ __forceinline__ void touch_block(const GridAcc& a, int64_t b) {
    if (a.touched[b] == 0u && atomicExch(a.touched + b, 1u) == 0u) a.list[atomicAdd(a.count, 1)] = (int32_t)b;
}

// Marks the 4^3 blocks covered by the stencil nodes of non-zero 1-D weight
// (base..base+2 per axis, the end nodes dropped when their weight is 0) as
// allocated (the reference allocates a block on the first get_node() of any
// node in it, spgrid_cpu.h:78-91) and as holding data in `a`.
__device__ __forceinline__ void mark_stencil_blocks(const GridDesc& g, const GridAcc& a, uint8_t* alloc,
                                                    const int base[3], const float wx[3], const float wy[3],
                                                    const float wz[3]) {
    const int lo0 = base[0] + (wx[0] == 0.0f), hi0 = base[0] + 2 - (wx[2] == 0.0f);
    const int lo1 = base[1] + (wy[0] == 0.0f), hi1 = base[1] + 2 - (wy[2] == 0.0f);
    const int lo2 = base[2] + (wz[0] == 0.0f), hi2 = base[2] + 2 - (wz[2] == 0.0f);
    for (int i = (lo0 - g.ox) >> 2; i <= (hi0 - g.ox) >> 2; ++i)
        for (int j = (lo1 - g.oy) >> 2; j <= (hi1 - g.oy) >> 2; ++j)
            for (int k = (lo2 - g.oz) >> 2; k <= (hi2 - g.oz) >> 2; ++k) {
                if ((unsigned)i < (unsigned)g.nbx && (unsigned)j < (unsigned)g.nby && (unsigned)k < (unsigned)g.nbz) {
                    const int64_t blk = g.block_of(i, j, k);
                    if (alloc[blk] == 0) alloc[blk] = 1;
                    touch_block(a, blk);
                }
            }
}

// Sort keys of one scene: bins of 2^bin_shift nodes per axis in grid order,
// plus one key for particles outside the box.
__host__ __device__ __forceinline__ int64_t sort_keys_of(const GridDesc& g, int bin_shift) {
    const int m = (1 << bin_shift) - 1;
    return (int64_t)((g.ex() + m) >> bin_shift) * ((g.ey() + m) >> bin_shift) * ((g.ez() + m) >> bin_shift) + 1;
}

// Shared arrays of the counting sort (keys of all scenes, scene by scene:
// scene s owns keys [key_base, key_base + sort_keys_of(g, bin_shift)), the
// last one for particles outside its box).
struct SortBuffers {
    int32_t* count;      // nkeys
    int32_t* start;      // nkeys + 1
    int64_t* tile_sum;   // per scan tile
    int64_t nkeys;
};
int64_t scan_tiles(int64_t nkeys);

// ---- launchers (bm_kernels.cu) ----------------------------------------------------
// cur = accumulation buffer of the current step; sel = current particle store;
// n_ctas = per-particle CTAs of the table (cta_prefix[n_scenes]).
// only_fresh: skip scenes whose `fresh` flag is 0 (newly admitted scenes of
// a running table get their first P2G while the others keep theirs).
void launch_p2g(const SceneTable& t, int64_t n_ctas, int cur, int sel, cudaStream_t st, bool only_fresh = false);
// Device words of a World's grid update (kWorldWords: [0] set by the grid
// update when a scene found a light-node suspect, [1], [2] finished-CTA
// counts of the grid update and of the repair's update, [3] of the
// single-body M1 launch) and what the light-node repair's standalone P2G
// needs (the table's per-particle CTAs and the current particle store).
constexpr int kWorldWords = 4;
struct LightRepair {
    uint32_t* word;
    int64_t n_ctas;
    int sel;
    int num_sms;
};
// folded: acc[cur].mv holds momentum + force * dt (the force channel only
// holds the contributions of w*m <= 1e-6 particle-node pairs); scenes whose
// `fresh` flag is set are always treated as unfolded. With a folded grid, a
// scene with a light-node suspect has this step's grid redone from its
// particles unfolded (standalone P2G, update_grid), on the device.
void launch_grid_update(const SceneTable& t, int64_t max_blocks, int cur, bool folded, cudaStream_t st,
                        const LightRepair* repair);
void launch_g2p(const SceneTable& t, int64_t n_ctas, int cur, int sel, cudaStream_t st);
// Fused G2P of this step + P2G of the next (into acc[1-cur]), in one of the
// compiled launch shapes.
int fused_variant_count();
const char* fused_variant_name(int v);
// Index of the launch variant with this shape and lane order (0 if none).
int fused_variant_index(int threads, int min_blocks, int interleave);
// The fused kernel's view of one scene with the buffer choice (cur, sel)
// resolved: exactly the fields it touches, no runtime-indexed arrays.
struct FusedScene {
    float* base;          // store[sel] planes
    int64_t cap, n;
    GridDesc g;
    const float4* cur_mv;  // acc[cur].mv: this step's grid velocities
    GridAcc next;          // acc[1-cur]: the next step's P2G
    uint8_t* alloc;
    float mu, lambda, neg_alpha_koh, dt;
    uint32_t* status;
    unsigned long long* escaped;
    __host__ __device__ __forceinline__ float* plane(int p) const { return base + (int64_t)p * cap; }
};
FusedScene fused_view(const SceneDev& d, int cur, int sel);
// Views of up to kPackScenes scenes and their 128-thread units, passed to the
// many-scene fused kernel as one kernel parameter (kernel parameters of up to
// 32,764 bytes: CUDA 12.1 and later).
constexpr int kPackScenes = 160;
struct FusedPack {
    int64_t prefix[kPackScenes + 1];  // units before each scene of the pack
    FusedScene v[kPackScenes];
    int n;
};
static_assert(sizeof(FusedPack) <= 32000, "the pack fits the kernel-parameter limit");
// Single scene, its view passed by value; many scenes, host arrays of the
// views (one per scene) for this (cur, sel) and the table's CTA prefix: one
// launch per pack of scenes.
// `reverse` runs the CTAs in the opposite order (alternated step by step).
void launch_g2p2g_one(const FusedScene& scene, bool fast_math, int variant, bool reverse, cudaStream_t st);
void launch_g2p2g_many(const FusedScene* views, const int64_t* prefix, int n_scenes, bool fast_math, int variant,
                       bool reverse, cudaStream_t st);
// Counting sort of every scene's particles by stencil base node, from
// store[sel] into store[1-sel].
void launch_sort(const SceneTable& t, int64_t n_ctas, int sel, const SortBuffers& sb, cudaStream_t st);
void launch_gather_rows(const ParticleSoA& ps, int plane0, int width, float* out_add_order, cudaStream_t st);
void launch_scatter_rows(const ParticleSoA& ps, int plane0, int width, const float* in_rows, int64_t first,
                         int64_t n, const int32_t* inv, cudaStream_t st);
void launch_inverse_pid(const ParticleSoA& ps, int32_t* inv, cudaStream_t st);
// Particles [n0, n0 + n) of a store from device rows (pos n x 3, vel n x 3 or
// NULL, mass n or NULL): F = I, C = 0, V0 = m / density, pid = slot.
void launch_fill_particles(const ParticleSoA& s, int64_t n0, int64_t n, const float* pos, const float* vel,
                           const float* mass, float density, cudaStream_t st);

// ---- coupler and bodies (bm_m1.cu) ------------------------------------------------
// M1 parameters of one body for one step, computed on the host
// (m1_prepare) or on the device from the body state (batched form).
struct M1Params {
    float R[9];          // body-to-world rotation, row-major
    float c[3], vl[3], w[3];
    float he[3];
    float lo[3], hi[3];  // world AABB of the box formula
    float mb;            // per-node body mass
    float mb_over_dt;
    float friction;      // the body's friction (M0)
    int shape;
    int scene;           // scene whose grid the body couples to
    int active;          // 0: dt <= 0 or AABB outside the box -> no work
    int bi0, bj0, bk0, nbi, nbj, nbk;  // candidate block range (relative to box)
};
bool m1_prepare(const GridDesc& g, const bm_collider_t& b, float dt, int scene, M1Params* out);
// M0 for one body over `candidates` blocks of the M1 frame (m1_prepare):
// Dirichlet exchange on the nodes inside, reaction added into d_acc.
void launch_m0(const SceneTable& t, const M1Params* d_param, int64_t candidates, int cur, float dt, double* d_acc,
               cudaStream_t st);
// M4.5a frame of one body of scene 0: the shape's tight AABB in lo/hi, the
// body's mass in mb.
bool m45a_prepare(const GridDesc& g, const bm_collider_t& b, float dt, M1Params* out);
// The two passes of the sweep couplers for one body over `candidates` blocks
// (P.nbi * P.nbj * P.nbk): Sigma frac into *d_frac_sum (zeroed by the
// caller), then the exchange with the rule of layer 0 = M4.5a, 1 = M4.5b,
// 2 = M4.5, reaction added into d_acc (7 doubles, zeroed by the caller).
void launch_m45(const SceneTable& t, const M1Params* d_param, int64_t candidates, int cur, float dt,
                double* d_frac_sum, double* d_acc, int layer, cudaStream_t st);
// True when the candidate block ranges of two bodies of one scene intersect
// (they may then write the same nodes).
inline bool m1_blocks_overlap(const M1Params& a, const M1Params& b) {
    return a.bi0 < b.bi0 + b.nbi && b.bi0 < a.bi0 + a.nbi && a.bj0 < b.bj0 + b.nbj && b.bj0 < a.bj0 + a.nbj &&
           a.bk0 < b.bk0 + b.nbk && b.bk0 < a.bk0 + a.nbk;
}
// Candidate blocks the AABB of a body with these half extents can span.
int64_t m1_max_candidates(const GridDesc& g, const float half_extents[3]);
// One CTA of 64 threads per candidate block: grid (max_candidates, n_bodies).
void launch_m1(const SceneTable& t, const M1Params* d_params, int n_bodies, int64_t max_candidates, int cur,
               double* d_acc, cudaStream_t st);
// Flat grid: body b owns CTAs [d_cand_prefix[b], d_cand_prefix[b+1]) (each an
// upper bound of its candidate blocks, e.g. m1_max_candidates), total CTAs.
void launch_m1_flat(const SceneTable& t, const M1Params* d_params, int n_bodies, const int64_t* d_cand_prefix,
                    int64_t total_candidates, int cur, double* d_acc, cudaStream_t st);
// The FP64 sums of n_bodies bodies -> reactions in d_out; the sums are zeroed
// after reading (they start at zero for the next call).
void launch_reaction_finalize(double* d_acc, int n_bodies, bm_reaction_t* d_out, cudaStream_t st);
// One body of scene P.scene over its candidate blocks, P passed by value;
// the launch's last CTA writes the reaction to d_out and zeroes the sums
// (counter: a zero device word). Returns false, launching nothing, when the
// body has no candidate block (the caller finalizes then).
bool launch_m1_one(const SceneTable& t, const M1Params& P, int cur, double* d_acc, bm_reaction_t* d_out,
                   uint32_t* counter, cudaStream_t st);
// Loads the code of the M1 and reaction-finalize kernels on the current
// device (a no-op once loaded).
cudaError_t load_m1_kernels();

// Rigid bodies stepped on the device (batched and served forms), with the
// semi-implicit Euler update of include/basements/physics/dynamics/integrator.h:19-57.
struct BodyDev {
    bm_collider_t state;   // pose, velocities, extents, mass, shape
    float inv_mass;
    float inv_inertia[9];  // body-space inverse inertia (the reference integrator uses it as is)
    float gravity[3];
    float dt;
    int32_t dynamic;       // 0: kinematic (pose advanced by the velocities only)
    int32_t scene;
};
void launch_body_prepare(const SceneTable& t, const BodyDev* d_bodies, int n_bodies, M1Params* d_params,
                         cudaStream_t st);
void launch_body_integrate(BodyDev* d_bodies, int n_bodies, const double* d_acc, cudaStream_t st);
// out[k] = staged[k] with the state of old[src[k]] when src[k] >= 0.
void launch_body_remap(const BodyDev* d_old, BodyDev* d_out, const BodyDev* d_staged, const int32_t* d_src, int n,
                       cudaStream_t st);

// Dense (i,j,k) copies of one scene's grid (plain API).
void launch_grid_to_dense(const GridDesc& g, const GridAcc& a, const uint8_t* alloc, float* vel, float* force,
                          float* mass, uint8_t* active, uint8_t* balloc, cudaStream_t st);
void launch_dense_velocity_to_grid(const GridDesc& g, const GridAcc& a, const float* vel, cudaStream_t st);
void launch_seed_grid(const GridDesc& g, const GridAcc& a, uint8_t* alloc, int64_t n, const int32_t* ijk,
                      const float* vel, const float* mass, uint32_t* d_status, cudaStream_t st);

// Thread-local error text.
void set_last_error(const std::string& s);

}  // namespace bm
