// bm_kernels.cu — the MLS-MPM step kernels, over a table of scenes.
//
// Reference (2nugu/basements, include/basements/physics/mpm/mpm_solver.h):
//   step :71-87   p2g_single :168-248   update_grid :250-291
//   g2p_single :293-348   apply_plasticity :114-166
//
// Layout: particles are FP32 SoA planes (bm_internal.h, Plane); the grid is a
// dense box per scene with two float4 per node: (momentum, mass) and
// (force, 0). P2G scatters with 16-byte vector reductions into L2
// (red.global.add.v4.f32).
//
// Per-particle kernels map a CTA (or a 128-thread unit of it) to its scene by
// a binary search of the table's CTA prefix, so one launch covers scenes of
// any particle count; the grid update takes one grid row per scene.
//
// Step n of MPMSolver::step runs P2G(n), update_grid(n), G2P(n). P2G(n+1)
// only needs the particle state that G2P(n) produces, so the fused kernel
// k_g2p2g does G2P(n) and P2G(n+1) back to back while the particle is in
// registers: every particle is read once (x, F, m, V0) and written once
// (x, v, C, F) per step, and the Kirchhoff stress of P2G(n+1) comes from the
// SVD that the Drucker-Prager projection of G2P(n) already computed
// (F_new = U S V^T with known U and S), saving the reference's second SVD.
// Particles are kept in the order of their stencil base node
// floor(x/dx - 0.5) (grid order, k fastest) by a counting sort
// (warp-aggregated histogram, three-phase scan, permutation) that runs every
// few steps, so neighbouring threads share stencil nodes: the gather hits L1
// and a warp's reductions land on a few L2 lines. (A variant that
// accumulated each 4^3 bin's P2G in a shared-memory tile was 3.6x slower on
// B200: float atomics on shared memory are a compare-and-swap loop, and the
// per-bin barriers stalled the warps.)
#include <algorithm>
#include <cfloat>

#include "bm_internal.h"
#include "bm_math.cuh"

namespace bm {

namespace {

constexpr int kGridThreads = 256;
constexpr int kScanThreads = 1024;
constexpr int kScanTile = kScanThreads * 8;

// 16-byte vector reduction into global memory, no value returned. Written as
// PTX with the global state space: a pointer the compiler cannot prove
// global (one read from a scene table) otherwise becomes a generic atomic
// that returns its old value, which doubled the crossbar traffic and kept
// L1 busy checking the shared window.
__device__ __forceinline__ void red_v4(float4* a, float x, float y, float z, float w) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(a), "f"(x), "f"(y), "f"(z), "f"(w)
                 : "memory");
}

// Largest CTA of the fused kernel's launch shapes (its per-thread shared
// columns are sized for it).
constexpr int kMaxFusedThreads = 256;

// a[i] for a runtime i in {0,1,2} without indexing (keeps `a` in registers).
__device__ __forceinline__ float pick3(const float a[3], int i) { return i == 0 ? a[0] : (i == 1 ? a[1] : a[2]); }

__device__ __forceinline__ void report(const SceneDev& S, int dropped, bool finite) {
    if (!finite) atomicOr(S.status, ERR_NONFINITE);
    if (dropped) {
        atomicOr(S.status, ERR_ESCAPE);
        atomicAdd(S.escaped, (unsigned long long)dropped);
    }
}

// Particle handled by this thread: scene index and slot, or false.
struct PSlot {
    int s;
    int64_t p;
};
__device__ __forceinline__ bool particle_slot(const SceneTable& t, int sel, PSlot& out) {
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t unit = gtid / kParticleCTA;
    if (unit >= t.cta_prefix[t.n_scenes]) return false;
    const int s = scene_of_cta(t, unit);
    const int64_t p = (unit - t.cta_prefix[s]) * kParticleCTA + (gtid % kParticleCTA);
    if (p >= t.scenes[s].store[sel].n) return false;
    out.s = s;
    out.p = p;
    return true;
}

// ---- standalone P2G (grid.clear() + the P2G loop) --------------------------------

// The reference's P2G of one particle (mpm_solver.h:168-248) into acc[cur]:
// Kirchhoff stress from the SVD of F, momentum and force kept apart (N5).
// Returns the number of stencil writes dropped outside the box.
__device__ __forceinline__ int p2g_particle(const SceneDev& S, int cur, int sel, int64_t p) {
    const ParticleSoA ps = S.store[sel];
    const GridDesc g = S.g;
    const GridAcc acc = S.acc[cur];
    const float x[3] = {ps.plane(P_X)[p], ps.plane(P_X + 1)[p], ps.plane(P_X + 2)[p]};
    const float v[3] = {ps.plane(P_V)[p], ps.plane(P_V + 1)[p], ps.plane(P_V + 2)[p]};
    float F[9], Cm[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        F[q] = ps.plane(P_F + q)[p];
        Cm[q] = ps.plane(P_C + q)[p];
    }
    const float m = ps.plane(P_M)[p];
    const float vol = ps.plane(P_V0)[p];

    float fx[3], wgt[3][3];
    int base[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        fx[a] = x[a] * g.inv_dx - 0.5f;
        base[a] = (int)floorf(fx[a]);
        bspline_weights(fx[a] - (float)base[a], wgt[a]);
    }
    float tau[9];
    hencky_tau(F, S.mat.mu, S.mat.lambda, tau);
    const float ff = -4.0f * g.inv_dx * g.inv_dx * vol;
    float sk[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) sk[q] = tau[q] * ff;

    int dropped = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float w = wgt[0][i] * wgt[1][j] * wgt[2][k];
                if (w == 0.0f) continue;
                const int ni = base[0] + i, nj = base[1] + j, nk = base[2] + k;
                const float d0 = ((float)ni - fx[0] - 0.5f) * g.dx;
                const float d1 = ((float)nj - fx[1] - 0.5f) * g.dx;
                const float d2 = ((float)nk - fx[2] - 0.5f) * g.dx;
                const int64_t id = g.node(ni, nj, nk);
                if (id < 0) { ++dropped; continue; }
                const float a0 = (Cm[0] * d0 + Cm[1] * d1) + Cm[2] * d2;
                const float a1 = (Cm[3] * d0 + Cm[4] * d1) + Cm[5] * d2;
                const float a2 = (Cm[6] * d0 + Cm[7] * d1) + Cm[8] * d2;
                const float mc = w * m;
                const float s0 = (sk[0] * d0 + sk[1] * d1) + sk[2] * d2;
                const float s1 = (sk[3] * d0 + sk[4] * d1) + sk[5] * d2;
                const float s2 = (sk[6] * d0 + sk[7] * d1) + sk[8] * d2;
                red_v4(acc.mv + id, (v[0] + a0) * mc, (v[1] + a1) * mc, (v[2] + a2) * mc, mc);
                red_v4(acc.f + id, s0 * w, s1 * w, s2 * w, 0.0f);
            }
    mark_stencil_blocks(g, acc, S.alloc, base, wgt[0], wgt[1], wgt[2]);
    return dropped;
}

__global__ void __launch_bounds__(kParticleCTA) k_p2g(SceneTable t, int cur, int sel, bool only_fresh) {
    PSlot slot;
    if (!particle_slot(t, sel, slot)) return;
    const SceneDev& S = t.scenes[slot.s];
    if (only_fresh && !S.fresh) return;
    report(S, p2g_particle(S, cur, sel, slot.p), true);
}

// ---- grid update -------------------------------------------------------------------

// update_grid (mpm_solver.h:250-291) of node tt of listed block b of acc c.
// folded: the momentum already holds force * dt (the fused kernel's P2G).
__device__ __forceinline__ void update_node(const GridDesc& g, const GridAcc& c, const Material& mat, float dt,
                                            bool folded, int64_t b, int tt) {
    const int64_t id = g.node_of_block(b, tt);
    const float4 mv = c.mv[id];
    if (!(mv.w > 1e-6f)) {
        // inactive (mass 0) or mass <= 1e-6: the reference leaves the
        // momentum (without force) in place (mpm_solver.h:257)
        if (folded && (mv.w > 0.0f || mv.x != 0.0f || mv.y != 0.0f || mv.z != 0.0f)) {
            const float4 f = c.f[id];
            c.mv[id] = make_float4(mv.x - f.x * dt, mv.y - f.y * dt, mv.z - f.z * dt, mv.w);
        }
        return;
    }
    float v0, v1, v2;
    if (folded) {
        v0 = mv.x / mv.w;
        v1 = mv.y / mv.w;
        v2 = mv.z / mv.w;
    } else {
        const float4 f = c.f[id];
        v0 = (mv.x + f.x * dt) / mv.w;
        v1 = (mv.y + f.y * dt) / mv.w;
        v2 = (mv.z + f.z * dt) / mv.w;
    }
    v0 = v0 + mat.gx * dt;
    v1 = v1 + mat.gy * dt;
    v2 = v2 + mat.gz * dt;
    const int lj = (tt >> 2) & 3;
    const int bj = (int)(((unsigned)b / (unsigned)g.nbz) % (unsigned)g.nby);
    const int j = g.oy + 4 * bj + lj;
    const float node_y = ((float)j + 0.5f) * g.dx;
    if (node_y < g.dx && v1 < 0.0f) {
        const float vn = -v1;
        v1 = 0.0f;
        const float mag = sqrtf(v0 * v0 + v2 * v2);
        const float budget = mat.floor_friction * vn;
        if (mag > 1e-12f) {
            const float sc = smax(0.0f, (mag - budget) / mag);
            v0 = v0 * sc;
            v2 = v2 * sc;
        }
    }
    c.mv[id] = make_float4(v0, v1, v2, mv.w);
}

// update_grid over the blocks listed in acc[cur] of scene blockIdx.y (every
// other node of the box is empty, so skipping it is exact); the same launch
// zeroes the blocks listed in acc[1-cur] so that it can take the next P2G.
// Before zeroing a node of acc[1-cur] (the previous step's grid, particle
// mass in .w) it looks for light-node suspects: nodes whose particle mass
// was at least kHeavyNodeMass there and is in (0, 1e-6] in a folded
// acc[cur]. Only at such a node can the fused kernel have skipped a force
// record that update_grid needs (the mass lane of acc[cur] is not changed by
// this launch). A suspect is counted (escaped[1]) and marks its scene for
// the repair that follows (escaped[2], and repair[0] for the launch).
__global__ void __launch_bounds__(kGridThreads) k_grid_update(SceneTable t, int cur, bool folded_all,
                                                              uint32_t* words) {
    const SceneDev& S = t.scenes[blockIdx.y];
    const bool folded = folded_all && !S.fresh;
    const GridDesc g = S.g;
    const GridAcc c = S.acc[cur], o = S.acc[1 - cur];
    const Material mat = S.mat;
    const float dt = S.dt;
    const int n_cur = *c.count, n_other = *o.count;
    const int64_t total = (int64_t)(n_cur + n_other) * 64;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int slot = (int)(e >> 6), tt = (int)(e & 63);
        if (slot >= n_cur) {
            const int64_t b = o.list[slot - n_cur];
            const int64_t id = g.node_of_block(b, tt);
            if (folded && o.mv[id].w >= kHeavyNodeMass) {
                const float m_new = c.mv[id].w;
                if (m_new > 0.0f && m_new <= 1e-6f) {
                    atomicAdd(S.escaped + 1, 1ull);
                    S.escaped[2] = 1ull;
                    words[0] = 1u;
                }
            }
            o.mv[id] = make_float4(0.f, 0.f, 0.f, 0.f);
            o.f[id] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (tt == 0) o.touched[b] = 0u;
            continue;
        }
        update_node(g, c, mat, dt, folded, c.list[slot], tt);
    }
    // the last CTA: the zeroed acc[1-cur] of every scene takes the next P2G
    // (its list restarts), and a scene marked for the light-node repair has
    // its acc[cur] zeroed on the listed blocks (the list and the block flags
    // stay) for the repair's P2G
    if (!last_cta(words + 1)) return;
    for (int s = threadIdx.x; s < t.n_scenes; s += blockDim.x) *t.scenes[s].acc[1 - cur].count = 0;
    if (*(volatile uint32_t*)words == 0u) return;
    for (int s = 0; s < t.n_scenes; ++s) {
        const SceneDev& M = t.scenes[s];
        if (*(volatile unsigned long long*)(M.escaped + 2) == 0ull) continue;
        const GridAcc a = M.acc[cur];
        const int64_t n = (int64_t)(*a.count) * 64;
        for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
            const int64_t id = M.g.node_of_block(a.list[e >> 6], (int)(e & 63));
            a.mv[id] = make_float4(0.f, 0.f, 0.f, 0.f);
            a.f[id] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
}

// ---- exact repair of the light-node rule -----------------------------------------
//
// A scene marked by k_grid_update redoes this step's grid from its particles:
// acc[cur] is zeroed on its listed blocks (by the grid update's last CTA; the
// list and the block flags stay), the standalone P2G (momentum and force
// apart, stress from the SVD of F as in the reference) refills it, and
// update_grid runs unfolded. The result is the reference's grid for that
// step, N2 nodes included. Each kernel returns at once when words[0] is 0,
// the case of every step whose scenes saw no suspect.

// Standalone P2G of the marked scenes, CTAs striding over the table's
// 128-particle units (stencil writes outside the box were already counted by
// the fused kernel, so they are not counted again).
__global__ void __launch_bounds__(kParticleCTA) k_repair_p2g(SceneTable t, int cur, int sel, const uint32_t* words) {
    if (*words == 0u) return;
    const int64_t units = t.cta_prefix[t.n_scenes];
    for (int64_t unit = blockIdx.x; unit < units; unit += gridDim.x) {
        const int s = scene_of_cta(t, unit);
        const SceneDev& S = t.scenes[s];
        if (S.escaped[2] == 0ull) continue;
        const int64_t p = (unit - t.cta_prefix[s]) * kParticleCTA + threadIdx.x;
        if (p < S.store[sel].n) p2g_particle(S, cur, sel, p);
    }
}

// Unfolded update_grid of the marked scenes; the last CTA to finish clears
// the marks for the next step.
__global__ void __launch_bounds__(kGridThreads) k_repair_update(SceneTable t, int cur, uint32_t* words) {
    if (*words == 0u) return;
    const SceneDev& S = t.scenes[blockIdx.y];
    if (S.escaped[2] != 0ull) {
        const GridAcc c = S.acc[cur];
        const int64_t total = (int64_t)(*c.count) * 64;
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
             e += (int64_t)gridDim.x * blockDim.x)
            update_node(S.g, c, S.mat, S.dt, false, c.list[e >> 6], (int)(e & 63));
    }
    if (!last_cta(words + 2)) return;
    for (int s = threadIdx.x; s < t.n_scenes; s += blockDim.x) t.scenes[s].escaped[2] = 0ull;
    __syncthreads();
    if (threadIdx.x == 0) words[0] = 0u;
}

// ---- standalone G2P ---------------------------------------------------------------

__global__ void __launch_bounds__(kParticleCTA) k_g2p(SceneTable t, int cur, int sel) {
    PSlot slot;
    if (!particle_slot(t, sel, slot)) return;
    const SceneDev& S = t.scenes[slot.s];
    const ParticleSoA ps = S.store[sel];
    const GridDesc g = S.g;
    const GridAcc acc = S.acc[cur];
    const float dt = S.dt;
    const int64_t p = slot.p;
    float x[3] = {ps.plane(P_X)[p], ps.plane(P_X + 1)[p], ps.plane(P_X + 2)[p]};
    float F[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) F[q] = ps.plane(P_F + q)[p];
    float fx[3], wgt[3][3];
    int base[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        fx[a] = x[a] * g.inv_dx - 0.5f;
        base[a] = (int)floorf(fx[a]);
        bspline_weights(fx[a] - (float)base[a], wgt[a]);
    }
    const float cs = 4.0f * g.inv_dx * g.inv_dx;
    float v[3] = {0.0f, 0.0f, 0.0f};
    float Cm[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) Cm[q] = 0.0f;
    int dropped = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float w = wgt[0][i] * wgt[1][j] * wgt[2][k];
                if (w == 0.0f) continue;
                const int ni = base[0] + i, nj = base[1] + j, nk = base[2] + k;
                const int64_t id = g.node(ni, nj, nk);
                if (id < 0) { ++dropped; continue; }
                const float4 nv = acc.mv[id];
                const float d[3] = {((float)ni - fx[0] - 0.5f) * g.dx, ((float)nj - fx[1] - 0.5f) * g.dx,
                                    ((float)nk - fx[2] - 0.5f) * g.dx};
                const float wv[3] = {nv.x * w, nv.y * w, nv.z * w};
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    v[a] = v[a] + wv[a];
#pragma unroll
                    for (int c = 0; c < 3; ++c) Cm[3 * a + c] = Cm[3 * a + c] + (wv[a] * d[c]) * cs;
                }
            }
#pragma unroll
    for (int a = 0; a < 3; ++a) x[a] = x[a] + v[a] * dt;
    dp_project(F, Cm, dt, S.mat.neg_alpha_koh);
    if (x[1] < 0.0f) {
        x[1] = 0.0f;
        v[1] = 0.0f;
    }
    bool finite = isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]);
#pragma unroll
    for (int q = 0; q < 9; ++q) finite = finite && isfinite(F[q]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        ps.plane(P_X + a)[p] = x[a];
        ps.plane(P_V + a)[p] = v[a];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        ps.plane(P_F + q)[p] = F[q];
        ps.plane(P_C + q)[p] = Cm[q];
    }
    report(S, dropped, finite);
}

// ---- fused G2P(n) + P2G(n+1) ------------------------------------------------------

// Gather of G2P for a stencil inside the box: nodes at constant offsets from
// the base node, loaded one k-row (3 nodes) at a time. A zero weight
// multiplies instead of skipping, which is the same for finite grid values.
__device__ __forceinline__ void gather_inside(const float4* __restrict__ src, int64_t EYZ, int64_t EZ,
                                              const float wgt[3][3], const float dcs[3][3], float v[3],
                                              float Cm[9], uint32_t& light) {
    // separable in k: per (i, j) row, s = sum_k w_k v_k and t = sum_k w_k dk v_k,
    // then v += w_ij s and C += w_ij (di s, dj s, t). `light` takes one bit
    // per node, in stencil order (node n = 9 i + 3 j + k ends at bit 26 - n):
    // set when the node's particle mass is below kHeavyNodeMass. For two
    // non-negative floats a < b exactly when bits(a) - bits(b) is negative as
    // a signed integer, and the funnel shift moves that sign bit in.
    const float wd2[3] = {wgt[2][0] * dcs[2][0], wgt[2][1] * dcs[2][1], wgt[2][2] * dcs[2][2]};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float4* row = src + i * EYZ + j * EZ;
            const float4 n[3] = {row[0], row[1], row[2]};
#pragma unroll
            for (int k = 0; k < 3; ++k)
                light = __funnelshift_l(__float_as_uint(n[k].w) - __float_as_uint(kHeavyNodeMass), light, 1);
            const float sx = (n[0].x * wgt[2][0] + n[1].x * wgt[2][1]) + n[2].x * wgt[2][2];
            const float sy = (n[0].y * wgt[2][0] + n[1].y * wgt[2][1]) + n[2].y * wgt[2][2];
            const float sz = (n[0].z * wgt[2][0] + n[1].z * wgt[2][1]) + n[2].z * wgt[2][2];
            const float tx = (n[0].x * wd2[0] + n[1].x * wd2[1]) + n[2].x * wd2[2];
            const float ty = (n[0].y * wd2[0] + n[1].y * wd2[1]) + n[2].y * wd2[2];
            const float tz = (n[0].z * wd2[0] + n[1].z * wd2[1]) + n[2].z * wd2[2];
            const float wij = wgt[0][i] * wgt[1][j];
            const float wi0 = wij * dcs[0][i], wj1 = wij * dcs[1][j];
            const float sv[3] = {sx, sy, sz}, tv[3] = {tx, ty, tz};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                v[a] += wij * sv[a];
                Cm[3 * a + 0] += wi0 * sv[a];
                Cm[3 * a + 1] += wj1 * sv[a];
                Cm[3 * a + 2] += wij * tv[a];
            }
        }
}

// mark_stencil_blocks for particles in base-node order: a lane whose block
// range equals that of the lane before it leaves the marks to that lane, and
// the allocated flags are skipped when alloc_done (the blocks of a stencil the
// particle gathered from in full were allocated by its own scatter, or the
// lane that covered it, one step earlier). (A per-warp form, one block per
// lane of the warp's block box found by redux min/max and per-axis ballots,
// measured 8 us slower on the 2M wheel rut: the covered lanes of this form
// return at once.)
__device__ __forceinline__ void mark_stencil_blocks_warp(const GridDesc& g, const GridAcc& a, uint8_t* alloc,
                                                         const int base[3], const float wx[3], const float wy[3],
                                                         const float wz[3], bool alloc_done) {
    const int lo0 = base[0] + (wx[0] == 0.0f), hi0 = base[0] + 2 - (wx[2] == 0.0f);
    const int lo1 = base[1] + (wy[0] == 0.0f), hi1 = base[1] + 2 - (wy[2] == 0.0f);
    const int lo2 = base[2] + (wz[0] == 0.0f), hi2 = base[2] + 2 - (wz[2] == 0.0f);
    const int b0 = (lo0 - g.ox) >> 2, b1 = (lo1 - g.oy) >> 2, b2 = (lo2 - g.oz) >> 2;
    const int e0 = ((hi0 - g.ox) >> 2) - b0, e1 = ((hi1 - g.oy) >> 2) - b1, e2 = ((hi2 - g.oz) >> 2) - b2;
    const int lane = (int)(threadIdx.x & 31);
    // a 3-node stencil covers one or two blocks per axis (e in {0, 1}); block
    // indices far outside the box (a non-finite position) get a key of their
    // own so that they never stand in for another lane
    const bool near_box = (unsigned)(b0 + 1) <= (unsigned)(g.nbx + 1) && (unsigned)(b1 + 1) <= (unsigned)(g.nby + 1) &&
                          (unsigned)(b2 + 1) <= (unsigned)(g.nbz + 1);
    const unsigned long long key = near_box ? ((unsigned long long)(b0 & 0xFFFFF) << 43) |
                                                  ((unsigned long long)(b1 & 0xFFFFF) << 23) |
                                                  ((unsigned long long)(b2 & 0xFFFFF) << 3) |
                                                  (unsigned)(e0 << 2 | e1 << 1 | e2)
                                            : ~0ull - (unsigned long long)lane;
    const unsigned act = __activemask();
    const unsigned long long prev = __shfl_up_sync(act, key, 1);
    const bool covered = lane > 0 && ((act >> (lane - 1)) & 1u) && prev == key;
    if (covered) return;
    for (int i = b0; i <= b0 + e0; ++i)
        for (int j = b1; j <= b1 + e1; ++j)
            for (int k = b2; k <= b2 + e2; ++k) {
                if ((unsigned)i < (unsigned)g.nbx && (unsigned)j < (unsigned)g.nby && (unsigned)k < (unsigned)g.nbz) {
                    const int64_t blk = g.block_of(i, j, k);
                    if (!alloc_done && alloc[blk] == 0) alloc[blk] = 1;
                    touch_block(a, blk);
                }
            }
}

// One thread per particle, particles in base-node order. Reads x, F, m, V0;
// writes x, v, C, F; scatters P2G(n+1) with one 16-byte reduction per node:
// (momentum + force * dt, mass), the force folded in with the scene's dt. The
// reference keeps momentum without force at nodes of mass <= 1e-6
// (mpm_solver.h:257); every contribution to such a node has w*m <= 1e-6 on
// its own, so those light contributions also add their force to the force
// channel, and the grid update subtracts force * dt again there. A light
// contribution skips that record when its node held at least kHeavyNodeMass
// of particle mass in this step's grid and the particle's base node did not
// change (the node is then in both stencils); a node can only end light with
// a record missing if its mass fell from >= kHeavyNodeMass to <= 1e-6 in one
// step, and the grid update counts every such node (light-node suspects). A particle
// whose 3x3x3 stencil lies inside the box (all but escaping particles)
// addresses its nodes at constant offsets from the base node with one bounds
// check for the whole stencil, and its affine and stress terms are summed
// axis by axis (the three d components of a node depend on i, j and k
// separately).
template <bool Fast>
__device__ __forceinline__ void g2p2g_particle(const FusedScene& S, int64_t p) {
    const GridDesc& g = S.g;
    const FusedScene& ps = S;
    int dropped = 0;
    float x[3] = {ps.plane(P_X)[p], ps.plane(P_X + 1)[p], ps.plane(P_X + 2)[p]};
    float F[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) F[q] = ps.plane(P_F + q)[p];
    const float m = ps.plane(P_M)[p];
    const float vol = ps.plane(P_V0)[p];

    // ---- G2P(n): gather velocities of the 27 stencil nodes
    float fx[3], wgt[3][3], dd[3][3];
    int base[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        fx[a] = x[a] * g.inv_dx - 0.5f;
        base[a] = (int)floorf(fx[a]);
        bspline_weights(fx[a] - (float)base[a], wgt[a]);
#pragma unroll
        for (int i = 0; i < 3; ++i) dd[a][i] = ((float)(base[a] + i) - fx[a] - 0.5f) * g.dx;
    }
    float v[3] = {0.f, 0.f, 0.f};
    float Cm[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) Cm[q] = 0.0f;
    // bit 26 - n set: node n of the gathered stencil held less than
    // kHeavyNodeMass of particle mass (all set: not gathered in full)
    uint32_t light = 0x7FFFFFFu;
    const int gbase0 = base[0], gbase1 = base[1], gbase2 = base[2];
    // no end weight exactly 0: the gather stencil spans all of base..base+2
    const bool gather_full = wgt[0][0] != 0.0f && wgt[0][2] != 0.0f && wgt[1][0] != 0.0f && wgt[1][2] != 0.0f &&
                             wgt[2][0] != 0.0f && wgt[2][2] != 0.0f;
    {
        const float4* __restrict__ cur_mv = S.cur_mv;
        const float cs = 4.0f * g.inv_dx * g.inv_dx;
        const int r0 = base[0] - g.ox, r1 = base[1] - g.oy, r2 = base[2] - g.oz;
        const bool inside = (unsigned)r0 <= (unsigned)(g.ex() - 3) && (unsigned)r1 <= (unsigned)(g.ey() - 3) &&
                            (unsigned)r2 <= (unsigned)(g.ez() - 3);
        if (inside) {
            const int64_t EZ = g.ez(), EYZ = (int64_t)g.ey() * g.ez();
            float dcs[3][3];
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int i = 0; i < 3; ++i) dcs[a][i] = dd[a][i] * cs;
            light = 0u;
            gather_inside(cur_mv + g.node_rel(r0, r1, r2), EYZ, EZ, wgt, dcs, v, Cm, light);
        } else {
#pragma unroll 1
            for (int n = 0; n < 27; ++n) {
                const int i = n / 9, j = (n / 3) % 3, k = n % 3;
                const float w = pick3(wgt[0], i) * pick3(wgt[1], j) * pick3(wgt[2], k);
                if (w == 0.0f) continue;
                const int64_t id = g.node(base[0] + i, base[1] + j, base[2] + k);
                if (id < 0) { ++dropped; continue; }
                const float4 nv = cur_mv[id];
                const float wv[3] = {nv.x * w, nv.y * w, nv.z * w};
                const float d[3] = {pick3(dd[0], i), pick3(dd[1], j), pick3(dd[2], k)};
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    v[a] += wv[a];
#pragma unroll
                    for (int c = 0; c < 3; ++c) Cm[3 * a + c] += (wv[a] * d[c]) * cs;
                }
            }
        }
    }
    const float dt = S.dt;
#pragma unroll
    for (int a = 0; a < 3; ++a) x[a] = x[a] + v[a] * dt;
    float U[9], lnS[3];
    dp_project_keep<Fast>(F, Cm, dt, S.neg_alpha_koh, U, lnS);
    if (x[1] < 0.0f) {
        x[1] = 0.0f;
        v[1] = 0.0f;
    }
    bool fin = isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]);
#pragma unroll
    for (int q = 0; q < 9; ++q) fin = fin && isfinite(F[q]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        ps.plane(P_X + a)[p] = x[a];
        ps.plane(P_V + a)[p] = v[a];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        ps.plane(P_F + q)[p] = F[q];
        ps.plane(P_C + q)[p] = Cm[q];
    }

    // ---- P2G(n+1) from the new state; tau from the projection's SVD
    const float tr = (lnS[0] + lnS[1]) + lnS[2];
    const float mu = S.mu, lambda = S.lambda;
    const float td[3] = {2.0f * mu * lnS[0] + lambda * tr, 2.0f * mu * lnS[1] + lambda * tr,
                         2.0f * mu * lnS[2] + lambda * tr};
    float sk[9];
    u_diag_wt(U, td, U, sk);
    const float ff = -4.0f * g.inv_dx * g.inv_dx * vol;
#pragma unroll
    for (int q = 0; q < 9; ++q) sk[q] = sk[q] * ff;
    // the contribution to a node at offset d is w (m v + (m C + dt S) d)
    // (momentum plus force * dt), mass w m
    float Mq[9], Pm[3];
#pragma unroll
    for (int q = 0; q < 9; ++q) Mq[q] = m * Cm[q] + dt * sk[q];
#pragma unroll
    for (int a = 0; a < 3; ++a) Pm[a] = m * v[a];
    // S itself is needed again only for the (few) light-force records after
    // the unrolled scatter: park it in this thread's shared-memory column so
    // that it holds no registers through the loop
    __shared__ float sk_park[9 * kMaxFusedThreads];
#pragma unroll
    for (int q = 0; q < 9; ++q) sk_park[q * kMaxFusedThreads + threadIdx.x] = sk[q];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        fx[a] = x[a] * g.inv_dx - 0.5f;
        base[a] = (int)floorf(fx[a]);
        bspline_weights(fx[a] - (float)base[a], wgt[a]);
#pragma unroll
        for (int i = 0; i < 3; ++i) dd[a][i] = ((float)(base[a] + i) - fx[a] - 0.5f) * g.dx;
    }
    const bool same_base = base[0] == gbase0 && base[1] == gbase1 && base[2] == gbase2;
    // every node of the stencil was heavy in the gathered grid: no light
    // contribution of this particle needs its force record (the bulk case)
    const bool all_heavy = same_base && light == 0u;
    {
        const int r0 = base[0] - g.ox, r1 = base[1] - g.oy, r2 = base[2] - g.oz;
        const bool inside = (unsigned)r0 <= (unsigned)(g.ex() - 3) && (unsigned)r1 <= (unsigned)(g.ey() - 3) &&
                            (unsigned)r2 <= (unsigned)(g.ez() - 3);
        const GridAcc& next = S.next;
        const int64_t EZ = g.ez(), EYZ = (int64_t)g.ey() * g.ez();
        if (inside) {
            float4* dmv = next.mv + g.node_rel(r0, r1, r2);
            float4* df = next.f + g.node_rel(r0, r1, r2);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                // m v + (m C + dt S) d, summed axis by axis
                float ui[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) ui[a] = Pm[a] + Mq[3 * a] * dd[0][i];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    float uj[3];
#pragma unroll
                    for (int a = 0; a < 3; ++a) uj[a] = ui[a] + Mq[3 * a + 1] * dd[1][j];
                    const float wij = wgt[0][i] * wgt[1][j];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float w = wij * wgt[2][k];
                        const float mc = w * m;
                        const int64_t off = i * EYZ + j * EZ + k;
                        red_v4(dmv + off, (uj[0] + Mq[2] * dd[2][k]) * w, (uj[1] + Mq[5] * dd[2][k]) * w,
                               (uj[2] + Mq[8] * dd[2][k]) * w, mc);
                    }
                }
            }
            // the force records of light contributions (w m <= 1e-6, the same
            // product as the mass lane above) at nodes that were not heavy in
            // the gathered grid, off the unrolled loop: only particles at the
            // fringe of the material get here. The gathered masses come from
            // the gather's bits: no load, so the loop waits on nothing.
            if (!all_heavy) {
                // the nodes that take a record, as bits in stencil order (bit
                // 26 - n for node n): a light contribution (same product as
                // the scatter's mass lane) at a node that was not heavy; the
                // loop then visits only those (a fringe particle has a few of
                // its 27), where visiting all 27 held a fringe warp 3x longer
                const uint32_t not_heavy = same_base ? light : 0x7FFFFFFu;
                uint32_t rec = 0u;
#pragma unroll 1
                for (int i = 0; i < 3; ++i) {
                    const float wi = pick3(wgt[0], i);
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const float wij = wi * wgt[1][j];
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            const float w = wij * wgt[2][k];
                            rec = (rec << 1) | (w != 0.0f && w * m <= 1e-6f ? 1u : 0u);
                        }
                    }
                }
                rec &= not_heavy;
                while (rec) {
                    const int bit = 31 - __clz(rec);
                    rec &= ~(1u << bit);
                    const int n = 26 - bit;
                    const int i = n / 9, j = (n / 3) % 3, k = n % 3;
                    const float w = pick3(wgt[0], i) * pick3(wgt[1], j) * pick3(wgt[2], k);
                    const int64_t off = i * EYZ + j * EZ + k;
                    const float d0 = pick3(dd[0], i), d1 = pick3(dd[1], j), d2 = pick3(dd[2], k);
                    float S_[9];
#pragma unroll
                    for (int q = 0; q < 9; ++q) S_[q] = sk_park[q * kMaxFusedThreads + threadIdx.x];
                    red_v4(df + off, ((S_[0] * d0 + S_[1] * d1) + S_[2] * d2) * w,
                           ((S_[3] * d0 + S_[4] * d1) + S_[5] * d2) * w,
                           ((S_[6] * d0 + S_[7] * d1) + S_[8] * d2) * w, 0.0f);
                }
            }
        } else {
#pragma unroll 1
            for (int n = 0; n < 27; ++n) {
                const int i = n / 9, j = (n / 3) % 3, k = n % 3;
                const float w = pick3(wgt[0], i) * pick3(wgt[1], j) * pick3(wgt[2], k);
                if (w == 0.0f) continue;  // mpm_solver.h:223
                const int64_t id = g.node(base[0] + i, base[1] + j, base[2] + k);
                if (id < 0) { ++dropped; continue; }
                const float d0 = pick3(dd[0], i), d1 = pick3(dd[1], j), d2 = pick3(dd[2], k);
                const float mc = w * m;
                red_v4(next.mv + id, (Pm[0] + ((Mq[0] * d0 + Mq[1] * d1) + Mq[2] * d2)) * w,
                       (Pm[1] + ((Mq[3] * d0 + Mq[4] * d1) + Mq[5] * d2)) * w,
                       (Pm[2] + ((Mq[6] * d0 + Mq[7] * d1) + Mq[8] * d2)) * w, mc);
                if (mc <= 1e-6f) {
                    float S_[9];
#pragma unroll
                    for (int q = 0; q < 9; ++q) S_[q] = sk_park[q * kMaxFusedThreads + threadIdx.x];
                    red_v4(next.f + id, ((S_[0] * d0 + S_[1] * d1) + S_[2] * d2) * w,
                           ((S_[3] * d0 + S_[4] * d1) + S_[5] * d2) * w, ((S_[6] * d0 + S_[7] * d1) + S_[8] * d2) * w,
                           0.0f);
                }
            }
        }
    }
    mark_stencil_blocks_warp(g, S.next, S.alloc, base, wgt[0], wgt[1], wgt[2], same_base && gather_full);
    if (!fin) atomicOr(S.status, ERR_NONFINITE);
    if (dropped) {
        atomicOr(S.status, ERR_ESCAPE);
        atomicAdd(S.escaped, (unsigned long long)dropped);
    }
}

// Lane order inside a CTA. 0: thread t takes the CTA's particle t. 1: the
// warps of a CTA pair up and interleave, thread t of warp w taking particle
// 64 (w / 2) + 2 (t mod 32) + (w mod 2): a warp then holds every other
// particle of 64 consecutive ones, so at high particle counts per cell fewer
// of its lanes add into the same node in one reduction instruction (measured
// 3 % faster on the batched box drops at 8 particles per cell, 3 % slower on
// the wheel rut at 3). CTA sizes are multiples of 64.
__device__ __forceinline__ int lane_slot(int t, int interleave) {
    return interleave ? ((t >> 6) << 6) + ((t & 31) << 1) + ((t >> 5) & 1) : t;
}

// Many scenes: the views of up to kPackScenes scenes travel as one kernel
// parameter (FusedPack), so that, as in the single-scene kernel, every field
// of a scene is read through the constant bank rather than from memory. A
// 128-thread unit finds its scene by a binary search of the pack's prefix;
// with 128-thread CTAs the scene index is uniform over the CTA, and the
// fields can sit in uniform registers. (An earlier form copied each unit's
// view into shared memory: its fields were reloaded from there throughout the
// particle, short-scoreboard waits 2.75 per issue against 0.67 for the
// constant bank, and about 150 more instructions per particle.)
//
// `reverse` runs the CTAs in the opposite order (CTA b takes the work of CTA
// gridDim.x - 1 - b). The caller alternates it from one step to the next, so
// that a step starts with the particles the step before wrote last, whose
// planes are still in L2 (measured 1 % faster on the 2M-particle wheel rut).
// Results do not depend on it beyond the order of the float reductions.
template <bool Fast, int Threads, int MinBlocks>
__global__ void __launch_bounds__(Threads, MinBlocks) k_g2p2g_pack(const __grid_constant__ FusedPack P, int reverse,
                                                                  int interleave) {
    const int64_t b = reverse ? (int64_t)(gridDim.x - 1 - blockIdx.x) : (int64_t)blockIdx.x;
    const int64_t gtid = b * Threads + threadIdx.x;
    const int64_t unit = gtid / kParticleCTA;
    if (unit >= P.prefix[P.n]) return;
    int lo = 0, hi = P.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.prefix[mid] <= unit) lo = mid;
        else hi = mid - 1;
    }
    const FusedScene& S = P.v[lo];
    const int64_t p = (unit - P.prefix[lo]) * kParticleCTA + lane_slot((int)(gtid % kParticleCTA), interleave);
    if (p >= S.n) return;
    g2p2g_particle<Fast>(S, p);
}

// Single scene: the view is a kernel parameter (constant bank); `reverse` and
// `interleave` as for k_g2p2g_pack.
template <bool Fast, int Threads, int MinBlocks>
__global__ void __launch_bounds__(Threads, MinBlocks) k_g2p2g_one(const __grid_constant__ FusedScene S, int reverse,
                                                                 int interleave) {
    const int64_t b = reverse ? (int64_t)(gridDim.x - 1 - blockIdx.x) : (int64_t)blockIdx.x;
    const int64_t p = b * Threads + lane_slot((int)threadIdx.x, interleave);
    if (p >= S.n) return;
    g2p2g_particle<Fast>(S, p);
}

// ---- counting sort by stencil base node -------------------------------------------

__device__ __forceinline__ int key_of(const GridDesc& g, int shift, const float x[3]) {
    int r[3];
    const int o[3] = {g.ox, g.oy, g.oz};
    const int e[3] = {g.ex(), g.ey(), g.ez()};
    const int outside = (int)sort_keys_of(g, shift) - 1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float f = x[a] * g.inv_dx - 0.5f;
        if (!(f > -1e9f && f < 1e9f)) return outside;  // NaN or far outside
        r[a] = (int)floorf(f) - o[a];
        if ((unsigned)r[a] >= (unsigned)e[a]) return outside;
    }
    const int m = (1 << shift) - 1;
    const int ey = (e[1] + m) >> shift, ez = (e[2] + m) >> shift;
    return ((r[0] >> shift) * ey + (r[1] >> shift)) * ez + (r[2] >> shift);
}

__global__ void __launch_bounds__(kParticleCTA) k_sort_key(SceneTable t, int sel, int32_t* count) {
    PSlot slot;
    const bool valid = particle_slot(t, sel, slot);
    int key = -1;
    if (valid) {
        const SceneDev& S = t.scenes[slot.s];
        const ParticleSoA ps = S.store[sel];
        const float x[3] = {ps.plane(P_X)[slot.p], ps.plane(P_X + 1)[slot.p], ps.plane(P_X + 2)[slot.p]};
        key = (int)(S.key_base + key_of(S.g, S.bin_shift, x));
    }
    // warp-aggregated histogram: one atomic per distinct key in the warp
    const unsigned grp = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(grp) - 1;
    int base = 0;
    if (valid && lane == leader) base = atomicAdd(count + key, __popc(grp));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (valid) {
        const SceneDev& S = t.scenes[slot.s];
        S.key[slot.p] = key;
        S.rank[slot.p] = base + __popc(grp & ((1u << lane) - 1u));
    }
}

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* s_warp, long long* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        long long w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        s_warp[lane] = w;
    }
    __syncthreads();
    const long long before = (warp > 0 ? s_warp[warp - 1] : 0) + x - v;
    *total = s_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

// Scan phase 1: per-tile sums of count[0..n).
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int32_t* count, int64_t n, int64_t* tile_sum) {
    const int64_t t0 = (int64_t)blockIdx.x * kScanTile;
    long long s = 0;
    for (int q = threadIdx.x; q < kScanTile; q += kScanThreads) {
        const int64_t i = t0 + q;
        if (i < n) s += count[i];
    }
    __shared__ long long s_warp[32];
    long long total;
    block_exclusive_scan(s, s_warp, &total);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// Scan phase 2: exclusive scan of the tile sums (one CTA).
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(int64_t* tile_sum, int64_t n_tiles) {
    __shared__ long long s_warp[32];
    long long carry = 0;
    for (int64_t b = 0; b < n_tiles; b += kScanThreads) {
        const int64_t i = b + threadIdx.x;
        const long long v = i < n_tiles ? tile_sum[i] : 0;
        long long total;
        const long long ex = block_exclusive_scan(v, s_warp, &total);
        if (i < n_tiles) tile_sum[i] = carry + ex;
        carry += total;
    }
}

// Scan phase 3: start[i] = exclusive prefix of count; start[n] = total.
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int32_t* count, int64_t n,
                                                             const int64_t* tile_sum, int32_t* start) {
    const int64_t t0 = (int64_t)blockIdx.x * kScanTile;
    constexpr int per = kScanTile / kScanThreads;
    const int64_t i0 = t0 + (int64_t)threadIdx.x * per;
    int32_t c[per];
    long long s = 0;
#pragma unroll
    for (int q = 0; q < per; ++q) {
        c[q] = (i0 + q < n) ? count[i0 + q] : 0;
        s += c[q];
    }
    __shared__ long long s_warp[32];
    long long total;
    long long run = tile_sum[blockIdx.x] + block_exclusive_scan(s, s_warp, &total);
#pragma unroll
    for (int q = 0; q < per; ++q) {
        if (i0 + q < n) start[i0 + q] = (int32_t)run;
        run += c[q];
    }
    if (i0 + per >= n && i0 < n) start[n] = (int32_t)run;
}

// Moves each particle of store[sel] to its sorted slot of store[1-sel]
// (slots are relative to the scene's first key).
__global__ void __launch_bounds__(kParticleCTA) k_sort_permute(SceneTable t, int sel, const int32_t* start) {
    PSlot slot;
    if (!particle_slot(t, sel, slot)) return;
    const SceneDev& S = t.scenes[slot.s];
    const ParticleSoA src = S.store[sel], dst = S.store[1 - sel];
    const int64_t p = slot.p;
    const int64_t d = (int64_t)start[S.key[p]] + S.rank[p] - start[S.key_base];
#pragma unroll
    for (int c = 0; c < N_PLANES; ++c) dst.plane(c)[d] = src.plane(c)[p];
    dst.pid[d] = src.pid[p];
}

// ---- particle rows in add order ------------------------------------------------

__global__ void k_gather_rows(ParticleSoA ps, int plane0, int width, float* out) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ps.n) return;
    const int64_t a = ps.pid[p];
    for (int c = 0; c < width; ++c) out[a * width + c] = ps.plane(plane0 + c)[p];
}

__global__ void k_scatter_rows(ParticleSoA ps, int plane0, int width, const float* in, int64_t first, int64_t n,
                               const int32_t* inv) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int64_t p = inv[first + q];
    for (int c = 0; c < width; ++c) ps.plane(plane0 + c)[p] = in[q * width + c];
}

__global__ void k_inverse_pid(ParticleSoA ps, int32_t* inv) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ps.n) return;
    inv[ps.pid[p]] = (int32_t)p;
}

// New particles [n0, n0 + n) of a store from the caller's rows: F = I,
// C = 0, V0 = m / rho (mpm_solver.h:23-34, the reference's add_particle).
// vel / mass NULL: zero velocity / mass 1.
__global__ void k_fill_particles(ParticleSoA s, int64_t n0, int64_t n, const float* __restrict__ pos,
                                 const float* __restrict__ vel, const float* __restrict__ mass, float density) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int64_t p = n0 + q;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        s.plane(P_X + a)[p] = pos[3 * q + a];
        s.plane(P_V + a)[p] = vel ? vel[3 * q + a] : 0.0f;
    }
#pragma unroll
    for (int a = 0; a < 9; ++a) {
        s.plane(P_F + a)[p] = (a % 4 == 0) ? 1.0f : 0.0f;
        s.plane(P_C + a)[p] = 0.0f;
    }
    const float m = mass ? mass[q] : 1.0f;
    s.plane(P_M)[p] = m;
    s.plane(P_V0)[p] = (density > 1e-12f) ? (m / density) : 1.0f;
    s.pid[p] = (int32_t)p;
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// Compiled launch shapes of the fused kernel: threads per CTA and the
// minimum CTAs per SM given to the register allocator.
struct FusedVariant {
    const char* name;
    int threads, min_blocks, interleave;
    void (*pack[2])(const FusedPack, int, int);
    void (*one[2])(const FusedScene, int, int);
};

// The launch shapes, then the same shapes with interleaved lanes (lane_slot).
#define BM_FUSED(T, B, I, SUFFIX)                                                            \
    {#T "x" #B SUFFIX, T, B, I, {k_g2p2g_pack<false, T, B>, k_g2p2g_pack<true, T, B>},      \
     {k_g2p2g_one<false, T, B>, k_g2p2g_one<true, T, B>}}
#define BM_SHAPES(I, SUFFIX)                                                                                \
    BM_FUSED(128, 4, I, SUFFIX), BM_FUSED(128, 5, I, SUFFIX), BM_FUSED(128, 6, I, SUFFIX),                  \
        BM_FUSED(256, 2, I, SUFFIX), BM_FUSED(256, 3, I, SUFFIX), BM_FUSED(64, 10, I, SUFFIX),              \
        BM_FUSED(128, 8, I, SUFFIX), BM_FUSED(128, 7, I, SUFFIX)
const FusedVariant kFused[] = {BM_SHAPES(0, ""), BM_SHAPES(1, "/i2")};
#undef BM_SHAPES
#undef BM_FUSED
constexpr int kNumFused = sizeof(kFused) / sizeof(kFused[0]);

}  // namespace

int64_t scan_tiles(int64_t nkeys) { return (nkeys + kScanTile - 1) / kScanTile; }

int fused_variant_count() { return kNumFused; }
int fused_variant_index(int threads, int min_blocks, int interleave) {
    for (int v = 0; v < kNumFused; ++v)
        if (kFused[v].threads == threads && kFused[v].min_blocks == min_blocks && kFused[v].interleave == interleave)
            return v;
    return 0;
}
const char* fused_variant_name(int v) { return (v >= 0 && v < kNumFused) ? kFused[v].name : "?"; }

void launch_p2g(const SceneTable& t, int64_t n_ctas, int cur, int sel, cudaStream_t st, bool only_fresh) {
    if (n_ctas <= 0) return;
    k_p2g<<<(unsigned)n_ctas, kParticleCTA, 0, st>>>(t, cur, sel, only_fresh);
}

void launch_grid_update(const SceneTable& t, int64_t max_blocks, int cur, bool folded, cudaStream_t st,
                        const LightRepair* repair) {
    if (t.n_scenes <= 0) return;
    // one grid row per scene; a row needs no more CTAs than the largest
    // scene's listed nodes (both accumulators) fill, and at least 32 CTAs per
    // scene keep a table of many scenes balanced (a scene with fewer listed
    // blocks leaves its extra CTAs idle at once)
    const int64_t want = (2 * max_blocks * 64 + kGridThreads - 1) / kGridThreads;
    const int64_t cap = std::max<int64_t>(32, 148 * 8 / t.n_scenes);
    const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, cap));
    const dim3 grid(gx, (unsigned)t.n_scenes);
    k_grid_update<<<grid, kGridThreads, 0, st>>>(t, cur, folded, repair->word);
    if (!folded) return;
    // (grids sized for a quick return: the repair is rare, the launch is not)
    if (repair->n_ctas > 0) {
        const int64_t ctas = std::min<int64_t>(repair->n_ctas, (int64_t)repair->num_sms * 2);
        k_repair_p2g<<<(unsigned)ctas, kParticleCTA, 0, st>>>(t, cur, repair->sel, repair->word);
    }
    k_repair_update<<<dim3(std::min(gx, 16u), (unsigned)t.n_scenes), kGridThreads, 0, st>>>(t, cur, repair->word);
}

void launch_g2p(const SceneTable& t, int64_t n_ctas, int cur, int sel, cudaStream_t st) {
    if (n_ctas <= 0) return;
    k_g2p<<<(unsigned)n_ctas, kParticleCTA, 0, st>>>(t, cur, sel);
}

FusedScene fused_view(const SceneDev& d, int cur, int sel) {
    FusedScene v;
    v.base = d.store[sel].base;
    v.cap = d.store[sel].cap;
    v.n = d.store[sel].n;
    v.g = d.g;
    v.cur_mv = d.acc[cur].mv;
    v.next = d.acc[1 - cur];
    v.alloc = d.alloc;
    v.mu = d.mat.mu;
    v.lambda = d.mat.lambda;
    v.neg_alpha_koh = d.mat.neg_alpha_koh;
    v.dt = d.dt;
    v.status = d.status;
    v.escaped = d.escaped;
    return v;
}

void launch_g2p2g_one(const FusedScene& scene, bool fast_math, int variant, bool reverse, cudaStream_t st) {
    if (scene.n <= 0) return;
    const FusedVariant& v = kFused[(variant >= 0 && variant < kNumFused) ? variant : 0];
    v.one[fast_math ? 1 : 0]<<<nblk(scene.n, v.threads), v.threads, 0, st>>>(scene, reverse ? 1 : 0, v.interleave);
}

void launch_g2p2g_many(const FusedScene* views, const int64_t* prefix, int n_scenes, bool fast_math, int variant,
                       bool reverse, cudaStream_t st) {
    if (n_scenes <= 0) return;
    const FusedVariant& v = kFused[(variant >= 0 && variant < kNumFused) ? variant : 0];
    // one launch per pack of up to kPackScenes consecutive scenes
    static thread_local FusedPack pack;
    for (int first = 0; first < n_scenes; first += kPackScenes) {
        const int n = std::min(kPackScenes, n_scenes - first);
        const int64_t units = prefix[first + n] - prefix[first];
        if (units <= 0) continue;
        pack.n = n;
        for (int q = 0; q < n; ++q) {
            pack.v[q] = views[first + q];
            pack.prefix[q] = prefix[first + q] - prefix[first];
        }
        pack.prefix[n] = units;
        v.pack[fast_math ? 1 : 0]<<<nblk(units * kParticleCTA, v.threads), v.threads, 0, st>>>(pack, reverse ? 1 : 0,
                                                                                                v.interleave);
    }
}

void launch_sort(const SceneTable& t, int64_t n_ctas, int sel, const SortBuffers& sb, cudaStream_t st) {
    if (n_ctas <= 0) return;
    const int64_t n = sb.nkeys;
    const int64_t tiles = scan_tiles(n);
    cudaMemsetAsync(sb.count, 0, sizeof(int32_t) * n, st);
    k_sort_key<<<(unsigned)n_ctas, kParticleCTA, 0, st>>>(t, sel, sb.count);
    k_scan_reduce<<<(unsigned)tiles, kScanThreads, 0, st>>>(sb.count, n, sb.tile_sum);
    k_scan_tiles<<<1, kScanThreads, 0, st>>>(sb.tile_sum, tiles);
    k_scan_apply<<<(unsigned)tiles, kScanThreads, 0, st>>>(sb.count, n, sb.tile_sum, sb.start);
    k_sort_permute<<<(unsigned)n_ctas, kParticleCTA, 0, st>>>(t, sel, sb.start);
}

void launch_gather_rows(const ParticleSoA& ps, int plane0, int width, float* out, cudaStream_t st) {
    if (ps.n == 0) return;
    k_gather_rows<<<nblk(ps.n, 256), 256, 0, st>>>(ps, plane0, width, out);
}

void launch_scatter_rows(const ParticleSoA& ps, int plane0, int width, const float* in, int64_t first, int64_t n,
                         const int32_t* inv, cudaStream_t st) {
    if (n == 0) return;
    k_scatter_rows<<<nblk(n, 256), 256, 0, st>>>(ps, plane0, width, in, first, n, inv);
}

void launch_fill_particles(const ParticleSoA& s, int64_t n0, int64_t n, const float* pos, const float* vel,
                           const float* mass, float density, cudaStream_t st) {
    if (n <= 0) return;
    k_fill_particles<<<nblk(n, 256), 256, 0, st>>>(s, n0, n, pos, vel, mass, density);
}

void launch_inverse_pid(const ParticleSoA& ps, int32_t* inv, cudaStream_t st) {
    if (ps.n == 0) return;
    k_inverse_pid<<<nblk(ps.n, 256), 256, 0, st>>>(ps, inv);
}

}  // namespace bm
