// bm_fused.cu — binned particle order and the fused G2P + next-step P2G kernel.
//
// Reference (2nugu/basements, include/basements/physics/mpm/mpm_solver.h):
//   step        :71-87     g2p_single :293-348   apply_plasticity :114-166
//   p2g_single  :168-248
//
// Step n of MPMSolver::step runs P2G(n), update_grid(n), G2P(n). P2G(n+1)
// only needs the particle state that G2P(n) produces, so one kernel does
// G2P(n) and P2G(n+1) back to back while the particle is in registers:
// every particle is read once (x, F, m, V0) and written once (x, v, C, F) per
// step, and the Kirchhoff stress of P2G(n+1) comes from the SVD that the
// Drucker-Prager projection of G2P(n) already computed (F_new = U S V^T with
// known U and S), saving the second SVD of the reference.
//
// Particles are kept in the order of their stencil base node floor(x/dx -
// 0.5) (grid order, k fastest) by a counting sort (warp-aggregated
// histogram, three-phase scan, permutation) that runs every few steps. Neighbouring threads then work on neighbouring particles: the
// 27-node gather hits L1 and the 16-byte P2G reductions of a warp land on a
// few L2 lines. (A variant that accumulated each bin's P2G in a shared-memory
// tile was 3.6x slower on B200: float atomics on shared memory are a
// compare-and-swap loop, and the per-bin barriers stalled the warps.)
#include <algorithm>

#include "bm_internal.h"
#include "bm_math.cuh"

namespace bm {

namespace {

constexpr int kSortThreads = 256;
constexpr int kFusedThreads = 128;
constexpr int kFusedMinBlocks = 6;

// ---- particle order: counting sort by stencil base node ---------------------------

constexpr int kScanThreads = 1024;
constexpr int kScanTile = kScanThreads * 8;

__device__ __forceinline__ int key_of(const GridDesc& g, const float x[3], int64_t nkeys) {
    int r[3];
    const int o[3] = {g.ox, g.oy, g.oz};
    const int e[3] = {g.ex(), g.ey(), g.ez()};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float f = x[a] * g.inv_dx - 0.5f;
        if (!(f > -1e9f && f < 1e9f)) return (int)nkeys;  // NaN or far outside
        r[a] = (int)floorf(f) - o[a];
        if ((unsigned)r[a] >= (unsigned)e[a]) return (int)nkeys;
    }
    return (int)g.node_rel(r[0], r[1], r[2]);
}

__global__ void __launch_bounds__(kSortThreads) k_bin_key(ParticleSoA ps, GridDesc g, BinBuffers bb) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < ps.n;
    int key = -1;
    if (valid) {
        const float x[3] = {ps.plane(P_X)[p], ps.plane(P_X + 1)[p], ps.plane(P_X + 2)[p]};
        key = key_of(g, x, bb.nkeys);
    }
    // warp-aggregated histogram: one atomic per distinct key in the warp
    const unsigned grp = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(grp) - 1;
    int base = 0;
    if (valid && lane == leader) base = atomicAdd(bb.count + key, __popc(grp));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (valid) {
        bb.key[p] = key;
        bb.rank[p] = base + __popc(grp & ((1u << lane) - 1u));
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

__global__ void __launch_bounds__(kSortThreads) k_bin_permute(ParticleSoA src, ParticleSoA dst, BinBuffers bb) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= src.n) return;
    const int64_t d = (int64_t)bb.start[bb.key[p]] + bb.rank[p];
#pragma unroll
    for (int c = 0; c < N_PLANES; ++c) dst.plane(c)[d] = src.plane(c)[p];
    dst.pid[d] = src.pid[p];
}

// ---- fused G2P(n) + P2G(n+1) ------------------------------------------------------

__device__ __forceinline__ void red_v4(float4* a, float x, float y, float z, float w) {
    atomicAdd(a, make_float4(x, y, z, w));
}

// a[i] for a runtime i in {0,1,2} without indexing (keeps `a` in registers).
__device__ __forceinline__ float pick3(const float a[3], int i) { return i == 0 ? a[0] : (i == 1 ? a[1] : a[2]); }

// Gather of G2P for a stencil inside the box: nodes at constant offsets from
// the base node, loaded one k-row (3 nodes) at a time. A zero weight
// multiplies instead of skipping, which is the same for finite grid values.
__device__ __forceinline__ void gather_inside(const float4* __restrict__ src, int64_t EYZ, int64_t EZ,
                                              const float wgt[3][3], const float dcs[3][3], float v[3],
                                              float Cm[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float4* row = src + i * EYZ + j * EZ;
            const float4 n[3] = {row[0], row[1], row[2]};
            const float wij = wgt[0][i] * wgt[1][j];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float w = wij * wgt[2][k];
                const float wv[3] = {n[k].x * w, n[k].y * w, n[k].z * w};
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    v[a] += wv[a];
                    Cm[3 * a + 0] += wv[a] * dcs[0][i];
                    Cm[3 * a + 1] += wv[a] * dcs[1][j];
                    Cm[3 * a + 2] += wv[a] * dcs[2][k];
                }
            }
        }
}

// One thread per particle, particles in base-node order (neighbouring threads
// share stencil nodes, so the gather hits L1 and the reductions of a warp land
// on a few L2 lines). Reads x, F, m, V0; writes x, v, C, F; scatters P2G(n+1)
// with one 16-byte reduction per node: (momentum + force * dt_next, mass),
// the force folded in with the next step's dt. The reference keeps momentum
// without force at nodes of mass <= 1e-6 (mpm_solver.h:257); every
// contribution to such a node has w*m <= 1e-6 on its own, so exactly those
// contributions also add their force to the force channel, and the grid
// update subtracts force * dt again there. A particle whose 3x3x3 stencil lies
// inside the box (all but escaping particles) addresses its nodes at constant
// offsets from the base node with one bounds check for the whole stencil, and
// its affine and stress terms are summed axis by axis (the three d components
// of a node depend on i, j and k separately).
template <bool Fast>
__global__ void __launch_bounds__(kFusedThreads, kFusedMinBlocks)
    k_g2p2g(ParticleSoA ps, GridDesc g, GridAcc cur, GridAcc next, uint8_t* alloc, Material mat, float dt,
            float dt_next, uint32_t* status, unsigned long long* escaped) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ps.n) return;
    const float cs = 4.0f * g.inv_dx * g.inv_dx;
    const int64_t EZ = g.ez(), EYZ = (int64_t)g.ey() * g.ez();
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
    {
        const int r0 = base[0] - g.ox, r1 = base[1] - g.oy, r2 = base[2] - g.oz;
        const bool inside = (unsigned)r0 <= (unsigned)(g.ex() - 3) && (unsigned)r1 <= (unsigned)(g.ey() - 3) &&
                            (unsigned)r2 <= (unsigned)(g.ez() - 3);
        if (inside) {
            float dcs[3][3];
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int i = 0; i < 3; ++i) dcs[a][i] = dd[a][i] * cs;
            gather_inside(cur.mv + g.node_rel(r0, r1, r2), EYZ, EZ, wgt, dcs, v, Cm);
        } else {
#pragma unroll 1
            for (int n = 0; n < 27; ++n) {
                const int i = n / 9, j = (n / 3) % 3, k = n % 3;
                const float w = pick3(wgt[0], i) * pick3(wgt[1], j) * pick3(wgt[2], k);
                if (w == 0.0f) continue;
                const int64_t id = g.node(base[0] + i, base[1] + j, base[2] + k);
                if (id < 0) { ++dropped; continue; }
                const float4 nv = cur.mv[id];
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
#pragma unroll
    for (int a = 0; a < 3; ++a) x[a] = x[a] + v[a] * dt;
    float U[9], lnS[3];
    dp_project_keep<Fast>(F, Cm, dt, mat.neg_alpha_koh, U, lnS);
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
    const float td[3] = {2.0f * mat.mu * lnS[0] + mat.lambda * tr, 2.0f * mat.mu * lnS[1] + mat.lambda * tr,
                         2.0f * mat.mu * lnS[2] + mat.lambda * tr};
    float sk[9];
    u_diag_wt(U, td, U, sk);
    const float ff = -4.0f * g.inv_dx * g.inv_dx * vol;
#pragma unroll
    for (int q = 0; q < 9; ++q) sk[q] = sk[q] * ff;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        fx[a] = x[a] * g.inv_dx - 0.5f;
        base[a] = (int)floorf(fx[a]);
        bspline_weights(fx[a] - (float)base[a], wgt[a]);
#pragma unroll
        for (int i = 0; i < 3; ++i) dd[a][i] = ((float)(base[a] + i) - fx[a] - 0.5f) * g.dx;
    }
    {
        const int r0 = base[0] - g.ox, r1 = base[1] - g.oy, r2 = base[2] - g.oz;
        const bool inside = (unsigned)r0 <= (unsigned)(g.ex() - 3) && (unsigned)r1 <= (unsigned)(g.ey() - 3) &&
                            (unsigned)r2 <= (unsigned)(g.ez() - 3);
        if (inside) {
            float4* dmv = next.mv + g.node_rel(r0, r1, r2);
            float4* df = next.f + g.node_rel(r0, r1, r2);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                // momentum direction v + C d and stress S d, summed axis by axis
                float qi[3], si[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    qi[a] = v[a] + Cm[3 * a] * dd[0][i];
                    si[a] = sk[3 * a] * dd[0][i];
                }
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    float qj[3], sj[3];
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        qj[a] = qi[a] + Cm[3 * a + 1] * dd[1][j];
                        sj[a] = si[a] + sk[3 * a + 1] * dd[1][j];
                    }
                    const float wij = wgt[0][i] * wgt[1][j];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float w = wij * wgt[2][k];
                        const float mc = w * m;
                        const float wdt = w * dt_next;
                        const int64_t off = i * EYZ + j * EZ + k;
                        const float s0 = sj[0] + sk[2] * dd[2][k], s1 = sj[1] + sk[5] * dd[2][k],
                                    s2 = sj[2] + sk[8] * dd[2][k];
                        red_v4(dmv + off, (qj[0] + Cm[2] * dd[2][k]) * mc + s0 * wdt,
                               (qj[1] + Cm[5] * dd[2][k]) * mc + s1 * wdt, (qj[2] + Cm[8] * dd[2][k]) * mc + s2 * wdt,
                               mc);
                        if (mc <= 1e-6f) red_v4(df + off, s0 * w, s1 * w, s2 * w, 0.0f);
                    }
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
                const float s0 = (sk[0] * d0 + sk[1] * d1) + sk[2] * d2;
                const float s1 = (sk[3] * d0 + sk[4] * d1) + sk[5] * d2;
                const float s2 = (sk[6] * d0 + sk[7] * d1) + sk[8] * d2;
                const float wdt = w * dt_next;
                red_v4(next.mv + id, (v[0] + ((Cm[0] * d0 + Cm[1] * d1) + Cm[2] * d2)) * mc + s0 * wdt,
                       (v[1] + ((Cm[3] * d0 + Cm[4] * d1) + Cm[5] * d2)) * mc + s1 * wdt,
                       (v[2] + ((Cm[6] * d0 + Cm[7] * d1) + Cm[8] * d2)) * mc + s2 * wdt, mc);
                if (mc <= 1e-6f) red_v4(next.f + id, s0 * w, s1 * w, s2 * w, 0.0f);
            }
        }
    }
    mark_stencil_blocks(g, next, alloc, base, wgt[0], wgt[1], wgt[2]);
    if (!fin) atomicOr(status, ERR_NONFINITE);
    if (dropped) {
        atomicOr(status, ERR_ESCAPE);
        atomicAdd(escaped, (unsigned long long)dropped);
    }
}

}  // namespace

int64_t scan_tiles(int64_t nkeys) { return (nkeys + 1 + kScanTile - 1) / kScanTile; }

void launch_bin_sort(const ParticleSoA& src, const ParticleSoA& dst, const GridDesc& g, const BinBuffers& bb,
                     cudaStream_t st) {
    if (src.n == 0) return;
    const int64_t n = bb.nkeys + 1;
    const int64_t tiles = scan_tiles(bb.nkeys);
    cudaMemsetAsync(bb.count, 0, sizeof(int32_t) * n, st);
    const unsigned pb = (unsigned)((src.n + kSortThreads - 1) / kSortThreads);
    k_bin_key<<<pb, kSortThreads, 0, st>>>(src, g, bb);
    k_scan_reduce<<<(unsigned)tiles, kScanThreads, 0, st>>>(bb.count, n, bb.tile_sum);
    k_scan_tiles<<<1, kScanThreads, 0, st>>>(bb.tile_sum, tiles);
    k_scan_apply<<<(unsigned)tiles, kScanThreads, 0, st>>>(bb.count, n, bb.tile_sum, bb.start);
    k_bin_permute<<<pb, kSortThreads, 0, st>>>(src, dst, bb);
}

void launch_g2p2g(const ParticleSoA& ps, const GridDesc& g, const GridAcc& cur, const GridAcc& next, uint8_t* alloc,
                  const Material& mat, float dt, float dt_next, bool fast_math, uint32_t* d_status,
                  unsigned long long* d_escaped, cudaStream_t st) {
    if (ps.n == 0) return;
    const unsigned grid = (unsigned)((ps.n + kFusedThreads - 1) / kFusedThreads);
    if (fast_math)
        k_g2p2g<true><<<grid, kFusedThreads, 0, st>>>(ps, g, cur, next, alloc, mat, dt, dt_next, d_status, d_escaped);
    else
        k_g2p2g<false><<<grid, kFusedThreads, 0, st>>>(ps, g, cur, next, alloc, mat, dt, dt_next, d_status,
                                                        d_escaped);
}

}  // namespace bm
