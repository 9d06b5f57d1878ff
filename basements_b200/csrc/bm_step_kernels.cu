// bm_step_kernels.cu — P2G, grid update and G2P of the MLS-MPM soil step.
//
// Reference (2nugu/basements, include/basements/physics/mpm/mpm_solver.h):
//   p2g_single  :168-248   update_grid  :250-291   g2p_single  :293-348
//   apply_plasticity :114-166
//
// Layout: particles are FP32 SoA planes (bm_internal.h, Plane); the grid is a
// dense box of 4^3-node blocks holding two float4 per node: (momentum, mass)
// and (force, 0). P2G scatters with 16-byte vector reductions into L2
// (red.global.add.v4.f32), two per particle-node pair.
#include <algorithm>

#include "bm_internal.h"
#include "bm_math.cuh"

namespace bm {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void red_add_v4(float4* addr, float a, float b, float c, float d) {
    atomicAdd(addr, make_float4(a, b, c, d));
}

__global__ void __launch_bounds__(kThreads) k_p2g(ParticleSoA ps, GridDesc g, GridBuffers gb, Material mat,
                                                  uint32_t* status, unsigned long long* escaped) {
    // One thread per particle; scatter with 16-byte vector reductions.
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ps.n) return;
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
    hencky_tau(F, mat.mu, mat.lambda, tau);
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
                red_add_v4(gb.acc.mv + id, (v[0] + a0) * mc, (v[1] + a1) * mc, (v[2] + a2) * mc, mc);
                red_add_v4(gb.acc.f + id, s0 * w, s1 * w, s2 * w, 0.0f);
            }
    mark_stencil_blocks(g, gb.acc, gb.alloc, base, wgt[0], wgt[1], wgt[2]);
    if (dropped) {
        atomicOr(status, ERR_ESCAPE);
        atomicAdd(escaped, (unsigned long long)dropped);
    }
}

// update_grid over the blocks listed in `cur` (every other node of the box is
// empty, so skipping it is exact); the same launch zeroes the blocks listed in
// `other` so that it can take the next P2G.
__global__ void __launch_bounds__(kThreads) k_grid_update(GridDesc g, GridAcc cur, GridAcc other, Material mat,
                                                          float dt, bool folded) {
    const int n_cur = *cur.count, n_other = *other.count;
    const int64_t total = (int64_t)(n_cur + n_other) * 64;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int slot = (int)(e >> 6), t = (int)(e & 63);
        if (slot >= n_cur) {
            const int64_t b = other.list[slot - n_cur];
            const int64_t id = g.node_of_block(b, t);
            other.mv[id] = make_float4(0.f, 0.f, 0.f, 0.f);
            other.f[id] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (t == 0) other.touched[b] = 0u;
            continue;
        }
        const int64_t b = cur.list[slot];
        const int64_t id = g.node_of_block(b, t);
        const float4 mv = cur.mv[id];
        if (!(mv.w > 1e-6f)) {
            // inactive (mass 0) or mass <= 1e-6: the reference leaves the
            // momentum (without force) in place
            if (folded && (mv.w > 0.0f || mv.x != 0.0f || mv.y != 0.0f || mv.z != 0.0f)) {
                const float4 f = cur.f[id];
                cur.mv[id] = make_float4(mv.x - f.x * dt, mv.y - f.y * dt, mv.z - f.z * dt, mv.w);
            }
            continue;
        }
        float v0, v1, v2;
        if (folded) {
            v0 = mv.x / mv.w;
            v1 = mv.y / mv.w;
            v2 = mv.z / mv.w;
        } else {
            const float4 f = cur.f[id];
            v0 = (mv.x + f.x * dt) / mv.w;
            v1 = (mv.y + f.y * dt) / mv.w;
            v2 = (mv.z + f.z * dt) / mv.w;
        }
        v0 = v0 + mat.gx * dt;
        v1 = v1 + mat.gy * dt;
        v2 = v2 + mat.gz * dt;
        const int lj = (t >> 2) & 3;
        const int bj = (int)((b / g.nbz) % g.nby);
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
        cur.mv[id] = make_float4(v0, v1, v2, mv.w);
    }
}

__global__ void __launch_bounds__(kThreads) k_g2p(ParticleSoA ps, GridDesc g, GridBuffers gb, Material mat, float dt,
                                                  uint32_t* status, unsigned long long* escaped) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ps.n) return;
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
                const float4 nv = gb.acc.mv[id];
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
    dp_project(F, Cm, dt, mat.neg_alpha_koh);
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
    if (!finite) atomicOr(status, ERR_NONFINITE);
    if (dropped) {
        atomicOr(status, ERR_ESCAPE);
        atomicAdd(escaped, (unsigned long long)dropped);
    }
}

inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

}  // namespace

void launch_p2g(const ParticleSoA& ps, const GridDesc& g, const GridBuffers& gb, const Material& mat,
                uint32_t* d_status, unsigned long long* d_escaped, cudaStream_t st) {
    if (ps.n == 0) return;
    k_p2g<<<blocks_for(ps.n), kThreads, 0, st>>>(ps, g, gb, mat, d_status, d_escaped);
}

void launch_grid_update(const GridDesc& g, const GridAcc& cur, const GridAcc& other, const Material& mat, float dt,
                        bool folded, int64_t max_blocks, cudaStream_t st) {
    const int64_t want = (2 * max_blocks * 64 + kThreads - 1) / kThreads;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, 148 * 16));
    k_grid_update<<<grid, kThreads, 0, st>>>(g, cur, other, mat, dt, folded);
}

void launch_g2p(const ParticleSoA& ps, const GridDesc& g, const GridBuffers& gb, const Material& mat, float dt,
                uint32_t* d_status, unsigned long long* d_escaped, cudaStream_t st) {
    if (ps.n == 0) return;
    k_g2p<<<blocks_for(ps.n), kThreads, 0, st>>>(ps, g, gb, mat, dt, d_status, d_escaped);
}

// ---- particle rows in add order ------------------------------------------------

namespace {

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

}  // namespace

void launch_gather_rows(const ParticleSoA& ps, int plane0, int width, float* out, cudaStream_t st) {
    if (ps.n == 0) return;
    k_gather_rows<<<blocks_for(ps.n), kThreads, 0, st>>>(ps, plane0, width, out);
}

void launch_scatter_rows(const ParticleSoA& ps, int plane0, int width, const float* in, int64_t first, int64_t n,
                         const int32_t* inv, cudaStream_t st) {
    if (n == 0) return;
    k_scatter_rows<<<blocks_for(n), kThreads, 0, st>>>(ps, plane0, width, in, first, n, inv);
}

void launch_inverse_pid(const ParticleSoA& ps, int32_t* inv, cudaStream_t st) {
    if (ps.n == 0) return;
    k_inverse_pid<<<blocks_for(ps.n), kThreads, 0, st>>>(ps, inv);
}

}  // namespace bm
