// bm_m1.cu — M1 PIC-rigid coupler and grid copy/seed kernels.
//
// Reference (2nugu/basements):
//   MPMRigidCouplerPIC::apply  include/basements/physics/coupling/mpm_rigid_coupler_pic.h:88-184
//   shape_inside               include/basements/physics/coupling/mpm_rigid_coupler.h:90-103
//   Matrix3::from_quaternion   include/basements/core/math/matrix3.h:432-447
//
// One CTA of 64 threads per candidate 4^3 block of the body's AABB (one
// thread per node). The reference visits only blocks its hash grid has
// allocated and whose node-centre span overlaps the AABB; the same two tests
// run here on the block-allocated flags. Node arithmetic uses explicit
// round-to-nearest intrinsics (no FMA contraction) so that the inside test
// and the exchanged velocities match the reference bit for bit. Force, torque
// and the node count are reduced per CTA in double and added into a per-body
// accumulator.
#include <cmath>

#include "bm_internal.h"
#include "bm_math.cuh"

namespace bm {

namespace {

__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

__global__ void __launch_bounds__(64) k_m1(GridDesc g, GridBuffers gb, M1Params P, double* acc) {
    const int cb = blockIdx.x;
    const int bk = P.bk0 + cb % P.nbk;
    const int bj = P.bj0 + (cb / P.nbk) % P.nbj;
    const int bi = P.bi0 + cb / (P.nbk * P.nbj);
    const int64_t blin = ((int64_t)bi * g.nby + bj) * g.nbz + bk;
    const int t = threadIdx.x;

    double f0 = 0, f1 = 0, f2 = 0, t0 = 0, t1 = 0, t2 = 0, cnt = 0;
    const int ox = g.ox + 4 * bi, oy = g.oy + 4 * bj, oz = g.oz + 4 * bk;
    const float dx = g.dx;
    bool visit = gb.alloc[blin] != 0;
    if (visit) {
        const float blo0 = mul((float)ox + 0.5f, dx), bhi0 = mul((float)(ox + 3) + 0.5f, dx);
        const float blo1 = mul((float)oy + 0.5f, dx), bhi1 = mul((float)(oy + 3) + 0.5f, dx);
        const float blo2 = mul((float)oz + 0.5f, dx), bhi2 = mul((float)(oz + 3) + 0.5f, dx);
        if (bhi0 < P.lo[0] || blo0 > P.hi[0]) visit = false;
        if (bhi1 < P.lo[1] || blo1 > P.hi[1]) visit = false;
        if (bhi2 < P.lo[2] || blo2 > P.hi[2]) visit = false;
    }
    if (visit) {
        const int li = t >> 4, lj = (t >> 2) & 3, lk = t & 3;
        const int64_t id = g.node_of_block(blin, t);
        const float xn[3] = {mul((float)(ox + li) + 0.5f, dx), mul((float)(oy + lj) + 0.5f, dx),
                             mul((float)(oz + lk) + 0.5f, dx)};
        const float r[3] = {sub(xn[0], P.c[0]), sub(xn[1], P.c[1]), sub(xn[2], P.c[2])};
        float l[3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
            l[a] = add(add(mul(P.R[a], r[0]), mul(P.R[3 + a], r[1])), mul(P.R[6 + a], r[2]));
        bool inside;
        if (P.shape == 1) {
            const float r2 = add(mul(l[0], l[0]), mul(l[2], l[2]));
            inside = fabsf(l[1]) <= P.he[1] && r2 <= mul(P.he[0], P.he[0]);
        } else {
            inside = fabsf(l[0]) <= P.he[0] && fabsf(l[1]) <= P.he[1] && fabsf(l[2]) <= P.he[2];
        }
        if (inside) {
            const float vb[3] = {add(P.vl[0], sub(mul(P.w[1], r[2]), mul(P.w[2], r[1]))),
                                 add(P.vl[1], sub(mul(P.w[2], r[0]), mul(P.w[0], r[2]))),
                                 add(P.vl[2], sub(mul(P.w[0], r[1]), mul(P.w[1], r[0])))};
            float4 nv = gb.acc.mv[id];
            float va[3];
            if (!(nv.w >= 1e-9f)) {  // inactive (mass 0) or mass < 1e-9: body claims the node
                va[0] = vb[0]; va[1] = vb[1]; va[2] = vb[2];
                nv = make_float4(vb[0], vb[1], vb[2], P.mb);
            } else {
                const float mn = add(nv.w, P.mb);
                const float pa[3] = {add(mul(nv.x, nv.w), mul(vb[0], P.mb)), add(mul(nv.y, nv.w), mul(vb[1], P.mb)),
                                     add(mul(nv.z, nv.w), mul(vb[2], P.mb))};
                if (fabsf(mn) < 1e-6f) {  // Vec3 division guard of the reference
                    va[0] = va[1] = va[2] = 0.0f;
                } else {
                    va[0] = __fdiv_rn(pa[0], mn); va[1] = __fdiv_rn(pa[1], mn); va[2] = __fdiv_rn(pa[2], mn);
                }
                nv = make_float4(va[0], va[1], va[2], mn);
            }
            gb.acc.mv[id] = nv;
            touch_block(gb.acc, blin);
            const float dF[3] = {mul(sub(va[0], vb[0]), P.mb_over_dt), mul(sub(va[1], vb[1]), P.mb_over_dt),
                                 mul(sub(va[2], vb[2]), P.mb_over_dt)};
            f0 = dF[0]; f1 = dF[1]; f2 = dF[2];
            t0 = sub(mul(r[1], dF[2]), mul(r[2], dF[1]));
            t1 = sub(mul(r[2], dF[0]), mul(r[0], dF[2]));
            t2 = sub(mul(r[0], dF[1]), mul(r[1], dF[0]));
            cnt = 1;
        }
    }
    // 64 threads = 2 warps: shuffle-reduce, then combine through shared memory.
    double vals[7] = {f0, f1, f2, t0, t1, t2, cnt};
#pragma unroll
    for (int q = 0; q < 7; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vals[q] += __shfl_down_sync(0xffffffffu, vals[q], o);
    __shared__ double part[2][7];
    if ((t & 31) == 0) {
#pragma unroll
        for (int q = 0; q < 7; ++q) part[t >> 5][q] = vals[q];
    }
    __syncthreads();
    if (t < 7) {
        const double s = part[0][t] + part[1][t];
        if (s != 0.0) atomicAdd(acc + t, s);
    }
}

__global__ void k_reaction_finalize(const double* acc, int n, bm_reaction_t* out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const double* a = acc + 7 * b;
    bm_reaction_t r;
    for (int q = 0; q < 3; ++q) {
        r.force[q] = (float)a[q];
        r.torque[q] = (float)a[3 + q];
    }
    r.nodes_inside = (int32_t)a[6];
    out[b] = r;
}

__global__ void k_grid_to_dense(GridDesc g, GridBuffers gb, float* vel, float* force, float* mass, uint8_t* active,
                                uint8_t* balloc) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ez = (int64_t)g.nbz * 4, ey = (int64_t)g.nby * 4;
    if (q >= g.num_nodes()) return;
    const int k = (int)(q % ez), j = (int)((q / ez) % ey), i = (int)(q / (ez * ey));
    const int64_t id = g.node(g.ox + i, g.oy + j, g.oz + k);
    const float4 mv = gb.acc.mv[id];
    if (vel) { vel[3 * q] = mv.x; vel[3 * q + 1] = mv.y; vel[3 * q + 2] = mv.z; }
    if (force) {
        const float4 f = gb.acc.f[id];
        force[3 * q] = f.x; force[3 * q + 1] = f.y; force[3 * q + 2] = f.z;
    }
    if (mass) mass[q] = mv.w;
    if (active) active[q] = mv.w > 0.0f ? 1 : 0;
    if (balloc) balloc[q] = gb.alloc[g.block_of_node(id)];
}

__global__ void k_dense_velocity_to_grid(GridDesc g, GridBuffers gb, const float* vel) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ez = (int64_t)g.nbz * 4, ey = (int64_t)g.nby * 4;
    if (q >= g.num_nodes()) return;
    const int k = (int)(q % ez), j = (int)((q / ez) % ey), i = (int)(q / (ez * ey));
    const int64_t id = g.node(g.ox + i, g.oy + j, g.oz + k);
    float4 mv = gb.acc.mv[id];
    mv.x = vel[3 * q]; mv.y = vel[3 * q + 1]; mv.z = vel[3 * q + 2];
    gb.acc.mv[id] = mv;
    if (mv.x != 0.0f || mv.y != 0.0f || mv.z != 0.0f || mv.w != 0.0f) touch_block(gb.acc, g.block_of_node(id));
}

__global__ void k_seed(GridDesc g, GridBuffers gb, int64_t n, const int32_t* ijk, const float* vel, const float* mass,
                       uint32_t* status) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int64_t id = g.node(ijk[3 * q], ijk[3 * q + 1], ijk[3 * q + 2]);
    if (id < 0) {
        atomicOr(status, ERR_ESCAPE);
        return;
    }
    gb.acc.mv[id] = make_float4(vel[3 * q], vel[3 * q + 1], vel[3 * q + 2], mass[q]);
    gb.alloc[g.block_of_node(id)] = 1;
    touch_block(gb.acc, g.block_of_node(id));
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// Host-side preparation in plain float (host code is compiled without FMA
// contraction), following mpm_rigid_coupler_pic.h:100-117.
bool m1_prepare(const GridDesc& g, const bm_collider_t& b, float dt, M1Params* P) {
    if (!(dt > 0.0f)) return false;
    const float w = b.orientation[0], x = b.orientation[1], y = b.orientation[2], z = b.orientation[3];
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
    const float wx = w * x, wy = w * y, wz = w * z;
    float* R = P->R;
    R[0] = 1.0f - 2.0f * (yy + zz); R[1] = 2.0f * (xy - wz);        R[2] = 2.0f * (xz + wy);
    R[3] = 2.0f * (xy + wz);        R[4] = 1.0f - 2.0f * (xx + zz); R[5] = 2.0f * (yz - wx);
    R[6] = 2.0f * (xz - wy);        R[7] = 2.0f * (yz + wx);        R[8] = 1.0f - 2.0f * (xx + yy);
    const float hx = b.half_extents[0], hy = b.half_extents[1], hz = b.half_extents[2];
    const float dx = g.dx;
    const float vol = 8.0f * hx * hy * hz;
    const int approx = std::max(1, (int)std::round(vol / (dx * dx * dx)));
    P->mb = b.mass / (float)approx;
    P->mb_over_dt = P->mb / dt;
    for (int a = 0; a < 3; ++a) {
        const float h = std::fabs(R[3 * a]) * hx + std::fabs(R[3 * a + 1]) * hy + std::fabs(R[3 * a + 2]) * hz;
        P->lo[a] = b.center[a] - h;
        P->hi[a] = b.center[a] + h;
        P->c[a] = b.center[a];
        P->vl[a] = b.linear_velocity[a];
        P->w[a] = b.angular_velocity[a];
        P->he[a] = b.half_extents[a];
    }
    P->shape = b.shape;
    // Conservative candidate block range (the exact float test runs per block).
    const int org[3] = {g.ox, g.oy, g.oz};
    const int nb[3] = {g.nbx, g.nby, g.nbz};
    int b0[3], n[3];
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(P->lo[a]) || !std::isfinite(P->hi[a])) return false;
        const double lo_node = std::floor((double)P->lo[a] / dx - 0.5) - 4;
        const double hi_node = std::ceil((double)P->hi[a] / dx - 0.5) + 4;
        long lo_b = (long)std::floor((lo_node - org[a]) / 4.0);
        long hi_b = (long)std::floor((hi_node - org[a]) / 4.0);
        lo_b = std::max(lo_b, 0L);
        hi_b = std::min(hi_b, (long)nb[a] - 1);
        if (hi_b < lo_b) return false;
        b0[a] = (int)lo_b;
        n[a] = (int)(hi_b - lo_b + 1);
    }
    P->bi0 = b0[0]; P->bj0 = b0[1]; P->bk0 = b0[2];
    P->nbi = n[0]; P->nbj = n[1]; P->nbk = n[2];
    return true;
}

void launch_m1(const GridDesc& g, const GridBuffers& gb, const M1Params& p, double* d_acc, cudaStream_t st) {
    const int64_t nblocks = (int64_t)p.nbi * p.nbj * p.nbk;
    if (nblocks <= 0) return;
    k_m1<<<(unsigned)nblocks, 64, 0, st>>>(g, gb, p, d_acc);
}

void launch_reaction_finalize(const double* d_acc, int n_bodies, bm_reaction_t* d_out, cudaStream_t st) {
    if (n_bodies <= 0) return;
    k_reaction_finalize<<<nblk(n_bodies, 64), 64, 0, st>>>(d_acc, n_bodies, d_out);
}

void launch_grid_to_dense(const GridDesc& g, const GridBuffers& gb, float* vel, float* force, float* mass,
                          uint8_t* active, uint8_t* balloc, cudaStream_t st) {
    k_grid_to_dense<<<nblk(g.num_nodes(), 256), 256, 0, st>>>(g, gb, vel, force, mass, active, balloc);
}

void launch_dense_velocity_to_grid(const GridDesc& g, const GridBuffers& gb, const float* vel, cudaStream_t st) {
    k_dense_velocity_to_grid<<<nblk(g.num_nodes(), 256), 256, 0, st>>>(g, gb, vel);
}

void launch_seed_grid(const GridDesc& g, const GridBuffers& gb, int64_t n, const int32_t* ijk, const float* vel,
                      const float* mass, uint32_t* d_status, cudaStream_t st) {
    if (n <= 0) return;
    k_seed<<<nblk(n, 256), 256, 0, st>>>(g, gb, n, ijk, vel, mass, d_status);
}

}  // namespace bm
