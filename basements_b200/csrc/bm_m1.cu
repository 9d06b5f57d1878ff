// bm_m1.cu — M1 PIC-rigid coupler, device rigid-body update, grid copies.
//
// Reference (2nugu/basements):
//   MPMRigidCouplerPIC::apply  include/basements/physics/coupling/mpm_rigid_coupler_pic.h:88-184
//   shape_inside               include/basements/physics/coupling/mpm_rigid_coupler.h:90-103
//   Matrix3::from_quaternion   include/basements/core/math/matrix3.h:432-447
//   TimeIntegrator::integrate  include/basements/physics/dynamics/integrator.h:19-57
//
// One CTA of 64 threads per candidate 4^3 block of a body's AABB (one thread
// per node), one grid row per body. The reference visits only blocks its hash
// grid has allocated and whose node-centre span overlaps the AABB; the same
// two tests run here on the block-allocated flags. Node arithmetic is written
// with explicit round-to-nearest operations (no FMA contraction) so that the
// inside test and the exchanged velocities match the reference bit for bit.
// Force, torque and the node count are reduced per CTA in double and added
// into a per-body accumulator.
#include <cmath>

#include "bm_internal.h"
#include "bm_m1.cuh"
#include "bm_math.cuh"

namespace bm {

namespace {

using namespace rn;

// Matrix3::from_quaternion (matrix3.h:432-447), row-major.
__host__ __device__ void body_rotation(const bm_collider_t& b, float R[9]) {
    const float w = b.orientation[0], x = b.orientation[1], y = b.orientation[2], z = b.orientation[3];
    const float xx = mul(x, x), yy = mul(y, y), zz = mul(z, z), xy = mul(x, y), xz = mul(x, z), yz = mul(y, z);
    const float wx = mul(w, x), wy = mul(w, y), wz = mul(w, z);
    R[0] = sub(1.0f, mul(2.0f, add(yy, zz))); R[1] = mul(2.0f, sub(xy, wz)); R[2] = mul(2.0f, add(xz, wy));
    R[3] = mul(2.0f, add(xy, wz)); R[4] = sub(1.0f, mul(2.0f, add(xx, zz))); R[5] = mul(2.0f, sub(yz, wx));
    R[6] = mul(2.0f, sub(xz, wy)); R[7] = mul(2.0f, add(yz, wx)); R[8] = sub(1.0f, mul(2.0f, add(xx, yy)));
}

// Conservative candidate block range of P's AABB (lo, hi) in the box (the
// exact float test runs per block); false when it misses the box.
__host__ __device__ bool candidate_range(const GridDesc& g, M1Params* P) {
    const float dx = g.dx;
    const int org[3] = {g.ox, g.oy, g.oz};
    const int nb[3] = {g.nbx, g.nby, g.nbz};
    int b0[3], n[3];
    for (int a = 0; a < 3; ++a) {
        if (!(P->lo[a] > -1e30f && P->hi[a] < 1e30f)) return false;
        // one node of slack on each side for the float/double rounding
        const double lo_node = floor((double)P->lo[a] / dx - 0.5) - 1;
        const double hi_node = ceil((double)P->hi[a] / dx - 0.5) + 1;
        double lo_b = floor((lo_node - org[a]) / 4.0);
        double hi_b = floor((hi_node - org[a]) / 4.0);
        lo_b = lo_b < 0.0 ? 0.0 : lo_b;
        hi_b = hi_b > (double)(nb[a] - 1) ? (double)(nb[a] - 1) : hi_b;
        if (hi_b < lo_b) return false;
        b0[a] = (int)lo_b;
        n[a] = (int)(hi_b - lo_b) + 1;
    }
    P->bi0 = b0[0]; P->bj0 = b0[1]; P->bk0 = b0[2];
    P->nbi = n[0]; P->nbj = n[1]; P->nbk = n[2];
    return true;
}

// mpm_rigid_coupler_pic.h:100-117 plus the candidate block range.
__host__ __device__ bool m1_params(const GridDesc& g, const bm_collider_t& b, float dt, int scene, M1Params* P) {
    P->scene = scene;
    P->active = 0;
    P->nbi = P->nbj = P->nbk = 0;
    P->bi0 = P->bj0 = P->bk0 = 0;
    if (!(dt > 0.0f)) return false;
    float* R = P->R;
    body_rotation(b, R);
    const float hx = b.half_extents[0], hy = b.half_extents[1], hz = b.half_extents[2];
    const float dx = g.dx;
    const float vol = mul(mul(mul(8.0f, hx), hy), hz);
    const int approx = (int)roundf(dvd(vol, mul(mul(dx, dx), dx)));
    P->mb = dvd(b.mass, (float)(approx > 1 ? approx : 1));
    P->mb_over_dt = dvd(P->mb, dt);
    for (int a = 0; a < 3; ++a) {
        const float h = add(add(mul(fabsf(R[3 * a]), hx), mul(fabsf(R[3 * a + 1]), hy)), mul(fabsf(R[3 * a + 2]), hz));
        P->lo[a] = sub(b.center[a], h);
        P->hi[a] = add(b.center[a], h);
        P->c[a] = b.center[a];
        P->vl[a] = b.linear_velocity[a];
        P->w[a] = b.angular_velocity[a];
        P->he[a] = b.half_extents[a];
    }
    P->shape = b.shape;
    P->friction = b.friction;
    if (!candidate_range(g, P)) return false;
    P->active = 1;
    return true;
}

// m4_5_hybrid.h:113-120: the M4.5a frame of one body. P->lo/hi is the
// shape's tight AABB (shape_world_aabb_half, mpm_rigid_coupler.h:167-200) and
// P->mb holds the body's mass (the per-node share is set by the sweep).
bool m45a_params(const GridDesc& g, const bm_collider_t& b, float dt, M1Params* P) {
    P->scene = 0;
    P->active = 0;
    P->nbi = P->nbj = P->nbk = 0;
    P->bi0 = P->bj0 = P->bk0 = 0;
    if (!(dt > 0.0f)) return false;
    float* R = P->R;
    body_rotation(b, R);
    const float hx = b.half_extents[0], hy = b.half_extents[1], hz = b.half_extents[2];
    for (int a = 0; a < 3; ++a) {
        float h;
        if (b.shape == 1) {
            // |a_i| L + sqrt(max(0, 1 - a_i^2)) R, a = the body's y axis in world
            const float ai = R[3 * a + 1];
            const float s = sub(1.0f, mul(ai, ai));
            const float perp = s > 0.0f ? std::sqrt(s) : 0.0f;
            h = add(mul(fabsf(ai), hy), mul(perp, hx));
        } else {
            h = add(add(mul(fabsf(R[3 * a]), hx), mul(fabsf(R[3 * a + 1]), hy)), mul(fabsf(R[3 * a + 2]), hz));
        }
        P->lo[a] = sub(b.center[a], h);
        P->hi[a] = add(b.center[a], h);
        P->c[a] = b.center[a];
        P->vl[a] = b.linear_velocity[a];
        P->w[a] = b.angular_velocity[a];
        P->he[a] = b.half_extents[a];
    }
    P->shape = b.shape;
    P->friction = b.friction;
    P->mb = b.mass;
    P->mb_over_dt = 0.0f;
    if (!candidate_range(g, P)) return false;
    P->active = 1;
    return true;
}

// Candidate block (cb) of body P in scene S: its (bi, bj, bk) and linear id.
__device__ __forceinline__ void candidate_block(const M1Params& P, const GridDesc& g, int64_t cb, int& bi, int& bj,
                                                int& bk) {
    bk = P.bk0 + (int)(cb % P.nbk);
    bj = P.bj0 + (int)((cb / P.nbk) % P.nbj);
    bi = P.bi0 + (int)(cb / ((int64_t)P.nbk * P.nbj));
}

// Sum over the 64 threads (2 warps) of a CTA, added to *out when non-zero.
template <int N>
__device__ __forceinline__ void cta64_add(double (&vals)[N], double* out) {
#pragma unroll
    for (int q = 0; q < N; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vals[q] += __shfl_down_sync(0xffffffffu, vals[q], o);
    __shared__ double part[2][N];
    const int tt = threadIdx.x;
    if ((tt & 31) == 0) {
#pragma unroll
        for (int q = 0; q < N; ++q) part[tt >> 5][q] = vals[q];
    }
    __syncthreads();
    if (tt < N) {
        const double s = part[0][tt] + part[1][tt];
        if (s != 0.0) atomicAdd(out + tt, s);
    }
}

// shape_outward_normal_local (mpm_rigid_coupler.h:106-132): the outward
// normal of the closest face in the body frame.
__device__ __forceinline__ void outward_normal_local(const M1Params& P, const float l[3], float n[3]) {
    n[0] = n[1] = n[2] = 0.0f;
    if (P.shape == 1) {
        const float r = __fsqrt_rn(add(mul(l[0], l[0]), mul(l[2], l[2])));
        const float axial = sub(P.he[1], fabsf(l[1]));
        const float radial = sub(P.he[0], r);
        if (axial < radial) {
            n[1] = l[1] >= 0.0f ? 1.0f : -1.0f;
        } else if (r > 1e-9f) {
            n[0] = dvd(l[0], r);
            n[2] = dvd(l[2], r);
        } else {
            n[0] = 1.0f;
        }
        return;
    }
    const float d0 = sub(P.he[0], fabsf(l[0])), d1 = sub(P.he[1], fabsf(l[1])), d2 = sub(P.he[2], fabsf(l[2]));
    if (d0 <= d1 && d0 <= d2) n[0] = l[0] >= 0.0f ? 1.0f : -1.0f;
    else if (d1 <= d2) n[1] = l[1] >= 0.0f ? 1.0f : -1.0f;
    else n[2] = l[2] >= 0.0f ? 1.0f : -1.0f;
}

__device__ __forceinline__ float dot3(const float a[3], const float b[3]) {
    return add(add(mul(a[0], b[0]), mul(a[1], b[1])), mul(a[2], b[2]));
}

// (R_l2w * shape_outward_normal_local).normalized() (Vec3::normalized: zero
// below length 1e-6).
__device__ __forceinline__ void world_face_normal(const M1Params& P, const float l[3], float nw[3]) {
    float nl[3];
    outward_normal_local(P, l, nl);
#pragma unroll
    for (int a = 0; a < 3; ++a)
        nw[a] = add(add(mul(P.R[3 * a], nl[0]), mul(P.R[3 * a + 1], nl[1])), mul(P.R[3 * a + 2], nl[2]));
    const float len = __fsqrt_rn(dot3(nw, nw));
#pragma unroll
    for (int a = 0; a < 3; ++a) nw[a] = len < 1e-6f ? 0.0f : dvd(nw[a], len);
}

// apply_friction_tangent (m4_5_hybrid.h:225-232): keep the normal part of v,
// blend its tangential part toward the body's by min(1, friction).
__device__ __forceinline__ void friction_tangent(float v[3], const float vb[3], const float n[3], float friction) {
    const float vn = dot3(v, n), vbn = dot3(vb, n);
    const float fr = friction < 1.0f ? friction : 1.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float vt = sub(v[a], mul(n[a], vn));
        const float vtb = sub(vb[a], mul(n[a], vbn));
        v[a] = add(mul(n[a], vn), add(vt, mul(sub(vtb, vt), fr)));
    }
}

// bspline1d (m4_5_hybrid.h:58-63): the quadratic B-spline, 0 beyond 1.5.
__device__ __forceinline__ float bspline1d(float xi) {
    const float a = fabsf(xi);
    if (a < 0.5f) return sub(0.75f, mul(a, a));
    if (a < 1.5f) {
        const float t = sub(1.5f, a);
        return mul(mul(0.5f, t), t);
    }
    return 0.0f;
}

// M0, MPMRigidCoupler::apply (mpm_rigid_coupler.cpp:58-143): over the
// visited blocks of the M1 frame, a node with mass > 1e-8 inside the shape
// keeps its normal velocity no slower outward than the body's (n = the
// closest face's normal in world, normalised) and blends its tangential
// velocity toward the body's by min(1, friction); its mass is unchanged. The
// reaction is -dp/dt and its moment, per CTA in double into acc.
__global__ void __launch_bounds__(64) k_m0(SceneTable t, const M1Params* params, int cur, float dt, double* acc) {
    const M1Params& P = params[0];
    if (!P.active) return;
    const int64_t cb = blockIdx.x;
    if (cb >= (int64_t)P.nbi * P.nbj * P.nbk) return;
    const SceneDev& S = t.scenes[P.scene];
    const GridDesc g = S.g;
    const GridAcc A = S.acc[cur];
    int bi, bj, bk;
    candidate_block(P, g, cb, bi, bj, bk);
    const int64_t blin = g.block_of(bi, bj, bk);
    const int tt = threadIdx.x;
    double vals[7] = {0, 0, 0, 0, 0, 0, 0};
    if (m1_block_visited(P, g, S.alloc, bi, bj, bk)) {
        const int64_t id = g.node_of_block(blin, tt);
        float4 nv = A.mv[id];
        const float m = node_total_mass(nv, A.f[id]);
        float r[3], l[3];
        if (m > 1e-8f && coupler_node_local(P, g.dx, g.ox + 4 * bi + (tt >> 4), g.oy + 4 * bj + ((tt >> 2) & 3),
                                            g.oz + 4 * bk + (tt & 3), r, l)) {
            const float vb[3] = {add(P.vl[0], sub(mul(P.w[1], r[2]), mul(P.w[2], r[1]))),
                                 add(P.vl[1], sub(mul(P.w[2], r[0]), mul(P.w[0], r[2]))),
                                 add(P.vl[2], sub(mul(P.w[0], r[1]), mul(P.w[1], r[0])))};
            float nw[3];
            world_face_normal(P, l, nw);
            const float v[3] = {nv.x, nv.y, nv.z};
            const float vn_node = dot3(v, nw), vn_body = dot3(vb, nw);
            const float vn_cl = vn_node < vn_body ? vn_body : vn_node;
            const float fr = P.friction < 1.0f ? P.friction : 1.0f;
            float va[3], dp[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float vt_node = sub(v[a], mul(nw[a], vn_node));
                const float vt_body = sub(vb[a], mul(nw[a], vn_body));
                const float vt_new = add(vt_node, mul(sub(vt_body, vt_node), fr));
                va[a] = add(mul(nw[a], vn_cl), vt_new);
                dp[a] = mul(sub(va[a], v[a]), m);
            }
            nv.x = va[0]; nv.y = va[1]; nv.z = va[2];
            A.mv[id] = nv;
            const bool tiny = fabsf(dt) < 1e-6f;  // Vec3 division guard of the reference
            const float tq[3] = {sub(mul(r[1], dp[2]), mul(r[2], dp[1])), sub(mul(r[2], dp[0]), mul(r[0], dp[2])),
                                 sub(mul(r[0], dp[1]), mul(r[1], dp[0]))};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                vals[a] = tiny ? 0.0f : -dvd(dp[a], dt);
                vals[3 + a] = tiny ? 0.0f : -dvd(tq[a], dt);
            }
            vals[6] = 1;
        }
    }
    cta64_add<7>(vals, acc);
}

// M4.5a pass 1 (m4_5_hybrid.h:126-146): the overlap fraction summed over the
// nodes inside the shape, per CTA in double, into *frac_sum.
__global__ void __launch_bounds__(64) k_m45a_sum(SceneTable t, const M1Params* params, int cur, double* frac_sum) {
    const M1Params& P = params[0];
    if (!P.active) return;
    const int64_t cb = blockIdx.x;
    if (cb >= (int64_t)P.nbi * P.nbj * P.nbk) return;
    const SceneDev& S = t.scenes[P.scene];
    const GridDesc g = S.g;
    int bi, bj, bk;
    candidate_block(P, g, cb, bi, bj, bk);
    const int tt = threadIdx.x;
    double vals[1] = {0.0};
    if (m1_block_visited(P, g, S.alloc, bi, bj, bk)) {
        float r[3], l[3];
        if (coupler_node_local(P, g.dx, g.ox + 4 * bi + (tt >> 4), g.oy + 4 * bj + ((tt >> 2) & 3),
                               g.oz + 4 * bk + (tt & 3), r, l))
            vals[0] = coupler_overlap_fraction(P, l);
    }
    cta64_add<1>(vals, frac_sum);
}

// Sweep pass 2 (m4_5_hybrid.h:148-208) with the rule of Layer 0 = M4_5a
// (:242-257), 1 = M4_5b (:259-275), 2 = M4_5c (:282-305): each inside node
// gets m_b = M frac / sum (skipped when m_b <= 0; layer c scales it by the
// B-spline weight of (x_node - centre) / dx and, below 1e-6, gives the node
// the body velocity and no mass) and the mass-weighted average of node and
// body velocity, as in M1; layers b and c then blend its tangential part
// toward the body's about the closest face's normal. Reaction into acc
// (force, torque, count) per CTA in double. The sum arrives in double and is
// used in float, the type of the reference's accumulator.
template <int Layer>
__global__ void __launch_bounds__(64) k_m45(SceneTable t, const M1Params* params, int cur, float dt,
                                            const double* frac_sum, double* acc) {
    const M1Params& P = params[0];
    if (!P.active) return;
    const int64_t cb = blockIdx.x;
    if (cb >= (int64_t)P.nbi * P.nbj * P.nbk) return;
    const float fs = (float)*frac_sum;
    if (fs < 1e-9f) return;  // no overlap at all (m4_5_hybrid.h:147)
    const float per_frac = dvd(P.mb, fs);
    const SceneDev& S = t.scenes[P.scene];
    const GridDesc g = S.g;
    const GridAcc A = S.acc[cur];
    int bi, bj, bk;
    candidate_block(P, g, cb, bi, bj, bk);
    const int64_t blin = g.block_of(bi, bj, bk);
    const int tt = threadIdx.x;
    double vals[7] = {0, 0, 0, 0, 0, 0, 0};
    if (m1_block_visited(P, g, S.alloc, bi, bj, bk)) {
        float r[3], l[3];
        if (coupler_node_local(P, g.dx, g.ox + 4 * bi + (tt >> 4), g.oy + 4 * bj + ((tt >> 2) & 3),
                               g.oz + 4 * bk + (tt & 3), r, l)) {
            float mb = mul(per_frac, coupler_overlap_fraction(P, l));
            if (!(mb <= 0.0f)) {
                const float vb[3] = {add(P.vl[0], sub(mul(P.w[1], r[2]), mul(P.w[2], r[1]))),
                                     add(P.vl[1], sub(mul(P.w[2], r[0]), mul(P.w[0], r[2]))),
                                     add(P.vl[2], sub(mul(P.w[0], r[1]), mul(P.w[1], r[0])))};
                bool rule = true;
                if (Layer == 2) {
                    const float k = mul(mul(bspline1d(dvd(r[0], g.dx)), bspline1d(dvd(r[1], g.dx))),
                                        bspline1d(dvd(r[2], g.dx)));
                    if (k < 1e-6f) {
                        mb = 0.0f;
                        rule = false;
                    } else {
                        mb = mul(mb, k);
                    }
                }
                const int64_t id = g.node_of_block(blin, tt);
                float4 nv = A.mv[id];
                float4 nf = A.f[id];
                const float m_tot = node_total_mass(nv, nf);
                float va[3] = {vb[0], vb[1], vb[2]};
                const bool was_active = m_tot >= 1e-9f;  // else the node's mass is dropped (old_mass = 0)
                if (rule && was_active) {
                    const float mn = add(m_tot, mb);
                    const float pa[3] = {add(mul(nv.x, m_tot), mul(vb[0], mb)), add(mul(nv.y, m_tot), mul(vb[1], mb)),
                                         add(mul(nv.z, m_tot), mul(vb[2], mb))};
                    if (fabsf(mn) < 1e-6f) {  // Vec3 division guard of the reference
                        va[0] = va[1] = va[2] = 0.0f;
                    } else {
                        va[0] = dvd(pa[0], mn); va[1] = dvd(pa[1], mn); va[2] = dvd(pa[2], mn);
                    }
                }
                if (Layer >= 1 && rule) {
                    float nw[3];
                    world_face_normal(P, l, nw);
                    friction_tangent(va, vb, nw, P.friction);
                }
                nv = make_float4(va[0], va[1], va[2], was_active ? nv.w : 0.0f);
                nf.w = was_active ? add(m_tot, mb) : mb;
                A.mv[id] = nv;
                A.f[id] = nf;
                touch_block(A, blin);
                const float mbdt = dvd(mb, dt);
                const float dF[3] = {mul(sub(va[0], vb[0]), mbdt), mul(sub(va[1], vb[1]), mbdt),
                                     mul(sub(va[2], vb[2]), mbdt)};
                vals[0] = dF[0]; vals[1] = dF[1]; vals[2] = dF[2];
                vals[3] = sub(mul(r[1], dF[2]), mul(r[2], dF[1]));
                vals[4] = sub(mul(r[2], dF[0]), mul(r[0], dF[2]));
                vals[5] = sub(mul(r[0], dF[1]), mul(r[1], dF[0]));
                vals[6] = 1;
            }
        }
    }
    cta64_add<7>(vals, acc);
}

// cand_prefix NULL: grid (max candidates, bodies), body = blockIdx.y.
// Otherwise a flat grid over the bodies' candidate bounds: body b owns CTAs
// [cand_prefix[b], cand_prefix[b+1]).
// Candidate block cb of body P (one CTA of 64 threads, one node each); the
// CTA's reaction is added to acc (7 doubles).
__device__ __forceinline__ void m1_candidate_block(const SceneTable& t, const M1Params& P, int64_t cb, int cur,
                                                   double* acc) {
    if (!P.active) return;
    const int64_t ncand = (int64_t)P.nbi * P.nbj * P.nbk;
    if (cb >= ncand) return;
    const SceneDev& S = t.scenes[P.scene];
    const GridDesc g = S.g;
    const GridAcc A = S.acc[cur];
    const int bk = P.bk0 + (int)(cb % P.nbk);
    const int bj = P.bj0 + (int)((cb / P.nbk) % P.nbj);
    const int bi = P.bi0 + (int)(cb / ((int64_t)P.nbk * P.nbj));
    const int64_t blin = g.block_of(bi, bj, bk);
    const int tt = threadIdx.x;

    double f0 = 0, f1 = 0, f2 = 0, t0 = 0, t1 = 0, t2 = 0, cnt = 0;
    const int ox = g.ox + 4 * bi, oy = g.oy + 4 * bj, oz = g.oz + 4 * bk;
    const float dx = g.dx;
    if (m1_block_visited(P, g, S.alloc, bi, bj, bk)) {
        const int li = tt >> 4, lj = (tt >> 2) & 3, lk = tt & 3;
        const int64_t id = g.node_of_block(blin, tt);
        float r[3], vb[3];
        if (m1_node_inside(P, dx, ox + li, oy + lj, oz + lk, r, vb)) {
            // the node's mass is its particle mass (mv.w) plus what couplers
            // added this step; the new total goes to f.w, mv.w keeps the
            // particle mass (the fused kernel's light-contribution rule reads it)
            float4 nv = A.mv[id];
            float4 nf = A.f[id];
            const float m_tot = node_total_mass(nv, nf);
            float va[3];
            if (!(m_tot >= 1e-9f)) {  // inactive (mass 0) or mass < 1e-9: body claims the node
                va[0] = vb[0]; va[1] = vb[1]; va[2] = vb[2];
                nv = make_float4(vb[0], vb[1], vb[2], 0.0f);
                nf.w = P.mb;
            } else {
                const float mn = add(m_tot, P.mb);
                const float pa[3] = {add(mul(nv.x, m_tot), mul(vb[0], P.mb)), add(mul(nv.y, m_tot), mul(vb[1], P.mb)),
                                     add(mul(nv.z, m_tot), mul(vb[2], P.mb))};
                if (fabsf(mn) < 1e-6f) {  // Vec3 division guard of the reference
                    va[0] = va[1] = va[2] = 0.0f;
                } else {
                    va[0] = dvd(pa[0], mn); va[1] = dvd(pa[1], mn); va[2] = dvd(pa[2], mn);
                }
                nv = make_float4(va[0], va[1], va[2], nv.w);
                nf.w = mn;
            }
            A.mv[id] = nv;
            A.f[id] = nf;
            touch_block(A, blin);
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
    if ((tt & 31) == 0) {
#pragma unroll
        for (int q = 0; q < 7; ++q) part[tt >> 5][q] = vals[q];
    }
    __syncthreads();
    if (tt < 7) {
        const double s = part[0][tt] + part[1][tt];
        if (s != 0.0) atomicAdd(acc + tt, s);
    }
}

__global__ void __launch_bounds__(64) k_m1(SceneTable t, const M1Params* params, int cur, double* acc_all,
                                           const int64_t* __restrict__ cand_prefix, int n_bodies) {
    int body = blockIdx.y;
    int64_t cb = blockIdx.x;
    if (cand_prefix) {
        int lo = 0, hi = n_bodies - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (cand_prefix[mid] <= (int64_t)blockIdx.x) lo = mid;
            else hi = mid - 1;
        }
        body = lo;
        cb = (int64_t)blockIdx.x - cand_prefix[lo];
    }
    m1_candidate_block(t, params[body], cb, cur, acc_all + 7 * body);
}

// One body, its parameters passed by value (no upload before the launch);
// the last CTA turns the sums into the reaction and zeroes them.
__global__ void __launch_bounds__(64) k_m1_one(SceneTable t, const __grid_constant__ M1Params P, int cur,
                                               double* acc, bm_reaction_t* out, uint32_t* counter) {
    m1_candidate_block(t, P, blockIdx.x, cur, acc);
    if (!last_cta(counter)) return;
    if (threadIdx.x == 0) {
        volatile double* a = acc;
        bm_reaction_t r;
        for (int q = 0; q < 3; ++q) {
            r.force[q] = (float)a[q];
            r.torque[q] = (float)a[3 + q];
        }
        r.nodes_inside = (int32_t)a[6];
        *out = r;
        for (int q = 0; q < 7; ++q) a[q] = 0.0;
    }
}

// The reactions from the FP64 sums, which are zeroed after reading so that
// the next call's sums start from zero.
__global__ void k_reaction_finalize(double* acc, int n, bm_reaction_t* out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    double* a = acc + 7 * b;
    bm_reaction_t r;
    for (int q = 0; q < 3; ++q) {
        r.force[q] = (float)a[q];
        r.torque[q] = (float)a[3 + q];
    }
    r.nodes_inside = (int32_t)a[6];
    out[b] = r;
    for (int q = 0; q < 7; ++q) a[q] = 0.0;
}

__global__ void k_body_prepare(SceneTable t, const BodyDev* bodies, int n, M1Params* params) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const BodyDev& B = bodies[b];
    m1_params(t.scenes[B.scene].g, B.state, B.dt, B.scene, params + b);
}

// integrator.h:19-57 for one body, with the body's weight applied as an
// external force (the research harness applies m*g before the coupler,
// bench_compare_all.cpp:97-98) and the coupler reaction added to it.
__global__ void k_body_integrate(BodyDev* bodies, int n, const double* acc) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    BodyDev& B = bodies[b];
    bm_collider_t& s = B.state;
    const float dt = B.dt;
    if (B.dynamic) {
        const double* a = acc + 7 * b;
        const float force[3] = {add(mul(B.gravity[0], s.mass), (float)a[0]), add(mul(B.gravity[1], s.mass), (float)a[1]),
                                add(mul(B.gravity[2], s.mass), (float)a[2])};
        const float torque[3] = {(float)a[3], (float)a[4], (float)a[5]};
        for (int q = 0; q < 3; ++q)
            s.linear_velocity[q] = add(s.linear_velocity[q], mul(mul(force[q], B.inv_mass), dt));
        for (int q = 0; q < 3; ++q) {
            const float it = add(add(mul(B.inv_inertia[3 * q], torque[0]), mul(B.inv_inertia[3 * q + 1], torque[1])),
                                 mul(B.inv_inertia[3 * q + 2], torque[2]));
            s.angular_velocity[q] = add(s.angular_velocity[q], mul(it, dt));
        }
    }
    for (int q = 0; q < 3; ++q) s.center[q] = add(s.center[q], mul(s.linear_velocity[q], dt));
    if (B.dynamic) {
        // q += 0.5 dt (0, w) * q, then normalise (quaternion.h: Hamilton product)
        const float qw = s.orientation[0], qx = s.orientation[1], qy = s.orientation[2], qz = s.orientation[3];
        const float wx = s.angular_velocity[0], wy = s.angular_velocity[1], wz = s.angular_velocity[2];
        const float dq[4] = {sub(sub(sub(mul(0.0f, qw), mul(wx, qx)), mul(wy, qy)), mul(wz, qz)),
                             sub(add(add(mul(0.0f, qx), mul(wx, qw)), mul(wy, qz)), mul(wz, qy)),
                             add(add(sub(mul(0.0f, qy), mul(wx, qz)), mul(wy, qw)), mul(wz, qx)),
                             add(sub(add(mul(0.0f, qz), mul(wx, qy)), mul(wy, qx)), mul(wz, qw))};
        const float h = mul(0.5f, dt);
        float q[4];
        for (int k = 0; k < 4; ++k) q[k] = add(s.orientation[k], mul(dq[k], h));
        const float nrm = sqrtf(add(add(add(mul(q[0], q[0]), mul(q[1], q[1])), mul(q[2], q[2])), mul(q[3], q[3])));
        if (nrm < 1e-6f) {
            s.orientation[0] = 1.0f; s.orientation[1] = s.orientation[2] = s.orientation[3] = 0.0f;
        } else {
            const float inv = dvd(1.0f, nrm);
            for (int k = 0; k < 4; ++k) s.orientation[k] = mul(q[k], inv);
        }
    }
}

__global__ void k_grid_to_dense(GridDesc g, GridAcc a, const uint8_t* alloc, float* vel, float* force, float* mass,
                                uint8_t* active, uint8_t* balloc) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.num_nodes()) return;  // the flat layout is the dense (i,j,k) order
    const float4 mv = a.mv[q];
    const float4 f = a.f[q];
    const float m = node_total_mass(mv, f);
    if (vel) { vel[3 * q] = mv.x; vel[3 * q + 1] = mv.y; vel[3 * q + 2] = mv.z; }
    if (force) { force[3 * q] = f.x; force[3 * q + 1] = f.y; force[3 * q + 2] = f.z; }
    if (mass) mass[q] = m;
    if (active) active[q] = m > 0.0f ? 1 : 0;
    if (balloc) balloc[q] = alloc[g.block_of_node(q)];
}

__global__ void k_dense_velocity_to_grid(GridDesc g, GridAcc a, const float* vel) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.num_nodes()) return;
    float4 mv = a.mv[q];
    mv.x = vel[3 * q]; mv.y = vel[3 * q + 1]; mv.z = vel[3 * q + 2];
    a.mv[q] = mv;
    if (mv.x != 0.0f || mv.y != 0.0f || mv.z != 0.0f || node_total_mass(mv, a.f[q]) != 0.0f)
        touch_block(a, g.block_of_node(q));
}

__global__ void k_seed(GridDesc g, GridAcc a, uint8_t* alloc, int64_t n, const int32_t* ijk, const float* vel,
                       const float* mass, uint32_t* status) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int64_t id = g.node(ijk[3 * q], ijk[3 * q + 1], ijk[3 * q + 2]);
    if (id < 0) {
        atomicOr(status, ERR_ESCAPE);
        return;
    }
    a.mv[id] = make_float4(vel[3 * q], vel[3 * q + 1], vel[3 * q + 2], mass[q]);
    a.f[id].w = 0.0f;  // the seeded mass is the node's whole mass
    const int64_t b = g.block_of_node(id);
    alloc[b] = 1;
    touch_block(a, b);
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

bool m1_prepare(const GridDesc& g, const bm_collider_t& b, float dt, int scene, M1Params* P) {
    return m1_params(g, b, dt, scene, P);
}

bool m45a_prepare(const GridDesc& g, const bm_collider_t& b, float dt, M1Params* P) {
    return m45a_params(g, b, dt, P);
}

void launch_m0(const SceneTable& t, const M1Params* d_param, int64_t candidates, int cur, float dt, double* d_acc,
               cudaStream_t st) {
    if (candidates <= 0) return;
    k_m0<<<(unsigned)candidates, 64, 0, st>>>(t, d_param, cur, dt, d_acc);
}

void launch_m45(const SceneTable& t, const M1Params* d_param, int64_t candidates, int cur, float dt,
                double* d_frac_sum, double* d_acc, int layer, cudaStream_t st) {
    if (candidates <= 0) return;
    k_m45a_sum<<<(unsigned)candidates, 64, 0, st>>>(t, d_param, cur, d_frac_sum);
    if (layer == 2) k_m45<2><<<(unsigned)candidates, 64, 0, st>>>(t, d_param, cur, dt, d_frac_sum, d_acc);
    else if (layer == 1) k_m45<1><<<(unsigned)candidates, 64, 0, st>>>(t, d_param, cur, dt, d_frac_sum, d_acc);
    else k_m45<0><<<(unsigned)candidates, 64, 0, st>>>(t, d_param, cur, dt, d_frac_sum, d_acc);
}

int64_t m1_max_candidates(const GridDesc& g, const float he[3]) {
    // each AABB half side is sum_j |R_aj| h_j <= |h| (a row of R has unit
    // length); the candidate nodes span at most 2 |h| / dx + 4 (rounding and
    // one node of slack each side), i.e. span / 4 + 2 blocks per axis
    const double h = std::sqrt((double)he[0] * he[0] + (double)he[1] * he[1] + (double)he[2] * he[2]) * (1.0 + 1e-6);
    const double nodes = 2.0 * h / g.dx + 4.0;
    const int64_t per = (int64_t)std::ceil(nodes / 4.0) + 2;
    const int64_t a = std::min<int64_t>(per, g.nbx), b = std::min<int64_t>(per, g.nby), c = std::min<int64_t>(per, g.nbz);
    return std::max<int64_t>(1, a * b * c);
}

void launch_m1(const SceneTable& t, const M1Params* d_params, int n_bodies, int64_t max_candidates, int cur,
               double* d_acc, cudaStream_t st) {
    if (n_bodies <= 0 || max_candidates <= 0) return;
    k_m1<<<dim3((unsigned)max_candidates, (unsigned)n_bodies), 64, 0, st>>>(t, d_params, cur, d_acc, nullptr,
                                                                             n_bodies);
}

bool launch_m1_one(const SceneTable& t, const M1Params& P, int cur, double* d_acc, bm_reaction_t* d_out,
                   uint32_t* counter, cudaStream_t st) {
    const int64_t cand = (int64_t)P.nbi * P.nbj * P.nbk;
    if (!P.active || cand <= 0) return false;
    k_m1_one<<<(unsigned)cand, 64, 0, st>>>(t, P, cur, d_acc, d_out, counter);
    return true;
}

void launch_m1_flat(const SceneTable& t, const M1Params* d_params, int n_bodies, const int64_t* d_cand_prefix,
                    int64_t total_candidates, int cur, double* d_acc, cudaStream_t st) {
    if (n_bodies <= 0 || total_candidates <= 0) return;
    k_m1<<<(unsigned)total_candidates, 64, 0, st>>>(t, d_params, cur, d_acc, d_cand_prefix, n_bodies);
}

cudaError_t load_m1_kernels() {
    // under CUDA's lazy module loading a kernel's code is loaded on its first
    // use, and querying its attributes is such a use
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, k_m1);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_reaction_finalize);
    return e;
}

void launch_reaction_finalize(double* d_acc, int n_bodies, bm_reaction_t* d_out, cudaStream_t st) {
    if (n_bodies <= 0) return;
    k_reaction_finalize<<<nblk(n_bodies, 64), 64, 0, st>>>(d_acc, n_bodies, d_out);
}

// The body array of the served form after its scene set changed: body k
// takes its pose and velocities from old[src[k]] (a scene that stays) and
// everything else from staged[k] (built on the host; its state is the initial
// one for a new scene, src[k] < 0).
__global__ void k_body_remap(const BodyDev* __restrict__ old, BodyDev* __restrict__ out,
                             const BodyDev* __restrict__ staged, const int32_t* __restrict__ src, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    BodyDev B = staged[k];
    if (src[k] >= 0) B.state = old[src[k]].state;
    out[k] = B;
}

void launch_body_remap(const BodyDev* d_old, BodyDev* d_out, const BodyDev* d_staged, const int32_t* d_src, int n,
                       cudaStream_t st) {
    if (n <= 0) return;
    k_body_remap<<<nblk(n, 64), 64, 0, st>>>(d_old, d_out, d_staged, d_src, n);
}

void launch_body_prepare(const SceneTable& t, const BodyDev* d_bodies, int n_bodies, M1Params* d_params,
                         cudaStream_t st) {
    if (n_bodies <= 0) return;
    k_body_prepare<<<nblk(n_bodies, 64), 64, 0, st>>>(t, d_bodies, n_bodies, d_params);
}

void launch_body_integrate(BodyDev* d_bodies, int n_bodies, const double* d_acc, cudaStream_t st) {
    if (n_bodies <= 0) return;
    k_body_integrate<<<nblk(n_bodies, 64), 64, 0, st>>>(d_bodies, n_bodies, d_acc);
}

void launch_grid_to_dense(const GridDesc& g, const GridAcc& a, const uint8_t* alloc, float* vel, float* force,
                          float* mass, uint8_t* active, uint8_t* balloc, cudaStream_t st) {
    k_grid_to_dense<<<nblk(g.num_nodes(), 256), 256, 0, st>>>(g, a, alloc, vel, force, mass, active, balloc);
}

void launch_dense_velocity_to_grid(const GridDesc& g, const GridAcc& a, const float* vel, cudaStream_t st) {
    k_dense_velocity_to_grid<<<nblk(g.num_nodes(), 256), 256, 0, st>>>(g, a, vel);
}

void launch_seed_grid(const GridDesc& g, const GridAcc& a, uint8_t* alloc, int64_t n, const int32_t* ijk,
                      const float* vel, const float* mass, uint32_t* d_status, cudaStream_t st) {
    if (n <= 0) return;
    k_seed<<<nblk(n, 256), 256, 0, st>>>(g, a, alloc, n, ijk, vel, mass, d_status);
}

}  // namespace bm
