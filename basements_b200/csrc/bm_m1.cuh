// bm_m1.cuh — the per-node test of the M1 PIC-rigid coupler, shared by the
// coupler kernel (bm_m1.cu) and its adjoint (bm_adjoint.cu).
//
// Reference (2nugu/basements):
//   MPMRigidCouplerPIC::apply  include/basements/physics/coupling/mpm_rigid_coupler_pic.h:119-160
//   shape_inside               include/basements/physics/coupling/mpm_rigid_coupler.h:90-103
//
// Node arithmetic uses explicit round-to-nearest operations (never contracted
// into FMA) so that the inside test and the body velocity at the node match
// the reference bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "bm_internal.h"

namespace bm {
namespace rn {

// Round-to-nearest float arithmetic that is never contracted into FMA: the
// intrinsics on the device, plain operators on the host (host code is built
// with -ffp-contract=off).
__host__ __device__ __forceinline__ float mul(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ float add(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ __forceinline__ float sub(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ __forceinline__ float dvd(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}

}  // namespace rn

// Block (bi, bj, bk) (box-relative) is visited by the coupler: allocated, and
// its node-centre span overlaps the body's AABB (pic.h:122-131).
__device__ __forceinline__ bool m1_block_visited(const M1Params& P, const GridDesc& g, const uint8_t* alloc, int bi,
                                                 int bj, int bk) {
    using namespace rn;
    if (alloc[g.block_of(bi, bj, bk)] == 0) return false;
    const int ox = g.ox + 4 * bi, oy = g.oy + 4 * bj, oz = g.oz + 4 * bk;
    const float dx = g.dx;
    const float blo0 = mul((float)ox + 0.5f, dx), bhi0 = mul((float)(ox + 3) + 0.5f, dx);
    const float blo1 = mul((float)oy + 0.5f, dx), bhi1 = mul((float)(oy + 3) + 0.5f, dx);
    const float blo2 = mul((float)oz + 0.5f, dx), bhi2 = mul((float)(oz + 3) + 0.5f, dx);
    if (bhi0 < P.lo[0] || blo0 > P.hi[0]) return false;
    if (bhi1 < P.lo[1] || blo1 > P.hi[1]) return false;
    if (bhi2 < P.lo[2] || blo2 > P.hi[2]) return false;
    return true;
}

// Node (i, j, k) (absolute indices) is inside the body's shape; on true, r is
// the node centre relative to the body centre and vb the body velocity there
// (v + w x r).
__device__ __forceinline__ bool m1_node_inside(const M1Params& P, float dx, int i, int j, int k, float r[3],
                                               float vb[3]) {
    using namespace rn;
    const float xn[3] = {mul((float)i + 0.5f, dx), mul((float)j + 0.5f, dx), mul((float)k + 0.5f, dx)};
    r[0] = sub(xn[0], P.c[0]);
    r[1] = sub(xn[1], P.c[1]);
    r[2] = sub(xn[2], P.c[2]);
    float l[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) l[a] = add(add(mul(P.R[a], r[0]), mul(P.R[3 + a], r[1])), mul(P.R[6 + a], r[2]));
    bool inside;
    if (P.shape == 1) {
        const float r2 = add(mul(l[0], l[0]), mul(l[2], l[2]));
        inside = fabsf(l[1]) <= P.he[1] && r2 <= mul(P.he[0], P.he[0]);
    } else {
        inside = fabsf(l[0]) <= P.he[0] && fabsf(l[1]) <= P.he[1] && fabsf(l[2]) <= P.he[2];
    }
    if (inside) {
        vb[0] = add(P.vl[0], sub(mul(P.w[1], r[2]), mul(P.w[2], r[1])));
        vb[1] = add(P.vl[1], sub(mul(P.w[2], r[0]), mul(P.w[0], r[2])));
        vb[2] = add(P.vl[2], sub(mul(P.w[0], r[1]), mul(P.w[1], r[0])));
    }
    return inside;
}

// The node (i, j, k) in the body frame: r its centre relative to the body
// centre, l = R^T r; true when it is inside the shape (the test of
// m1_node_inside, for couplers that also need l).
__device__ __forceinline__ bool coupler_node_local(const M1Params& P, float dx, int i, int j, int k, float r[3],
                                                   float l[3]) {
    using namespace rn;
    const float xn[3] = {mul((float)i + 0.5f, dx), mul((float)j + 0.5f, dx), mul((float)k + 0.5f, dx)};
    r[0] = sub(xn[0], P.c[0]);
    r[1] = sub(xn[1], P.c[1]);
    r[2] = sub(xn[2], P.c[2]);
#pragma unroll
    for (int a = 0; a < 3; ++a) l[a] = add(add(mul(P.R[a], r[0]), mul(P.R[3 + a], r[1])), mul(P.R[6 + a], r[2]));
    if (P.shape == 1) {
        const float r2 = add(mul(l[0], l[0]), mul(l[2], l[2]));
        return fabsf(l[1]) <= P.he[1] && r2 <= mul(P.he[0], P.he[0]);
    }
    return fabsf(l[0]) <= P.he[0] && fabsf(l[1]) <= P.he[1] && fabsf(l[2]) <= P.he[2];
}

// shape_cell_overlap_fraction (mpm_rigid_coupler.h:139-164): 1 at the centre,
// 0 at the surface; box (1-|x|/hx)(1-|y|/hy)(1-|z|/hz), cylinder
// (1-|y|/L)(1-r/R), each factor clamped to [0, 1].
__device__ __forceinline__ float coupler_overlap_fraction(const M1Params& P, const float l[3]) {
    using namespace rn;
    auto clamp01 = [](float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); };
    if (P.shape == 1) {
        const float r = __fsqrt_rn(add(mul(l[0], l[0]), mul(l[2], l[2])));
        const float axial = sub(1.0f, dvd(fabsf(l[1]), fmaxf(P.he[1], 1e-9f)));
        const float radial = sub(1.0f, dvd(r, fmaxf(P.he[0], 1e-9f)));
        return mul(clamp01(axial), clamp01(radial));
    }
    const float ux = clamp01(sub(1.0f, dvd(fabsf(l[0]), fmaxf(P.he[0], 1e-9f))));
    const float uy = clamp01(sub(1.0f, dvd(fabsf(l[1]), fmaxf(P.he[1], 1e-9f))));
    const float uz = clamp01(sub(1.0f, dvd(fabsf(l[2]), fmaxf(P.he[2], 1e-9f))));
    return mul(mul(ux, uy), uz);
}

}  // namespace bm
