// bm_adjoint.cu — the differentiable run: a tape of the plain split step and
// its hand-written adjoint kernels.
//
// The reference declares a tape (AutodiffTape, mpm_autodiff_tape.h:37-92,
// passed to MPMSolver::step(dt, tape*), mpm_solver.h:71-87) that records
// nothing; there is no reference gradient. This file gives the split step
// P2G -> update_grid -> M1 -> G2P (the same kernels as bm_solver_p2g /
// _grid_update / bm_coupler_m1_apply / _g2p) a reverse pass:
//
//   forward:  from the solver's particle state, n steps; the particle state
//             (x, v, F, C) is saved every K steps (checkpoints).
//   backward: for each K-step segment, last first: restore its checkpoint,
//             re-run the segment saving every step's state, then for each step
//             in reverse recompute its grid (P2G, update, M1) and run
//               k_adj_g2p   G2P adjoint: gathers the post-coupler velocities,
//                           rebuilds v, C, F_trial, runs the DP/SVD adjoint,
//                           scatters dL/dv_node and forms dL/dx through the
//                           B-spline weights;
//               k_adj_grid  per node: M1 blend adjoint (and dL/d body
//                           velocity), floor boundary and update_grid adjoint;
//               k_adj_p2g   P2G adjoint: gathers dL/d(momentum, mass, force),
//                           forms dL/dv, dL/dC, dL/dx and dL/dF through the
//                           Hencky stress adjoint.
//
// The body follows a piecewise-linear path through waypoints; its velocity
// on each step is the slope of the path segment, so dL/d waypoint is the sum
// of dL/d(body velocity) over the steps of the two adjacent segments.
// The inside test of the coupler and the mass thresholds of update_grid are
// piecewise constant: their derivative is zero almost everywhere, as here.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bm_adjoint.cuh"
#include "bm_m1.cuh"
#include "bm_solver_impl.h"

using namespace bm;
using namespace bm::sol;

namespace {

constexpr int kStatePlanes = 24;  // x, v, F, C (planes 0..23 of the store)
constexpr int kAdjThreads = 128;

// What the adjoint kernels read and write for one step.
struct AdjStep {
    const float* st;      // state of step n: kStatePlanes planes of `cap`
    const float* mass;    // store plane P_M
    const float* vol;     // store plane P_V0
    int64_t cap, n;
    GridDesc g;
    const float4* gv;      // node velocities after update + coupler
    const float4* pre_mv;  // P2G output: (momentum, mass)
    const float4* pre_f;   // P2G output: (force, 0)
    float4* adj_gv;        // dL/d(node velocity after the coupler)
    float4* adj_pm;        // dL/d(momentum, mass)
    float4* adj_f;         // dL/d(force)
    const float* adj_in;   // dL/d(state of step n+1)
    float* adj_out;        // dL/d(state of step n)
    float mu, lambda, nak, dt;
    float gx, gy, gz, floor_friction;
    const uint8_t* alloc;  // per block: allocated (the coupler visits these only)
    const M1Params* body;  // NULL: no body
    double* body_adj;      // 6 doubles: dL/d(linear velocity), dL/d(angular velocity)
};

__device__ __forceinline__ float ld(const float* base, int64_t cap, int plane, int64_t p) {
    return base[(int64_t)plane * cap + p];
}

// ---- G2P adjoint ------------------------------------------------------------------

__global__ void __launch_bounds__(kAdjThreads) k_adj_g2p(AdjStep A) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n) return;
    const GridDesc g = A.g;
    const float dt = A.dt;
    float x[3], F[9];
#pragma unroll
    for (int a = 0; a < 3; ++a) x[a] = ld(A.st, A.cap, P_X + a, p);
#pragma unroll
    for (int q = 0; q < 9; ++q) F[q] = ld(A.st, A.cap, P_F + q, p);
    float fx[3], wgt[3][3], dwg[3][3];
    int base[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        fx[a] = x[a] * g.inv_dx - 0.5f;
        base[a] = (int)floorf(fx[a]);
        bspline_weights(fx[a] - (float)base[a], wgt[a]);
        adj::bspline_dweights(fx[a] - (float)base[a], dwg[a]);
    }
    const float cs = 4.0f * g.inv_dx * g.inv_dx;
    // forward gather (the arithmetic of k_g2p)
    float v[3] = {0.0f, 0.0f, 0.0f};
    float Cm[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) Cm[q] = 0.0f;
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
                if (id < 0) continue;
                const float4 nv = A.gv[id];
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
    const float ynew = x[1] + v[1] * dt;
    const bool clamped = ynew < 0.0f;
    // incoming adjoints of x, v, F, C after the step
    float xb[3], vb[3], Fnb[9], Cb[9];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        xb[a] = ld(A.adj_in, A.cap, P_X + a, p);
        vb[a] = ld(A.adj_in, A.cap, P_V + a, p);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        Fnb[q] = ld(A.adj_in, A.cap, P_F + q, p);
        Cb[q] = ld(A.adj_in, A.cap, P_C + q, p);
    }
    if (clamped) {  // x.y = 0 and v.y = 0 after the floor clamp
        xb[1] = 0.0f;
        vb[1] = 0.0f;
    }
    // x_new = x + v dt
#pragma unroll
    for (int a = 0; a < 3; ++a) vb[a] += dt * xb[a];
    // F_new = DP((I + C dt) F), F_tr formed in double for the DP/SVD adjoint
    double Am[9], Ft[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) Am[q] = ((q % 4 == 0) ? 1.0 : 0.0) + (double)Cm[q] * dt;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            Ft[3 * i + j] = Am[3 * i] * F[j] + Am[3 * i + 1] * F[3 + j] + Am[3 * i + 2] * F[6 + j];
    double Ftb[9];
    adj::dp_project_adjoint(Ft, A.nak, Fnb, Ftb);
    // C_bar += dt Ft_bar F^T ; F_bar = A^T Ft_bar
    float Fb[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Cb[3 * i + j] += (float)(dt * (Ftb[3 * i] * F[3 * j] + Ftb[3 * i + 1] * F[3 * j + 1] +
                                           Ftb[3 * i + 2] * F[3 * j + 2]));
            Fb[3 * i + j] = (float)(Am[i] * Ftb[j] + Am[3 + i] * Ftb[3 + j] + Am[6 + i] * Ftb[6 + j]);
        }
    // scatter to the nodes, and the position adjoint through the weights
    float xo[3] = {xb[0], xb[1], xb[2]};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float w = wgt[0][i] * wgt[1][j] * wgt[2][k];
                const int ni = base[0] + i, nj = base[1] + j, nk = base[2] + k;
                const int64_t id = g.node(ni, nj, nk);
                if (id < 0) continue;
                const float gw[3] = {dwg[0][i] * wgt[1][j] * wgt[2][k] * g.inv_dx,
                                     wgt[0][i] * dwg[1][j] * wgt[2][k] * g.inv_dx,
                                     wgt[0][i] * wgt[1][j] * dwg[2][k] * g.inv_dx};
                const float d[3] = {((float)ni - fx[0] - 0.5f) * g.dx, ((float)nj - fx[1] - 0.5f) * g.dx,
                                    ((float)nk - fx[2] - 0.5f) * g.dx};
                const float4 nv = A.gv[id];
                const float vi[3] = {nv.x, nv.y, nv.z};
                float Cd[3], CTv[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    Cd[a] = Cb[3 * a] * d[0] + Cb[3 * a + 1] * d[1] + Cb[3 * a + 2] * d[2];
                    CTv[a] = Cb[a] * vi[0] + Cb[3 + a] * vi[1] + Cb[6 + a] * vi[2];
                }
                if (w != 0.0f)
                    atomicAdd(A.adj_gv + id, make_float4(w * (vb[0] + cs * Cd[0]), w * (vb[1] + cs * Cd[1]),
                                                         w * (vb[2] + cs * Cd[2]), 0.0f));
                // v = sum w v_i, C = cs sum w v_i d^T, d = x_i - x
                const float sdot = (vi[0] * vb[0] + vi[1] * vb[1] + vi[2] * vb[2]) +
                                   cs * (vi[0] * Cd[0] + vi[1] * Cd[1] + vi[2] * Cd[2]);
#pragma unroll
                for (int a = 0; a < 3; ++a) xo[a] += gw[a] * sdot - w * cs * CTv[a];
            }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        A.adj_out[(int64_t)(P_X + a) * A.cap + p] = xo[a];
        A.adj_out[(int64_t)(P_V + a) * A.cap + p] = 0.0f;
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        A.adj_out[(int64_t)(P_F + q) * A.cap + p] = Fb[q];
        A.adj_out[(int64_t)(P_C + q) * A.cap + p] = 0.0f;
    }
}

// ---- grid adjoint: coupler, floor boundary, update_grid --------------------------

__global__ void __launch_bounds__(256) k_adj_grid(AdjStep A) {
    const GridDesc g = A.g;
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double bl[6] = {0, 0, 0, 0, 0, 0};
    if (id < g.num_nodes()) {
        const float4 pm = A.pre_mv[id];
        const float4 f = A.pre_f[id];
        const float4 gb4 = A.adj_gv[id];
        float gv[3] = {gb4.x, gb4.y, gb4.z};  // becomes dL/d(velocity before the coupler)
        const float m = pm.w;
        const float dt = A.dt;
        const int64_t ez = g.ez(), ey = g.ey();
        const int rk = (int)(id % ez), rj = (int)((id / ez) % ey), ri = (int)(id / (ez * ey));
        const int ni = g.ox + ri, nj = g.oy + rj, nk = g.oz + rk;
        // forward update_grid (the arithmetic of k_grid_update, unfolded)
        const bool live = m > 1e-6f;
        float v[3], vt0 = 0.0f, vt2 = 0.0f;
        bool bc = false;
        float mag = 0.0f, budget = 0.0f;
        if (live) {
            v[0] = (pm.x + f.x * dt) / m;
            v[1] = (pm.y + f.y * dt) / m;
            v[2] = (pm.z + f.z * dt) / m;
            v[0] = v[0] + A.gx * dt;
            v[1] = v[1] + A.gy * dt;
            v[2] = v[2] + A.gz * dt;
            const float node_y = ((float)nj + 0.5f) * g.dx;
            if (node_y < g.dx && v[1] < 0.0f) {
                bc = true;
                const float vn = -v[1];
                v[1] = 0.0f;
                vt0 = v[0];
                vt2 = v[2];
                mag = sqrtf(v[0] * v[0] + v[2] * v[2]);
                budget = A.floor_friction * vn;
                if (mag > 1e-12f) {
                    const float sc = smax(0.0f, (mag - budget) / mag);
                    v[0] = v[0] * sc;
                    v[2] = v[2] * sc;
                }
            }
        } else {
            v[0] = pm.x; v[1] = pm.y; v[2] = pm.z;  // mass <= 1e-6: momentum kept, no force, no gravity
        }
        float mbar = 0.0f;
        // coupler on this node (k_m1's visit and inside tests)
        if (A.body) {
            const M1Params& P = *A.body;
            const int bi = ri >> 2, bj = rj >> 2, bk = rk >> 2;
            float r[3], vb[3];
            if (P.active && bi >= P.bi0 && bi < P.bi0 + P.nbi && bj >= P.bj0 && bj < P.bj0 + P.nbj &&
                bk >= P.bk0 && bk < P.bk0 + P.nbk && m1_block_visited(P, g, A.alloc, bi, bj, bk) &&
                m1_node_inside(P, g.dx, ni, nj, nk, r, vb)) {
                float gbody[3] = {0.0f, 0.0f, 0.0f};
                if (!(m >= 1e-9f)) {  // v' = v_body
                    gbody[0] = gv[0]; gbody[1] = gv[1]; gbody[2] = gv[2];
                    gv[0] = gv[1] = gv[2] = 0.0f;
                } else {
                    const float mn = m + P.mb;
                    if (fabsf(mn) < 1e-6f) {  // v' = 0
                        gv[0] = gv[1] = gv[2] = 0.0f;
                    } else {
                        // v' = (m v + mb v_body) / (m + mb)
                        float vp[3];
#pragma unroll
                        for (int a = 0; a < 3; ++a) vp[a] = (m * v[a] + P.mb * vb[a]) / mn;
                        mbar += ((gv[0] * (v[0] - vp[0]) + gv[1] * (v[1] - vp[1])) + gv[2] * (v[2] - vp[2])) / mn;
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            gbody[a] = gv[a] * (P.mb / mn);
                            gv[a] = gv[a] * (m / mn);
                        }
                    }
                }
                bl[0] = gbody[0]; bl[1] = gbody[1]; bl[2] = gbody[2];
                // v_body = v + w x r: dL/dw = r x dL/dv_body
                bl[3] = (double)r[1] * gbody[2] - (double)r[2] * gbody[1];
                bl[4] = (double)r[2] * gbody[0] - (double)r[0] * gbody[2];
                bl[5] = (double)r[0] * gbody[1] - (double)r[1] * gbody[0];
            }
        }
        // floor boundary: v_y' = 0, v_t' = v_t max(0, 1 - mu |v_y| / |v_t|)
        // (v_t kept as is when |v_t| <= 1e-12). At rest (v_t = 0 and a
        // positive friction budget) every neighbouring state sticks, so the
        // derivative there is the sticking one (zero), not the identity.
        if (bc) {
            const float g0 = gv[0], g2 = gv[2];
            float gy = 0.0f;
            if (mag > budget) {
                if (mag > 1e-12f) {
                    const float t0 = vt0 / mag, t2 = vt2 / mag;
                    const float tg = t0 * g0 + t2 * g2;
                    const float k = budget / mag;
                    gv[0] = g0 - k * (g0 - t0 * tg);
                    gv[2] = g2 - k * (g2 - t2 * tg);
                    gy = A.floor_friction * tg;
                }
            } else {
                gv[0] = 0.0f;
                gv[2] = 0.0f;
            }
            gv[1] = gy;
        }
        // update_grid: v = (p + f dt) / m + g dt
        float4 apm, af;
        if (live) {
            const float im = 1.0f / m;
            const float pf[3] = {pm.x + f.x * dt, pm.y + f.y * dt, pm.z + f.z * dt};
            mbar -= ((gv[0] * pf[0] + gv[1] * pf[1]) + gv[2] * pf[2]) * im * im;
            apm = make_float4(gv[0] * im, gv[1] * im, gv[2] * im, mbar);
            af = make_float4(gv[0] * im * dt, gv[1] * im * dt, gv[2] * im * dt, 0.0f);
        } else {
            apm = make_float4(gv[0], gv[1], gv[2], mbar);
            af = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        A.adj_pm[id] = apm;
        A.adj_f[id] = af;
    }
    if (!A.body) return;  // uniform across the block: A is a kernel parameter
    // dL/d body velocity: warp shuffle, then one double atomic per warp
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double x = bl[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0 && x != 0.0) atomicAdd(A.body_adj + q, x);
    }
}

// ---- P2G adjoint ------------------------------------------------------------------

__global__ void __launch_bounds__(kAdjThreads) k_adj_p2g(AdjStep A) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n) return;
    const GridDesc g = A.g;
    float x[3], v[3], F[9], Cm[9];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        x[a] = ld(A.st, A.cap, P_X + a, p);
        v[a] = ld(A.st, A.cap, P_V + a, p);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        F[q] = ld(A.st, A.cap, P_F + q, p);
        Cm[q] = ld(A.st, A.cap, P_C + q, p);
    }
    const float m = A.mass[p];
    const float vol = A.vol[p];
    float fx[3], wgt[3][3], dwg[3][3];
    int base[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        fx[a] = x[a] * g.inv_dx - 0.5f;
        base[a] = (int)floorf(fx[a]);
        bspline_weights(fx[a] - (float)base[a], wgt[a]);
        adj::bspline_dweights(fx[a] - (float)base[a], dwg[a]);
    }
    float tau[9];
    hencky_tau(F, A.mu, A.lambda, tau);
    const float ff = -4.0f * g.inv_dx * g.inv_dx * vol;
    float sk[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) sk[q] = tau[q] * ff;
    float vbar[3] = {0.0f, 0.0f, 0.0f}, xbar[3] = {0.0f, 0.0f, 0.0f};
    float Cbar[9], skbar[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        Cbar[q] = 0.0f;
        skbar[q] = 0.0f;
    }
    // momentum_i += w m (v + C d), mass_i += w m, force_i += w sk d, d = x_i - x
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
                if (id < 0) continue;
                const float4 apm = A.adj_pm[id];
                const float4 af = A.adj_f[id];
                const float pb[3] = {apm.x, apm.y, apm.z}, fb[3] = {af.x, af.y, af.z};
                const float d[3] = {((float)ni - fx[0] - 0.5f) * g.dx, ((float)nj - fx[1] - 0.5f) * g.dx,
                                    ((float)nk - fx[2] - 0.5f) * g.dx};
                const float gw[3] = {dwg[0][i] * wgt[1][j] * wgt[2][k] * g.inv_dx,
                                     wgt[0][i] * dwg[1][j] * wgt[2][k] * g.inv_dx,
                                     wgt[0][i] * wgt[1][j] * dwg[2][k] * g.inv_dx};
                float Cd[3], skd[3], CTp[3], skTf[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    Cd[a] = Cm[3 * a] * d[0] + Cm[3 * a + 1] * d[1] + Cm[3 * a + 2] * d[2];
                    skd[a] = sk[3 * a] * d[0] + sk[3 * a + 1] * d[1] + sk[3 * a + 2] * d[2];
                    CTp[a] = Cm[a] * pb[0] + Cm[3 + a] * pb[1] + Cm[6 + a] * pb[2];
                    skTf[a] = sk[a] * fb[0] + sk[3 + a] * fb[1] + sk[6 + a] * fb[2];
                }
                const float wm = w * m;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    vbar[a] += wm * pb[a];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        Cbar[3 * a + c] += wm * pb[a] * d[c];
                        skbar[3 * a + c] += w * fb[a] * d[c];
                    }
                }
                const float sdot = m * apm.w +
                                   m * ((pb[0] * (v[0] + Cd[0]) + pb[1] * (v[1] + Cd[1])) + pb[2] * (v[2] + Cd[2])) +
                                   ((fb[0] * skd[0] + fb[1] * skd[1]) + fb[2] * skd[2]);
#pragma unroll
                for (int a = 0; a < 3; ++a) xbar[a] += gw[a] * sdot - w * (m * CTp[a] + skTf[a]);
            }
    float taub[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) taub[q] = ff * skbar[q];
    float Fb[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) Fb[q] = 0.0f;
    adj::hencky_tau_adjoint(F, A.mu, A.lambda, taub, Fb);
    float* o = A.adj_out;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        o[(int64_t)(P_X + a) * A.cap + p] += xbar[a];
        o[(int64_t)(P_V + a) * A.cap + p] = vbar[a];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        o[(int64_t)(P_F + q) * A.cap + p] += Fb[q];
        o[(int64_t)(P_C + q) * A.cap + p] = Cbar[q];
    }
}

int64_t nblk(int64_t n, int t) { return (n + t - 1) / t; }

}  // namespace

// ---- the tape -----------------------------------------------------------------------

struct bm_tape {
    bm_solver* s = nullptr;
    int device = 0;  // the solver's device (destroy may run after the solver is gone)
    int32_t K = 20;
    float dt = 0.0f;
    int32_t n_steps = 0;
    bool has_body = false;
    bm_collider_t body{};
    std::vector<double> wp;  // n_wp x 3
    int32_t n_wp = 0;
    bool recorded = false;
    int64_t cap = 0, n = 0, nodes = 0;
    int n_ckpt = 0;            // states at steps 0, K, 2K, ... plus the final state
    float* d_ckpt = nullptr;   // n_ckpt x kStatePlanes x cap
    float* d_seg = nullptr;    // K x kStatePlanes x cap
    float* d_adj[2] = {nullptr, nullptr};
    float4* d_pre = nullptr;   // 2 x nodes: P2G (momentum, mass), (force, 0)
    float4* d_gadj = nullptr;  // 3 x nodes: adj_gv, adj_pm, adj_f
    double* d_body_adj = nullptr;  // n_steps x 6
    float* d_rows = nullptr;       // n x 9 (add order)
    int32_t* d_inv = nullptr;      // store slot of each add-order index
    std::vector<double> h_body_adj;
};

namespace {

void tape_free(bm_tape* t) {
    cudaFree(t->d_ckpt);
    cudaFree(t->d_seg);
    cudaFree(t->d_adj[0]);
    cudaFree(t->d_adj[1]);
    cudaFree(t->d_pre);
    cudaFree(t->d_gadj);
    cudaFree(t->d_body_adj);
    cudaFree(t->d_rows);
    cudaFree(t->d_inv);
    t->d_ckpt = t->d_seg = t->d_adj[0] = t->d_adj[1] = t->d_rows = nullptr;
    t->d_pre = t->d_gadj = nullptr;
    t->d_body_adj = nullptr;
    t->d_inv = nullptr;
}

template <typename T>
bm_status_t dalloc(T** p, size_t count) {
    if (cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        set_last_error("out of device memory for the tape");
        return BM_ERR_OUT_OF_MEMORY;
    }
    return BM_OK;
}

// Waypoint segment of step n and its length (the body path spans n_steps * dt).
void path_segment(const bm_tape* t, int n, int* k, double* seg, double* tn) {
    const double T = (double)t->n_steps * (double)t->dt;
    *seg = T / (double)(t->n_wp - 1);
    *tn = (double)n * (double)t->dt;
    const int kk = (int)std::floor(*tn / *seg);
    *k = std::min(std::max(kk, 0), t->n_wp - 2);
}

bm_collider_t body_at(const bm_tape* t, int n) {
    bm_collider_t b = t->body;
    int k;
    double seg, tn;
    path_segment(t, n, &k, &seg, &tn);
    for (int a = 0; a < 3; ++a) {
        const double w0 = t->wp[3 * k + a], w1 = t->wp[3 * (k + 1) + a];
        const double v = (w1 - w0) / seg;
        b.linear_velocity[a] = (float)v;
        b.center[a] = (float)(w0 + (tn - (double)k * seg) * v);
    }
    return b;
}

ParticleSoA& store_of(bm_tape* t) { return t->s->sc().dev.store[t->s->w.sel]; }

bm_status_t copy_state(bm_tape* t, float* dst, const float* src) {
    BM_CHECK_CUDA(cudaMemcpyAsync(dst, src, sizeof(float) * kStatePlanes * t->cap, cudaMemcpyDeviceToDevice,
                                  t->s->w.stream));
    return BM_OK;
}

float* ckpt(bm_tape* t, int i) { return t->d_ckpt + (int64_t)i * kStatePlanes * t->cap; }
float* seg_state(bm_tape* t, int j) { return t->d_seg + (int64_t)j * kStatePlanes * t->cap; }

// One split step of the recorded run.
bm_status_t run_step(bm_tape* t, int n) {
    bm_solver* s = t->s;
    bm_status_t st = do_p2g(s);
    if (st == BM_OK) st = do_grid_update(s, t->dt);
    if (st == BM_OK && t->has_body) {
        const bm_collider_t b = body_at(t, n);
        st = do_m1(s, 1, &b, t->dt);
    }
    if (st == BM_OK) st = do_g2p(s, t->dt);
    return st;
}

// The state fields of a particles view with their first plane and width.
struct Field {
    int plane, width;
};
constexpr Field kFields[4] = {{P_X, 3}, {P_V, 3}, {P_F, 9}, {P_C, 9}};
float* view_field(const bm_particles_view_t* v, int f) {
    if (!v) return nullptr;
    return f == 0 ? v->position : f == 1 ? v->velocity : f == 2 ? v->F : v->C;
}

bm_status_t backward(bm_tape* t, const bm_particles_view_t* dfinal, float* dL_dwaypoints,
                     const bm_particles_view_t* dinitial) {
    if (!t->recorded) {
        set_last_error("bm_adjoint_backward needs a recorded bm_tape_forward");
        return BM_ERR_STATE;
    }
    bm_solver* s = t->s;
    bm_status_t st = prepare(s);
    if (st != BM_OK) return st;
    ParticleSoA& ps = store_of(t);
    if (ps.n != t->n || ps.cap != t->cap || s->sc().dev.g.num_nodes() != t->nodes) {
        set_last_error("the solver changed since bm_tape_forward");
        return BM_ERR_STATE;
    }
    cudaStream_t stream = s->w.stream;
    const size_t state = (size_t)kStatePlanes * t->cap;
    int cur = 0;
    BM_CHECK_CUDA(cudaMemsetAsync(t->d_adj[cur], 0, sizeof(float) * state, stream));
    BM_CHECK_CUDA(cudaMemsetAsync(t->d_body_adj, 0, sizeof(double) * 6 * t->n_steps, stream));
    if (t->n > 0) {
        launch_inverse_pid(ps, t->d_inv, stream);
        ParticleSoA av{t->d_adj[cur], ps.pid, t->cap, t->n};
        for (int f = 0; f < 4; ++f) {
            const float* src = view_field(dfinal, f);
            if (!src) continue;
            BM_CHECK_CUDA(cudaMemcpyAsync(t->d_rows, src, sizeof(float) * kFields[f].width * t->n,
                                          cudaMemcpyHostToDevice, stream));
            launch_scatter_rows(av, kFields[f].plane, kFields[f].width, t->d_rows, 0, t->n, t->d_inv, stream);
        }
    }
    const int n_seg = (t->n_steps + t->K - 1) / t->K;
    const GridDesc g = s->sc().dev.g;
    float4* adj_gv = t->d_gadj;
    float4* adj_pm = t->d_gadj + t->nodes;
    float4* adj_f = t->d_gadj + 2 * t->nodes;
    for (int sg = n_seg - 1; sg >= 0 && st == BM_OK; --sg) {
        const int first = sg * t->K;
        const int len = std::min(t->K, t->n_steps - first);
        if ((st = copy_state(t, ps.base, ckpt(t, sg))) != BM_OK) break;
        for (int j = 0; j < len && st == BM_OK; ++j) {
            if ((st = copy_state(t, seg_state(t, j), ps.base)) != BM_OK) break;
            st = run_step(t, first + j);
        }
        for (int j = len - 1; j >= 0 && st == BM_OK; --j) {
            const int n = first + j;
            if ((st = copy_state(t, ps.base, seg_state(t, j))) != BM_OK) break;
            if ((st = do_p2g(s)) != BM_OK) break;
            const GridAcc acc = s->sc().dev.acc[s->w.cur];
            BM_CHECK_CUDA(cudaMemcpyAsync(t->d_pre, acc.mv, sizeof(float4) * t->nodes, cudaMemcpyDeviceToDevice,
                                          stream));
            BM_CHECK_CUDA(cudaMemcpyAsync(t->d_pre + t->nodes, acc.f, sizeof(float4) * t->nodes,
                                          cudaMemcpyDeviceToDevice, stream));
            if ((st = do_grid_update(s, t->dt)) != BM_OK) break;
            if (t->has_body) {
                const bm_collider_t b = body_at(t, n);
                if ((st = do_m1(s, 1, &b, t->dt)) != BM_OK) break;
                // the adjoint kernels read this step's M1 parameters on the
                // device (the one-body coupler passes them by value)
                BM_CHECK_CUDA(cudaMemcpyAsync(s->d_params, s->h_params.data(), sizeof(M1Params),
                                              cudaMemcpyHostToDevice, stream));
            }
            BM_CHECK_CUDA(cudaMemsetAsync(adj_gv, 0, sizeof(float4) * t->nodes, stream));
            const Material& mat = s->sc().dev.mat;
            AdjStep A{};
            A.st = seg_state(t, j);
            A.mass = ps.plane(P_M);
            A.vol = ps.plane(P_V0);
            A.cap = t->cap;
            A.n = t->n;
            A.g = g;
            A.gv = s->sc().dev.acc[s->w.cur].mv;
            A.pre_mv = t->d_pre;
            A.pre_f = t->d_pre + t->nodes;
            A.adj_gv = adj_gv;
            A.adj_pm = adj_pm;
            A.adj_f = adj_f;
            A.adj_in = t->d_adj[cur];
            A.adj_out = t->d_adj[1 - cur];
            A.mu = mat.mu;
            A.lambda = mat.lambda;
            A.nak = mat.neg_alpha_koh;
            A.dt = t->dt;
            A.gx = mat.gx;
            A.gy = mat.gy;
            A.gz = mat.gz;
            A.floor_friction = mat.floor_friction;
            A.alloc = s->sc().dev.alloc;
            A.body = t->has_body ? s->d_params : nullptr;
            A.body_adj = t->d_body_adj + 6 * (int64_t)n;
            if (t->n > 0) k_adj_g2p<<<(unsigned)nblk(t->n, kAdjThreads), kAdjThreads, 0, stream>>>(A);
            k_adj_grid<<<(unsigned)nblk(t->nodes, 256), 256, 0, stream>>>(A);
            if (t->n > 0) k_adj_p2g<<<(unsigned)nblk(t->n, kAdjThreads), kAdjThreads, 0, stream>>>(A);
            st = launch_status("adjoint step");
            cur = 1 - cur;
        }
    }
    // leave the solver in the recorded final state
    const bm_status_t st2 = copy_state(t, ps.base, ckpt(t, t->n_ckpt - 1));
    invalidate_state(s);
    if (st == BM_OK) st = st2;
    if (st != BM_OK) return st;
    t->h_body_adj.assign(6 * (size_t)t->n_steps, 0.0);
    BM_CHECK_CUDA(cudaMemcpyAsync(t->h_body_adj.data(), t->d_body_adj, sizeof(double) * 6 * t->n_steps,
                                  cudaMemcpyDeviceToHost, stream));
    if (t->n > 0 && dinitial) {
        ParticleSoA av{t->d_adj[cur], ps.pid, t->cap, t->n};
        for (int f = 0; f < 4; ++f) {
            float* dst = view_field(dinitial, f);
            if (!dst) continue;
            launch_gather_rows(av, kFields[f].plane, kFields[f].width, t->d_rows, stream);
            BM_CHECK_CUDA(cudaMemcpyAsync(dst, t->d_rows, sizeof(float) * kFields[f].width * t->n,
                                          cudaMemcpyDeviceToHost, stream));
            BM_CHECK_CUDA(cudaStreamSynchronize(stream));
        }
    }
    BM_CHECK_CUDA(cudaStreamSynchronize(stream));
    if (dL_dwaypoints && t->has_body) {
        std::vector<double> gw(3 * (size_t)t->n_wp, 0.0);
        for (int n = 0; n < t->n_steps; ++n) {
            int k;
            double seg, tn;
            path_segment(t, n, &k, &seg, &tn);
            for (int a = 0; a < 3; ++a) {
                // v = (w_{k+1} - w_k) / seg; the centre's dependence is the
                // coupler's inside test (zero almost everywhere)
                const double gvel = t->h_body_adj[6 * (size_t)n + a];
                gw[3 * (k + 1) + a] += gvel / seg;
                gw[3 * k + a] -= gvel / seg;
            }
        }
        for (size_t q = 0; q < gw.size(); ++q) dL_dwaypoints[q] = (float)gw[q];
    }
    return BM_OK;
}

}  // namespace

extern "C" {

BM_API bm_status_t bm_tape_create(bm_solver_t* s, int32_t checkpoint_every, bm_tape_t** out) {
    if (!s || !out) return invalid_arg("NULL argument");
    *out = nullptr;
    if (checkpoint_every < 1) return invalid_arg("checkpoint_every must be >= 1");
    bm_tape* t = new bm_tape();
    t->s = s;
    t->device = s->w.device;
    t->K = checkpoint_every;
    *out = t;
    return BM_OK;
}

BM_API bm_status_t bm_tape_destroy(bm_tape_t* t) {
    if (!t) return BM_OK;
    DeviceGuard dg(t->device);  // only the tape's own buffers: the solver may already be destroyed
    tape_free(t);
    delete t;
    return BM_OK;
}

BM_API bm_status_t bm_tape_forward(bm_tape_t* t, float dt, int32_t n_steps, const bm_collider_t* body,
                                   int32_t n_waypoints, const float* waypoints) {
    if (!t) return invalid_arg("NULL tape");
    if (!(dt > 0.0f) || !std::isfinite(dt)) return invalid_arg("dt must be positive and finite");
    if (n_steps < 1) return invalid_arg("n_steps must be >= 1");
    if (body && (n_waypoints < 2 || !waypoints)) return invalid_arg("a body needs >= 2 waypoints");
    bm_solver* s = t->s;
    DeviceGuard dg(s->w.device);
    t->recorded = false;
    bm_status_t st = prepare(s);
    if (st != BM_OK) return st;
    t->dt = dt;
    t->n_steps = n_steps;
    t->has_body = body != nullptr;
    if (body) {
        t->body = *body;
        t->n_wp = n_waypoints;
        t->wp.assign(waypoints, waypoints + 3 * (size_t)n_waypoints);
    } else {
        t->n_wp = 0;
        t->wp.clear();
    }
    const ParticleSoA& ps = store_of(t);
    tape_free(t);
    t->cap = ps.cap;
    t->n = ps.n;
    t->nodes = s->sc().dev.g.num_nodes();
    t->n_ckpt = (n_steps + t->K - 1) / t->K + 1;
    const size_t state = (size_t)kStatePlanes * t->cap;
    if ((st = dalloc(&t->d_ckpt, state * t->n_ckpt)) != BM_OK) return st;
    if ((st = dalloc(&t->d_seg, state * t->K)) != BM_OK) return st;
    if ((st = dalloc(&t->d_adj[0], state)) != BM_OK) return st;
    if ((st = dalloc(&t->d_adj[1], state)) != BM_OK) return st;
    if ((st = dalloc(&t->d_pre, 2 * (size_t)t->nodes)) != BM_OK) return st;
    if ((st = dalloc(&t->d_gadj, 3 * (size_t)t->nodes)) != BM_OK) return st;
    if ((st = dalloc(&t->d_body_adj, 6 * (size_t)n_steps)) != BM_OK) return st;
    if ((st = dalloc(&t->d_rows, 9 * (size_t)std::max<int64_t>(t->n, 1))) != BM_OK) return st;
    if ((st = dalloc(&t->d_inv, (size_t)std::max<int64_t>(t->n, 1))) != BM_OK) return st;
    if ((st = copy_state(t, ckpt(t, 0), ps.base)) != BM_OK) return st;
    for (int n = 0; n < n_steps; ++n) {
        if (n > 0 && n % t->K == 0 && (st = copy_state(t, ckpt(t, n / t->K), store_of(t).base)) != BM_OK) return st;
        if ((st = run_step(t, n)) != BM_OK) return st;
    }
    if ((st = copy_state(t, ckpt(t, t->n_ckpt - 1), store_of(t).base)) != BM_OK) return st;
    t->recorded = true;
    return launch_status("tape forward");
}

BM_API bm_status_t bm_adjoint_backward(bm_tape_t* t, const float* dL_dx, const float* dL_dv, float* dL_dwaypoints,
                                       float* dL_dx0, float* dL_dv0) {
    if (!t) return invalid_arg("NULL tape");
    if (!dL_dx) return invalid_arg("dL_dx is NULL");
    DeviceGuard dg(t->s->w.device);
    bm_particles_view_t in{};
    in.position = const_cast<float*>(dL_dx);
    in.velocity = const_cast<float*>(dL_dv);
    bm_particles_view_t out{};
    out.position = dL_dx0;
    out.velocity = dL_dv0;
    return backward(t, &in, dL_dwaypoints, (dL_dx0 || dL_dv0) ? &out : nullptr);
}

BM_API bm_status_t bm_adjoint_backward_state(bm_tape_t* t, const bm_particles_view_t* dL_dfinal,
                                             float* dL_dwaypoints, const bm_particles_view_t* dL_dinitial) {
    if (!t || !dL_dfinal) return invalid_arg("NULL argument");
    DeviceGuard dg(t->s->w.device);
    return backward(t, dL_dfinal, dL_dwaypoints, dL_dinitial);
}

BM_API bm_status_t bm_tape_body_grad(bm_tape_t* t, int32_t n_steps, double* out) {
    if (!t || !out) return invalid_arg("NULL argument");
    if (n_steps != t->n_steps || t->h_body_adj.size() != 6 * (size_t)n_steps) {
        set_last_error("bm_tape_body_grad needs the step count of a finished bm_adjoint_backward");
        return BM_ERR_STATE;
    }
    std::memcpy(out, t->h_body_adj.data(), sizeof(double) * 6 * n_steps);
    return BM_OK;
}

}  // extern "C"
