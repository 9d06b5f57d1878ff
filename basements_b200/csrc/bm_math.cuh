// bm_math.cuh — per-thread 3x3 math for the MLS-MPM kernels (sm_100a).
//
// Matrices are row-major float[9] kept in registers (every index below is a
// compile-time constant after unrolling). The arithmetic follows the order of
// the reference so that FP32 results agree with it to rounding; the compiler
// is allowed to contract a*b+c into FMA here (the trajectory is insensitive
// to that at the 1e-5*dx level over 1000 steps).
//
// Reference (2nugu/basements):
//   SVD          include/basements/core/math/svd.h:18-108
//   weights      include/basements/physics/mpm/mpm_solver.h:170-184
//   Hencky tau   include/basements/physics/mpm/mpm_solver.h:191-217
//   DP return    include/basements/physics/mpm/mpm_solver.h:114-166
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace bm {

// std::max semantics ((a < b) ? b : a), including NaN handling.
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }

// Quadratic B-spline weights for fractional offset f in [0, 1).
__device__ __forceinline__ void bspline_weights(float f, float w[3]) {
    w[0] = 0.5f * (1.0f - f) * (1.0f - f);
    w[1] = 0.75f - (f - 0.5f) * (f - 0.5f);
    w[2] = 0.5f * f * f;
}

__device__ __forceinline__ void matmul3(const float a[9], const float b[9], float r[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            r[3 * i + j] = (a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j]) + a[3 * i + 2] * b[6 + j];
}

// Division and square roots of the Jacobi rotation. Fast: the tangent t of
// the rotation angle uses the hardware approximations (about 1-2 ulp) -- an
// error in t only picks a slightly different angle, the rotation stays
// orthonormal because c and s are derived from t -- while c = 1/sqrt(1+t^2)
// and 1/sigma use correctly rounded intrinsics: an approximation there is
// biased and would scale F by the same tiny factor every step.
template <bool Fast> __device__ __forceinline__ float rcp_(float x) { return Fast ? __fdividef(1.0f, x) : 1.0f / x; }
template <bool Fast> __device__ __forceinline__ float div_(float a, float b) { return Fast ? __fdividef(a, b) : a / b; }
template <bool Fast> __device__ __forceinline__ float sqrt_(float x) { return Fast ? x * rsqrtf(x) : sqrtf(x); }
template <bool Fast> __device__ __forceinline__ float rsqrt_(float x) { return Fast ? __frsqrt_rn(x) : 1.0f / sqrtf(x); }

// One Jacobi rotation on the symmetric A (upper triangle kept in sync with
// the lower) for the pair (I, J); K is the third index.
template <int I, int J, int K, bool Fast = false>
__device__ __forceinline__ void jacobi_rotate(float A[9], float V[9], float& max_off) {
    const float a_ij = A[3 * I + J], a_ii = A[3 * I + I], a_jj = A[3 * J + J];
    max_off = smax(max_off, fabsf(a_ij));
    if (fabsf(a_ij) < 1e-6f) return;
    const float tau = div_<Fast>(a_jj - a_ii, 2.0f * a_ij);
    float t;
    if (tau >= 0.0f) t = rcp_<Fast>(tau + sqrt_<Fast>(1.0f + tau * tau));
    else             t = -rcp_<Fast>(-tau + sqrt_<Fast>(1.0f + tau * tau));
    const float c = rsqrt_<Fast>(1.0f + t * t);
    const float s = c * t;
    const float n_ii = c * c * a_ii - 2.0f * s * c * a_ij + s * s * a_jj;
    const float n_jj = s * s * a_ii + 2.0f * s * c * a_ij + c * c * a_jj;
    A[3 * I + I] = n_ii;
    A[3 * J + J] = n_jj;
    A[3 * I + J] = 0.0f;
    A[3 * J + I] = 0.0f;
    const float aik = A[3 * I + K], ajk = A[3 * J + K];
    const float nik = c * aik - s * ajk;
    const float njk = s * aik + c * ajk;
    A[3 * I + K] = nik; A[3 * K + I] = nik;
    A[3 * J + K] = njk; A[3 * K + J] = njk;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const float vri = V[3 * r + I], vrj = V[3 * r + J];
        V[3 * r + I] = c * vri - s * vrj;
        V[3 * r + J] = s * vri + c * vrj;
    }
}

// F = U diag(S) V^T by cyclic Jacobi on F^T F (at most 5 sweeps, pair skipped
// below 1e-6, stop when the sweep's largest off-diagonal is below 1e-5).
// Singular values unsorted, no sign fix; U column c = (F V)_c / S_c, or the
// unit axis when S_c <= 1e-6.
template <bool Fast = false>
__device__ __forceinline__ void svd3(const float F[9], float U[9], float S[3], float V[9]) {
    float A[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            A[3 * i + j] = (F[i] * F[j] + F[3 + i] * F[3 + j]) + F[6 + i] * F[6 + j];
#pragma unroll
    for (int q = 0; q < 9; ++q) V[q] = (q % 4 == 0) ? 1.0f : 0.0f;
#pragma unroll 1
    for (int sweep = 0; sweep < 5; ++sweep) {
        float max_off = 0.0f;
        jacobi_rotate<0, 1, 2, Fast>(A, V, max_off);
        jacobi_rotate<0, 2, 1, Fast>(A, V, max_off);
        jacobi_rotate<1, 2, 0, Fast>(A, V, max_off);
        if (max_off < 1e-5f) break;
    }
    S[0] = sqrtf(smax(0.0f, A[0]));
    S[1] = sqrtf(smax(0.0f, A[4]));
    S[2] = sqrtf(smax(0.0f, A[8]));
    float FV[9];
    matmul3(F, V, FV);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (S[c] > 1e-6f) {
            // Vec3 / s with the reference's |s| < 1e-6 guard (never taken here).
            if (Fast) {
                const float inv = __frcp_rn(S[c]);
                U[c] = FV[c] * inv;
                U[3 + c] = FV[3 + c] * inv;
                U[6 + c] = FV[6 + c] * inv;
            } else {
                U[c] = FV[c] / S[c];
                U[3 + c] = FV[3 + c] / S[c];
                U[6 + c] = FV[6 + c] / S[c];
            }
        } else {
            U[c] = (c == 0) ? 1.0f : 0.0f;
            U[3 + c] = (c == 1) ? 1.0f : 0.0f;
            U[6 + c] = (c == 2) ? 1.0f : 0.0f;
        }
    }
}

// M = U diag(d) W^T (the reference forms U * Matrix3::scale(d) * W^T; the
// zero products of the diagonal matrix add exactly nothing).
__device__ __forceinline__ void u_diag_wt(const float U[9], const float d[3], const float W[9], float M[9]) {
    float Ud[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Ud[3 * i + j] = U[3 * i + j] * d[j];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            M[3 * i + j] = (Ud[3 * i] * W[3 * j] + Ud[3 * i + 1] * W[3 * j + 1]) + Ud[3 * i + 2] * W[3 * j + 2];
}

// Kirchhoff stress tau = U diag(2 mu ln s + lambda tr(ln s)) U^T from F.
__device__ __forceinline__ void hencky_tau(const float F[9], float mu, float lambda, float tau[9]) {
    float U[9], S[3], V[9];
    svd3(F, U, S, V);
    const float lx = logf(smax(S[0], 1e-6f));
    const float ly = logf(smax(S[1], 1e-6f));
    const float lz = logf(smax(S[2], 1e-6f));
    const float tr = (lx + ly) + lz;
    const float d[3] = {2.0f * mu * lx + lambda * tr, 2.0f * mu * ly + lambda * tr, 2.0f * mu * lz + lambda * tr};
    u_diag_wt(U, d, U, tau);
}

// Drucker-Prager return map of F_trial = (I + C dt) F in log-strain space.
// cone = alpha * (3 lambda + 2 mu) / (2 mu), precomputed on the host.
__device__ __forceinline__ void dp_project(float F[9], const float Cm[9], float dt, float neg_alpha_koh) {
    float A[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) A[q] = ((q % 4 == 0) ? 1.0f : 0.0f) + Cm[q] * dt;
    float Ft[9];
    matmul3(A, F, Ft);
    float U[9], S[3], V[9];
    svd3(Ft, U, S, V);
    S[0] = smax(S[0], 1e-6f);
    S[1] = smax(S[1], 1e-6f);
    S[2] = smax(S[2], 1e-6f);
    float e0 = logf(S[0]), e1 = logf(S[1]), e2 = logf(S[2]);
    const float tr = (e0 + e1) + e2;
    const float m3 = tr / 3.0f;
    float h0 = e0 - m3, h1 = e1 - m3, h2 = e2 - m3;
    const float hn = sqrtf((h0 * h0 + h1 * h1) + h2 * h2);
    if (tr > 0.0f) {
        S[0] = 1.0f; S[1] = 1.0f; S[2] = 1.0f;
    } else {
        const float limit = neg_alpha_koh * tr;
        if (hn > limit) {
            const float sc = limit / hn;
            h0 = h0 * sc; h1 = h1 * sc; h2 = h2 * sc;
            S[0] = expf(h0 + m3);
            S[1] = expf(h1 + m3);
            S[2] = expf(h2 + m3);
        }
    }
    u_diag_wt(U, S, V, F);
}

// dp_project that also returns U and the log of the final singular values,
// so that the Kirchhoff stress of the next P2G is U diag(2 mu lnS + lambda
// tr lnS) U^T without a second SVD of the projected F (= U diag(S) V^T).
// lnS is 0 on the tension tip, the scaled log-strain on the cone, and
// log(max(S, 1e-6)) otherwise.
template <bool Fast = false>
__device__ __forceinline__ void dp_project_keep(float F[9], const float Cm[9], float dt, float neg_alpha_koh,
                                                float U[9], float lnS[3]) {
    float A[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) A[q] = ((q % 4 == 0) ? 1.0f : 0.0f) + Cm[q] * dt;
    float Ft[9];
    matmul3(A, F, Ft);
    float S[3], V[9];
    svd3<Fast>(Ft, U, S, V);
    S[0] = smax(S[0], 1e-6f);
    S[1] = smax(S[1], 1e-6f);
    S[2] = smax(S[2], 1e-6f);
    const float e0 = logf(S[0]), e1 = logf(S[1]), e2 = logf(S[2]);
    const float tr = (e0 + e1) + e2;
    const float m3 = tr / 3.0f;
    float h0 = e0 - m3, h1 = e1 - m3, h2 = e2 - m3;
    const float hn = sqrtf((h0 * h0 + h1 * h1) + h2 * h2);
    lnS[0] = e0; lnS[1] = e1; lnS[2] = e2;
    if (tr > 0.0f) {
        S[0] = 1.0f; S[1] = 1.0f; S[2] = 1.0f;
        lnS[0] = 0.0f; lnS[1] = 0.0f; lnS[2] = 0.0f;
    } else {
        const float limit = neg_alpha_koh * tr;
        if (hn > limit) {
            const float sc = limit / hn;
            h0 = h0 * sc; h1 = h1 * sc; h2 = h2 * sc;
            lnS[0] = h0 + m3; lnS[1] = h1 + m3; lnS[2] = h2 + m3;
            S[0] = expf(lnS[0]);
            S[1] = expf(lnS[1]);
            S[2] = expf(lnS[2]);
        }
    }
    u_diag_wt(U, S, V, F);
}

}  // namespace bm
