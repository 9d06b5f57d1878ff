// bm_adjoint.cuh — per-thread adjoints of the 3x3 constitutive maps.
//
// Both maps go through the reference's Jacobi SVD (svd.h:18-108) of a 3x3 F:
//
//   Hencky stress  tau(F)   = U diag(t) U^T,  t_k = 2 mu ln s_k + lambda sum_j ln s_j
//                             (mpm_solver.h:191-212)
//   DP return map  F'(F_tr) = U diag(g) V^T,  g = exp(projected log-strain)
//                             (mpm_solver.h:114-166)
//
// The SVD stops early: a rotation is skipped when |a_ij| < 1e-6 and the
// sweeps stop once the largest off-diagonal of F^T F is below 1e-5. Near
// F = I, the state of sand at rest, that residual is comparable to the gaps
// between the singular values, so U and V are far from the exact singular
// vectors, and the derivative of the exact SVD is not the derivative of what
// the step computes: at strains of 1e-5 they differ by tens of percent. The
// adjoint therefore differentiates the algorithm itself: the rotations are
// replayed with the same thresholds and the reverse pass goes back through
// them one by one (between two decisions the computed function is smooth and
// this is its exact derivative). The forward records each rotation and the
// reverse pass undoes them in turn. Both run in double: their terms scale
// with 1/a_ij and cancel, and in float the result loses percents at small
// strains. They follow the algorithm as the FP64 path runs it, at the state
// the FP32 forward produced.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "bm_math.cuh"

namespace bm {
namespace adj {

// Unique-entry index of the symmetric A (upper triangle).
template <int a, int b> __device__ __forceinline__ constexpr int uix() { return a < b ? 3 * a + b : 3 * b + a; }

// One Jacobi rotation of svd3 (bm_math.cuh, jacobi_rotate) in double.
// Returns whether it rotated, and then its (c, s).
template <int I, int J, int K>
__device__ __forceinline__ bool jacobi_rotate_d(double A[9], double V[9], double& max_off, double& c_out,
                                                double& s_out) {
    const double a_ij = A[3 * I + J], a_ii = A[3 * I + I], a_jj = A[3 * J + J];
    max_off = fmax(max_off, fabs(a_ij));
    if (fabs(a_ij) < 1e-6) return false;
    const double tau = (a_jj - a_ii) / (2.0 * a_ij);
    const double t = tau >= 0.0 ? 1.0 / (tau + sqrt(1.0 + tau * tau)) : -1.0 / (-tau + sqrt(1.0 + tau * tau));
    const double c = 1.0 / sqrt(1.0 + t * t);
    const double s = c * t;
    const double n_ii = c * c * a_ii - 2.0 * s * c * a_ij + s * s * a_jj;
    const double n_jj = s * s * a_ii + 2.0 * s * c * a_ij + c * c * a_jj;
    A[3 * I + I] = n_ii;
    A[3 * J + J] = n_jj;
    A[3 * I + J] = 0.0;
    A[3 * J + I] = 0.0;
    const double aik = A[3 * I + K], ajk = A[3 * J + K];
    const double nik = c * aik - s * ajk;
    const double njk = s * aik + c * ajk;
    A[3 * I + K] = nik;
    A[3 * K + I] = nik;
    A[3 * J + K] = njk;
    A[3 * K + J] = njk;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const double vri = V[3 * r + I], vrj = V[3 * r + J];
        V[3 * r + I] = c * vri - s * vrj;
        V[3 * r + J] = s * vri + c * vrj;
    }    c_out = c;
    s_out = s;
    return true;
}

// Undoes a rotation of jacobi_rotate_d from its (c, s). The rotation is the
// similarity A' = G^T A G, V' = V G with G = [[c, s], [-s, c]] in the (I, J)
// plane, so A = G A' G^T and V = V' G^T (one rounding in double; the
// rotation's own zero of a'_ij is what that similarity gives up to rounding).
template <int I, int J, int K>
__device__ __forceinline__ void jacobi_unrotate_d(double A[9], double V[9], double c, double s) {
    const double a_ii = A[3 * I + I], a_jj = A[3 * J + J], a_ij = A[3 * I + J];
    const double cc = c * c, ss = s * s, cs = c * s;
    const double o_ij = cs * (a_jj - a_ii) + (cc - ss) * a_ij;
    A[3 * I + I] = cc * a_ii + 2.0 * cs * a_ij + ss * a_jj;
    A[3 * J + J] = ss * a_ii - 2.0 * cs * a_ij + cc * a_jj;
    A[3 * I + J] = o_ij;
    A[3 * J + I] = o_ij;
    const double nik = A[3 * I + K], njk = A[3 * J + K];
    const double aik = c * nik + s * njk, ajk = -s * nik + c * njk;
    A[3 * I + K] = aik;
    A[3 * K + I] = aik;
    A[3 * J + K] = ajk;
    A[3 * K + J] = ajk;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const double vi = V[3 * r + I], vj = V[3 * r + J];
        V[3 * r + I] = c * vi + s * vj;
        V[3 * r + J] = -s * vi + c * vj;
    }
}

// Reverse of one jacobi_rotate_d<I,J,K> applied to (A, V) (the state before
// it): Ab (unique entries) and Vb hold the adjoints after the rotation on
// entry and before it on return. The rotation sets a_ij to 0, so the adjoint
// of the output a_ij does not flow back.
template <int I, int J, int K>
__device__ __forceinline__ void jacobi_rotate_adjoint(const double A[9], const double V[9], double Ab[9],
                                                      double Vb[9]) {
    const double a_ij = A[3 * I + J], a_ii = A[3 * I + I], a_jj = A[3 * J + J];
    if (fabs(a_ij) < 1e-6) return;  // skipped: the identity
    const double tau = (a_jj - a_ii) / (2.0 * a_ij);
    const double r = sqrt(1.0 + tau * tau);
    const double t = tau >= 0.0 ? 1.0 / (tau + r) : -1.0 / (-tau + r);
    const double c = 1.0 / sqrt(1.0 + t * t);
    const double s = c * t;
    const double aik = A[uix<I, K>()], ajk = A[uix<J, K>()];
    const double bii = Ab[4 * I], bjj = Ab[4 * J], bik = Ab[uix<I, K>()], bjk = Ab[uix<J, K>()];
    double cb = bii * (2.0 * c * a_ii - 2.0 * s * a_ij) + bjj * (2.0 * c * a_jj + 2.0 * s * a_ij) + bik * aik +
                bjk * ajk;
    double sb = bii * (2.0 * s * a_jj - 2.0 * c * a_ij) + bjj * (2.0 * s * a_ii + 2.0 * c * a_ij) - bik * ajk +
                bjk * aik;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double gI = Vb[3 * q + I], gJ = Vb[3 * q + J];
        const double vI = V[3 * q + I], vJ = V[3 * q + J];
        cb += gI * vI + gJ * vJ;
        sb += gJ * vI - gI * vJ;
        Vb[3 * q + I] = c * gI + s * gJ;
        Vb[3 * q + J] = c * gJ - s * gI;
    }
    Ab[4 * I] = bii * c * c + bjj * s * s;
    Ab[4 * J] = bii * s * s + bjj * c * c;
    Ab[uix<I, J>()] = 2.0 * s * c * (bjj - bii);
    Ab[uix<I, K>()] = c * bik + s * bjk;
    Ab[uix<J, K>()] = c * bjk - s * bik;
    // (c, s) from t: dc/dt = -t c^3, ds/dt = c^3; t from tau: dt/dtau = -|t| / r;
    // tau from (a_ii, a_jj, a_ij)
    const double tb = c * c * c * (sb - t * cb);
    const double taub = -tb * fabs(t) / r;
    Ab[4 * J] += taub / (2.0 * a_ij);
    Ab[4 * I] -= taub / (2.0 * a_ij);
    Ab[uix<I, J>()] -= taub * tau / a_ij;
}

// The SVD forward with what its adjoint needs: the final A and V, and the
// rotation of every slot (slot q = 3 * sweep + pair), so that the reverse
// pass undoes the rotations one by one instead of replaying the sweeps.
struct SvdD {
    double A[9], V[9], U[9], S[3];
    double c[15], s[15];  // (c, s) of slot q when it rotated
    unsigned applied;     // bit q: slot q rotated (else it was skipped, the identity)
    int n;                // rotation slots reached
};

// A = F^T F, V = I and the sweeps of svd3 (at most 5, a pair skipped below
// 1e-6, stopped when the sweep's largest off-diagonal is below 1e-5).
__device__ __forceinline__ void svd_forward(const double F[9], SvdD& f) {
    double* A = f.A;
    double* V = f.V;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) A[3 * i + j] = (F[i] * F[j] + F[3 + i] * F[3 + j]) + F[6 + i] * F[6 + j];
#pragma unroll
    for (int q = 0; q < 9; ++q) V[q] = (q % 4 == 0) ? 1.0 : 0.0;
    f.applied = 0u;
    int q = 0;
#pragma unroll 1
    for (int sweep = 0; sweep < 5; ++sweep) {
        double max_off = 0.0;
        if (jacobi_rotate_d<0, 1, 2>(A, V, max_off, f.c[q], f.s[q])) f.applied |= 1u << q;
        ++q;
        if (jacobi_rotate_d<0, 2, 1>(A, V, max_off, f.c[q], f.s[q])) f.applied |= 1u << q;
        ++q;
        if (jacobi_rotate_d<1, 2, 0>(A, V, max_off, f.c[q], f.s[q])) f.applied |= 1u << q;
        ++q;
        if (max_off < 1e-5) break;
    }
    f.n = q;
#pragma unroll
    for (int k = 0; k < 3; ++k) f.S[k] = sqrt(fmax(0.0, f.A[4 * k]));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double fv = F[3 * i] * f.V[c] + F[3 * i + 1] * f.V[3 + c] + F[3 * i + 2] * f.V[6 + c];
            f.U[3 * i + c] = f.S[c] > 1e-6 ? fv / f.S[c] : (i == c ? 1.0 : 0.0);
        }
    }
}

// Given the adjoints of U, S, V (all three are consumed), adds dL/dF into Fb.
__device__ __forceinline__ void svd_adjoint(const double F[9], const SvdD& f, const double Ub[9], double Sb[3],
                                            double Vb[9], double Fb[9]) {
    // U_c = (F V)_c / S_c
    double FVb[9];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (f.S[c] > 1e-6) {
            const double inv = 1.0 / f.S[c];
            FVb[c] = Ub[c] * inv;
            FVb[3 + c] = Ub[3 + c] * inv;
            FVb[6 + c] = Ub[6 + c] * inv;
            Sb[c] -= (Ub[c] * f.U[c] + Ub[3 + c] * f.U[3 + c] + Ub[6 + c] * f.U[6 + c]) * inv;
        } else {
            FVb[c] = FVb[3 + c] = FVb[6 + c] = 0.0;
        }
    }
    // F_bar += FV_bar V^T ; V_bar += F^T FV_bar
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Fb[3 * i + j] += FVb[3 * i] * f.V[3 * j] + FVb[3 * i + 1] * f.V[3 * j + 1] + FVb[3 * i + 2] * f.V[3 * j + 2];
            Vb[3 * i + j] += F[i] * FVb[j] + F[3 + i] * FVb[3 + j] + F[6 + i] * FVb[6 + j];
        }
    // S_k = sqrt(max(0, A_kk))
    double Ab[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) Ab[q] = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (f.A[4 * k] > 0.0 && f.S[k] > 0.0) Ab[4 * k] = Sb[k] / (2.0 * f.S[k]);
    // back through the rotations, last first: undo slot q to get the state
    // before it, then take its adjoint there (a skipped slot is the identity)
    double Ap[9], Vp[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        Ap[q] = f.A[q];
        Vp[q] = f.V[q];
    }
#pragma unroll 1
    for (int q = f.n - 1; q >= 0; --q) {
        if (!((f.applied >> q) & 1u)) continue;
        const int pair = q % 3;
        if (pair == 0) {
            jacobi_unrotate_d<0, 1, 2>(Ap, Vp, f.c[q], f.s[q]);
            jacobi_rotate_adjoint<0, 1, 2>(Ap, Vp, Ab, Vb);
        } else if (pair == 1) {
            jacobi_unrotate_d<0, 2, 1>(Ap, Vp, f.c[q], f.s[q]);
            jacobi_rotate_adjoint<0, 2, 1>(Ap, Vp, Ab, Vb);
        } else {
            jacobi_unrotate_d<1, 2, 0>(Ap, Vp, f.c[q], f.s[q]);
            jacobi_rotate_adjoint<1, 2, 0>(Ap, Vp, Ab, Vb);
        }
    }
    // A = F^T F (unique entries)
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const double f0 = F[3 * r], f1 = F[3 * r + 1], f2 = F[3 * r + 2];
        Fb[3 * r] += 2.0 * f0 * Ab[0] + f1 * Ab[1] + f2 * Ab[2];
        Fb[3 * r + 1] += 2.0 * f1 * Ab[4] + f0 * Ab[1] + f2 * Ab[5];
        Fb[3 * r + 2] += 2.0 * f2 * Ab[8] + f0 * Ab[2] + f1 * Ab[5];
    }
}

// Adjoint of hencky_tau: tau = U diag(2 mu e + lambda tr e) U^T with
// e = ln max(S, 1e-6). Adds dL/dF into Fb.
__device__ __forceinline__ void hencky_tau_adjoint(const float Ff[9], float mu, float lambda, const float tau_bar[9],
                                                   float Fb[9]) {
    double F[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) F[q] = Ff[q];
    SvdD f;
    svd_forward(F, f);
    double e[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) e[k] = log(fmax(f.S[k], 1e-6));
    const double tr = (e[0] + e[1]) + e[2];
    double d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = 2.0 * mu * e[k] + (double)lambda * tr;
    // tau_ij = sum_k U_ik d_k U_jk: U_bar = (tau_bar + tau_bar^T) U diag(d),
    // d_bar_k = (U^T tau_bar U)_kk
    double Ub[9], db[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double acc = 0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) acc += ((double)tau_bar[3 * i + j] + tau_bar[3 * j + i]) * f.U[3 * j + k];
            Ub[3 * i + k] = acc * d[k];
        }
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) db[k] += f.U[3 * i + k] * tau_bar[3 * i + j] * f.U[3 * j + k];
    const double sdb = (db[0] + db[1]) + db[2];
    double Sb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) Sb[k] = f.S[k] > 1e-6 ? (2.0 * mu * db[k] + (double)lambda * sdb) / f.S[k] : 0.0;
    double Vb[9], Fbd[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        Vb[q] = 0.0;
        Fbd[q] = 0.0;
    }
    svd_adjoint(F, f, Ub, Sb, Vb, Fbd);
#pragma unroll
    for (int q = 0; q < 9; ++q) Fb[q] += (float)Fbd[q];
}

// Adjoint of the Drucker-Prager return map F_new = U diag(g(S)) V^T of F_tr
// (dp_project): tension tip (tr ln S > 0: g = 1), cone (the deviatoric
// log-strain scaled onto the cone), elastic (g = max(S, 1e-6)). Ft is F_tr
// in double; writes dL/dF_tr into Ftb.
__device__ __forceinline__ void dp_project_adjoint(const double Ft[9], float neg_alpha_koh, const float Fnb[9],
                                                   double Ftb[9]) {
    SvdD f;
    svd_forward(Ft, f);
    const double nak = neg_alpha_koh;
    double s[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) s[k] = fmax(f.S[k], 1e-6);
    const double e[3] = {log(s[0]), log(s[1]), log(s[2])};
    const double tr = (e[0] + e[1]) + e[2];
    const double m3 = tr / 3.0;
    const double h[3] = {e[0] - m3, e[1] - m3, e[2] - m3};
    const double hn = sqrt((h[0] * h[0] + h[1] * h[1]) + h[2] * h[2]);
    const double limit = nak * tr;
    double g[3], dg[9];  // dg[3k+j] = dg_k/dS_j
    if (tr > 0.0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) g[k] = 1.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) dg[q] = 0.0;
    } else if (hn > limit) {
        // e* = m3 + (nak tr / hn) h:  de*_k/de_j = 1/3 + nak (n_k + (tr/hn)(delta_kj - 1/3 - n_k n_j))
        const double sc = limit / hn, q = tr / hn;
        double n[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            n[k] = h[k] / hn;
            g[k] = exp(h[k] * sc + m3);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double J = 1.0 / 3.0 + nak * (n[k] + q * (((k == j) ? 1.0 : 0.0) - 1.0 / 3.0 - n[k] * n[j]));
                dg[3 * k + j] = f.S[j] > 1e-6 ? g[k] * J / s[j] : 0.0;
            }
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) g[k] = s[k];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j) dg[3 * k + j] = (k == j && f.S[j] > 1e-6) ? 1.0 : 0.0;
    }
    // F_new_ij = sum_k U_ik g_k V_jk: U_bar = Fnb V diag(g), V_bar = Fnb^T U diag(g),
    // g_bar_k = (U^T Fnb V)_kk
    double Ub[9], Vb[9], gb[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double u = 0.0, v = 0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                u += (double)Fnb[3 * i + j] * f.V[3 * j + k];
                v += (double)Fnb[3 * j + i] * f.U[3 * j + k];
            }
            Ub[3 * i + k] = u * g[k];
            Vb[3 * i + k] = v * g[k];
        }
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) gb[k] += f.U[3 * i + k] * Fnb[3 * i + j] * f.V[3 * j + k];
    double Sb[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) Sb[j] = (gb[0] * dg[j] + gb[1] * dg[3 + j]) + gb[2] * dg[6 + j];
#pragma unroll
    for (int q = 0; q < 9; ++q) Ftb[q] = 0.0;
    svd_adjoint(Ft, f, Ub, Sb, Vb, Ftb);
}

// Derivatives of the quadratic B-spline weights with respect to the
// fractional offset f (w = bspline_weights(f)).
__device__ __forceinline__ void bspline_dweights(float f, float dw[3]) {
    dw[0] = f - 1.0f;
    dw[1] = 1.0f - 2.0f * f;
    dw[2] = f;
}

}  // namespace adj
}  // namespace bm
