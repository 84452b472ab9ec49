// Face features and labels of the troubled-cell indicator.
//
// For the face between cells i-1 and i (x faces; y faces alike along j), with
// the 6-point WENO stencil i-3 .. i+2 and the left eigenvectors at the face
// average (ProjectLeftEig.cpp:47-66):
//   features: for the characteristic fields k = 0, 1, 2, 4 (field 3, rho w, is
//     zero in 2D), the 5 undivided differences D_k,s = w_k(s+1) - w_k(s) of
//     w = L q, each divided by max(max_s |D_k,s|, FEAT_FLOOR): 20 values;
//   label: 1 when, for any of those fields and either split direction, the
//     WENO5-JS weights of the reconstructed values gp / gm
//     (ConstructL.cpp:179-192) depart from the linear weights d = (0.1, 0.6,
//     0.3) by more than 10 %: max_j |w_j - d_j| / d_j > 0.1
//     (lib/WenoReconstruct.cpp:104, 131-134).
// FEAT_FLOOR = 1e-3 (the square root of the default WENO epsilon 1e-6): a
// field whose differences stay below it cannot move the weights (beta ~ D^2
// stays below epsilon), so its features stay small instead of being
// normalised up to O(1).
#pragma once
#include "fin_device.cuh"
#include "fin_weno_face.cuh"

namespace fin {
namespace ind {

constexpr int NFEAT = 20;
constexpr float FEAT_FLOOR = 1e-3f;

// Global face index -> (direction, i, j): x faces first ((mx+1) x my, j
// fastest), then y faces (mx x (my+1)).
__device__ __forceinline__ void face_of(long long f, int mx, int my, bool& isx, int& i, int& j)
{
    const long long nx = (long long)(mx + 1) * my;
    if (f < nx) {
        isx = true;
        i = int(f / my);
        j = int(f - (long long)i * my);
    } else {
        isx = false;
        const long long g = f - nx;
        i = int(g / (my + 1));
        j = int(g - (long long)i * (my + 1));
    }
}

// Stencil point s (0..5) of face (isx, i, j) -> remapped cell index.
__device__ __forceinline__ size_t stencil_cell(bool isx, int i, int j, int s, int mx, int my, const int* bc)
{
    const int ci = isx ? i + s - 3 : i, cj = isx ? j : j + s - 3;
    return size_t(bc_remap(ci, mx, bc[0], bc[1])) * my + bc_remap(cj, my, bc[2], bc[3]);
}

// Features of one face in arithmetic R from its 6-point stencil Q[s][m]
// (normal frame: rho, m_n, m_t, m_w, E).
template <class R>
__device__ __forceinline__ void stencil_features(const R (&Q)[6][MEQN], R gamma, float* x)
{
    R Qa[MEQN];
#pragma unroll
    for (int m = 0; m < MEQN; m++) Qa[m] = R(0.5) * (Q[3][m] + Q[2][m]);
    const typename Euler::Eig<R> e = Euler::eig(gamma, Qa);
    const typename Euler::Rows<R> rw = Euler::rows(e);
    R w[4][6];
#ifndef FIN_X2_FEAT
#define FIN_X2_FEAT 1
#endif
    if constexpr (sizeof(R) == 4 && FIN_X2_FEAT) {
        // FP32: two stencil points per f32x2 pair (the same rows lane by lane)
#pragma unroll
        for (int s = 0; s < 6; s += 2) {
            f2 v[MEQN], w0, w4;
#pragma unroll
            for (int m = 0; m < MEQN; m++) v[m] = f2_make(Q[s][m], Q[s + 1][m]);
            left04_x2(e, rw, v, w0, w4);
            const f2 w1 = left1_x2(e, rw, v);
            const f2 w2 = f2_fma(f2_splat(-e.u2), v[0], v[2]);
            w[0][s] = f2_lo(w0); w[0][s + 1] = f2_hi(w0);
            w[1][s] = f2_lo(w1); w[1][s + 1] = f2_hi(w1);
            w[2][s] = f2_lo(w2); w[2][s + 1] = f2_hi(w2);
            w[3][s] = f2_lo(w4); w[3][s + 1] = f2_hi(w4);
        }
    } else {
#pragma unroll
        for (int s = 0; s < 6; s++) {
            R w0, w4;
            Euler::left04(e, rw, Q[s], w0, w4);
            w[0][s] = w0;
            w[1][s] = Euler::left1(e, rw, Q[s]);
            w[2][s] = Q[s][2] - e.u2 * Q[s][0];
            w[3][s] = w4;
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        R d[5], mmax = R(FEAT_FLOOR);
#pragma unroll
        for (int s = 0; s < 5; s++) {
            d[s] = w[k][s + 1] - w[k][s];
            mmax = Max(mmax, R(fabs(d[s])));
        }
        // FP32: the hardware reciprocal (rcp.approx, within 1 ulp; mmax >=
        // FEAT_FLOOR is a normal number) instead of the IEEE division's
        // instruction sequence; the features are rounded to BF16 next
        const R inv = sizeof(R) == 4 ? rcp(mmax) : R(1) / mmax;
#pragma unroll
        for (int s = 0; s < 5; s++) x[k * 5 + s] = float(d[s] * inv);
    }
}

// Features of one face in arithmetic R from the state planes q.
template <class R>
__device__ __forceinline__ void face_features(const double* q, size_t plane, int mx, int my, const int* bc, R gamma,
                                              bool isx, int i, int j, float* x)
{
    const int cn = isx ? 1 : 2, ct = isx ? 2 : 1;
    R Q[6][MEQN];
#pragma unroll
    for (int s = 0; s < 6; s++) {
        const size_t c = stencil_cell(isx, i, j, s, mx, my, bc);
        Q[s][0] = R(__ldg(q + c));
        Q[s][1] = R(__ldg(q + cn * plane + c));
        Q[s][2] = R(__ldg(q + ct * plane + c));
        Q[s][3] = R(__ldg(q + 3 * plane + c));
        Q[s][4] = R(__ldg(q + 4 * plane + c));
    }
    stencil_features<R>(Q, gamma, x);
}

// WENO5-JS weights departure of one 5-point stencil: max_j |w_j - d_j| / d_j.
__device__ __forceinline__ double js5_departure(const double* u, double eps, double pw)
{
    double b0, b1, b2, c0, c1, c2;
    weno5_parts(u, b0, b1, b2, c0, c1, c2);
    const double o0 = 0.1 * pow(eps + b0, -pw), o1 = 0.6 * pow(eps + b1, -pw), o2 = 0.3 * pow(eps + b2, -pw);
    const double s = o0 + o1 + o2;
    return Max(fabs(o0 / s - 0.1) / 0.1, Max(fabs(o1 / s - 0.6) / 0.6, fabs(o2 / s - 0.3) / 0.3));
}

// Label of one face (FP64): the reference's own split and WENO5-JS weights.
__device__ __forceinline__ unsigned char face_label(const double* q, size_t plane, int mx, int my, const int* bc,
                                                   double gamma, double eps, double pw, double ascale, double alpha_g,
                                                   bool isx, int i, int j)
{
    const int cn = isx ? 1 : 2, ct = isx ? 2 : 1;
    double Q[6][MEQN], F[6][MEQN];
#pragma unroll
    for (int s = 0; s < 6; s++) {
        const size_t c = stencil_cell(isx, i, j, s, mx, my, bc);
        const double Qp[MEQN] = {q[c], q[plane + c], q[2 * plane + c], q[3 * plane + c], q[4 * plane + c]};
        double f[MEQN], g[MEQN];
        Euler::flux(gamma, Qp, f, g);
        const double* fn = isx ? f : g;
        const int ml[MEQN] = {0, cn, ct, 3, 4};
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            Q[s][m] = Qp[ml[m]];
            F[s][m] = fn[ml[m]];
        }
    }
    double Qa[MEQN];
#pragma unroll
    for (int m = 0; m < MEQN; m++) Qa[m] = 0.5 * (Q[3][m] + Q[2][m]);
    const Euler::Cell<double> cl = Euler::cell(gamma, Q[2]), cr = Euler::cell(gamma, Q[3]);
    bool neg = false;
    const double alpha = Max(alpha_g, Euler::speed(gamma, cl, cr, &neg));
    const double la = ascale * alpha;
    const typename Euler::Eig<double> e = Euler::eig(gamma, Qa);
    double W[6][MEQN], G[6][MEQN];
#pragma unroll
    for (int s = 0; s < 6; s++) {
        Euler::left(e, Q[s], W[s]);
        Euler::left(e, F[s], G[s]);
    }
    double dep = 0.0;
    const int fields[4] = {0, 1, 2, 4};
#pragma unroll
    for (int t = 0; t < 4; t++) {
        const int k = fields[t];
        double gp[5], gm[5];
#pragma unroll
        for (int s = 0; s < 5; s++) {
            gp[s] = 0.5 * (G[s][k] + la * W[s][k]);
            gm[s] = 0.5 * (G[5 - s][k] - la * W[5 - s][k]);
        }
        dep = Max(dep, Max(js5_departure(gp, eps, pw), js5_departure(gm, eps, pw)));
    }
    return dep > 0.1 ? 1 : 0;
}

}  // namespace ind
}  // namespace fin
