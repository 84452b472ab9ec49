// Time-integrated fluxes of the Lax-Wendroff / two-stage multiderivative
// path (ConstructIntegratedR, lib/2d/ConstructIntegratedR.cpp): for every cell
// of the domain and its 3-cell ghost frame,
//   1-state:  F = f + dt/2 (f_t + dt/3 f_tt)                     (:59-296)
//   2-state:  F = a1 f(q1) + dt b1 f_t(q1) + a2 f(q2) + dt b2 f_t(q2)   (:525-606)
//   2-state with f_tt (the overload of :608-700, time_order 5 of FinSolveMD):
//             F = a1 f(q1) + dt (b1 f_t(q1) + c1 dt f_tt(q1))
//               + a2 f(q2) + dt (b2 f_t(q2) + c2 dt f_tt(q2)),
//             its f_tt by LocalIntegrate (:298-524), whose mixed derivatives
//             take a 4th-order stencil (:427-442) where the 1-state form
//             takes a 2nd-order one
// with f_t = -A (f_x + g_y) and, when time_order > 2 in the 1-state form,
//   f_tt = A (f_x+g_y)_t + f''[w, w],
//   (f_x+g_y)_t = f''[q_x, w] + g''[q_y, w] + A (f_xx + g_xy) + B (f_xy + g_yy),
// w = f_x + g_y, derivatives by the 5-point central differences Diff1/Diff2
// (lib/WenoReconstruct.cpp:702-716, :791-806) and the 2nd-order mixed stencil
// of :202-213.  The reference multiplies tabulated 5x5 Jacobians and 5x5x5
// Hessians (apps/2d/euler/lib/DFluxFunc.cpp, D2FluxFunc.cpp); here each
// product is a closed-form directional derivative of the Euler flux, which
// equals the tabulated product for every 2D state (rho w = 0).  The
// reference's Hessian leaves the pressure's E dependence out of the energy
// flux's E cross terms; dflux2 reproduces that.
//
// One block computes a TI x TJ tile of output cells; q is staged with a
// 2-cell halo (boundary conditions by remap), f and g are evaluated once per
// staged cell, then one thread per output cell forms F and G.  Output arrays
// are ghosted planes of (mx+6) x (my+6): cell (i, j), i in [-3, mx+3), sits at
// (i+3)*(my+6) + (j+3).
#pragma once
#include "fin_device.cuh"

namespace fin {

struct IntFluxArgs {
    const double* q1;       // state planes (q^n)
    const double* q2;       // second state for the 2-state form (q*), else nullptr
    double* F;              // ghosted output planes
    double* G;
    size_t plane;           // state plane stride
    size_t gplane;          // F/G plane stride (>= (mx+6)*(my+6))
    int mx, my;
    double dx, dy, gamma;
    double dt;              // 1-state: the dt argument of ConstructIntegratedR
    double a1, b1, a2, b2;  // 2-state coefficients
    double c1, c2;          // f_tt coefficients of the three-coefficient form
    int bc[4];
};

// Per-cell state for the directional derivatives.
struct DCell {
    double rho, ir, u[3], E, p, m[3];
};

__device__ __forceinline__ DCell dcell(double gamma, const double* Q)
{
    DCell c;
    c.rho = Q[0];
    c.ir = rcp(Q[0]);
    c.m[0] = Q[1]; c.m[1] = Q[2]; c.m[2] = Q[3];
    c.u[0] = Q[1] * c.ir; c.u[1] = Q[2] * c.ir; c.u[2] = Q[3] * c.ir;
    c.E = Q[4];
    c.p = (gamma - 1.0) * (Q[4] - 0.5 * c.rho * (c.u[0] * c.u[0] + c.u[1] * c.u[1] + c.u[2] * c.u[2]));
    return c;
}

// First variation of u and p along a: du_k = (a_k - u_k a_0)/rho,
// dp = (gamma-1)(a_4 - u.a_m + |u|^2 a_0 / 2); dpe = dp without its a_4 term.
struct DVar { double du[3], dp, dpe; };

__device__ __forceinline__ DVar dvar(double gamma, const DCell& c, const double* a)
{
    DVar v;
    v.du[0] = (a[1] - c.u[0] * a[0]) * c.ir;
    v.du[1] = (a[2] - c.u[1] * a[0]) * c.ir;
    v.du[2] = (a[3] - c.u[2] * a[0]) * c.ir;
    const double uu = c.u[0] * c.u[0] + c.u[1] * c.u[1] + c.u[2] * c.u[2];
    v.dpe = (gamma - 1.0) * (-(c.u[0] * a[1] + c.u[1] * a[2] + c.u[2] * a[3]) + 0.5 * uu * a[0]);
    v.dp = v.dpe + (gamma - 1.0) * a[4];
    return v;
}

// A a (n = 1: f, n = 2: g):  f_0 = m_n, f_k = m_n u_k + delta_kn p, f_4 = (E+p) u_n.
__device__ __forceinline__ void dflux1(int n, const DCell& c, const double* a, const DVar& va, double* out)
{
    out[0] = a[n];
#pragma unroll
    for (int k = 0; k < 3; k++) out[k + 1] = a[n] * c.u[k] + c.m[n - 1] * va.du[k] + (k + 1 == n ? va.dp : 0.0);
    out[4] = (a[4] + va.dp) * c.u[n - 1] + (c.E + c.p) * va.du[n - 1];
}

// Hessian product f''[a, b] in the reference's convention (see the header).
__device__ __forceinline__ void dflux2(double gamma, int n, const DCell& c, const double* a, const DVar& va,
                                       const double* b, const DVar& vb, double* out)
{
    double d2u[3];
#pragma unroll
    for (int k = 0; k < 3; k++) d2u[k] = -(va.du[k] * b[0] + vb.du[k] * a[0]) * c.ir;
    const double d2p = -(gamma - 1.0) * c.rho * (va.du[0] * vb.du[0] + va.du[1] * vb.du[1] + va.du[2] * vb.du[2]);
    out[0] = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++)
        out[k + 1] = a[n] * vb.du[k] + b[n] * va.du[k] + c.m[n - 1] * d2u[k] + (k + 1 == n ? d2p : 0.0);
    out[4] = (a[4] + va.dpe) * vb.du[n - 1] + (b[4] + vb.dpe) * va.du[n - 1] + d2p * c.u[n - 1] +
             (c.E + c.p) * d2u[n - 1];
}

__device__ __forceinline__ double diff1(double rdx, double f0, double f1, double f3, double f4)
{
    double tmp = (f0 - f4) * (1.0 / 12.0);
    tmp += (-f1 + f3) * (2.0 / 3.0);
    return tmp * rdx;
}
__device__ __forceinline__ double diff2(double rdx2, double f0, double f1, double f2, double f3, double f4)
{
    double tmp = (-f0 - f4) * (1.0 / 12.0);
    tmp += (f1 + f3) * (4.0 / 3.0);
    tmp += (-f2) * (5.0 / 2.0);
    return tmp * rdx2;
}

// MODE 0: 1-state, f_t only (time_order <= 2); 1: 1-state with f_tt; 2: 2-state;
// 3: 2-state with f_tt (q2 null: the second state's terms, all with zero
// coefficients, add nothing).
template <int MODE, int TI, int TJ>
__global__ void __launch_bounds__(TI * TJ) k_intflux(const IntFluxArgs a)
{
    constexpr int HB = 2, BI = TI + 2 * HB, BJ = TJ + 2 * HB, PB = BI * BJ;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double* qb = reinterpret_cast<double*>(smem_raw);   // [5][BI][BJ]
    double* fb = qb + MEQN * PB;                       // [5][BI][BJ]  f
    double* gb = fb + MEQN * PB;                       // [5][BI][BJ]  g
    const int tid = threadIdx.x;
    const int i0 = int(blockIdx.y) * TI - 3, j0 = int(blockIdx.x) * TJ - 3;   // extended-domain origin
    const int ci = tid / TJ, cj = tid - ci * TJ;
    const int i = i0 + ci, j = j0 + cj;                // this thread's output cell
    const bool out_ok = i < a.mx + 3 && j < a.my + 3;
    const double rdx = 1.0 / a.dx, rdy = 1.0 / a.dy;
    double Fo[MEQN] = {0, 0, 0, 0, 0}, Go[MEQN] = {0, 0, 0, 0, 0};

    const int nstate = (MODE == 2 || (MODE == 3 && a.q2)) ? 2 : 1;
    for (int st = 0; st < nstate; st++) {
        const double* q = st == 0 ? a.q1 : a.q2;
        if (st) __syncthreads();
        // all of a thread's loads before its flux evaluations and stores
        // (one memory round trip per block, not one per pass over the box)
        constexpr int NIT = (PB + TI * TJ - 1) / (TI * TJ);
        double Qv[NIT][MEQN];
#pragma unroll
        for (int it = 0; it < NIT; it++) {
            const int e = tid + it * TI * TJ;
            if (e < PB) {
                const int ii = e / BJ, jj = e - ii * BJ;
                const int gi = bc_remap(i0 - HB + ii, a.mx, a.bc[0], a.bc[1]);
                const int gj = bc_remap(j0 - HB + jj, a.my, a.bc[2], a.bc[3]);
                const size_t g = size_t(gi) * a.my + gj;
#pragma unroll
                for (int m = 0; m < MEQN; m++) Qv[it][m] = __ldg(q + m * a.plane + g);
            }
        }
#pragma unroll
        for (int it = 0; it < NIT; it++) {
            const int e = tid + it * TI * TJ;
            if (e < PB) {
                double f[MEQN], gg[MEQN];
                Euler::flux(a.gamma, Qv[it], f, gg);
#pragma unroll
                for (int m = 0; m < MEQN; m++) {
                    qb[m * PB + e] = Qv[it][m];
                    fb[m * PB + e] = f[m];
                    gb[m * PB + e] = gg[m];
                }
            }
        }
        __syncthreads();
        const int c0 = (ci + HB) * BJ + (cj + HB);
#define AT(arr, m, di, dj) arr[(m) * PB + c0 + (di) * BJ + (dj)]
        double Q[MEQN], w[MEQN], qx[MEQN], qy[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            Q[m] = AT(qb, m, 0, 0);
            const double fx = diff1(rdx, AT(fb, m, -2, 0), AT(fb, m, -1, 0), AT(fb, m, 1, 0), AT(fb, m, 2, 0));
            const double gy = diff1(rdy, AT(gb, m, 0, -2), AT(gb, m, 0, -1), AT(gb, m, 0, 1), AT(gb, m, 0, 2));
            w[m] = fx + gy;
            if (MODE == 1 || MODE == 3) {
                qx[m] = diff1(rdx, AT(qb, m, -2, 0), AT(qb, m, -1, 0), AT(qb, m, 1, 0), AT(qb, m, 2, 0));
                qy[m] = diff1(rdy, AT(qb, m, 0, -2), AT(qb, m, 0, -1), AT(qb, m, 0, 1), AT(qb, m, 0, 2));
            }
        }
        const DCell c = dcell(a.gamma, Q);
        const DVar vw = dvar(a.gamma, c, w);
        double ft[MEQN], gt[MEQN];
        dflux1(1, c, w, vw, ft);
        dflux1(2, c, w, vw, gt);
        if (MODE == 2) {
            const double al = st == 0 ? a.a1 : a.a2, be = st == 0 ? a.b1 : a.b2;
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                // F = a1 R1 + dt (b1 f1_t) + a2 R2 + dt (b2 f2_t), left to right
                Fo[m] = Fo[m] + al * AT(fb, m, 0, 0) + a.dt * (be * -ft[m]);
                Go[m] = Go[m] + al * AT(gb, m, 0, 0) + a.dt * (be * -gt[m]);
            }
        } else {
            double ftt[MEQN] = {0, 0, 0, 0, 0}, gtt[MEQN] = {0, 0, 0, 0, 0};
            if (MODE == 1 || MODE == 3) {
                double h1[MEQN], h2[MEQN], fpg[MEQN], v1[MEQN], v2[MEQN], t1[MEQN], t2[MEQN];
                const DVar vx = dvar(a.gamma, c, qx), vy = dvar(a.gamma, c, qy);
                dflux2(a.gamma, 1, c, qx, vx, w, vw, h1);
                dflux2(a.gamma, 2, c, qy, vy, w, vw, h2);
#pragma unroll
                for (int m = 0; m < MEQN; m++) {
                    const double fxx = diff2(rdx * rdx, AT(fb, m, -2, 0), AT(fb, m, -1, 0), AT(fb, m, 0, 0),
                                             AT(fb, m, 1, 0), AT(fb, m, 2, 0));
                    const double gyy = diff2(rdy * rdy, AT(gb, m, 0, -2), AT(gb, m, 0, -1), AT(gb, m, 0, 0),
                                             AT(gb, m, 0, 1), AT(gb, m, 0, 2));
                    double fxy, gxy;
                    if (MODE == 3) {
                        // 4th-order mixed derivative of LocalIntegrate, ConstructIntegratedR.cpp:427-442
                        auto mixed = [&](const double* r) {
                            double t = 0.25 * (AT(r, m, 1, 1) - AT(r, m, -1, 1) - AT(r, m, 1, -1) + AT(r, m, -1, -1));
                            t -= (1. / 24.) * (AT(r, m, 2, 1) + AT(r, m, -2, -1) - AT(r, m, 2, -1) - AT(r, m, -2, 1) -
                                               AT(r, m, 1, 2) - AT(r, m, -1, -2) + AT(r, m, 1, -2) + AT(r, m, -1, 2));
                            return t * (1. / (a.dx * a.dy));
                        };
                        fxy = mixed(fb);
                        gxy = mixed(gb);
                    } else {
                        // 2nd-order mixed derivative, ConstructIntegratedR.cpp:204-211
                        fxy = 0.5 * (AT(fb, m, 1, 1) - AT(fb, m, -1, 1)) * rdx;
                        fxy -= 0.5 * (AT(fb, m, 1, -1) - AT(fb, m, -1, -1)) * rdx;
                        fxy *= 0.5 * rdy;
                        gxy = 0.5 * (AT(gb, m, 1, 1) - AT(gb, m, -1, 1)) * rdx;
                        gxy -= 0.5 * (AT(gb, m, 1, -1) - AT(gb, m, -1, -1)) * rdx;
                        gxy *= 0.5 * rdy;
                    }
                    v1[m] = fxx + gxy;
                    v2[m] = fxy + gyy;
                }
                const DVar v1v = dvar(a.gamma, c, v1), v2v = dvar(a.gamma, c, v2);
                dflux1(1, c, v1, v1v, t1);
                dflux1(2, c, v2, v2v, t2);
#pragma unroll
                for (int m = 0; m < MEQN; m++) fpg[m] = h1[m] + h2[m] + t1[m] + t2[m];
                const DVar vf = dvar(a.gamma, c, fpg);
                dflux1(1, c, fpg, vf, ftt);
                dflux1(2, c, fpg, vf, gtt);
                dflux2(a.gamma, 1, c, w, vw, w, vw, h1);
                dflux2(a.gamma, 2, c, w, vw, w, vw, h2);
#pragma unroll
                for (int m = 0; m < MEQN; m++) {
                    ftt[m] += h1[m];
                    gtt[m] += h2[m];
                }
            }
            if (MODE == 3) {
                const double al = st == 0 ? a.a1 : a.a2, be = st == 0 ? a.b1 : a.b2, ch = st == 0 ? a.c1 : a.c2;
#pragma unroll
                for (int m = 0; m < MEQN; m++) {
                    // ConstructIntegratedR.cpp:685-692, left to right
                    Fo[m] = Fo[m] + al * AT(fb, m, 0, 0) + a.dt * (be * -ft[m] + ch * a.dt * ftt[m]);
                    Go[m] = Go[m] + al * AT(gb, m, 0, 0) + a.dt * (be * -gt[m] + ch * a.dt * gtt[m]);
                }
            } else {
#pragma unroll
                for (int m = 0; m < MEQN; m++) {
                    Fo[m] = AT(fb, m, 0, 0) + 0.5 * a.dt * (-ft[m] + a.dt / 3.0 * ftt[m]);
                    Go[m] = AT(gb, m, 0, 0) + 0.5 * a.dt * (-gt[m] + a.dt / 3.0 * gtt[m]);
                }
            }
        }
#undef AT
    }
    if (out_ok) {
        const size_t o = size_t(i + 3) * (a.my + 6) + (j + 3);
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            a.F[m * a.gplane + o] = Fo[m];
            a.G[m * a.gplane + o] = Go[m];
        }
    }
}

}  // namespace fin
