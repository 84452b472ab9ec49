// The maximum-principle-preserving (positivity) limiter of the Lax-Wendroff
// step, FinSolveLxW.cpp:126-158: the high-order face fluxes fhat, ghat of
// ConstructLxWL (written by the stage kernel in its flux-only mode), the
// Lax-Friedrichs fluxes of ConstructLFL.cpp:92-108, ApplyMPPLimiter2D
// (apps/2d/euler/lib/ApplyMPPLimiter2D.cpp:27-285) and the conservative
// update of FinSolveLxW.cpp:143-151.
//
// Two kernels, one thread per cell:
//   k_mpp_limit   the cell's four limiting factors amin[k] (k = left, right,
//                 bottom, top face): the density step (:57-92) and the
//                 pressure step over the 16 on/off combinations of the faces
//                 with its 9-step bisection (:97-217);
//   k_mpp_update  the face factors theta = min of the two cells' (one-sided
//                 at the domain boundary, :222-243), the limited fluxes
//                 theta (fhat - fLF) + fLF (:248-270), the update, and the
//                 new state's global wave speeds (GlobalWaveSpd.cpp:71-76).
// The Lax-Friedrichs fluxes are recomputed where needed (cheap) instead of
// stored.  Every operation follows the reference's order with correctly
// rounded IEEE operations (no contraction), so equal inputs give equal
// results.
#pragma once
#include "fin_stage.cuh"

namespace fin {
namespace mpp {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }
// dog_math.h:18-22
__device__ __forceinline__ double Mn(double a, double b) { return a < b ? a : b; }

struct MppArgs {
    const double* q;      // q^n planes
    double* qout;         // q^{n+1} planes
    size_t plane;
    int mx, my;
    int bc[4];
    const double* fhat;   // [m][mx+1][my]  high-order x-face fluxes (face i between cells i-1, i)
    const double* ghat;   // [m][mx][my+1]  high-order y-face fluxes
    double* amin;         // [4][mx][my]
    const double* alpha;  // [2] global wave speeds of q^n (GlobalWaveSpd, ConstructLFL.cpp:62-65)
    double dt, dx, dy, gamma;
    double* alpha_out;    // [2] GlobalWaveSpd of q^{n+1}
    unsigned int* status; // bit 0: non-finite wave speed of q^{n+1}
};

// FluxFunc.cpp:19-42, component m of direction d (0: f, 1: g).
__device__ __forceinline__ double flux_comp(const double* Q, double gamma, int d, int m)
{
    const double rho = Q[0];
    const double u1 = dvd(Q[1], rho), u2 = dvd(Q[2], rho), u3 = dvd(Q[3], rho);
    const double energy = Q[4];
    const double ke = add(add(mul(u1, u1), mul(u2, u2)), mul(u3, u3));
    const double press = mul(sub(gamma, 1.0e0), sub(energy, mul(mul(0.5e0, rho), ke)));
    const double un = d == 0 ? u1 : u2;
    switch (m) {
    case 0: return mul(rho, un);
    case 1: return d == 0 ? add(mul(mul(rho, u1), u1), press) : mul(mul(rho, u2), u1);
    case 2: return d == 0 ? mul(mul(rho, u1), u2) : add(mul(mul(rho, u2), u2), press);
    case 3: return mul(mul(rho, un), u3);
    default: return mul(un, add(energy, press));
    }
}

__device__ __forceinline__ void load_cell(const MppArgs& a, int i, int j, double* Q)
{
    const size_t g = size_t(bc_remap(i, a.mx, a.bc[0], a.bc[1])) * a.my + bc_remap(j, a.my, a.bc[2], a.bc[3]);
#pragma unroll
    for (int m = 0; m < MEQN; m++) Q[m] = a.q[m * a.plane + g];
}

// Lax-Friedrichs flux of the face between cells L and R (ConstructLFL.cpp:
// 92-108): 0.5 (f(L) + f(R)) + 0.5 alpha (q_L - q_R), all components.
__device__ __forceinline__ void lf_flux(const double* QL, const double* QR, double gamma, int d, double alpha,
                                        double* out)
{
#pragma unroll
    for (int m = 0; m < MEQN; m++) {
        const double fl = flux_comp(QL, gamma, d, m), fr = flux_comp(QR, gamma, d, m);
        out[m] = add(mul(0.5, add(fl, fr)), mul(mul(0.5, alpha), sub(QL[m], QR[m])));
    }
}

// The four faces of cell (i, j): high-order and Lax-Friedrichs fluxes
// (k = 0: x face i, 1: x face i+1, 2: y face j, 3: y face j+1).
__device__ __forceinline__ void cell_faces(const MppArgs& a, int i, int j, double (&fh)[4][MEQN],
                                           double (&fl)[4][MEQN], double (&qc)[MEQN])
{
    const int mx = a.mx, my = a.my;
    double Qn[MEQN];
    load_cell(a, i, j, qc);
    load_cell(a, i - 1, j, Qn);
    lf_flux(Qn, qc, a.gamma, 0, a.alpha[0], fl[0]);
    load_cell(a, i + 1, j, Qn);
    lf_flux(qc, Qn, a.gamma, 0, a.alpha[0], fl[1]);
    load_cell(a, i, j - 1, Qn);
    lf_flux(Qn, qc, a.gamma, 1, a.alpha[1], fl[2]);
    load_cell(a, i, j + 1, Qn);
    lf_flux(qc, Qn, a.gamma, 1, a.alpha[1], fl[3]);
#pragma unroll
    for (int m = 0; m < MEQN; m++) {
        fh[0][m] = a.fhat[(size_t(m) * (mx + 1) + i) * my + j];
        fh[1][m] = a.fhat[(size_t(m) * (mx + 1) + i + 1) * my + j];
        fh[2][m] = a.ghat[(size_t(m) * mx + i) * (my + 1) + j];
        fh[3][m] = a.ghat[(size_t(m) * mx + i) * (my + 1) + j + 1];
    }
}

// Pressure of a state, ApplyMPPLimiter2D.cpp:108-113.
__device__ __forceinline__ double pressure(const double* Q, double gm1)
{
    const double rho = Q[0];
    const double u1 = dvd(Q[1], rho), u2 = dvd(Q[2], rho), u3 = dvd(Q[3], rho);
    const double ke = add(add(mul(u1, u1), mul(u2, u2)), mul(u3, u3));
    return mul(gm1, sub(Q[4], mul(mul(0.5, rho), ke)));
}

__global__ void __launch_bounds__(128) k_mpp_limit(const MppArgs a)
{
    const int mx = a.mx, my = a.my;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= (long long)mx * my) return;
    const int i = int(c / my), j = int(c - (long long)i * my);
    double fh[4][MEQN], fl[4][MEQN], qc[MEQN];
    cell_faces(a, i, j, fh, fl, qc);
    const double eps = 1.0e-12, rho_min = eps;
    const double dtx = dvd(a.dt, a.dx), dty = dvd(a.dt, a.dy);
    const double gm1 = sub(a.gamma, 1.0);
    // ---- step 1: density (:57-92) ----
    const double gmin = sub(rho_min, add(add(qc[0], mul(dtx, sub(fl[0][0], fl[1][0]))),
                                         mul(dty, sub(fl[2][0], fl[3][0]))));
    double ff[4], amin[4];
    ff[0] = mul(dtx, sub(fh[0][0], fl[0][0]));
    ff[1] = mul(-dtx, sub(fh[1][0], fl[1][0]));
    ff[2] = mul(dty, sub(fh[2][0], fl[2][0]));
    ff[3] = mul(-dty, sub(fh[3][0], fl[3][0]));
    int isgn[4];
#pragma unroll
    for (int k = 0; k < 4; k++) isgn[k] = ff[k] < 0.0 ? 1 : 0;
    double ffsum = mul(double(isgn[0]), ff[0]);
#pragma unroll
    for (int k = 1; k < 4; k++) ffsum = add(ffsum, mul(double(isgn[k]), ff[k]));
#pragma unroll
    for (int k = 0; k < 4; k++) amin[k] = isgn[k] == 1 ? Mn(dvd(gmin, sub(ffsum, eps)), 1.e0) : 1.e0;
    // ---- step 2: pressure (:97-217) ----
    double qlf[MEQN];
#pragma unroll
    for (int m = 0; m < MEQN; m++)
        qlf[m] = add(add(qc[m], mul(dtx, sub(fl[0][m], fl[1][m]))), mul(dty, sub(fl[2][m], fl[3][m])));
    if (pressure(qlf, gm1) < 0.0) atomicOr(a.status, 2u);   // "Negative solution in Lax-Friedrich's flux"
    double rescale[16];
#pragma unroll 1
    for (int combo = 0; combo < 16; combo++) {
        // combo bits (i1 i2 i3 i4) with i1 the most significant, as the
        // reference's nested loops enumerate them
        const int on[4] = {(combo >> 3) & 1, (combo >> 2) & 1, (combo >> 1) & 1, combo & 1};
        double aa[4], qh[MEQN];
#pragma unroll
        for (int k = 0; k < 4; k++) aa[k] = mul(double(on[k]), amin[k]);
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            double f4[4];
#pragma unroll
            for (int k = 0; k < 4; k++) f4[k] = add(mul(aa[k], fh[k][m]), mul(sub(1.0, aa[k]), fl[k][m]));
            qh[m] = add(add(qc[m], mul(dtx, sub(f4[0], f4[1]))), mul(dty, sub(f4[2], f4[3])));
        }
        double phigh = pressure(qh, gm1);
        double r = 1.0;
        if (phigh < 0.0) {
            double root1 = 0.0, root2 = 1.0, rate = 0.0;
#pragma unroll 1
            for (int nn = 1; nn < 10; nn++) {
                rate = dvd(add(root1, root2), 2.0);
                double q2[MEQN];
#pragma unroll
                for (int m = 0; m < MEQN; m++) q2[m] = add(mul(rate, qh[m]), mul(sub(1.0, rate), qlf[m]));
                phigh = pressure(q2, gm1);
                if (phigh < 0.0) root2 = rate;
                else root1 = rate;
            }
            r = phigh > 0.0 ? rate : root1;
        }
        rescale[combo] = r;
    }
    double rescale2[4] = {1.0, 1.0, 1.0, 1.0};
#pragma unroll 1
    for (int t = 0; t < 8; t++) {   // (i1, i2, i3) of :220-227, i3 fastest
        const int b1 = (t >> 2) & 1, b2 = (t >> 1) & 1, b3 = t & 1;
        rescale2[0] = Mn(rescale2[0], rescale[8 | (b1 << 2) | (b2 << 1) | b3]);
        rescale2[1] = Mn(rescale2[1], rescale[(b1 << 3) | 4 | (b2 << 1) | b3]);
        rescale2[2] = Mn(rescale2[2], rescale[(b1 << 3) | (b2 << 2) | 2 | b3]);
        rescale2[3] = Mn(rescale2[3], rescale[(b1 << 3) | (b2 << 2) | (b3 << 1) | 1]);
    }
    const size_t nc = size_t(mx) * my;
#pragma unroll
    for (int k = 0; k < 4; k++) a.amin[k * nc + c] = mul(rescale2[k], amin[k]);
}

__global__ void __launch_bounds__(128) k_mpp_update(const MppArgs a)
{
    __shared__ double red[2][4];
    const int mx = a.mx, my = a.my;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double sx = 0.0, sy = 0.0;
    bool nonfinite = false;
    if (c < (long long)mx * my) {
        const int i = int(c / my), j = int(c - (long long)i * my);
        const size_t nc = size_t(mx) * my;
        double fh[4][MEQN], fl[4][MEQN], qc[MEQN];
        cell_faces(a, i, j, fh, fl, qc);
        // face factors (:222-243): min of the two cells' entries, the
        // cell's own at the domain boundary
        const double* am = a.amin;
        double th[4];
        th[0] = i > 0 ? Mn(am[0 * nc + c], am[1 * nc + (c - my)]) : am[0 * nc + c];
        th[1] = i < mx - 1 ? Mn(am[0 * nc + (c + my)], am[1 * nc + c]) : am[1 * nc + c];
        th[2] = j > 0 ? Mn(am[2 * nc + c], am[3 * nc + (c - 1)]) : am[2 * nc + c];
        th[3] = j < my - 1 ? Mn(am[2 * nc + (c + 1)], am[3 * nc + c]) : am[3 * nc + c];
        const double dtdx = dvd(a.dt, a.dx), dtdy = dvd(a.dt, a.dy);
        double qn[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            double f[4];
#pragma unroll
            for (int k = 0; k < 4; k++) f[k] = add(mul(th[k], sub(fh[k][m], fl[k][m])), fl[k][m]);
            // FinSolveLxW.cpp:145-148
            double v = sub(qc[m], mul(dtdx, sub(f[1], f[0])));
            v = sub(v, mul(dtdy, sub(f[3], f[2])));
            qn[m] = v;
            a.qout[m * a.plane + (size_t(i) * my + j)] = v;
        }
        // GlobalWaveSpd.cpp:71-76 on the new state
        const double rho = qn[0];
        const double u1 = dvd(qn[1], rho), u2 = dvd(qn[2], rho), u3 = dvd(qn[3], rho);
        const double ke = add(add(mul(u1, u1), mul(u2, u2)), mul(u3, u3));
        const double press = mul(sub(a.gamma, 1.0), sub(qn[4], mul(mul(0.5, rho), ke)));
        const double cs = sqrt(fabs(dvd(mul(a.gamma, press), rho)));
        sx = add(fabs(u1), cs);
        sy = add(fabs(u2), cs);
        if (!(sx <= 1e300) || !(sy <= 1e300)) nonfinite = true;
        if (!(sx <= 1e300)) sx = 0.0;
        if (!(sy <= 1e300)) sy = 0.0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sx = Max(sx, __shfl_xor_sync(0xffffffffu, sx, o));
        sy = Max(sy, __shfl_xor_sync(0xffffffffu, sy, o));
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = sx;
        red[1][threadIdx.x >> 5] = sy;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 4; w++) {
            sx = Max(sx, red[0][w]);
            sy = Max(sy, red[1][w]);
        }
        if (a.alpha_out) {
            atomic_max_nonneg(a.alpha_out, sx);
            atomic_max_nonneg(a.alpha_out + 1, sy);
        }
    }
    if (nonfinite) atomicOr(a.status, 1u);
}

}  // namespace mpp
}  // namespace fin
