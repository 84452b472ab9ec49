// The fused stage kernel: one launch computes, for a TI x TJ tile of cells,
//   L(q_in)   (ConstructL, lib/2d/ConstructL.cpp:62-401)
//   q_out = a1*A + a2*B + (beta*dt)*L     (UpdateSoln, lib/2d/UpdateSoln.cpp:29-35)
// and, in its epilogue, the two maxima the next stage and the CFL need:
//   * the wave-speed maxima alpha1/alpha2 of q_out over interior cells
//     (GlobalWaveSpd, lib/2d/GlobalWaveSpd.cpp:52-78), which the *next*
//     stage uses as its global alpha, so no stage needs a separate pass over
//     its own input;
//   * the maxima of the face speeds over the faces GetCFL reads
//     (lib/2d/GetCFL.cpp:54-59 reads smax(i,j,.) for i<=mx, j<=my).
// Maxima are exact, so computing them in a different order or place than the
// reference changes no bit of the result.
//
// Data layout in HBM: one plane per component, plane m holds mx*my values
// with j (y) fastest -- the reference's own axis order (x slowest,
// lib/tensors.h:267-273) without its ghost frame.  Ghost values are produced
// on load by the boundary remap (no ghost writes, no BC pass).
//
// Per block, shared memory holds (R = double or float):
//   qs  [M][TI+6][TJ+6]   stage input with a 3-cell halo (corners unused)
//   fs  [M][TI+6][TJ]     x flux f at the x-stencil cells
//   gs  [M][TI][TJ+6]     y flux g at the y-stencil cells
//   Fh  [M][TI+1][TJ]     x-face numerical fluxes
//   Gh  [M][TI][TJ+1]     y-face numerical fluxes
// Phases: load (coalesced along j) -> flux per cell (FluxFunc once per cell,
// not six times per face as the reference does) -> one thread per face, x
// and y faces in one work list (projection, LLF split, two WENO5, back
// projection, all in registers) -> per cell flux difference + RK update +
// next-stage wave speed -> block max -> one atomicMax per block.
#pragma once
#include "fin_device.cuh"

namespace fin {

struct StageArgs {
    const double* qin;     // stage input planes
    const double* A;       // a1 term (may alias qin); nullptr = term absent
    const double* B;       // a2 term; nullptr = term absent
    double* qout;          // output planes (never aliases qin)
    double a1, a2, bdt;    // bdt = beta*dt
    int mx, my;
    size_t plane;          // elements per component plane (>= mx*my)
    double rdx, rdy;       // 1/dx, 1/dy
    double gamma, eps, pw, alpha_scaling;
    const double* alpha_in;   // [2] global alpha of q_in (x, y); nullptr = local LLF
    double* alpha_out;        // [2] max cell speed of q_out; nullptr = skip
    double* smax_out;         // [2] max face speed over GetCFL's faces; nullptr = skip
    double* face_alpha_x;     // optional per-face alpha, (mx+1)*my, face-major i then j
    double* face_alpha_y;     // optional per-face alpha, mx*(my+1)
    unsigned int* status;     // bit 0: non-finite speed, bit 1: negative p or rho
    int bc[4];                // xlow, xhigh, ylow, yhigh
};

template <int TI_, int TJ_, int NT_>
struct TileCfg {
    static constexpr int TI = TI_, TJ = TJ_, NT = NT_, H = 3;
    static constexpr int RI = TI + 2 * H, RJ = TJ + 2 * H;
    static constexpr int NFX = (TI + 1) * TJ, NFY = TI * (TJ + 1);
    // byte offset of the reduction scratch (after the five arrays, 16-B aligned)
    template <class R>
    __host__ __device__ static constexpr size_t red_offset()
    {
        return (sizeof(R) * MEQN * (size_t(RI) * RJ + size_t(RI) * TJ + size_t(TI) * RJ +
                                    size_t(TI + 1) * TJ + size_t(TI) * (TJ + 1)) + 15) / 16 * 16;
    }
    template <class R>
    __host__ __device__ static constexpr size_t smem_bytes() { return red_offset<R>() + 4 * (NT / 32) * sizeof(double); }
};

template <class R, int VER, bool P2, class Cfg>
__global__ void __launch_bounds__(Cfg::NT, 1) k_stage(const StageArgs a)
{
    constexpr int TI = Cfg::TI, TJ = Cfg::TJ, NT = Cfg::NT, H = Cfg::H;
    constexpr int RI = Cfg::RI, RJ = Cfg::RJ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* qs = reinterpret_cast<R*>(smem_raw);
    R* fs = qs + MEQN * RI * RJ;
    R* gs = fs + MEQN * RI * TJ;
    R* Fh = gs + MEQN * TI * RJ;
    R* Gh = Fh + MEQN * (TI + 1) * TJ;
    double* red = reinterpret_cast<double*>(smem_raw + Cfg::template red_offset<R>());

    const int tid = threadIdx.x;
    const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
    const int mx = a.mx, my = a.my;
    const R gamma = R(a.gamma);

    // ---- phase 0: load the tile + halo, boundary conditions by remap ----
    for (int e = tid; e < RI * RJ; e += NT) {
        const int ii = e / RJ, jj = e - ii * RJ;
        const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
        if (!xin && !yin) continue;
        const int gi = bc_remap(i0 + ii - H, mx, a.bc[0], a.bc[1]);
        const int gj = bc_remap(j0 + jj - H, my, a.bc[2], a.bc[3]);
        const size_t g = size_t(gi) * my + gj;
#pragma unroll
        for (int m = 0; m < MEQN; m++) qs[m * RI * RJ + e] = R(__ldg(a.qin + m * a.plane + g));
    }
    __syncthreads();

    // ---- phase 1: FluxFunc once per cell of the cross-shaped stencil region ----
    for (int e = tid; e < RI * RJ; e += NT) {
        const int ii = e / RJ, jj = e - ii * RJ;
        const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
        if (!xin && !yin) continue;
        R Q[MEQN], f[MEQN], g[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) Q[m] = qs[m * RI * RJ + e];
        Euler::flux(gamma, Q, f, g);
        if (yin) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) fs[m * RI * TJ + ii * TJ + (jj - H)] = f[m];
        }
        if (xin) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) gs[m * TI * RJ + (ii - H) * RJ + jj] = g[m];
        }
    }
    __syncthreads();

    // ---- phase 2: one thread per face (x faces then y faces) ----
    const R eps = R(a.eps), pw = R(a.pw), ascale = R(a.alpha_scaling);
    const R ag1 = a.alpha_in ? R(a.alpha_in[0]) : R(0);
    const R ag2 = a.alpha_in ? R(a.alpha_in[1]) : R(0);
    R smax_x = R(0), smax_y = R(0);
    bool neg = false, nonfinite = false;
    for (int w = tid; w < Cfg::NFX + Cfg::NFY; w += NT) {
        const bool isx = w < Cfg::NFX;
        int fi, fj, qbase, qstr, fbase, fstr, fplane;
        const R* fl;
        if (isx) {
            fi = w / TJ; fj = w - fi * TJ;            // face between rows fi-1, fi of the tile
            qbase = (H + fi) * RJ + (H + fj); qstr = RJ;
            fl = fs; fbase = (H + fi) * TJ + fj; fstr = TJ; fplane = RI * TJ;
        } else {
            const int v = w - Cfg::NFX;
            fi = v / (TJ + 1); fj = v - fi * (TJ + 1);  // face between cols fj-1, fj
            qbase = (H + fi) * RJ + (H + fj); qstr = 1;
            fl = gs; fbase = fi * RJ + (H + fj); fstr = 1; fplane = TI * RJ;
        }
        const int cn = isx ? 1 : 2, ct = isx ? 2 : 1;   // normal / tangential momentum
        // Face average (ConstructL.cpp:72-77) in the normal frame.
        R Ql[MEQN], Qr[MEQN], Qa[MEQN];
        {
            const int ml[MEQN] = {0, cn, ct, 3, 4};
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                Qr[m] = qs[ml[m] * RI * RJ + qbase];
                Ql[m] = qs[ml[m] * RI * RJ + qbase - qstr];
                Qa[m] = R(0.5) * (Qr[m] + Ql[m]);
            }
        }
        // Local wave speed (SetWaveSpd.cpp) and LLF alpha (ConstructL.cpp:172-174).
        const typename Euler::Cell<R> cl = Euler::cell(gamma, Ql), cr = Euler::cell(gamma, Qr);
        const R sloc = Euler::speed(gamma, cl, cr, &neg);
        const R alpha = Max(isx ? ag1 : ag2, sloc);
        if (!(alpha <= R(1e30))) nonfinite = true;
        const R la = ascale * alpha;
        const typename Euler::Eig<R> ev = Euler::eig(gamma, Qa);
        // Project the 6-point stencil (ConstructL.cpp:140-141) and split
        // (:179-185): gp_k(s) uses points s = 0..4, gm_k(s) points 5-s.
        R gp[MEQN][5], gm[MEQN][5];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            R Q[MEQN], F[MEQN], W[MEQN], G[MEQN];
            const int ml[MEQN] = {0, cn, ct, 3, 4};
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                Q[m] = qs[ml[m] * RI * RJ + qbase + (s - 3) * qstr];
                F[m] = fl[ml[m] * fplane + fbase + (s - 3) * fstr];
            }
            Euler::left(ev, Q, W);
            Euler::left(ev, F, G);
#pragma unroll
            for (int k = 0; k < MEQN; k++) {
                if (s < 5) gp[k][s] = R(0.5) * (G[k] + la * W[k]);
                if (s > 0) gm[k][5 - s] = R(0.5) * (G[k] - la * W[k]);
            }
        }
        R gh[MEQN], fh[MEQN];
#pragma unroll
        for (int k = 0; k < MEQN; k++)
            gh[k] = weno5<R, VER, P2>(gp[k], eps, pw) + weno5<R, VER, P2>(gm[k], eps, pw);
        Euler::right(ev, gh, fh);
        // Back to (rho, rho u, rho v, rho w, E) and store.
        if (isx) {
            const R o[MEQN] = {fh[0], fh[1], fh[2], fh[3], fh[4]};
#pragma unroll
            for (int m = 0; m < MEQN; m++) Fh[m * (TI + 1) * TJ + fi * TJ + fj] = o[m];
            const int gfi = i0 + fi, gj = j0 + fj;
            // GetCFL's Max skips NaN entries (Max(NaN, c) = c), so only
            // finite face speeds enter the CFL maximum.
            if (gfi < mx && gj < my && alpha <= R(1e30)) smax_x = Max(smax_x, alpha);
            if (a.face_alpha_x && gfi <= mx && gj < my) a.face_alpha_x[size_t(gfi) * my + gj] = double(alpha);
        } else {
            const R o[MEQN] = {fh[0], fh[2], fh[1], fh[3], fh[4]};
#pragma unroll
            for (int m = 0; m < MEQN; m++) Gh[m * TI * (TJ + 1) + fi * (TJ + 1) + fj] = o[m];
            const int gi = i0 + fi, gfj = j0 + fj;
            if (gi < mx && gfj < my && alpha <= R(1e30)) smax_y = Max(smax_y, alpha);
            if (a.face_alpha_y && gi < mx && gfj <= my) a.face_alpha_y[size_t(gi) * (my + 1) + gfj] = double(alpha);
        }
    }
    __syncthreads();

    // ---- phase 3: flux difference, stage update, next-stage wave speed ----
    double cs_x = 0.0, cs_y = 0.0;
    const double gam = a.gamma;
    for (int c = tid; c < TI * TJ; c += NT) {
        const int ci = c / TJ, cj = c - ci * TJ;
        const int gi = i0 + ci, gj = j0 + cj;
        if (gi >= mx || gj >= my) continue;
        const size_t g = size_t(gi) * my + gj;
        double qn[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            // ConstructL.cpp:396-398
            const double f1 = Fh[m * (TI + 1) * TJ + (ci + 1) * TJ + cj], f0 = Fh[m * (TI + 1) * TJ + ci * TJ + cj];
            const double g1 = Gh[m * TI * (TJ + 1) + ci * (TJ + 1) + cj + 1], g0 = Gh[m * TI * (TJ + 1) + ci * (TJ + 1) + cj];
            double L = -(f1 - f0) * a.rdx;
            L = L - (g1 - g0) * a.rdy;
            double v = 0.0;
            if (a.A) v = a.a1 * a.A[m * a.plane + g];
            if (a.B) v = v + a.a2 * a.B[m * a.plane + g];
            v = v + a.bdt * L;
            qn[m] = v;
            a.qout[m * a.plane + g] = v;
        }
        if (a.alpha_out) {
            // GlobalWaveSpd.cpp:71-76 on the new state, both directions.
            const double qy[MEQN] = {qn[0], qn[2], qn[1], qn[3], qn[4]};
            const double sx = Euler::cell_speed(Euler::cell(gam, qn));
            const double sy = Euler::cell_speed(Euler::cell(gam, qy));
            if (!(sx <= 1e300) || !(sy <= 1e300)) nonfinite = true;
            if (sx <= 1e300) cs_x = Max(cs_x, sx);
            if (sy <= 1e300) cs_y = Max(cs_y, sy);
        }
    }

    // ---- block reductions of the four maxima, one atomic each ----
    double v4[4] = {double(smax_x), double(smax_y), cs_x, cs_y};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        // Non-finite speeds were flagged per value above (a NaN does not
        // survive Max(NaN, b) = b), so the reduction only sees finite ones.
        double v = v4[k] <= 1e300 ? v4[k] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = Max(v, __shfl_xor_sync(0xffffffffu, v, o));
        v4[k] = v;
    }
    if ((tid & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) red[(tid >> 5) * 4 + k] = v4[k];
    }
    if (neg) atomicOr(a.status, 2u);
    if (nonfinite) atomicOr(a.status, 1u);
    __syncthreads();
    if (tid < 4) {
        double v = 0.0;
        for (int wv = 0; wv < NT / 32; wv++) v = Max(v, red[wv * 4 + tid]);
        double* dst = tid < 2 ? a.smax_out : a.alpha_out;
        if (dst) atomic_max_nonneg(dst + (tid & 1), v);
    }
}

// GlobalWaveSpd (lib/2d/GlobalWaveSpd.cpp:52-78) on a state already in HBM:
// grid-stride over interior cells, block max, one atomicMax per block.
__global__ void k_wave_spd_max(const double* q, int mx, int my, size_t plane, double gamma,
                               double* alpha_out, unsigned int* status);

// Reference ghosted AoS (i, j, m) <-> device planes.
__global__ void k_aos_to_planes(const double* aos, double* planes, int mx, int my, int mbc, size_t plane);
__global__ void k_planes_to_aos(const double* planes, double* aos, int mx, int my, int mbc, size_t plane,
                                int bc0, int bc1, int bc2, int bc3);

}  // namespace fin
