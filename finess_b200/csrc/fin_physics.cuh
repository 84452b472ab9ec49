// The application callback surface on the device: ConstructL + UpdateSoln
// templated on a physics policy that an application writes.
//
// FINESS applications supply FluxFunc, SetWaveSpd, ProjectLeftEig and
// ProjectRightEig (lib/2d/ConstructL.h:8-23) and link them into lib/2d's
// ConstructL.  Here an application supplies the same callbacks as a policy
// struct of __device__ member functions, point by point, and instantiates
// k_phys_stage<Policy, ...> (and the host driver of fin_physics_host.h) in
// its own translation unit:
//
//   struct MyPhysics {
//       static constexpr int MEQN = ...;                    // meqn
//       // FluxFunc (ConstructL.h:8) at one point (x, y): both flux
//       // components, f = flux(:,:,1), g = flux(:,:,2)
//       __device__ void flux(double x, double y, const double* q, double* f, double* g) const;
//       // SetWaveSpd (ConstructL.h:20-23): the speeds s1 <= s2 at the face
//       // with unit normal (nx, ny) at xedge = (x, y) between states ql, qr
//       __device__ void wave_speed(double nx, double ny, double x, double y, const double* ql,
//                                  const double* qr, double& s1, double& s2) const;
//       // ProjectLeftEig / ProjectRightEig (ConstructL.h:12-15) at the face
//       // average qa in direction ixy (1: x, 2: y), split into the per-face
//       // set-up and the per-point projection:
//       struct Face { ... };
//       __device__ Face face(int ixy, const double* qa) const;
//       __device__ void left(const Face& f, const double* v, double* w) const;    // w = L v
//       __device__ void right(const Face& f, const double* w, double* v) const;   // v = R w
//   };
//
// The policy object is passed by value to the kernels, so its fields carry
// the application's parameters (the reference reads them from
// global_ini_params).  Aux arrays are not carried (maux = 0).
//
// The stage follows lib/2d/ConstructL.cpp:62-401 step by step for every face
// (x faces :62-208, y faces :214-358): the face average Qavg = 0.5 (q_i +
// q_{i-1}), the six-point stencil's w = L q and g = L f, the local speed and
// alpha = max(alpha_global, |s1|, |s2|), gp = 0.5 (g + l w) on points 0..4 and
// gm = 0.5 (g - l w) on points 5..1 with l = alpha_scaling alpha, the WENO5
// reconstructions of every field, Fhat = R (WENO(gp) + WENO(gm)); then
// L = -(F_{i+1} - F_i)/dx - (G_{j+1} - G_j)/dy (:390-401) and the update
// q_out = a1 A + a2 B + (beta dt) L (UpdateSoln.cpp:29-35), with the face-speed
// maxima for GetCFL and the next stage's global alpha (GlobalWaveSpd.cpp:
// 52-78) in the epilogue.  FP64.  One 16 x 16 tile per CTA staged in shared
// memory with a 3-cell halo (boundary conditions as an index remap), FluxFunc
// once per cell, one thread per face.
//
// This is the general path: the library's own Euler and MHD physics run
// through hand-specialised kernels (fin_stage.cuh, fin_mhd.cuh) and the Euler
// callbacks are also given below as a policy (EulerPhys) that runs through
// this template.
#pragma once
#include <cuda_runtime.h>
#include "fin_device.cuh"

namespace fin {
namespace phys {

struct StageArgs {
    const double* qin;   // stage input planes, plane m at qin + m * plane, cell (i, j) at i * my + j
    const double* A;     // a1 term (nullptr: absent)
    const double* B;     // a2 term (nullptr: absent)
    double* qout;
    double a1, a2, bdt;
    int mx, my;
    size_t plane;
    double xlow, ylow, dx, dy;
    double eps, pw, alpha_scaling;
    const double* alpha_in;   // [2] global alpha of qin; nullptr: local LLF
    double* alpha_out;        // [2] GlobalWaveSpd of qout; nullptr: skip
    double* smax_out;         // [2] face-speed maxima over GetCFL's faces
    double* face_alpha_x;     // optional per-face alpha, (mx+1) x my
    double* face_alpha_y;     // optional per-face alpha, mx x (my+1)
    unsigned* status;         // bit 0: non-finite speed
    int bc[4];
};

template <int M>
struct Tile {
    static constexpr int TI = 16, TJ = 16, H = 3, RI = TI + 2 * H, RJ = TJ + 2 * H, NT = 256;
    static constexpr int NFX = (TI + 1) * TJ, NFY = TI * (TJ + 1);
    static constexpr size_t Q = 0;                                 // [M][RI][RJ]
    static constexpr size_t F = Q + size_t(M) * RI * RJ;           // [M][RI][TJ]   f of the x stencils
    static constexpr size_t G = F + size_t(M) * RI * TJ;           // [M][TI][RJ]   g of the y stencils
    static constexpr size_t FH = G + size_t(M) * TI * RJ;          // [M][TI+1][TJ]
    static constexpr size_t GH = FH + size_t(M) * (TI + 1) * TJ;   // [M][TI][TJ+1]
    static constexpr size_t RED = GH + size_t(M) * TI * (TJ + 1);  // [NT/32][4]
    static constexpr size_t BYTES = (RED + 4 * (NT / 32)) * sizeof(double);
};

// The WENO5 reconstruction the parameters name (lib/WenoReconstruct.cpp:
// JS5 90-141, Z5 385-438, FD5 580-616).
template <int VER, bool P2>
__device__ __forceinline__ double weno(const double* u, double eps, double pw)
{
    return weno5<double, VER, P2>(u, eps, pw);
}

template <class Phys, int VER, bool P2>
__global__ void __launch_bounds__(256, 1) k_phys_stage(const __grid_constant__ StageArgs a, const Phys phys)
{
    constexpr int M = Phys::MEQN;
    using T = Tile<M>;
    constexpr int TI = T::TI, TJ = T::TJ, H = T::H, RI = T::RI, RJ = T::RJ, NT = T::NT;
    constexpr int PQ = RI * RJ;
    extern __shared__ __align__(16) double sm[];
    double* qs = sm + T::Q;
    double* fs = sm + T::F;
    double* gs = sm + T::G;
    double* Fh = sm + T::FH;
    double* Gh = sm + T::GH;
    double* red = sm + T::RED;
    const int tid = threadIdx.x;
    const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
    const int mx = a.mx, my = a.my;

    // ---- the tile + halo (the cross region), boundary conditions by remap ----
    for (int e = tid; e < PQ; e += NT) {
        const int ii = e / RJ, jj = e - ii * RJ;
        const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
        if (!xin && !yin) continue;
        const int gi = bc_remap(i0 + ii - H, mx, a.bc[0], a.bc[1]);
        const int gj = bc_remap(j0 + jj - H, my, a.bc[2], a.bc[3]);
        const size_t g = size_t(gi) * my + gj;
        for (int m = 0; m < M; m++) qs[m * PQ + e] = a.qin[m * a.plane + g];
    }
    __syncthreads();
    // ---- FluxFunc once per cell of the cross region, at its cell centre ----
    for (int e = tid; e < PQ; e += NT) {
        const int ii = e / RJ, jj = e - ii * RJ;
        const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
        if (!xin && !yin) continue;
        double q[M], f[M], g[M];
        for (int m = 0; m < M; m++) q[m] = qs[m * PQ + e];
        // ConstructL.cpp:100-101: xlow + double(is)*dx - 0.5*dx (1-based is)
        const int ci = i0 + ii - H + 1, cj = j0 + jj - H + 1;
        const double x = a.xlow + double(ci) * a.dx - 0.5 * a.dx, y = a.ylow + double(cj) * a.dy - 0.5 * a.dy;
        phys.flux(x, y, q, f, g);
        if (yin)
            for (int m = 0; m < M; m++) fs[m * RI * TJ + ii * TJ + (jj - H)] = f[m];
        if (xin)
            for (int m = 0; m < M; m++) gs[m * TI * RJ + (ii - H) * RJ + jj] = g[m];
    }
    __syncthreads();
    // ---- one thread per face ----
    const double ag1 = a.alpha_in ? a.alpha_in[0] : 0.0, ag2 = a.alpha_in ? a.alpha_in[1] : 0.0;
    double smax_x = 0.0, smax_y = 0.0;
    bool nonfinite = false;
    for (int w = tid; w < T::NFX + T::NFY; w += NT) {
        const bool isx = w < T::NFX;
        int fi, fj, qb, qst, fb, fst, fpl;
        const double* fl;
        if (isx) {
            fi = w / TJ; fj = w - fi * TJ;            // face between rows fi-1 and fi
            qb = (H + fi) * RJ + (H + fj); qst = RJ;
            fl = fs; fb = (H + fi) * TJ + fj; fst = TJ; fpl = RI * TJ;
        } else {
            const int v = w - T::NFX;
            fi = v / (TJ + 1); fj = v - fi * (TJ + 1);   // face between columns fj-1 and fj
            qb = (H + fi) * RJ + (H + fj); qst = 1;
            fl = gs; fb = fi * RJ + (H + fj); fst = 1; fpl = TI * RJ;
        }
        const int gi = i0 + fi, gj = j0 + fj;           // 0-based global face index
        double ql[M], qr[M], qa[M];
        for (int m = 0; m < M; m++) {
            qr[m] = qs[m * PQ + qb];
            ql[m] = qs[m * PQ + qb - qst];
            qa[m] = 0.5 * (qr[m] + ql[m]);              // ConstructL.cpp:73-77
        }
        // xedge of ConstructL.cpp:153-154 (x faces) / :303-304 (y faces)
        const double xe = a.xlow + double(gi + 1) * a.dx - 0.5 * a.dx;
        const double ye = a.ylow + double(gj + 1) * a.dy - 0.5 * a.dy;
        double s1, s2;
        phys.wave_speed(isx ? 1.0 : 0.0, isx ? 0.0 : 1.0, xe, ye, ql, qr, s1, s2);
        const double alpha = Max(isx ? ag1 : ag2, Max(fabs(s1), fabs(s2)));
        if (!(alpha <= 1e300)) nonfinite = true;
        const double la = a.alpha_scaling * alpha;
        const typename Phys::Face fc = phys.face(isx ? 1 : 2, qa);
        double gp[M][5], gm[M][5];
        for (int s = 0; s < 6; s++) {
            double q[M], f[M], wv[M], gv[M];
            for (int m = 0; m < M; m++) {
                q[m] = qs[m * PQ + qb + (s - 3) * qst];
                f[m] = fl[m * fpl + fb + (s - 3) * fst];
            }
            phys.left(fc, q, wv);
            phys.left(fc, f, gv);
            // ConstructL.cpp:179-185
            for (int m = 0; m < M; m++) {
                if (s < 5) gp[m][s] = 0.5 * (gv[m] + la * wv[m]);
                if (s > 0) gm[m][5 - s] = 0.5 * (gv[m] - la * wv[m]);
            }
        }
        double gh[M], fh[M];
        for (int m = 0; m < M; m++)
            gh[m] = weno<VER, P2>(gp[m], a.eps, a.pw) + weno<VER, P2>(gm[m], a.eps, a.pw);
        phys.right(fc, gh, fh);
        if (isx) {
            for (int m = 0; m < M; m++) Fh[m * (TI + 1) * TJ + fi * TJ + fj] = fh[m];
            if (gi < mx && gj < my && alpha <= 1e300) smax_x = Max(smax_x, alpha);
            if (a.face_alpha_x && gi <= mx && gj < my) a.face_alpha_x[size_t(gi) * my + gj] = alpha;
        } else {
            for (int m = 0; m < M; m++) Gh[m * TI * (TJ + 1) + fi * (TJ + 1) + fj] = fh[m];
            if (gi < mx && gj < my && alpha <= 1e300) smax_y = Max(smax_y, alpha);
            if (a.face_alpha_y && gi < mx && gj <= my) a.face_alpha_y[size_t(gi) * (my + 1) + gj] = alpha;
        }
    }
    __syncthreads();
    // ---- flux difference, update, next-stage wave speed ----
    double cs_x = 0.0, cs_y = 0.0;
    for (int c = tid; c < TI * TJ; c += NT) {
        const int ci = c / TJ, cj = c - ci * TJ;
        const int gi = i0 + ci, gj = j0 + cj;
        if (gi >= mx || gj >= my) continue;
        const size_t g = size_t(gi) * my + gj;
        // operand loads ahead of the first store (qout may alias A or B as
        // far as the compiler knows)
        double va[M], vb[M];
        for (int m = 0; m < M; m++) {
            va[m] = a.A ? a.A[m * a.plane + g] : 0.0;
            vb[m] = a.B ? a.B[m * a.plane + g] : 0.0;
        }
        double qn[M];
        for (int m = 0; m < M; m++) {
            const double f1 = Fh[m * (TI + 1) * TJ + (ci + 1) * TJ + cj], f0 = Fh[m * (TI + 1) * TJ + ci * TJ + cj];
            const double g1 = Gh[m * TI * (TJ + 1) + ci * (TJ + 1) + cj + 1], g0 = Gh[m * TI * (TJ + 1) + ci * (TJ + 1) + cj];
            // ConstructL.cpp:396-398: divisions, in this order
            double L = __ddiv_rn(-__dsub_rn(f1, f0), a.dx);
            L = __dsub_rn(L, __ddiv_rn(__dsub_rn(g1, g0), a.dy));
            double v = 0.0;
            if (a.A) v = __dmul_rn(a.a1, va[m]);
            if (a.B) v = __dadd_rn(v, __dmul_rn(a.a2, vb[m]));
            v = __dadd_rn(v, __dmul_rn(a.bdt, L));
            qn[m] = v;
            a.qout[m * a.plane + g] = v;
        }
        if (a.alpha_out) {
            // GlobalWaveSpd.cpp:64-76 with Ql = Qr = the new state
            const double x = a.xlow + double(gi + 1) * a.dx - 0.5 * a.dx;
            const double y = a.ylow + double(gj + 1) * a.dy - 0.5 * a.dy;
            double s1, s2;
            phys.wave_speed(1.0, 0.0, x, y, qn, qn, s1, s2);
            const double sx = Max(fabs(s1), fabs(s2));
            phys.wave_speed(0.0, 1.0, x, y, qn, qn, s1, s2);
            const double sy = Max(fabs(s1), fabs(s2));
            if (!(sx <= 1e300) || !(sy <= 1e300)) nonfinite = true;
            if (sx <= 1e300) cs_x = Max(cs_x, sx);
            if (sy <= 1e300) cs_y = Max(cs_y, sy);
        }
    }
    // ---- block maxima, one atomic each ----
    double v4[4] = {smax_x, smax_y, cs_x, cs_y};
    for (int k = 0; k < 4; k++) {
        double v = v4[k];
        for (int o = 16; o > 0; o >>= 1) v = Max(v, __shfl_xor_sync(0xffffffffu, v, o));
        v4[k] = v;
    }
    if ((tid & 31) == 0)
        for (int k = 0; k < 4; k++) red[(tid >> 5) * 4 + k] = v4[k];
    if (nonfinite) atomicOr(a.status, 1u);
    __syncthreads();
    if (tid < 4) {
        double v = 0.0;
        for (int wv = 0; wv < NT / 32; wv++) v = Max(v, red[wv * 4 + tid]);
        double* dst = tid < 2 ? a.smax_out : a.alpha_out;
        if (dst) atomic_max_nonneg(dst + (tid & 1), v);
    }
}

// GlobalWaveSpd (lib/2d/GlobalWaveSpd.cpp:52-78) of a state: SetWaveSpd with
// Ql = Qr = q_ij at every interior cell, both directions; block max, one
// atomic per block.
template <class Phys>
__global__ void k_phys_wave_spd(const Phys phys, const double* q, int mx, int my, size_t plane, double xlow,
                                double ylow, double dx, double dy, double* alpha_out, unsigned* status)
{
    constexpr int M = Phys::MEQN;
    __shared__ double red[2][32];
    double ax = 0.0, ay = 0.0;
    bool nonfinite = false;
    const size_t n = size_t(mx) * my;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const int i = int(g / my), j = int(g - size_t(i) * my);
        double Q[M];
        for (int m = 0; m < M; m++) Q[m] = q[m * plane + g];
        const double x = xlow + double(i + 1) * dx - 0.5 * dx, y = ylow + double(j + 1) * dy - 0.5 * dy;
        double s1, s2;
        phys.wave_speed(1.0, 0.0, x, y, Q, Q, s1, s2);
        const double sx = Max(fabs(s1), fabs(s2));
        phys.wave_speed(0.0, 1.0, x, y, Q, Q, s1, s2);
        const double sy = Max(fabs(s1), fabs(s2));
        if (!(sx <= 1e300) || !(sy <= 1e300)) nonfinite = true;
        if (sx <= 1e300) ax = Max(ax, sx);
        if (sy <= 1e300) ay = Max(ay, sy);
    }
    for (int o = 16; o > 0; o >>= 1) {
        ax = Max(ax, __shfl_xor_sync(0xffffffffu, ax, o));
        ay = Max(ay, __shfl_xor_sync(0xffffffffu, ay, o));
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = ax; red[1][w] = ay; }
    if (nonfinite) atomicOr(status, 1u);
    __syncthreads();
    if (threadIdx.x < 2) {
        double v = 0.0;
        for (int k = 0; k < nw; k++) v = Max(v, red[threadIdx.x][k]);
        atomic_max_nonneg(alpha_out + threadIdx.x, v);
    }
}

// The library's Euler callbacks (apps/2d/euler/lib/FluxFunc.cpp:9-43,
// SetWaveSpd.cpp:11-69, ProjectLeftEig.cpp:9-68, ProjectRightEig.cpp:9-64)
// as a policy: the same device functions the specialised stage kernel uses,
// in the normal frame (rho, m_n, m_t, m_w, E), i.e. with the reference's
// mu/mv swap for ixy = 2 (ProjectLeftEig.cpp:20-32).
struct EulerPhys {
    static constexpr int MEQN = 5;
    double gamma;
    struct Face {
        Euler::Eig<double> e;
        bool swap;
    };
    __device__ void flux(double, double, const double* q, double* f, double* g) const { Euler::flux(gamma, q, f, g); }
    __device__ void wave_speed(double nx, double, double, double, const double* ql, const double* qr, double& s1,
                               double& s2) const
    {
        const bool sw = nx == 0.0;
        const double ln[5] = {ql[0], sw ? ql[2] : ql[1], sw ? ql[1] : ql[2], ql[3], ql[4]};
        const double rn[5] = {qr[0], sw ? qr[2] : qr[1], sw ? qr[1] : qr[2], qr[3], qr[4]};
        const Euler::Cell<double> l = Euler::cell(gamma, ln), r = Euler::cell(gamma, rn);
        // SetWaveSpd.cpp:39-68: arithmetic-mean state, nmag = 1
        const double rho = 0.5 * (l.rho + r.rho), un = 0.5 * (l.un + r.un), press = 0.5 * (l.p + r.p);
        const double c = fsqrt(fabs(gamma * press * rcp(rho)));
        s1 = Min(l.un - l.c, un - c);
        s2 = Max(r.un + r.c, un + c);
    }
    __device__ Face face(int ixy, const double* qa) const
    {
        Face f;
        f.swap = ixy == 2;
        const double qn[5] = {qa[0], f.swap ? qa[2] : qa[1], f.swap ? qa[1] : qa[2], qa[3], qa[4]};
        f.e = Euler::eig(gamma, qn);
        return f;
    }
    __device__ void left(const Face& f, const double* v, double* w) const
    {
        const double vn[5] = {v[0], f.swap ? v[2] : v[1], f.swap ? v[1] : v[2], v[3], v[4]};
        Euler::left(f.e, vn, w);
    }
    __device__ void right(const Face& f, const double* w, double* v) const
    {
        double vn[5];
        Euler::right(f.e, w, vn);
        v[0] = vn[0];
        v[1] = f.swap ? vn[2] : vn[1];
        v[2] = f.swap ? vn[1] : vn[2];
        v[3] = vn[3];
        v[4] = vn[4];
    }
};

}  // namespace phys
}  // namespace fin
