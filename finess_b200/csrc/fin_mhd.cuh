// Ideal MHD stage kernel: one launch per SSP-RK3 stage of the reference's
// MHD application (apps/2d/mhd/lib/FinSolveRK.cpp:176-219) computes, for a
// TI x TJ tile of cells,
//   L(q_in)     ConstructL (lib/2d/ConstructL.cpp:62-401) with the MHD
//               callbacks: FluxFunc.cpp:19-54, SetWaveSpd.cpp:11-90 and the
//               8 x 8 eigenvector projections of ProjectLeftEig.cpp /
//               ProjectRightEig.cpp;
//   Laux(q_in)  ConstructHJ_L_Order1 (ConstructHJ_L.cpp:29-113): WENO
//               Hamilton-Jacobi right-hand side of the potential A3;
//   q_out, A3_out = a1*A + a2*B + (beta*dt)*(L, Laux)   (UpdateSoln.cpp:21-58);
//   B1, B2 of q_out rebuilt from A3_out (AfterStep.cpp:31-56, constrained
//               transport), which needs A3_out two cells beyond the tile: the
//               kernel updates A3 on the tile plus a 2-cell cross halo (the
//               halo values are recomputed by the neighbouring tiles with the
//               same arithmetic, so they agree bit for bit);
// and, in its epilogue, the maxima the next stage needs: the GlobalWaveSpd
// maxima of q_out (lib/2d/GlobalWaveSpd.cpp:52-78), the HJ speeds max|u1|,
// max|u2| of q_out (ConstructHJ_L.cpp:472-497), and the face-speed maxima
// over the faces GetCFL reads (apps/2d/mhd/lib/GetCFL.cpp:54-59).
//
// State in HBM: 9 planes of mx*my FP64 values (j fastest): rho, rho u1,
// rho u2, rho u3, E, B1, B2, B3 and A3.  Boundaries are doubly periodic
// (apps/2d/mhd/orszag_tang/SetBndValues.cpp), applied as an index remap on
// load.
//
// The projections are not the reference's dense 8 x 8 products: with
//   z = (v0, (v_n - u_n v0)/rho, (v_t - u_t v0)/rho, (v_w - u_w v0)/rho,
//        (gamma-1) P, v_bn, v_bt, v_bw),
//   P = |u|^2/2 v0 - u.v_m + v_E - B.v_B,
// the reference's Lmat v (ProjectLeftEig.cpp:179-206) equals ru z, ru being
// its primitive eigenvector rows, and ru has 35 nonzeros in pairs that share
// terms (fast -/+, slow -/+, Alfven -/+), so each row costs a few operations;
// the right projection (ProjectRightEig.cpp:176-203) is the transposed form.
// The per-face scalars are those of ProjectLeftEig.cpp:34-86, in FP64
// evaluated with the reference's own rounding (see mhd_eig_scalars).
#pragma once
#include "fin_device.cuh"
#include "fin_stage.cuh"   // flag masks (flag_wx, row_bits) and linear_face

namespace fin {

constexpr int MHD_NQ = 8;   // rho, rho u1, rho u2, rho u3, E, B1, B2, B3
constexpr int MHD_NP = 9;   // + A3

struct MhdArgs {
    const double* qin;     // stage input (9 planes)
    const double* A;       // a1 operand (9 planes); nullptr = term absent
    const double* B;       // a2 operand; nullptr = term absent
    double* qout;          // output (9 planes; never aliases qin)
    double a1, a2, bdt;    // bdt = beta*dt
    int mx, my;
    size_t plane;
    double rdx, rdy;       // 1/dx, 1/dy
    double ct_y, ct_x;     // 1.0/(12.0*dy), -1.0/(12.0*dx)  (AfterStep.cpp:39-48)
    int ct;                // constrained transport on
    double gamma, eps, pw, alpha_scaling;
    float gamma_f, eps_f, pw_f, alpha_scaling_f;
    double r_sqrt2;        // 1.0/sqrt(2.0)
    double alf_deg, als_deg;   // sin(atan(1.0)/2.0), cos(atan(1.0)/2.0) (ProjectLeftEig.cpp:78-79)
    const double* alpha_in;    // [2] global alpha of q_in (x, y); nullptr = local LLF
    const double* hj_in;       // [2] max |u1|, |u2| of q_in
    double* alpha_out;         // [2] max cell speed of q_out; nullptr = skip
    double* hj_out;            // [2] max |u1|, |u2| of q_out; nullptr = skip
    double* smax_out;          // [2] max face speed over GetCFL's faces
    double* face_alpha_x;      // optional per-face alpha, (mx+1) x my, i-major
    double* face_alpha_y;      // optional per-face alpha, mx x (my+1)
    unsigned int* status;      // bit 0: non-finite speed, bit 1: negative p or rho, bit 2: a tensor-core
                               // wait ran out (indicator)
    const unsigned* flags;     // hybrid form: troubled-face bit masks (flag_wx / flag_wy layout of fin_stage.cuh)
};

// Periodic index wrap: one add or subtract for the indices a tile reaches
// (at most one period outside), the general remap otherwise (grids smaller
// than a tile and its halo).
__device__ __forceinline__ int pwrap(int k, int n)
{
    if (k < 0) k += n;
    else if (k >= n) k -= n;
    if (unsigned(k) >= unsigned(n)) k = bc_remap(k, n, FIN_BC_PERIODIC, FIN_BC_PERIODIC);
    return k;
}

template <class R> struct MPar;
template <> struct MPar<double> {
    __device__ static double gamma(const MhdArgs& a) { return a.gamma; }
    __device__ static double eps(const MhdArgs& a) { return a.eps; }
    __device__ static double pw(const MhdArgs& a) { return a.pw; }
    __device__ static double ascale(const MhdArgs& a) { return a.alpha_scaling; }
};
template <> struct MPar<float> {
    __device__ static float gamma(const MhdArgs& a) { return a.gamma_f; }
    __device__ static float eps(const MhdArgs& a) { return a.eps_f; }
    __device__ static float pw(const MhdArgs& a) { return a.pw_f; }
    __device__ static float ascale(const MhdArgs& a) { return a.alpha_scaling_f; }
};

// Products and sums with the reference's rounding (no contraction), for the
// branch conditions of ProjectLeftEig.cpp:58-86.
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }

// The scalars of ProjectLeftEig.cpp:34-86 at a face-average state Q (normal
// frame).  Near degenerate states the reference's alpha_f, alpha_s and c_s are
// differences of nearly equal numbers (where B_perp -> 0 its alpha_s is
// sqrt(c_f^2 - a^2) of a rounding-level difference); the eigenvectors, and
// through the nonlinear WENO weights the fluxes, follow those rounding bits.
// The FP64 form therefore evaluates this chain in the reference's order with
// IEEE operations and no contraction (EXACT), so that it takes the same
// values.  In FP32 the chain breaks down near the umbilic point (B_perp -> 0,
// a^2 -> B_n^2/rho): c_f^2 - c_s^2 = sqrt(disc) is resolved to ~3e-4 of d
// only, alpha_f and alpha_s become 0/0, and left times right eigenvectors
// departs from the identity (measured: NaN or 2e-4 in FP32, 1e-16 in FP64).
// The FP32 form recomputes such faces' scalars in FP64.
template <class R>
struct MhdEigScalars { R u1, u2, u3, um2, press, a2, cf, cs, af, as, b2, b3; };

template <class T, bool EXACT>
__device__ __forceinline__ void mhd_eig_core(T gamma, const T* Q, MhdEigScalars<T>& e, T& d, bool& umb)
{
    const T rho = Q[0], B1 = Q[5], B2 = Q[6], B3 = Q[7];
    const T bp2 = xadd(xmul(B2, B2), xmul(B3, B3));
    umb = false;
    if (EXACT) {
        e.u1 = xdiv(Q[1], rho); e.u2 = xdiv(Q[2], rho); e.u3 = xdiv(Q[3], rho);
        e.um2 = xmul(T(0.5), xadd(xadd(xmul(e.u1, e.u1), xmul(e.u2, e.u2)), xmul(e.u3, e.u3)));
        const T Bs = xadd(xadd(xmul(B1, B1), xmul(B2, B2)), xmul(B3, B3));
        e.press = xmul(xsub(gamma, T(1)), xsub(xsub(Q[4], xmul(rho, e.um2)), xmul(T(0.5), Bs)));
        e.a2 = xdiv(xmul(gamma, e.press), rho);
        d = xadd(e.a2, xdiv(Bs, rho));
        const T sq = sqrt(xsub(xmul(d, d), xdiv(xmul(xmul(xmul(T(4), e.a2), B1), B1), rho)));
        e.cf = sqrt(xmul(T(0.5), xadd(d, sq)));
        e.cs = sqrt(xmul(T(0.5), xsub(d, sq)));
        if (bp2 <= T(1.0e-12)) umb = fabs(xsub(e.a2, xdiv(xmul(B1, B1), rho))) <= T(1.0e-12);
        const T cf2 = xmul(e.cf, e.cf), cs2 = xmul(e.cs, e.cs);
        const T den = sqrt(fabs(xsub(cf2, cs2)));
        e.af = xdiv(sqrt(fabs(xsub(e.a2, cs2))), den);
        e.as = xdiv(sqrt(fabs(xsub(cf2, e.a2))), den);
    } else {
        const T ir = rcp(rho);
        e.u1 = Q[1] * ir; e.u2 = Q[2] * ir; e.u3 = Q[3] * ir;
        e.um2 = T(0.5) * (e.u1 * e.u1 + e.u2 * e.u2 + e.u3 * e.u3);
        const T Bs = B1 * B1 + B2 * B2 + B3 * B3;
        e.press = (gamma - T(1)) * (Q[4] - rho * e.um2 - T(0.5) * Bs);
        e.a2 = gamma * e.press * ir;
        d = e.a2 + Bs * ir;
        // clamped: an approximate square root may exceed d for d^2 minus a
        // tiny term (B_n -> 0)
        const T sq = fsqrt(Max(d * d - T(4) * e.a2 * (B1 * B1) * ir, T(0)));
        e.cf = fsqrt(T(0.5) * (d + sq));
        e.cs = fsqrt(Max(T(0.5) * (d - sq), T(0)));
        if (bp2 <= T(1.0e-12)) umb = fabs(e.a2 - B1 * B1 * ir) <= T(1.0e-12);
        const T cf2 = e.cf * e.cf, cs2 = e.cs * e.cs;
        const T iden = rcp(fsqrt(fabs(cf2 - cs2)));
        e.af = fsqrt(fabs(e.a2 - cs2)) * iden;
        e.as = fsqrt(fabs(cf2 - e.a2)) * iden;
    }
}

template <class R>
__device__ __forceinline__ MhdEigScalars<R> mhd_eig_scalars(const MhdArgs& a, R gamma, const R* Q)
{
    MhdEigScalars<R> e;
    R d;
    bool umb;
    if (sizeof(R) == 8) {
        mhd_eig_core<R, true>(gamma, Q, e, d, umb);
    } else {
        mhd_eig_core<R, false>(gamma, Q, e, d, umb);
        if (!(e.cf * e.cf - e.cs * e.cs > R(1.0e-2) * d)) {
            // near the umbilic point: the same scalars in FP64
            double Qd[MHD_NQ];
#pragma unroll
            for (int m = 0; m < MHD_NQ; m++) Qd[m] = double(Q[m]);
            MhdEigScalars<double> ed;
            double dd;
            mhd_eig_core<double, false>(a.gamma, Qd, ed, dd, umb);
            e.u1 = R(ed.u1); e.u2 = R(ed.u2); e.u3 = R(ed.u3); e.um2 = R(ed.um2);
            e.press = R(ed.press); e.a2 = R(ed.a2); e.cf = R(ed.cf); e.cs = R(ed.cs);
            e.af = R(ed.af); e.as = R(ed.as);
        }
    }
    const R B2 = Q[6], B3 = Q[7];
    const R rs2 = R(a.r_sqrt2);
    if (xadd(xmul(B2, B2), xmul(B3, B3)) <= R(1.0e-12)) {
        e.b2 = rs2;
        e.b3 = rs2;
    } else {
        const R ib = rcp(fsqrt(B2 * B2 + B3 * B3));
        e.b2 = B2 * ib;
        e.b3 = B3 * ib;
    }
    if (umb) {
        e.af = R(a.alf_deg);
        e.as = R(a.als_deg);
    }
    return e;
}

// Per-face coefficients of the left projection passes (normal frame; the
// density and (gamma-1) factors of z folded in).
template <class R>
struct MhdFace {
    R u1, u2, u3, um2, B1, B2, B3, b2, b3;
    R kfn, ksu, kfp, ksb;   // fast rows 0 / 7: dn, S_u, P, S_b
    R ksn, kfu, ksp, kfb;   // slow rows 2 / 5
    R ra, rb;               // Alfven rows 1 / 6: T_u, T_b
    R ie;                   // entropy row 3: v0 - ie P
};
// The right projection's coefficients, parked in shared memory while the
// left passes run.
enum { MR_RHO, MR_AF, MR_AS, MR_CF, MR_CS, MR_BETA1, MR_GP, MR_ASR, MR_SR2, MR_N };

template <class R>
__device__ __forceinline__ void mhd_face_setup(const MhdArgs& a, R gamma, const R* Q, MhdFace<R>& f, R* rec,
                                               int rstride, bool& neg)
{
    const R gm1 = gamma - R(1);
    const R rho = Q[0];
    const MhdEigScalars<R> e = mhd_eig_scalars<R>(a, gamma, Q);
    f.u1 = e.u1; f.u2 = e.u2; f.u3 = e.u3; f.um2 = e.um2;
    f.B1 = Q[5]; f.B2 = Q[6]; f.B3 = Q[7];
    f.b2 = e.b2; f.b3 = e.b3;
    if (e.press < R(0) || rho < R(0)) neg = true;
    const R ir = rcp(rho);
    const R asnd = fsqrt(e.a2);   // the reference's sqrt: NaN when a2 < 0
    const R beta1 = f.B1 < R(0) ? R(-1) : R(1);
    const R af = e.af, as = e.as, cf = e.cf, cs = e.cs;
    const R rs2 = R(a.r_sqrt2);
    const R rsq = fsqrt(rho);
    const R ia2 = rcp(e.a2);
    const R h = R(0.5) * ia2 * ir;             // 1/(2 a^2 rho)
    const R hb = R(0.5) * rcp(rsq * asnd);     // 1/(2 sqrt(rho) a)
    f.kfn = af * cf * h;
    f.ksu = as * cs * beta1 * h;
    f.kfp = af * h * gm1;
    f.ksb = as * hb;
    f.ksn = as * cs * h;
    f.kfu = af * cf * beta1 * h;
    f.ksp = as * h * gm1;
    f.kfb = af * hb;
    f.ra = rs2 * ir;
    f.rb = rs2 * rcp(rsq);
    f.ie = gm1 * ia2;
    if (!rec) return;
    rec[MR_RHO * rstride] = rho;
    rec[MR_AF * rstride] = af;
    rec[MR_AS * rstride] = as;
    rec[MR_CF * rstride] = cf;
    rec[MR_CS * rstride] = cs;
    rec[MR_BETA1 * rstride] = beta1;
    rec[MR_GP * rstride] = gamma * e.press;
    rec[MR_ASR * rstride] = asnd * rsq;
    rec[MR_SR2 * rstride] = rsq * rs2;
}

// Shared pieces of the projection of one normal-frame vector v.
template <class R>
__device__ __forceinline__ R mhd_P(const MhdFace<R>& f, const R* v)
{
    return f.um2 * v[0] - f.u1 * v[1] - f.u2 * v[2] - f.u3 * v[3] + v[4] - f.B1 * v[5] - f.B2 * v[6] - f.B3 * v[7];
}
// fast (k = 0) or slow (k = 1) pair of characteristic values (rows 0/7 or 2/5)
template <class R>
__device__ __forceinline__ void mhd_left_fs(const MhdFace<R>& f, int k, const R* v, R& wm, R& wp)
{
    const R dn = v[1] - f.u1 * v[0];
    const R dt = v[2] - f.u2 * v[0];
    const R dw = v[3] - f.u3 * v[0];
    const R P = mhd_P(f, v);
    const R Su = f.b2 * dt + f.b3 * dw;
    const R Sb = f.b2 * v[6] + f.b3 * v[7];
    if (k == 0) {
        const R s = f.kfp * P + f.ksb * Sb, t = f.ksu * Su - f.kfn * dn;
        wm = s + t;   // row 0
        wp = s - t;   // row 7
    } else {
        const R s = f.ksp * P - f.kfb * Sb, t = f.ksn * dn + f.kfu * Su;
        wm = s - t;   // row 2
        wp = s + t;   // row 5
    }
}
// both pairs at once (rows 0 / 7 and 2 / 5), sharing dn, S_u, P, S_b
template <class R>
__device__ __forceinline__ void mhd_left_fs4(const MhdFace<R>& f, const R* v, R& w0, R& w7, R& w2, R& w5)
{
    const R dn = v[1] - f.u1 * v[0];
    const R dt = v[2] - f.u2 * v[0];
    const R dw = v[3] - f.u3 * v[0];
    const R P = mhd_P(f, v);
    const R Su = f.b2 * dt + f.b3 * dw;
    const R Sb = f.b2 * v[6] + f.b3 * v[7];
    R s = f.kfp * P + f.ksb * Sb, t = f.ksu * Su - f.kfn * dn;
    w0 = s + t;
    w7 = s - t;
    s = f.ksp * P - f.kfb * Sb;
    t = f.ksn * dn + f.kfu * Su;
    w2 = s - t;
    w5 = s + t;
}
// Alfven pair (rows 1 / 6)
template <class R>
__device__ __forceinline__ void mhd_left_alf(const MhdFace<R>& f, const R* v, R& wm, R& wp)
{
    const R dt = v[2] - f.u2 * v[0];
    const R dw = v[3] - f.u3 * v[0];
    const R Tu = f.ra * (f.b2 * dw - f.b3 * dt);
    const R Tb = f.rb * (f.b2 * v[7] - f.b3 * v[6]);
    wm = Tu + Tb;
    wp = Tu - Tb;
}
// entropy and divergence rows (3 / 4)
template <class R>
__device__ __forceinline__ void mhd_left_ent(const MhdFace<R>& f, const R* v, R& w3, R& w4)
{
    w3 = v[0] - f.ie * mhd_P(f, v);
    w4 = v[5];
}

// The stencil of one face in shared memory: q and the half flux of the six
// points (normal-frame component order through perm).
template <class R>
struct MhdStencil {
    const R* qs;
    const R* fl;
    const int* perm;
    int qbase, qstr, fbase, fstr, fplane, PQ;
    R lah;
};

// One sweep over the stencil: K characteristic values of v+ = 0.5 f + lah q
// at points 0..4 into p, and of v- = 0.5 f - lah q at points 5..1 into m
// (reversed), as ConstructL.cpp:179-185 orders them.
template <class R, int K, class Left>
__device__ __forceinline__ void mhd_sweep(const MhdStencil<R>& st, const Left& left, R (&p)[K][5], R (&m)[K][5])
{
#pragma unroll
    for (int s = 0; s < 6; s++) {
        // keep the compiler from hoisting every point's loads ahead of the arithmetic
        asm volatile("" ::: "memory");
        const int oq = st.qbase + (s - 3) * st.qstr, of = st.fbase + (s - 3) * st.fstr;
        R q[MHD_NQ], fh[MHD_NQ];
#pragma unroll
        for (int c = 0; c < MHD_NQ; c++) {
            q[c] = st.qs[st.perm[c] * st.PQ + oq];
            fh[c] = st.fl[st.perm[c] * st.fplane + of];
        }
        if (s < 5) {
            R v[MHD_NQ], w[K];
#pragma unroll
            for (int c = 0; c < MHD_NQ; c++) v[c] = fh[c] + st.lah * q[c];
            left(v, w);
#pragma unroll
            for (int k = 0; k < K; k++) p[k][s] = w[k];
        }
        if (s > 0) {
            R v[MHD_NQ], w[K];
#pragma unroll
            for (int c = 0; c < MHD_NQ; c++) v[c] = fh[c] - st.lah * q[c];
            left(v, w);
#pragma unroll
            for (int k = 0; k < K; k++) m[k][5 - s] = w[k];
        }
    }
}

// ghat_k = WENO(p_k) + WENO(m_k) (ConstructL.cpp:191-199) for K fields,
// FIN_MHD_WGROUP fields at a time between scheduling fences.
#ifndef FIN_MHD_WGROUP
#define FIN_MHD_WGROUP 1
#endif
template <class R, int VER, bool P2, int K>
__device__ __forceinline__ void mhd_weno_fields(R (&p)[K][5], R (&m)[K][5], R eps, R pw, R* g)
{
    constexpr int G = FIN_MHD_WGROUP < K ? FIN_MHD_WGROUP : K;
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += G) {
#pragma unroll
        for (int k = k0; k < k0 + G; k++)
#pragma unroll
            for (int t = 0; t < 5; t++) { wfence(p[k][t]); wfence(m[k][t]); }
#pragma unroll
        for (int k = k0; k < k0 + G; k++) g[k] = weno5<R, VER, P2>(p[k], eps, pw) + weno5<R, VER, P2>(m[k], eps, pw);
#pragma unroll
        for (int k = k0; k < k0 + G; k++) wfence(g[k]);
    }
}

template <int TI_, int TJ_, int NT_, int MINB_ = 1>
struct MhdCfg {
    static constexpr int TI = TI_, TJ = TJ_, NT = NT_;
    static constexpr int MINB = MINB_;   // resident blocks per SM the registers are sized for
    static constexpr int H = 3;              // q halo of the WENO stencils
    static constexpr int HA = 5;             // A3 halo (HJ stencils of the 2-cell CT halo)
    static constexpr int HN = 2;             // CT halo of the updated A3
    static constexpr int RI = TI + 2 * H, RJ = TJ + 2 * H;
    static constexpr int PI = TI + 2, PJ = TJ + 2;      // per-cell speed data (halo 1)
    static constexpr int AI = TI + 2 * HA, AJ = TJ + 2 * HA;
    static constexpr int NI = TI + 2 * HN, NJ = TJ + 2 * HN;
    static constexpr int NFX = (TI + 1) * TJ, NFY = TI * (TJ + 1);
    // R arrays: qs [8][RI*RJ], fs [8][RI*TJ], gs [8][TI*RJ], pc [4][PI*PJ],
    // Fh [8][NFX], Gh [8][NFY], rec [MR_N][NT]; then FP64: as [AI*AJ],
    // an [NI*NJ], red [6][NT/32].
    // FP32 faces of a 15 x 16 tile go to threads so that the two half-warps
    // of a warp take face rows 8 apart (ROW8): 8 rows of RJ = 22 (PJ = 18)
    // words are 176 (144) words, 16 modulo 32, so the two rows' words fall
    // in opposite halves of the banks; the x-direction flux rows get a pitch
    // of FSJ = 18 for the same reason.  FP64 keeps the row-by-row order.
    template <class R>
    __host__ __device__ static constexpr bool ROW8() { return sizeof(R) == 4 && TI == 15 && TJ == 16; }
    template <class R>
    __host__ __device__ static constexpr int FSJ() { return ROW8<R>() ? TJ + 2 : TJ; }
    template <class R>
    __host__ __device__ static constexpr size_t NR()
    {
        return size_t(MHD_NQ) * (RI * RJ + RI * FSJ<R>() + TI * RJ + NFX + NFY) + 4 * PI * PJ + size_t(MR_N) * NT;
    }
    template <class R>
    __host__ __device__ static constexpr size_t dbl_offset() { return (NR<R>() * sizeof(R) + 15) / 16 * 16; }
    template <class R>
    __host__ __device__ static constexpr size_t smem_bytes()
    {
        return dbl_offset<R>() + sizeof(double) * (size_t(AI) * AJ + size_t(NI) * NJ + 6 * (NT / 32));
    }
    // Hybrid form, after the above: per-face speeds falpha [NF] (R), the
    // troubled-face list [NF] (short), its count, and the flag windows of the
    // 3 x 3 dilation as row masks (x faces: rows i0-1 .. i0+TI+1, bit c =
    // column j0-1+c, c < TJ+2; y faces: rows i0-1 .. i0+TI, c < TJ+3).
    static constexpr int NF = NFX + NFY;
    static constexpr int FXR = TI + 3, FXC = TJ + 2, FYR = TI + 2, FYC = TJ + 3;
    static_assert(FYC <= 32 && FXR <= 32 && FYR <= 32, "flag row masks are 32-bit words read by one warp each");
    template <class R>
    __host__ __device__ static constexpr size_t hyb_ntrb_offset() { return (NF * sizeof(R) + NF * 2 + 15) / 16 * 16; }
    template <class R>
    __host__ __device__ static constexpr size_t hyb_mask_offset() { return hyb_ntrb_offset<R>() + 16; }
    template <class R>
    __host__ __device__ static constexpr size_t smem_bytes_hyb()
    {
        return smem_bytes<R>() + hyb_mask_offset<R>() + 4 * (FXR + FYR);
    }
};

// Bits of columns c0 .. c0+nb-1 (nb <= 32) of one flag-mask row of nw words,
// columns taken modulo the period (periodic boundaries; the flag arrays hold
// columns 0 .. period-1, y faces also column period, equal to column 0).
__device__ __forceinline__ unsigned mask_row_wrapped(const unsigned* row, int nw, int c0, int nb, int period)
{
    if (c0 >= 0 && c0 + nb <= period) {
        const int k = c0 >> 5;
        const unsigned lo = __ldg(row + k), hi = k + 1 < nw ? __ldg(row + k + 1) : 0u;
        return row_bits(lo, hi, c0) & (nb >= 32 ? 0xffffffffu : ((1u << nb) - 1u));
    }
    unsigned m = 0;
    for (int b = 0; b < nb; b++) {
        int c = c0 + b;
        if (c < 0) c += period;
        else if (c >= period) c -= period;
        m |= ((__ldg(row + (c >> 5)) >> (c & 31)) & 1u) << b;
    }
    return m;
}

// Sweeps over the stencil per face: the fast and slow pairs share dn, S_u, P
// and S_b and take one sweep (40 live values); with FIN_MHD_SWEEPS = 2 the
// Alfven, entropy and divergence rows take a second (3: one sweep each for
// the Alfven pair and the entropy/divergence pair).  Stage ms on B200 at
// 2048^2, FP64 / FP32: a sweep per pair 2.98 / 1.78, three sweeps 2.63 /
// 1.49, two sweeps 2.36 / 1.26 (FP64 then spills ~130 B to L1, still faster).
// Evaluating the WENO pairs of two or four fields between one pair of
// scheduling fences (FIN_MHD_WGROUP) changed nothing measurable.
#ifndef FIN_MHD_SWEEPS
#define FIN_MHD_SWEEPS 2
#endif

template <class R, int VER, bool P2, class Cfg, bool HYB = false>
__global__ void __launch_bounds__(Cfg::NT, Cfg::MINB) k_mhd_stage(const __grid_constant__ MhdArgs a)
{
    constexpr int TI = Cfg::TI, TJ = Cfg::TJ, NT = Cfg::NT, H = Cfg::H;
    constexpr int RI = Cfg::RI, RJ = Cfg::RJ, PQ = RI * RJ;
    constexpr int PI = Cfg::PI, PJ = Cfg::PJ, PP = PI * PJ;
    constexpr int AJ = Cfg::AJ, NJ = Cfg::NJ;
    constexpr int HA = Cfg::HA, HN = Cfg::HN;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    R* qs = reinterpret_cast<R*>(smem_raw);          // [8][RI][RJ]
    R* fs = qs + MHD_NQ * PQ;                        // [8][RI][TJ]  0.5 f
    constexpr int FS = Cfg::template FSJ<R>();
    R* gs = fs + MHD_NQ * RI * FS;                   // [8][TI][RJ]  0.5 g
    R* pc = gs + MHD_NQ * TI * RJ;                   // [4][PI][PJ]  u1, u2, p, cf
    R* Fh = pc + 4 * PP;                             // [8][TI+1][TJ]
    R* Gh = Fh + MHD_NQ * Cfg::NFX;                  // [8][TI][TJ+1]
    R* rec = Gh + MHD_NQ * Cfg::NFY;                 // [MR_N][NT]
    double* as = reinterpret_cast<double*>(smem_raw + Cfg::template dbl_offset<R>());   // [AI][AJ]
    double* an = as + Cfg::AI * AJ;                  // [NI][NJ]
    double* red = an + Cfg::NI * NJ;                 // [NT/32][6]
    unsigned char* hyb_base = smem_raw + Cfg::template smem_bytes<R>();
    unsigned* fxm = reinterpret_cast<unsigned*>(hyb_base + Cfg::template hyb_mask_offset<R>());
    unsigned* fym = fxm + Cfg::FXR;

    const int tid = threadIdx.x;
    const int mx = a.mx, my = a.my;
    const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
    const R gamma = MPar<R>::gamma(a);
    bool neg = false, nonfinite = false;

    // ---- phase 0: q_in on the tile + 3-cell cross halo, A3 on the tile +
    // 5-cell frame (periodic remap) ----
    // All of a thread's loads (the state, A3 of q_in, and A3 of the other
    // stage operands for the update of phase 1b) are issued before its
    // stores: one memory round trip per tile, not one per pass over a region.
    // The operands' part of the A3 update, a1 A + a2 B (UpdateSoln.cpp:42-47),
    // is kept in an[] for phase 1b to add bdt L to.
    {
        constexpr int NQI = (PQ + NT - 1) / NT, NAI = (Cfg::AI * AJ + NT - 1) / NT;
        constexpr int NHI = (Cfg::NI * NJ + NT - 1) / NT;
        double vq[NQI][MHD_NQ], va[NAI], vab[NHI];
#pragma unroll
        for (int it = 0; it < NQI; it++) {
            const int e = tid + it * NT;
            const int ii = e / RJ, jj = e - ii * RJ;
            const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
            if (e < PQ && (xin || yin)) {
                const int gi = pwrap(i0 + ii - H, mx);
                const int gj = pwrap(j0 + jj - H, my);
                const size_t g = size_t(gi) * my + gj;
#pragma unroll
                for (int m = 0; m < MHD_NQ; m++) vq[it][m] = __ldg(a.qin + m * a.plane + g);
            }
        }
#pragma unroll
        for (int it = 0; it < NAI; it++) {
            const int e = tid + it * NT;
            if (e < Cfg::AI * AJ) {
                const int ii = e / AJ, jj = e - ii * AJ;
                const int gi = pwrap(i0 + ii - HA, mx);
                const int gj = pwrap(j0 + jj - HA, my);
                va[it] = __ldg(a.qin + 8 * a.plane + size_t(gi) * my + gj);
            }
        }
#pragma unroll
        for (int it = 0; it < NHI; it++) {
            const int e = tid + it * NT;
            const int ni = e / NJ, nj = e - ni * NJ;
            const int ci = ni - HN, cj = nj - HN;   // tile frame
            const bool xin = ci >= 0 && ci < TI, yin = cj >= 0 && cj < TJ;
            if (e < Cfg::NI * NJ && (xin || yin)) {
                const size_t g = 8 * a.plane + size_t(pwrap(i0 + ci, mx)) * my + pwrap(j0 + cj, my);
                double v = 0.0;
                if (a.A) v = a.a1 * __ldg(a.A + g);
                if (a.B) v = v + a.a2 * __ldg(a.B + g);
                vab[it] = v;
            }
        }
#pragma unroll
        for (int it = 0; it < NQI; it++) {
            const int e = tid + it * NT;
            const int ii = e / RJ, jj = e - ii * RJ;
            const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
            if (e < PQ && (xin || yin)) {
#pragma unroll
                for (int m = 0; m < MHD_NQ; m++) qs[m * PQ + e] = R(vq[it][m]);
            }
        }
#pragma unroll
        for (int it = 0; it < NHI; it++) {
            const int e = tid + it * NT;
            const int ni = e / NJ, nj = e - ni * NJ;
            const int ci = ni - HN, cj = nj - HN;
            const bool xin = ci >= 0 && ci < TI, yin = cj >= 0 && cj < TJ;
            if (e < Cfg::NI * NJ && (xin || yin)) an[e] = vab[it];
        }
#pragma unroll
        for (int it = 0; it < NAI; it++) {
            const int e = tid + it * NT;
            if (e < Cfg::AI * AJ) as[e] = va[it];
        }
    }
    if (HYB) {
        // the flag windows, rows and columns wrapped (doubly periodic), each
        // row dilated over 3 columns
        const int wx = flag_wx(my), wy = flag_wy(my);
        if (tid < Cfg::FXR) {
            int r = i0 - 1 + tid;   // x-face row (faces 0 .. mx, face mx = face 0)
            if (r < 0) r += mx;
            else if (r > mx) r -= mx;
            const unsigned m = mask_row_wrapped(a.flags + size_t(r) * wx, wx, j0 - 1, Cfg::FXC, my);
            fxm[tid] = m | (m >> 1) | (m >> 2);
        } else if (tid >= 32 && tid < 32 + Cfg::FYR) {
            int r = i0 - 1 + (tid - 32);   // y-face row (cell rows 0 .. mx-1)
            if (r < 0) r += mx;
            else if (r >= mx) r -= mx;
            const unsigned m =
                mask_row_wrapped(a.flags + size_t(mx + 1) * wx + size_t(r) * wy, wy, j0 - 1, Cfg::FYC, my);
            fym[tid - 32] = m | (m >> 1) | (m >> 2);
        }
        if (tid == 0) *reinterpret_cast<int*>(hyb_base + Cfg::template hyb_ntrb_offset<R>()) = 0;
    }
    __syncthreads();

    // ---- phase 1a: per cell of the cross region, FluxFunc (FluxFunc.cpp:
    // 19-54) halved for the LLF split, and for the cells next to the tile's
    // faces the per-cell terms of SetWaveSpd.cpp:24-72 ----
    for (int e = tid; e < PQ; e += NT) {
        const int ii = e / RJ, jj = e - ii * RJ;
        const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
        if (!xin && !yin) continue;
        const R rho = qs[e], m1 = qs[PQ + e], m2 = qs[2 * PQ + e], m3 = qs[3 * PQ + e], en = qs[4 * PQ + e];
        const R B1 = qs[5 * PQ + e], B2 = qs[6 * PQ + e], B3 = qs[7 * PQ + e];
        const R ir = rcp(rho);
        const R u1 = m1 * ir, u2 = m2 * ir, u3 = m3 * ir;
        const R Bsq = B1 * B1 + B2 * B2 + B3 * B3;
        const R press = (gamma - R(1)) * (en - R(0.5) * rho * (u1 * u1 + u2 * u2 + u3 * u3) - R(0.5) * Bsq);
        const R Bm = R(0.5) * Bsq;
        const R Bu = u1 * B1 + u2 * B2 + u3 * B3;
        const R eb = en + press + Bm;
        if (yin) {
            const int o = ii * FS + (jj - H);
            constexpr int S = RI * FS;
            fs[o] = R(0.5) * (rho * u1);
            fs[S + o] = R(0.5) * (rho * u1 * u1 + press + Bm - B1 * B1);
            fs[2 * S + o] = R(0.5) * (rho * u1 * u2 - B1 * B2);
            fs[3 * S + o] = R(0.5) * (rho * u1 * u3 - B1 * B3);
            fs[4 * S + o] = R(0.5) * (u1 * eb - B1 * Bu);
            fs[5 * S + o] = R(0);
            fs[6 * S + o] = R(0.5) * (u1 * B2 - u2 * B1);
            fs[7 * S + o] = R(0.5) * (u1 * B3 - u3 * B1);
        }
        if (xin) {
            const int o = (ii - H) * RJ + jj;
            constexpr int S = TI * RJ;
            gs[o] = R(0.5) * (rho * u2);
            gs[S + o] = R(0.5) * (rho * u1 * u2 - B2 * B1);
            gs[2 * S + o] = R(0.5) * (rho * u2 * u2 + press + Bm - B2 * B2);
            gs[3 * S + o] = R(0.5) * (rho * u2 * u3 - B2 * B3);
            gs[4 * S + o] = R(0.5) * (u2 * eb - B2 * Bu);
            gs[5 * S + o] = R(0.5) * (u2 * B1 - u1 * B2);
            gs[6 * S + o] = R(0);
            gs[7 * S + o] = R(0.5) * (u2 * B3 - u3 * B2);
        }
        if (ii >= H - 1 && ii <= H + TI && jj >= H - 1 && jj <= H + TJ) {
            const R a2c = fabs(gamma * press * ir);
            const R t = a2c + Bsq * ir;
            const R cfc = fsqrt(R(0.5) * (t + fsqrt(fabs(t * t - R(4) * a2c * (B1 * B1) * ir))));
            const int o = (ii - H + 1) * PJ + (jj - H + 1);
            pc[o] = u1;
            pc[PP + o] = u2;
            pc[2 * PP + o] = press;
            pc[3 * PP + o] = cfc;
        }
    }

    // ---- phase 1b: A3 on the tile + 2-cell cross halo: ConstructHJ_L_Order1
    // (ConstructHJ_L.cpp:62-111) and the update of UpdateSoln.cpp:42-47 ----
    {
        const double msx = Max(1e-15, a.hj_in[0]), msy = Max(1e-15, a.hj_in[1]);
        const R eps = MPar<R>::eps(a), pw = MPar<R>::pw(a);
        const double rdx = a.rdx, rdy = a.rdy;
        constexpr int NI = Cfg::NI;
        for (int e = tid; e < NI * NJ; e += NT) {
            const int ni = e / NJ, nj = e - ni * NJ;
            const int ci = ni - HN, cj = nj - HN;   // tile frame
            const bool xin = ci >= 0 && ci < TI, yin = cj >= 0 && cj < TJ;
            if (!xin && !yin) continue;
            const double* A = as + (ci + HA) * AJ + (cj + HA);
            R in[5];
#pragma unroll
            for (int k = 0; k < 5; k++) in[k] = R((A[(k - 2) * AJ] - A[(k - 3) * AJ]) * rdx);
            const R xm = weno5<R, VER, P2>(in, eps, pw);
#pragma unroll
            for (int k = 0; k < 5; k++) in[k] = R((A[(3 - k) * AJ] - A[(2 - k) * AJ]) * rdx);
            const R xp = weno5<R, VER, P2>(in, eps, pw);
#pragma unroll
            for (int k = 0; k < 5; k++) in[k] = R((A[k - 2] - A[k - 3]) * rdy);
            const R ym = weno5<R, VER, P2>(in, eps, pw);
#pragma unroll
            for (int k = 0; k < 5; k++) in[k] = R((A[3 - k] - A[2 - k]) * rdy);
            const R yp = weno5<R, VER, P2>(in, eps, pw);
            const int qe = (ci + H) * RJ + (cj + H);
            const R ir = rcp(qs[qe]);
            const R u1 = qs[PQ + qe] * ir, u2 = qs[2 * PQ + qe] * ir;
            const double La = double(-u1 * R(0.5) * (xm + xp) - u2 * R(0.5) * (ym + yp)) +
                              (msx * 0.5 * double(xp - xm) + msy * 0.5 * double(yp - ym));
            an[e] = an[e] + a.bdt * La;   // a1 A + a2 B from phase 0
        }
    }
    __syncthreads();

    // ---- phase 2: the faces (x faces then y faces).  Plain form: one thread
    // per face, the full characteristic WENO flux.  Hybrid form: pass A gives
    // every face its speed and the smooth faces (no troubled flag in the 3 x 3
    // window of same-direction faces) the linear FD5 flux, component by
    // component (linear_face, fin_stage.cuh); the troubled faces go to a list
    // that pass B works through with the full flux ----
    const R ag1 = a.alpha_in ? R(a.alpha_in[0]) : R(0);
    const R ag2 = a.alpha_in ? R(a.alpha_in[1]) : R(0);
    const R eps = MPar<R>::eps(a), pw = MPar<R>::pw(a);
    R smax_x = R(0), smax_y = R(0);
    const int nwork = Cfg::NFX + Cfg::NFY;
    struct Geom {
        bool isx;
        int fi, fj, qbase, qstr, fbase, fstr, fplane, pbase, pstr;
        const R* fl;
        int perm[MHD_NQ];
    };
    auto geom = [&](int w) {
        Geom g;
        g.isx = w < Cfg::NFX;
        if (g.isx) {
            // between tile rows fi-1 and fi
            if constexpr (Cfg::template ROW8<R>()) {
                g.fi = (w >> 5) + ((w >> 1) & 8); g.fj = w & 15;  // half-warps on rows r and r + 8
            } else {
                g.fi = w / TJ; g.fj = w - g.fi * TJ;
            }
            g.qbase = (H + g.fi) * RJ + (H + g.fj); g.qstr = RJ;
            g.fl = fs; g.fbase = (H + g.fi) * FS + g.fj; g.fstr = FS; g.fplane = RI * FS;
            g.pbase = (g.fi + 1) * PJ + (g.fj + 1); g.pstr = PJ;
        } else {
            const int v = w - Cfg::NFX;
            // between tile columns fj-1 and fj (FP32: half-warps on rows r and
            // r + 8, the last warp on row 7 and the last column)
            if constexpr (Cfg::template ROW8<R>()) {
                const int wv = v >> 5, ln = v & 31;
                if (wv < 7) { g.fi = wv + (ln & 16 ? 8 : 0); g.fj = ln & 15; }
                else if (ln < 16) { g.fi = 7; g.fj = ln; }
                else { g.fi = ln - 16; g.fj = TJ; }
            } else {
                g.fi = v / (TJ + 1); g.fj = v - g.fi * (TJ + 1);
            }
            g.qbase = (H + g.fi) * RJ + (H + g.fj); g.qstr = 1;
            g.fl = gs; g.fbase = g.fi * RJ + (H + g.fj); g.fstr = 1; g.fplane = TI * RJ;
            g.pbase = (g.fi + 1) * PJ + (g.fj + 1); g.pstr = 1;
        }
        // normal-frame component order: rho, m_n, m_t, m_w, E, B_n, B_t, B_w
        g.perm[0] = 0; g.perm[1] = g.isx ? 1 : 2; g.perm[2] = g.isx ? 2 : 1; g.perm[3] = 3; g.perm[4] = 4;
        g.perm[5] = g.isx ? 5 : 6; g.perm[6] = g.isx ? 6 : 5; g.perm[7] = 7;
        return g;
    };
    // SetWaveSpd.cpp:39-88 (nmag = 1; the fast speeds use B1, the x
    // component, for either normal), the LLF alpha of ConstructL.cpp:172-174,
    // and the face-speed maxima GetCFL reads.
    auto speed = [&](const Geom& g) -> R {
        const int pl = g.pbase - g.pstr, un = g.isx ? 0 : 1;
        const int ql = g.qbase - g.qstr;
        const R unl = pc[un * PP + pl], unr = pc[un * PP + g.pbase];
        const R pa = R(0.5) * (pc[2 * PP + pl] + pc[2 * PP + g.pbase]);
        const R rho = R(0.5) * (qs[g.qbase] + qs[ql]);
        const R b5 = R(0.5) * (qs[5 * PQ + g.qbase] + qs[5 * PQ + ql]);
        const R b6 = R(0.5) * (qs[6 * PQ + g.qbase] + qs[6 * PQ + ql]);
        const R b7 = R(0.5) * (qs[7 * PQ + g.qbase] + qs[7 * PQ + ql]);
        const R Bm2 = b5 * b5 + b6 * b6 + b7 * b7;
        const R ir = rcp(rho);
        const R a2 = fabs(gamma * pa * ir);
        const R t = a2 + Bm2 * ir;
        const R cf = fsqrt(R(0.5) * (t + fsqrt(fabs(t * t - R(4) * a2 * (b5 * b5) * ir))));
        const R ua = R(0.5) * (unl + unr);
        const R s1 = Min(unl - pc[3 * PP + pl], ua - cf);
        const R s2 = Max(unr + pc[3 * PP + g.pbase], ua + cf);
        const R alpha = Max(g.isx ? ag1 : ag2, Max(fabs(s1), fabs(s2)));
        if (!(alpha <= R(1e30))) nonfinite = true;
        if (g.isx) {
            const int gfi = i0 + g.fi, gj = j0 + g.fj;
            if (gfi < mx && gj < my && alpha <= R(1e30)) smax_x = Max(smax_x, alpha);
            if (a.face_alpha_x && gfi <= mx && gj < my) a.face_alpha_x[size_t(gfi) * my + gj] = double(alpha);
        } else {
            const int gi = i0 + g.fi, gfj = j0 + g.fj;
            if (gi < mx && gfj < my && alpha <= R(1e30)) smax_y = Max(smax_y, alpha);
            if (a.face_alpha_y && gi < mx && gfj <= my) a.face_alpha_y[size_t(gi) * (my + 1) + gfj] = double(alpha);
        }
        return alpha;
    };
    auto store_face = [&](const Geom& g, const R* Fo) {
        if (g.isx) {
#pragma unroll
            for (int m = 0; m < MHD_NQ; m++) Fh[g.perm[m] * Cfg::NFX + g.fi * TJ + g.fj] = Fo[m];
        } else {
#pragma unroll
            for (int m = 0; m < MHD_NQ; m++) Gh[g.perm[m] * Cfg::NFY + g.fi * (TJ + 1) + g.fj] = Fo[m];
        }
    };
    // The full characteristic WENO flux of one face (ConstructL.cpp:72-206 /
    // 224-356 with the MHD projections).
    auto full_face = [&](const Geom& g, R alpha) {
        const int* perm = g.perm;
        const int qbase = g.qbase, ql = g.qbase - g.qstr;
        R Qa[MHD_NQ];
#pragma unroll
        for (int m = 0; m < MHD_NQ; m++) Qa[m] = R(0.5) * (qs[perm[m] * PQ + qbase] + qs[perm[m] * PQ + ql]);
        const R lah = R(0.5) * MPar<R>::ascale(a) * alpha;
        const MhdStencil<R> st{qs, g.fl, perm, qbase, g.qstr, g.fbase, g.fstr, g.fplane, PQ, lah};
        MhdFace<R> f;
        mhd_face_setup<R>(a, gamma, Qa, f, rec + tid, NT, neg);

        // Characteristic WENO, field pair by field pair: gp from v+ = 0.5 f +
        // lah q at points 0..4, gm from v- = 0.5 f - lah q at points 5..1
        // (ConstructL.cpp:179-199); ghat[k] for the eight waves.
        R ghat[MHD_NQ];
        {
            // fast and slow pairs (rows 0, 7, 2, 5) in one sweep
            R p[4][5], m[4][5];
            mhd_sweep<R, 4>(st, [&](const R* v, R* w) { mhd_left_fs4<R>(f, v, w[0], w[1], w[2], w[3]); }, p, m);
            R gg[4];
            mhd_weno_fields<R, VER, P2, 4>(p, m, eps, pw, gg);
            ghat[0] = gg[0]; ghat[7] = gg[1]; ghat[2] = gg[2]; ghat[5] = gg[3];
        }
#if FIN_MHD_SWEEPS == 2
        {
            // Alfven, entropy and divergence rows (1, 6, 3, 4) in one sweep
            R p[4][5], m[4][5];
            mhd_sweep<R, 4>(st, [&](const R* v, R* w) {
                mhd_left_alf<R>(f, v, w[0], w[1]);
                mhd_left_ent<R>(f, v, w[2], w[3]);
            }, p, m);
            R gg[4];
            mhd_weno_fields<R, VER, P2, 4>(p, m, eps, pw, gg);
            ghat[1] = gg[0]; ghat[6] = gg[1]; ghat[3] = gg[2]; ghat[4] = gg[3];
        }
#else
        // the Alfven pair, then the entropy and divergence rows: one loop
        // body for both sweeps
#pragma unroll 1
        for (int pass = 0; pass < 2; pass++) {
            R p[2][5], m[2][5];
            mhd_sweep<R, 2>(st, [&](const R* v, R* w) {
                if (pass == 0) mhd_left_alf<R>(f, v, w[0], w[1]);
                else mhd_left_ent<R>(f, v, w[0], w[1]);
            }, p, m);
            R gg[2];
            mhd_weno_fields<R, VER, P2, 2>(p, m, eps, pw, gg);
            if (pass == 0) { ghat[1] = gg[0]; ghat[6] = gg[1]; }
            else { ghat[3] = gg[0]; ghat[4] = gg[1]; }
        }
#endif

        // Right projection (ProjectRightEig.cpp:89-203) in the normal frame.
        R Fo[MHD_NQ];
        {
            const R* rc = rec + tid;
            const R rho = rc[MR_RHO * NT], af = rc[MR_AF * NT], as_ = rc[MR_AS * NT];
            const R cf = rc[MR_CF * NT], cs = rc[MR_CS * NT], beta1 = rc[MR_BETA1 * NT];
            const R gp = rc[MR_GP * NT], asr = rc[MR_ASR * NT], sr2 = rc[MR_SR2 * NT];
            const R rs2 = R(a.r_sqrt2);
            const R Gp = ghat[0] + ghat[7], Gm = ghat[7] - ghat[0];
            const R Hp = ghat[2] + ghat[5], Hm = ghat[5] - ghat[2];
            const R Kp = ghat[1] + ghat[6], Km = ghat[6] - ghat[1];
            const R fsum = af * Gp + as_ * Hp;
            const R drho = rho * fsum + ghat[3];
            const R dun = af * cf * Gm + as_ * cs * Hm;
            const R X = beta1 * (af * cf * Hm - as_ * cs * Gm);
            const R dut = f.b2 * X - f.b3 * rs2 * Kp;
            const R duw = f.b3 * X + f.b2 * rs2 * Kp;
            const R dp = gp * fsum;
            const R dbn = ghat[4];
            const R Y = asr * (as_ * Gp - af * Hp);
            const R dbt = f.b2 * Y + f.b3 * sr2 * Km;
            const R dbw = f.b3 * Y - f.b2 * sr2 * Km;
            Fo[0] = drho;
            Fo[1] = rho * dun + f.u1 * drho;
            Fo[2] = rho * dut + f.u2 * drho;
            Fo[3] = rho * duw + f.u3 * drho;
            Fo[4] = f.um2 * drho + rho * (f.u1 * dun + f.u2 * dut + f.u3 * duw) + dp * rcp(gamma - R(1)) +
                    f.B1 * dbn + f.B2 * dbt + f.B3 * dbw;
            Fo[5] = dbn;
            Fo[6] = dbt;
            Fo[7] = dbw;
        }
        store_face(g, Fo);
    };
    if (HYB) {
        R* falpha = reinterpret_cast<R*>(hyb_base);                            // [NFX + NFY]
        short* tlist = reinterpret_cast<short*>(falpha + nwork);               // [NFX + NFY]
        int* ntrb = reinterpret_cast<int*>(hyb_base + Cfg::template hyb_ntrb_offset<R>());
#pragma unroll 1
        for (int wb = 0; wb < nwork; wb += NT) {
            const int w = wb + tid;
            bool push = false;
            if (w < nwork) {
                const Geom g = geom(w);
                const R alpha = speed(g);
                falpha[w] = alpha;
                const unsigned* fm = g.isx ? fxm : fym;
                push = (((fm[g.fi] | fm[g.fi + 1] | fm[g.fi + 2]) >> g.fj) & 1u) != 0;
                if (!push) {
                    const R lah = R(0.5) * MPar<R>::ascale(a) * alpha;
                    R Fo[MHD_NQ];
#pragma unroll
                    for (int m = 0; m < MHD_NQ; m++)
                        Fo[m] = linear_face<R>(g.fl + g.perm[m] * g.fplane + g.fbase, g.fstr,
                                               qs + g.perm[m] * PQ + g.qbase, g.qstr, lah);
                    store_face(g, Fo);
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, push);
            if (bal) {
                int base = 0;
                const int lead = __ffs(bal) - 1;
                if ((tid & 31) == lead) base = atomicAdd(ntrb, __popc(bal));
                base = __shfl_sync(0xffffffffu, base, lead);
                if (push) tlist[base + __popc(bal & ((1u << (tid & 31)) - 1u))] = short(w);
            }
        }
        __syncthreads();
        const int nt = *ntrb;
#pragma unroll 1
        for (int k = tid; k < nt; k += NT) {
            const int w = tlist[k];
            full_face(geom(w), falpha[w]);
        }
    } else {
#pragma unroll 1
        for (int w = tid; w < nwork; w += NT) {
            const Geom g = geom(w);
            full_face(g, speed(g));
        }
    }
    __syncthreads();

    // ---- phase 3: flux difference (ConstructL.cpp:390-401), stage update,
    // constrained transport, next-stage maxima ----
    double cs_x = 0.0, cs_y = 0.0, hx = 0.0, hy = 0.0;
    const double gam = a.gamma;
    for (int c = tid; c < TI * TJ; c += NT) {
        const int ci = c / TJ, cj = c - ci * TJ;
        const int gi = i0 + ci, gj = j0 + cj;
        if (gi >= mx || gj >= my) continue;
        const size_t g = size_t(gi) * my + gj;
        double qn[MHD_NQ];
#pragma unroll
        for (int m = 0; m < MHD_NQ; m++) {
            if (a.ct && (m == 5 || m == 6)) continue;
            const R f1 = Fh[m * Cfg::NFX + (ci + 1) * TJ + cj], f0 = Fh[m * Cfg::NFX + ci * TJ + cj];
            const R g1 = Gh[m * Cfg::NFY + ci * (TJ + 1) + cj + 1], g0 = Gh[m * Cfg::NFY + ci * (TJ + 1) + cj];
            R Lr = -(f1 - f0) * R(a.rdx);
            Lr = Lr - (g1 - g0) * R(a.rdy);
            double v = 0.0;
            if (a.A) v = a.a1 * a.A[m * a.plane + g];
            if (a.B) v = v + a.a2 * a.B[m * a.plane + g];
            qn[m] = v + a.bdt * double(Lr);
        }
        const double* N = an + (ci + HN) * NJ + (cj + HN);
        if (a.ct) {
            // AfterStep.cpp:39-48 on the updated potential
            qn[5] = a.ct_y * (N[-2] - 8 * N[-1] + 8 * N[1] - N[2]);
            qn[6] = a.ct_x * (N[-2 * NJ] - 8 * N[-NJ] + 8 * N[NJ] - N[2 * NJ]);
        }
#pragma unroll
        for (int m = 0; m < MHD_NQ; m++) a.qout[m * a.plane + g] = qn[m];
        a.qout[8 * a.plane + g] = N[0];
        // next stage's maxima: GlobalWaveSpd.cpp:71-76 with Ql = Qr (each
        // direction's speed is |u_n| + the cell's fast speed) and the HJ speeds
        const double ir = rcp(qn[0]);
        const double u1 = qn[1] * ir, u2 = qn[2] * ir, u3 = qn[3] * ir;
        if (a.alpha_out) {
            const R Bsq = R(qn[5] * qn[5] + qn[6] * qn[6] + qn[7] * qn[7]);
            const R press =
                R((gam - 1.0) * (qn[4] - 0.5 * qn[0] * (u1 * u1 + u2 * u2 + u3 * u3) - 0.5 * double(Bsq)));
            const R rir = R(ir);
            const R a2c = fabs(gamma * press * rir);
            const R t = a2c + Bsq * rir;
            const R B1 = R(qn[5]);
            const double cfc = double(fsqrt(R(0.5) * (t + fsqrt(fabs(t * t - R(4) * a2c * (B1 * B1) * rir)))));
            const double sx = Max(fabs(u1 - cfc), fabs(u1 + cfc));
            const double sy = Max(fabs(u2 - cfc), fabs(u2 + cfc));
            if (!(sx <= 1e300) || !(sy <= 1e300)) nonfinite = true;
            if (sx <= 1e300) cs_x = Max(cs_x, sx);
            if (sy <= 1e300) cs_y = Max(cs_y, sy);
        }
        if (a.hj_out) {
            // the HJ speeds of q_out, only where a stage produces a state (a
            // right-hand-side evaluation writes L there, whose density
            // entry may be exactly 0)
            const double ax = fabs(u1), ay = fabs(u2);
            if (ax <= 1e300) hx = Max(hx, ax); else nonfinite = true;
            if (ay <= 1e300) hy = Max(hy, ay); else nonfinite = true;
        }
    }

    // ---- block reductions, one atomic per maximum ----
    double v6[6] = {double(smax_x), double(smax_y), cs_x, cs_y, hx, hy};
#pragma unroll
    for (int k = 0; k < 6; k++) {
        double v = v6[k] <= 1e300 ? v6[k] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = Max(v, __shfl_xor_sync(0xffffffffu, v, o));
        v6[k] = v;
    }
    if ((tid & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 6; k++) red[(tid >> 5) * 6 + k] = v6[k];
    }
    if (neg) atomicOr(a.status, 2u);
    if (nonfinite) atomicOr(a.status, 1u);
    __syncthreads();
    if (tid < 6) {
        double v = 0.0;
        for (int wv = 0; wv < NT / 32; wv++) v = Max(v, red[wv * 6 + tid]);
        double* dst = tid < 2 ? a.smax_out : (tid < 4 ? a.alpha_out : a.hj_out);
        if (dst) atomic_max_nonneg(dst + (tid & 1), v);
    }
}

// The maxima of a state already in HBM (GlobalWaveSpd and the HJ speeds),
// for a state that no stage epilogue produced (after a host upload).
__global__ void k_mhd_state_max(const double* q, int mx, int my, size_t plane, double gamma, double* alpha_out,
                                double* hj_out, unsigned int* status);
// B1 = dA3/dy, B2 = -dA3/dx by AfterStep.cpp:39-48 (in place on a state).
__global__ void k_mhd_after_step(double* q, int mx, int my, size_t plane, double ct_y, double ct_x);
// max |D_x B1 + D_y B2| over the interior with D the 4th-order central
// difference of the constrained transport.
__global__ void k_mhd_div_b(const double* q, int mx, int my, size_t plane, double rdx, double rdy, double* out);

}  // namespace fin
