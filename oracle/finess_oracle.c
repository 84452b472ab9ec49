/*
 * finess_oracle.c -- CPU restatement (plain C, FP64) of the reference's 2D
 * WENO right-hand side and time steppers.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this library, and only as the checker.
 *
 * Every expression keeps the reference's operation order (left-to-right
 * evaluation, divisions where it divides) so that, built without FMA
 * contraction, it reproduces the reference bit for bit; tests pin that
 * against oracle/_ref/libfinref.so, the reference's own sources compiled
 * in place.  Each function cites the reference lines it restates.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "finess_oracle.h"

#define MEQN_MAX 8

/* dog_math.h:18-22 */
static double Max(double a, double b) { return a > b ? a : b; }
static double Min(double a, double b) { return a < b ? a : b; }

typedef struct {
    int mx, my, mbc, meqn, sy;   /* sy = my + 2*mbc */
} grid_t;

static grid_t grid_of(const fin_params* p, int mx, int my)
{
    grid_t g = {mx, my, p->mbc, p->meqn, my + 2 * p->mbc};
    return g;
}
/* lib/tensors.h:267-273 with b = 1-mbc */
static size_t IDX(const grid_t* g, int i, int j, int m)
{
    return ((size_t)(i + g->mbc - 1) * g->sy + (size_t)(j + g->mbc - 1)) * g->meqn + (m - 1);
}
static size_t numel(const grid_t* g)
{
    return (size_t)(g->mx + 2 * g->mbc) * g->sy * g->meqn;
}
static double get_dx(const fin_params* p) { return (p->xhigh - p->xlow) / p->mx; }
static double get_dy(const fin_params* p) { return (p->yhigh - p->ylow) / p->my; }

/* ---------------------------------------------------------------------- */
/* Euler callbacks                                                         */
/* ---------------------------------------------------------------------- */

/* apps/2d/euler/lib/FluxFunc.cpp:19-42, one point.  f = flux(.,1), g = flux(.,2) */
static void euler_flux(double gamma, const double* Q, double* f, double* g)
{
    const double rho = Q[0];
    const double u1 = Q[1] / rho;
    const double u2 = Q[2] / rho;
    const double u3 = Q[3] / rho;
    const double energy = Q[4];
    const double press = (gamma - 1.0e0) * (energy - 0.5e0 * rho * (u1 * u1 + u2 * u2 + u3 * u3));
    f[0] = rho * u1;
    f[1] = rho * u1 * u1 + press;
    f[2] = rho * u1 * u2;
    f[3] = rho * u1 * u3;
    f[4] = u1 * (energy + press);
    g[0] = rho * u2;
    g[1] = rho * u2 * u1;
    g[2] = rho * u2 * u2 + press;
    g[3] = rho * u2 * u3;
    g[4] = u2 * (energy + press);
}

/* Average-state quantities shared by both projections. */
typedef struct {
    int mu, mv, mw;               /* 0-based */
    double u1, u2, u3, umag2, c, H;
} eig_t;

/* apps/2d/euler/lib/ProjectLeftEig.cpp:20-44 (use_fabs = 0) and
 * ProjectRightEig.cpp:19-43 (use_fabs = 1: c = sqrt(fabs(...))). */
static eig_t euler_eig(int ixy, double gamma, const double* Qave, int use_fabs)
{
    eig_t e;
    if (ixy == 1) { e.mu = 1; e.mv = 2; e.mw = 3; }
    else { e.mu = 2; e.mv = 1; e.mw = 3; }
    const double rho = Qave[0];
    e.u1 = Qave[e.mu] / rho;
    e.u2 = Qave[e.mv] / rho;
    e.u3 = Qave[e.mw] / rho;
    const double energy = Qave[4];
    e.umag2 = (e.u1 * e.u1 + e.u2 * e.u2 + e.u3 * e.u3);
    const double press = (gamma - 1.0e0) * (energy - 0.5e0 * rho * e.umag2);
    e.c = use_fabs ? sqrt(fabs(gamma * press / rho)) : sqrt(gamma * press / rho);
    e.H = (energy + press) / rho;
    return e;
}

/* apps/2d/euler/lib/ProjectLeftEig.cpp:47-66, one point. */
static void euler_left(const eig_t* e, const double* Q, double* W)
{
    const double u1 = e->u1, u2 = e->u2, u3 = e->u3, umag2 = e->umag2, c = e->c, H = e->H;
    const int mu = e->mu, mv = e->mv, mw = e->mw;
    W[0] = ((umag2 / 2.0 - H - u1 * c) * Q[mu]
            + (umag2 / 2.0 * (c - u1) + H * u1) * Q[0]
            + c * (Q[4] - u2 * Q[mv] - u3 * Q[mw])) / (c * (2.0 * H - umag2));
    W[mu] = 2.0 * ((H - umag2) * Q[0] + u1 * Q[mu] + u2 * Q[mv] + u3 * Q[mw] - Q[4]) / (2.0 * H - umag2);
    W[mv] = Q[mv] - u2 * Q[0];
    W[mw] = Q[mw] - u3 * Q[0];
    W[4] = ((H - umag2 / 2.0 - u1 * c) * Q[mu]
            + (umag2 / 2.0 * (c + u1) - H * u1) * Q[0]
            + c * (Q[4] - u2 * Q[mv] - u3 * Q[mw])) / (c * (2.0 * H - umag2));
}

/* apps/2d/euler/lib/ProjectRightEig.cpp:46-62, one point. */
static void euler_right(const eig_t* e, const double* W, double* Q)
{
    const double u1 = e->u1, u2 = e->u2, u3 = e->u3, umag2 = e->umag2, c = e->c, H = e->H;
    const int mu = e->mu, mv = e->mv, mw = e->mw;
    Q[0] = W[0] + W[mu] + W[4];
    Q[mu] = (u1 - c) * W[0] + u1 * W[mu] + (u1 + c) * W[4];
    Q[mv] = u2 * (W[0] + W[mu] + W[4]) + W[mv];
    Q[mw] = u3 * (W[0] + W[mu] + W[4]) + W[mw];
    Q[4] = (H - u1 * c) * W[0] + umag2 / 2.0 * W[mu] + u2 * W[mv] + u3 * W[mw] + (H + u1 * c) * W[4];
}

/* apps/2d/euler/lib/SetWaveSpd.cpp:11-69 */
static void euler_wave_spd(double gamma, double n1, double n2, const double* Ql, const double* Qr,
                           double* s1, double* s2)
{
    const double rhol = Ql[0];
    const double u1l = Ql[1] / rhol;
    const double u2l = Ql[2] / rhol;
    const double u3l = Ql[3] / rhol;
    const double energyl = Ql[4];
    const double pressl = (gamma - 1.0e0) * (energyl - 0.5e0 * rhol * (u1l * u1l + u2l * u2l + u3l * u3l));
    const double rhor = Qr[0];
    const double u1r = Qr[1] / rhor;
    const double u2r = Qr[2] / rhor;
    const double u3r = Qr[3] / rhor;
    const double energyr = Qr[4];
    const double pressr = (gamma - 1.0e0) * (energyr - 0.5e0 * rhor * (u1r * u1r + u2r * u2r + u3r * u3r));
    const double rho = 0.5e0 * (rhol + rhor);
    const double u1 = 0.5e0 * (u1l + u1r);
    const double u2 = 0.5e0 * (u2l + u2r);
    (void)u3l; (void)u3r;
    const double press = 0.5e0 * (pressl + pressr);
    const double nmag = sqrt(n1 * n1 + n2 * n2);
    const double cl = nmag * sqrt(fabs(gamma * pressl / rhol));
    const double cr = nmag * sqrt(fabs(gamma * pressr / rhor));
    const double c = nmag * sqrt(fabs(gamma * press / rho));
    const double un = n1 * u1 + n2 * u2;
    const double unl = n1 * u1l + n2 * u2l;
    const double unr = n1 * u1r + n2 * u2r;
    *s1 = Min(unl - cl, un - c);
    *s2 = Max(unr + cr, un + c);
}

/* Directional derivatives of the Euler flux component d (0: f, 1: g) at Q.
 * The reference tabulates the Jacobian and Hessian entry by entry
 * (apps/2d/euler/lib/DFluxFunc.cpp:30-105, D2FluxFunc.cpp:44-300); for every
 * 2D state (rho w = 0) its Jacobian entries are the exact derivatives, and its
 * Hessian entries are exact except the energy-flux E cross terms (see
 * euler_d2flux_dir).  These closed forms produce them:
 *   du_k[a] = (a_k - u_k a_0)/rho,  dp[a] = (g-1)(a_4 - u.a_m + |u|^2 a_0/2),
 *   f_0 = m_n, f_k = m_n u_k + delta_kn p, f_4 = (E+p) u_n  (n = 1+d),
 *   d2u_k[a,b] = -(du_k[a] b_0 + du_k[b] a_0)/rho,
 *   d2p[a,b] = -(g-1) rho du[a].du[b]. */
static void euler_dflux_dir(double gamma, const double* Q, int d, const double* a, double* out)
{
    const int n = 1 + d;
    const double rho = Q[0], u[3] = {Q[1] / rho, Q[2] / rho, Q[3] / rho}, E = Q[4];
    const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const double p = (gamma - 1.0) * (E - 0.5 * rho * uu);
    double du[3];
    for (int k = 0; k < 3; k++) du[k] = (a[k + 1] - u[k] * a[0]) / rho;
    const double dp = (gamma - 1.0) * (a[4] - (u[0] * a[1] + u[1] * a[2] + u[2] * a[3]) + 0.5 * uu * a[0]);
    out[0] = a[n];
    for (int k = 0; k < 3; k++) out[k + 1] = a[n] * u[k] + Q[n] * du[k] + (k + 1 == n ? dp : 0.0);
    out[4] = (a[4] + dp) * u[n - 1] + (E + p) * du[n - 1];
}

static void euler_d2flux_dir(double gamma, const double* Q, int d, const double* a, const double* b, double* out)
{
    const int n = 1 + d;
    const double rho = Q[0], u[3] = {Q[1] / rho, Q[2] / rho, Q[3] / rho}, E = Q[4];
    const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const double p = (gamma - 1.0) * (E - 0.5 * rho * uu);
    double dua[3], dub[3], d2u[3];
    for (int k = 0; k < 3; k++) {
        dua[k] = (a[k + 1] - u[k] * a[0]) / rho;
        dub[k] = (b[k + 1] - u[k] * b[0]) / rho;
        d2u[k] = -(dua[k] * b[0] + dub[k] * a[0]) / rho;
    }
    const double dpa = (gamma - 1.0) * (a[4] - (u[0] * a[1] + u[1] * a[2] + u[2] * a[3]) + 0.5 * uu * a[0]);
    const double dpb = (gamma - 1.0) * (b[4] - (u[0] * b[1] + u[1] * b[2] + u[2] * b[3]) + 0.5 * uu * b[0]);
    const double d2p = -(gamma - 1.0) * rho * (dua[0] * dub[0] + dua[1] * dub[1] + dua[2] * dub[2]);
    out[0] = 0.0;
    for (int k = 0; k < 3; k++)
        out[k + 1] = a[n] * dub[k] + b[n] * dua[k] + Q[n] * d2u[k] + (k + 1 == n ? d2p : 0.0);
    /* The reference's energy-flux Hessian (D2FluxFunc.cpp, entries
     * D2flux(i,5,1,5,.), (i,5,2,5,.), (i,5,3,5,.) and their transposes) omits
     * the pressure's dependence on E in the E cross terms: its d2f5/dE dq_k is
     * d u_n/dq_k where the exact value is gamma d u_n/dq_k.  Reproduced here:
     * the E component of dp is left out of the two cross terms. */
    const double dpa_noE = dpa - (gamma - 1.0) * a[4];
    const double dpb_noE = dpb - (gamma - 1.0) * b[4];
    out[4] = (a[4] + dpa_noE) * dub[n - 1] + (b[4] + dpb_noE) * dua[n - 1] + d2p * u[n - 1] + (E + p) * d2u[n - 1];
}

void oracle_flux_derivs(double gamma, const double* Q, double* A, double* H);

/* Jacobian A[d][m][k] = d f^d_m / d q_k and Hessian H[d][m][k1][k2]
 * (DFluxFunc / D2FluxFunc's Dflux(1,m,k,d), D2flux(1,m,k1,k2,d)). */
static void euler_jac_hess(double gamma, const double* Q, double A[2][5][5], double H[2][5][5][5], int want_h)
{
    double e[5][5] = {{0}};
    for (int k = 0; k < 5; k++) e[k][k] = 1.0;
    for (int d = 0; d < 2; d++) {
        double col[5];
        for (int k = 0; k < 5; k++) {
            euler_dflux_dir(gamma, Q, d, e[k], col);
            for (int m = 0; m < 5; m++) A[d][m][k] = col[m];
        }
        if (!want_h) continue;
        for (int k1 = 0; k1 < 5; k1++)
            for (int k2 = 0; k2 < 5; k2++) {
                euler_d2flux_dir(gamma, Q, d, e[k1], e[k2], col);
                for (int m = 0; m < 5; m++) H[d][m][k1][k2] = col[m];
            }
    }
}

/* ---------------------------------------------------------------------- */
/* WENO reconstructions (lib/WenoReconstruct.cpp)                          */
/* ---------------------------------------------------------------------- */

/* :121-123, shared by JS5 and Z5 */
static void betas5(const double* u, double* b)
{
    const double uim2 = u[0], uim1 = u[1], ui = u[2], uip1 = u[3], uip2 = u[4];
    double t;
    t = uim2 - 2 * uim1 + ui;        b[0] = (13. / 12.) * (t * t);
    t = uim2 - 4 * uim1 + 3 * ui;    b[0] = b[0] + 0.25 * (t * t);
    t = uim1 - 2 * ui + uip1;        b[1] = (13. / 12.) * (t * t);
    t = uim1 - uip1;                 b[1] = b[1] + 0.25 * (t * t);
    t = ui - 2 * uip1 + uip2;        b[2] = (13. / 12.) * (t * t);
    t = 3 * ui - 4 * uip1 + uip2;    b[2] = b[2] + 0.25 * (t * t);
}
/* :126-128 */
static void cands5(const double* u, double* c)
{
    const double uim2 = u[0], uim1 = u[1], ui = u[2], uip1 = u[3], uip2 = u[4];
    c[0] = (1. / 3.) * uim2 - (7. / 6.) * uim1 + (11. / 6.) * ui;
    c[1] = (-1. / 6.) * uim1 + (5. / 6.) * ui + (1. / 3.) * uip1;
    c[2] = (1. / 3.) * ui + (5. / 6.) * uip1 - (1. / 6.) * uip2;
}

void oracle_weno_js5_weights(double eps, double power_param, const double u[5], double w[3])
{
    double b[3];
    betas5(u, b);
    const double omt0 = 0.1 * pow(eps + b[0], -power_param);
    const double omt1 = 0.6 * pow(eps + b[1], -power_param);
    const double omt2 = 0.3 * pow(eps + b[2], -power_param);
    const double omts = omt0 + omt1 + omt2;
    w[0] = omt0 / omts; w[1] = omt1 / omts; w[2] = omt2 / omts;
}

double oracle_weno5(int weno_version, double eps, double power_param, const double u[5])
{
    double c[3];
    cands5(u, c);
    if (weno_version == FIN_WENO_FD)         /* :580-616 */
        return 0.1 * c[0] + 0.6 * c[1] + 0.3 * c[2];
    double b[3], omt0, omt1, omt2;
    betas5(u, b);
    if (weno_version == FIN_WENO_JS) {       /* :90-141 */
        omt0 = 0.1 * pow(eps + b[0], -power_param);
        omt1 = 0.6 * pow(eps + b[1], -power_param);
        omt2 = 0.3 * pow(eps + b[2], -power_param);
    } else {                                 /* Z5, :385-438 */
        const double tau5 = fabs(b[0] - b[2]);
        omt0 = 0.1 * (1. + pow(tau5 / (eps + b[0]), power_param));
        omt1 = 0.6 * (1. + pow(tau5 / (eps + b[1]), power_param));
        omt2 = 0.3 * (1. + pow(tau5 / (eps + b[2]), power_param));
    }
    const double omts = omt0 + omt1 + omt2;
    return (omt0 * c[0] + omt1 * c[1] + omt2 * c[2]) / omts;
}

/* ---------------------------------------------------------------------- */
/* Boundary conditions and wave speeds                                     */
/* ---------------------------------------------------------------------- */

static int remap(int k, int n, int bc_lo, int bc_hi)
{
    if (k < 1) return bc_lo == FIN_BC_PERIODIC ? k + n : 1;
    if (k > n) return bc_hi == FIN_BC_PERIODIC ? k - n : n;
    return k;
}

/* Periodic: apps/2d/euler/test_exact2/SetBndValues.cpp:28-197 (corners by
 * wrap); transmissive: apps/2d/euler/riemann_test/SetBndValues.cpp:30-111
 * (zeroth-order extrapolation; corners filled here by the same clamp). */
void oracle_set_bnd(const fin_params* p, double* q)
{
    grid_t g = grid_of(p, p->mx, p->my);
    for (int i = 1 - g.mbc; i <= g.mx + g.mbc; i++)
        for (int j = 1 - g.mbc; j <= g.my + g.mbc; j++) {
            if (i >= 1 && i <= g.mx && j >= 1 && j <= g.my) continue;
            const int si = remap(i, g.mx, p->bc_xlow, p->bc_xhigh);
            const int sj = remap(j, g.my, p->bc_ylow, p->bc_yhigh);
            for (int m = 1; m <= g.meqn; m++) q[IDX(&g, i, j, m)] = q[IDX(&g, si, sj, m)];
        }
}

/* lib/2d/GlobalWaveSpd.cpp:41-78 (serial, i outer, j inner) */
void oracle_global_wave_spd(const fin_params* p, const double* q, double* alpha1, double* alpha2)
{
    grid_t g = grid_of(p, p->mx, p->my);
    double a1 = 0.0, a2 = 0.0, s1, s2;
    for (int i = 1; i <= g.mx; i++)
        for (int j = 1; j <= g.my; j++) {
            const double* Q = q + IDX(&g, i, j, 1);
            euler_wave_spd(p->gamma, 1.0, 0.0, Q, Q, &s1, &s2);
            a1 = Max(a1, Max(fabs(s1), fabs(s2)));
            euler_wave_spd(p->gamma, 0.0, 1.0, Q, Q, &s1, &s2);
            a2 = Max(a2, Max(fabs(s1), fabs(s2)));
        }
    *alpha1 = a1;
    *alpha2 = a2;
}

/* ---------------------------------------------------------------------- */
/* ConstructL (lib/2d/ConstructL.cpp)                                      */
/* ---------------------------------------------------------------------- */

/* One interface, both sweeps: ConstructL.cpp:72-206 (ixy = 1) and
 * :224-356 (ixy = 2).  qpts/fpts: the 6 stencil points' q and the normal
 * flux component (point-major, meqn each).  Qavg: face average.  Ql/Qr:
 * the two cells adjacent to the face.  Writes the face flux fhat[meqn] and
 * returns alpha (before alpha_scaling). */
static double face_flux(const fin_params* p, int ixy, double alpha_glob,
                        const double* Qavg, const double* Ql, const double* Qr,
                        const double qpts[6][MEQN_MAX], const double fpts[6][MEQN_MAX],
                        double* fhat)
{
    const int meqn = p->meqn;
    double w[6][MEQN_MAX], gv[6][MEQN_MAX];
    eig_t el = euler_eig(ixy, p->gamma, Qavg, 0);
    for (int s = 0; s < 6; s++) {
        euler_left(&el, qpts[s], w[s]);
        euler_left(&el, fpts[s], gv[s]);
    }
    double s1, s2;
    if (ixy == 1) euler_wave_spd(p->gamma, 1.0, 0.0, Ql, Qr, &s1, &s2);
    else euler_wave_spd(p->gamma, 0.0, 1.0, Ql, Qr, &s1, &s2);
    const double alpha = Max(alpha_glob, Max(fabs(s1), fabs(s2)));
    const double l_alpha = p->alpha_scaling * alpha;
    double ghat[MEQN_MAX];
    for (int m = 0; m < meqn; m++) {
        double gp[5], gm[5];
        for (int s = 1; s <= 5; s++) {
            gp[s - 1] = 0.5 * (gv[s - 1][m] + l_alpha * w[s - 1][m]);
            gm[s - 1] = 0.5 * (gv[5 - s + 1][m] - l_alpha * w[5 - s + 1][m]);
        }
        const double dGp = oracle_weno5(p->weno_version, p->epsilon, p->power_param, gp);
        const double dGm = oracle_weno5(p->weno_version, p->epsilon, p->power_param, gm);
        ghat[m] = dGp + dGm;
    }
    eig_t er = euler_eig(ixy, p->gamma, Qavg, 1);
    euler_right(&er, ghat, fhat);
    return alpha;
}

static int weno_supported(const fin_params* p)
{
    return p->space_order == 5 &&
           (p->weno_version == FIN_WENO_JS || p->weno_version == FIN_WENO_Z || p->weno_version == FIN_WENO_FD);
}

/* Shared sweep body of ConstructL and ConstructLxWL: fx/fy are the sampled
 * flux components at every ghosted cell (NULL = evaluate FluxFunc on q). */
static int construct_l_common(const fin_params* p, const double* q, const double* Fs, const double* Gs,
                              double* L, double* smax)
{
    if (!weno_supported(p) || p->meqn != 5) return FIN_ERR_ARG;
    const grid_t g = grid_of(p, p->mx, p->my);
    const grid_t gF = grid_of(p, p->mx + 1, p->my);
    const grid_t gG = grid_of(p, p->mx, p->my + 1);
    const grid_t gS = {p->mx + 1, p->my + 1, p->mbc, 2, p->my + 1 + 2 * p->mbc};
    const int meqn = g.meqn, mx = g.mx, my = g.my;
    const double dx = get_dx(p), dy = get_dy(p);
    double* Fhat = (double*)calloc(numel(&gF), sizeof(double));
    double* Ghat = (double*)calloc(numel(&gG), sizeof(double));
    double alpha1 = 0., alpha2 = 0.;
    if (p->global_alpha) oracle_global_wave_spd(p, q, &alpha1, &alpha2);

    for (int ixy = 1; ixy <= 2; ixy++) {
        const int imax = ixy == 1 ? mx + 1 : mx, jmax = ixy == 1 ? my : my + 1;
        for (int i = 1; i <= imax; i++)
            for (int j = 1; j <= jmax; j++) {
                const int di = ixy == 1 ? 1 : 0, dj = ixy == 1 ? 0 : 1;
                const double* Qr = q + IDX(&g, i, j, 1);
                const double* Ql = q + IDX(&g, i - di, j - dj, 1);
                double Qavg[MEQN_MAX], qpts[6][MEQN_MAX], fpts[6][MEQN_MAX], fhat[MEQN_MAX];
                for (int m = 0; m < meqn; m++) Qavg[m] = 0.5 * (Qr[m] + Ql[m]);
                for (int s = 1; s <= 6; s++) {
                    const int is = i + di * (s - 4), js = j + dj * (s - 4);
                    const double* Qs = q + IDX(&g, is, js, 1);
                    double fx[MEQN_MAX], fy[MEQN_MAX];
                    if (Fs) {
                        for (int m = 0; m < meqn; m++) {
                            fx[m] = Fs[IDX(&g, is, js, m + 1)];
                            fy[m] = Gs[IDX(&g, is, js, m + 1)];
                        }
                    } else {
                        euler_flux(p->gamma, Qs, fx, fy);
                    }
                    for (int m = 0; m < meqn; m++) {
                        qpts[s - 1][m] = Qs[m];
                        fpts[s - 1][m] = ixy == 1 ? fx[m] : fy[m];
                    }
                }
                const double alpha = face_flux(p, ixy, ixy == 1 ? alpha1 : alpha2, Qavg, Ql, Qr, qpts, fpts, fhat);
                double* sm = smax + IDX(&gS, i, j, ixy);
                *sm = Max(*sm, alpha);
                double* out = ixy == 1 ? Fhat + IDX(&gF, i, j, 1) : Ghat + IDX(&gG, i, j, 1);
                for (int m = 0; m < meqn; m++) out[m] = fhat[m];
            }
    }
    /* ConstructL.cpp:390-401 */
    for (int i = 1; i <= mx; i++)
        for (int j = 1; j <= my; j++)
            for (int m = 1; m <= meqn; m++) {
                double tmp = -(Fhat[IDX(&gF, i + 1, j, m)] - Fhat[IDX(&gF, i, j, m)]) / dx;
                tmp = tmp - (Ghat[IDX(&gG, i, j + 1, m)] - Ghat[IDX(&gG, i, j, m)]) / dy;
                L[IDX(&g, i, j, m)] = tmp;
            }
    free(Fhat);
    free(Ghat);
    return 0;
}

int oracle_construct_l(const fin_params* p, const double* q, double* L, double* smax)
{
    return construct_l_common(p, q, NULL, NULL, L, smax);
}

int oracle_construct_lxwl(const fin_params* p, const double* q, const double* F, const double* G,
                          double* L, double* smax)
{
    return construct_l_common(p, q, F, G, L, smax);
}

/* ---------------------------------------------------------------------- */
/* Time stepping                                                           */
/* ---------------------------------------------------------------------- */

/* lib/2d/UpdateSoln.cpp:29-35, interior only (ghosts are rebuilt by the BC). */
static void update_soln(const grid_t* g, double a1, double a2, double beta, double dt,
                        const double* qstar, const double* L, double* qnew)
{
    for (int i = 1; i <= g->mx; i++)
        for (int j = 1; j <= g->my; j++)
            for (int m = 1; m <= g->meqn; m++) {
                const size_t k = IDX(g, i, j, m);
                qnew[k] = a1 * qstar[k] + a2 * qnew[k] + beta * dt * L[k];
            }
}

/* lib/2d/GetCFL.cpp:31-73; returns FIN_OK or an error code. */
static int get_cfl(const fin_params* p, double dt, double dtmax, const double* smax, double* cfl_out)
{
    if (dt > dtmax) return FIN_ERR_DT_BOUNDS;
    const grid_t gS = {p->mx + 1, p->my + 1, p->mbc, 2, p->my + 1 + 2 * p->mbc};
    const double dx = get_dx(p), dy = get_dy(p);
    double cfl = -100.0;
    for (int i = 1; i <= p->mx; i++)
        for (int j = 1; j <= p->my; j++) {
            cfl = Max(dt * smax[IDX(&gS, i, j, 1)] / dx, cfl);
            cfl = Max(dt * smax[IDX(&gS, i, j, 2)] / dy, cfl);
        }
    if (cfl > 1.0e8) return FIN_ERR_CFL_BOUNDS;
    *cfl_out = cfl;
    return FIN_OK;
}

static int construct_integrated_r2(const fin_params* p, double dt, double a1, double b1, const double* q1,
                                   double a2, double b2, const double* q2, double* F, double* G);

typedef struct {
    grid_t g, gS;
    size_t n, nS;
    double *qold, *qstar, *L, *smax, *F, *G;
} work_t;

static void work_init(work_t* w, const fin_params* p)
{
    w->g = grid_of(p, p->mx, p->my);
    grid_t gS = {p->mx + 1, p->my + 1, p->mbc, 2, p->my + 1 + 2 * p->mbc};
    w->gS = gS;
    w->n = numel(&w->g);
    w->nS = numel(&w->gS);
    w->qold = (double*)calloc(w->n, sizeof(double));
    w->qstar = (double*)calloc(w->n, sizeof(double));
    w->L = (double*)calloc(w->n, sizeof(double));
    w->F = (double*)calloc(w->n, sizeof(double));
    w->G = (double*)calloc(w->n, sizeof(double));
    w->smax = (double*)calloc(w->nS, sizeof(double));
}
static void work_free(work_t* w)
{
    free(w->qold); free(w->qstar); free(w->L); free(w->F); free(w->G); free(w->smax);
}

/* The stages of one step of size dt from qnew (time *tnew); qstar/tstar are
 * the stage registers.  RK3: FinSolveRK.cpp:158-211 with SetRKinfo.cpp:50-64;
 * MD (time_order 4): FinSolveMD.cpp:116-170; LxW: FinSolveLxW.cpp:120-176. */
static int take_stages(const fin_params* p, work_t* w, double* q, double* tnew, double* tstar, double dt)
{
    const grid_t* g = &w->g;
    int rc;
    if (p->time_stepping_method == FIN_TS_RK) {
        if (p->time_order != 3) return FIN_ERR_UNSUPPORTED;
        static const double a1[3] = {1.0, 0.75, 2.0e0 / 3.0e0};
        static const double a2[3] = {0.0, 0.25, 1.0e0 / 3.0e0};
        static const double bt[3] = {1.0, 0.25, 2.0e0 / 3.0e0};
        /* stage 1: Qnew -> Qstar */
        oracle_set_bnd(p, q);
        if ((rc = oracle_construct_l(p, q, w->L, w->smax))) return rc;
        update_soln(g, a1[0], a2[0], bt[0], dt, q, w->L, w->qstar);
        *tstar = a1[0] * *tnew + a2[0] * *tstar + bt[0] * dt;
        /* stage 2: Qstar -> Qstar (with Qnew) */
        oracle_set_bnd(p, w->qstar);
        if ((rc = oracle_construct_l(p, w->qstar, w->L, w->smax))) return rc;
        update_soln(g, a1[1], a2[1], bt[1], dt, q, w->L, w->qstar);
        *tstar = a1[1] * *tnew + a2[1] * *tstar + bt[1] * dt;
        /* stage 3: Qstar -> Qnew */
        oracle_set_bnd(p, w->qstar);
        if ((rc = oracle_construct_l(p, w->qstar, w->L, w->smax))) return rc;
        update_soln(g, a1[2], a2[2], bt[2], dt, w->qstar, w->L, q);
        *tnew = a1[2] * *tstar + a2[2] * *tnew + bt[2] * dt;
        return FIN_OK;
    }
    if (p->time_stepping_method == FIN_TS_MD) {
        /* FinSolveMD.cpp:116-170 (time_order 4) */
        if (p->time_order != 4) return FIN_ERR_UNSUPPORTED;
        memcpy(w->qold, q, w->n * sizeof(double));   /* Qold: the step's starting state */
        oracle_set_bnd(p, q);
        if ((rc = oracle_construct_integrated_r(p, 0.5 * dt, q, w->F, w->G))) return rc;
        if ((rc = oracle_construct_lxwl(p, q, w->F, w->G, w->L, w->smax))) return rc;
        for (int i = 1; i <= g->mx; i++)
            for (int j = 1; j <= g->my; j++)
                for (int m = 1; m <= g->meqn; m++) {
                    const size_t k = IDX(g, i, j, m);
                    w->qstar[k] = q[k] + 0.5 * dt * w->L[k];
                }
        *tstar = *tnew + 0.5 * dt;
        oracle_set_bnd(p, q);
        oracle_set_bnd(p, w->qstar);
        if ((rc = construct_integrated_r2(p, dt, 1.0, (1.0 / 6.0), q, 0.0, (1.0 / 3.0), w->qstar, w->F, w->G)))
            return rc;
        if ((rc = oracle_construct_lxwl(p, w->qstar, w->F, w->G, w->L, w->smax))) return rc;
        /* q^{n+1} = q_old + dt L; q here still holds q_old (the stages never wrote it) */
        for (int i = 1; i <= g->mx; i++)
            for (int j = 1; j <= g->my; j++)
                for (int m = 1; m <= g->meqn; m++) {
                    const size_t k = IDX(g, i, j, m);
                    q[k] = w->qold[k] + dt * w->L[k];
                }
        *tnew = *tnew + dt;   /* Qold.get_t() + dt, Qold.t == Qnew.t at step start */
        return FIN_OK;
    }
    if (p->time_stepping_method == FIN_TS_LXW) {
        /* FinSolveLxW.cpp:120-176 (no MPP limiter) */
        oracle_set_bnd(p, q);
        if ((rc = oracle_construct_integrated_r(p, dt, q, w->F, w->G))) return rc;
        if ((rc = oracle_construct_lxwl(p, q, w->F, w->G, w->L, w->smax))) return rc;
        for (int i = 1; i <= g->mx; i++)
            for (int j = 1; j <= g->my; j++)
                for (int m = 1; m <= g->meqn; m++) {
                    const size_t k = IDX(g, i, j, m);
                    q[k] = q[k] + dt * w->L[k];
                }
        *tnew = *tnew + dt;
        return FIN_OK;
    }
    return FIN_ERR_UNSUPPORTED;
}

int oracle_step_fixed(const fin_params* p, double* q, double dt, double* cfl)
{
    work_t w;
    work_init(&w, p);
    memcpy(w.qstar, q, w.n * sizeof(double));
    double tnew = 0.0, tstar = 0.0;
    int rc = take_stages(p, &w, q, &tnew, &tstar, dt);
    if (rc == FIN_OK) rc = get_cfl(p, dt, 1e300, w.smax, cfl);
    work_free(&w);
    return rc;
}

/* lib/2d/FinSolveRK.cpp:13-371 (the driver loop is shared by FinSolveMD.cpp
 * :21-291 and FinSolveLxW.cpp:16-245). */
int oracle_finsolve(const fin_params* p, double* q, double* t_io, double tend, double* dtv, int* nsteps)
{
    work_t w;
    work_init(&w, p);
    const double CFL_max = p->max_cfl, CFL_target = p->desired_cfl;
    double t = *t_io, tq = *t_io;      /* t: driver time; tq: Qnew.get_t() */
    double dt = dtv[1], cfl = 0.0;
    double tstar = t, told_q = t;
    memcpy(w.qstar, q, w.n * sizeof(double));
    int n_step = 0, accepted = 0, rc = FIN_OK;
    while (t < tend) {
        int m_accept = 0;
        n_step = n_step + 1;
        if (n_step > p->nv) { rc = FIN_ERR_NSTEPS; break; }
        memcpy(w.qold, q, w.n * sizeof(double));
        told_q = tq;
        while (m_accept == 0) {
            tq = t;
            const double told = t;
            if (told + dt > tend) dt = tend - told;
            t = told + dt;
            memset(w.smax, 0, w.nS * sizeof(double));
            if ((rc = take_stages(p, &w, q, &tq, &tstar, dt))) goto done;
            if ((rc = get_cfl(p, dt, dtv[2], w.smax, &cfl))) goto done;
            if (cfl > 0.0) dt = Min(dtv[2], dt * CFL_target / cfl);
            else dt = dtv[2];
            if (cfl <= CFL_max) m_accept = 1;
            else {
                t = told;
                memcpy(q, w.qold, w.n * sizeof(double));
                tq = told_q;
            }
        }
        accepted++;
    }
    dtv[1] = dt;
done:
    *t_io = tq;
    if (nsteps) *nsteps = accepted;
    work_free(&w);
    return rc;
}

/* Flat copies of the Jacobian and Hessian at one state (for tests). */
void oracle_flux_derivs(double gamma, const double* Q, double* Aout, double* Hout)
{
    double A[2][5][5], H[2][5][5][5];
    euler_jac_hess(gamma, Q, A, H, 1);
    memcpy(Aout, A, sizeof(A));
    memcpy(Hout, H, sizeof(H));
}

/* Diff1 / Diff2 of lib/WenoReconstruct.cpp:702-716 and :791-806 (5 points). */
static double diff1(double dx, const double* f)
{
    double tmp = (f[0] - f[4]) * (1.0 / 12.0);
    tmp += (-f[1] + f[3]) * (2.0 / 3.0);
    return tmp / dx;
}
static double diff2(double dx, const double* f)
{
    double tmp = (-f[0] - f[4]) * (1.0 / 12.0);
    tmp += (f[1] + f[3]) * (4.0 / 3.0);
    tmp += (-f[2]) * (5.0 / 2.0);
    return tmp / (dx * dx);
}

/* R = FluxFunc sampled over the whole ghosted grid (SampleFunction,
 * lib/2d/SampleFunction.cpp:62-125): Rf, Rg ghosted (mx,my,meqn). */
static void sample_flux(const fin_params* p, const double* q, double* Rf, double* Rg)
{
    const grid_t g = grid_of(p, p->mx, p->my);
    for (int i = 1 - g.mbc; i <= g.mx + g.mbc; i++)
        for (int j = 1 - g.mbc; j <= g.my + g.mbc; j++)
            euler_flux(p->gamma, q + IDX(&g, i, j, 1), Rf + IDX(&g, i, j, 1), Rg + IDX(&g, i, j, 1));
}

/* f_t, g_t (and with nterms > 2, f_tt, g_tt) at one cell:
 * ConstructIntegratedR.cpp:106-284 (1-state, 2nd-order mixed derivatives,
 * mixed4 = 0) and LocalIntegrate :298-523 (4th-order mixed stencil, mixed4 = 1). */
static void local_time_derivs(const fin_params* p, const grid_t* g, int i, int j, const double* q,
                              const double* Rf, const double* Rg, int nterms, int mixed4,
                              double* f_t, double* g_t, double* f_tt, double* g_tt)
{
    const double dx = get_dx(p), dy = get_dy(p);
    const int meqn = 5;
    double fx[5], gy[5], qx[5], qy[5];
    for (int m = 0; m < meqn; m++) {
        double Fv[5], Gv[5], qxv[5], qyv[5];
        for (int r = 0; r < 5; r++) {
            const int s = r - 2;
            Fv[r] = Rf[IDX(g, i + s, j, m + 1)];
            Gv[r] = Rg[IDX(g, i, j + s, m + 1)];
            qxv[r] = q[IDX(g, i + s, j, m + 1)];
            qyv[r] = q[IDX(g, i, j + s, m + 1)];
        }
        fx[m] = diff1(dx, Fv);
        qx[m] = diff1(dx, qxv);
        gy[m] = diff1(dy, Gv);
        qy[m] = diff1(dy, qyv);
    }
    double A[2][5][5], H[2][5][5][5];
    euler_jac_hess(p->gamma, q + IDX(g, i, j, 1), A, H, nterms > 2);
    for (int m1 = 0; m1 < meqn; m1++) {
        double tmp1 = 0., tmp2 = 0.;
        for (int m2 = 0; m2 < meqn; m2++) {
            tmp1 += -(A[0][m1][m2]) * (fx[m2] + gy[m2]);
            tmp2 += -(A[1][m1][m2]) * (fx[m2] + gy[m2]);
        }
        f_t[m1] = tmp1;
        g_t[m1] = tmp2;
    }
    for (int m = 0; m < meqn; m++) f_tt[m] = g_tt[m] = 0.0;
    if (nterms <= 2) return;
    double w[5], fxx[5], gyy[5], fxy[5], gxy[5], fpg_t[5];
    for (int m = 0; m < meqn; m++) {
        w[m] = fx[m] + gy[m];
        double Fv[5], Gv[5];
        for (int r = 0; r < 5; r++) {
            Fv[r] = Rf[IDX(g, i + r - 2, j, m + 1)];
            Gv[r] = Rg[IDX(g, i, j + r - 2, m + 1)];
        }
        fxx[m] = diff2(dx, Fv);
        gyy[m] = diff2(dy, Gv);
    }
    for (int m = 0; m < meqn; m++) {
        for (int d = 0; d < 2; d++) {
            const double* R = d == 0 ? Rf : Rg;
#define RR(a, b) R[IDX(g, i + (a), j + (b), m + 1)]
            double tmp;
            if (!mixed4) {
                tmp = 0.5 * (RR(1, 1) - RR(-1, 1)) / dx;
                tmp -= 0.5 * (RR(1, -1) - RR(-1, -1)) / dx;
                tmp *= 0.5 / dy;
            } else {
                tmp = 0.25 * (RR(1, 1) - RR(-1, 1) - RR(1, -1) + RR(-1, -1));
                tmp -= (1. / 24.) * (RR(2, 1) + RR(-2, -1) - RR(2, -1) - RR(-2, 1) -
                                     RR(1, 2) - RR(-1, -2) + RR(1, -2) + RR(-1, 2));
                tmp *= (1. / (dx * dy));
            }
#undef RR
            if (d == 0) fxy[m] = tmp; else gxy[m] = tmp;
        }
    }
    for (int m = 0; m < meqn; m++) {
        double tmp = 0.;
        for (int m1 = 0; m1 < meqn; m1++)
            for (int m2 = 0; m2 < meqn; m2++) {
                tmp += H[0][m][m1][m2] * qx[m1] * w[m2];
                tmp += H[1][m][m1][m2] * qy[m1] * w[m2];
            }
        for (int m1 = 0; m1 < meqn; m1++) {
            tmp += A[0][m][m1] * (fxx[m1] + gxy[m1]);
            tmp += A[1][m][m1] * (fxy[m1] + gyy[m1]);
        }
        fpg_t[m] = tmp;
    }
    for (int m1 = 0; m1 < meqn; m1++) {
        double tmp1 = 0., tmp2 = 0.;
        for (int m2 = 0; m2 < meqn; m2++) {
            tmp1 += A[0][m1][m2] * fpg_t[m2];
            tmp2 += A[1][m1][m2] * fpg_t[m2];
        }
        f_tt[m1] = tmp1;
        g_tt[m1] = tmp2;
    }
    for (int m = 0; m < meqn; m++) {
        double tmp1 = 0., tmp2 = 0.;
        for (int m1 = 0; m1 < meqn; m1++)
            for (int m2 = 0; m2 < meqn; m2++) {
                tmp1 += H[0][m][m1][m2] * w[m1] * w[m2];
                tmp2 += H[1][m][m1][m2] * w[m1] * w[m2];
            }
        f_tt[m] = f_tt[m] + tmp1;
        g_tt[m] = g_tt[m] + tmp2;
    }
}

/* ConstructIntegratedR, 1-state (lib/2d/ConstructIntegratedR.cpp:59-296):
 * F = R + dt/2 (f_t + dt/3 f_tt) on [1-3, mx+3] x [1-3, my+3]; the Hessian
 * terms are present when time_order > 2 (:171). */
int oracle_construct_integrated_r(const fin_params* p, double dt, const double* q, double* F, double* G)
{
    if (p->meqn != 5 || p->mbc < 5) return FIN_ERR_ARG;
    const grid_t g = grid_of(p, p->mx, p->my);
    const size_t n = numel(&g);
    double* Rf = (double*)malloc(n * sizeof(double));
    double* Rg = (double*)malloc(n * sizeof(double));
    sample_flux(p, q, Rf, Rg);
    const int nterms = p->time_order > 2 ? 3 : 2;
    for (int i = 1 - 3; i <= g.mx + 3; i++)
        for (int j = 1 - 3; j <= g.my + 3; j++) {
            double f_t[5], g_t[5], f_tt[5], g_tt[5];
            local_time_derivs(p, &g, i, j, q, Rf, Rg, nterms, 0, f_t, g_t, f_tt, g_tt);
            for (int m = 1; m <= 5; m++) {
                const size_t k = IDX(&g, i, j, m);
                F[k] = Rf[k] + 0.5 * dt * (f_t[m - 1] + dt / 3.0 * f_tt[m - 1]);
                G[k] = Rg[k] + 0.5 * dt * (g_t[m - 1] + dt / 3.0 * g_tt[m - 1]);
            }
        }
    free(Rf);
    free(Rg);
    return FIN_OK;
}

/* ConstructIntegratedR, 2-state (lib/2d/ConstructIntegratedR.cpp:525-606):
 * F = a1 R1 + dt (b1 f1_t) + a2 R2 + dt (b2 f2_t), LocalIntegrate with nterms 2. */
static int construct_integrated_r2(const fin_params* p, double dt, double a1, double b1, const double* q1,
                                   double a2, double b2, const double* q2, double* F, double* G)
{
    if (p->meqn != 5 || (p->mbc + 1) / 2 != 3) return FIN_ERR_ARG;
    const grid_t g = grid_of(p, p->mx, p->my);
    const size_t n = numel(&g);
    double* R1f = (double*)malloc(n * sizeof(double));
    double* R1g = (double*)malloc(n * sizeof(double));
    double* R2f = (double*)malloc(n * sizeof(double));
    double* R2g = (double*)malloc(n * sizeof(double));
    sample_flux(p, q1, R1f, R1g);
    sample_flux(p, q2, R2f, R2g);
    for (int i = 1 - 3; i <= g.mx + 3; i++)
        for (int j = 1 - 3; j <= g.my + 3; j++) {
            double f1t[5], g1t[5], f2t[5], g2t[5], z1[5], z2[5];
            local_time_derivs(p, &g, i, j, q1, R1f, R1g, 2, 1, f1t, g1t, z1, z2);
            local_time_derivs(p, &g, i, j, q2, R2f, R2g, 2, 1, f2t, g2t, z1, z2);
            for (int m = 1; m <= 5; m++) {
                const size_t k = IDX(&g, i, j, m);
                F[k] = a1 * R1f[k] + dt * (b1 * f1t[m - 1]) + a2 * R2f[k] + dt * (b2 * f2t[m - 1]);
                G[k] = a1 * R1g[k] + dt * (b1 * g1t[m - 1]) + a2 * R2g[k] + dt * (b2 * g2t[m - 1]);
            }
        }
    free(R1f); free(R1g); free(R2f); free(R2g);
    return FIN_OK;
}

/* lib/2d/ConSoln.cpp:52-64 */
void oracle_conservation_totals(const fin_params* p, const double* q, double* totals)
{
    const grid_t g = grid_of(p, p->mx, p->my);
    const double dx = get_dx(p), dy = get_dy(p);
    for (int m = 1; m <= g.meqn; m++) {
        double s = 0.0;
        for (int i = 1; i <= g.mx; i++)
            for (int j = 1; j <= g.my; j++) s = s + dx * dy * q[IDX(&g, i, j, m)];
        totals[m - 1] = s;
    }
}


/* ---------------------------------------------------------------------- */
/* Troubled-cell indicator: features and labels of every face              */
/* ---------------------------------------------------------------------- */

/* x faces ((mx+1) x my, j fastest) then y faces (mx x (my+1)); face (i, j)
 * separates 0-based cells i-1 and i along its direction, stencil cells
 * i-3 .. i+2 (ConstructL.cpp:94-113).  q ghosted with BCs applied.
 *   X[f*20 + 5t + s]: (w_k(s+1) - w_k(s)) / max(max_s |.|, 1e-3), w = L q at
 *     the face average, fields k = 0, mu, mv, 4 (t = 0..3);
 *   y[f]: 1 if the WENO5-JS weights of gp or gm of any of those fields depart
 *     from (0.1, 0.6, 0.3) by more than 10 % (WenoReconstruct.cpp:104,131-134). */
void oracle_face_samples(const fin_params* p, const double* q, double* X, unsigned char* y)
{
    const grid_t g = grid_of(p, p->mx, p->my);
    double alpha1 = 0., alpha2 = 0.;
    if (p->global_alpha) oracle_global_wave_spd(p, q, &alpha1, &alpha2);
    long long f = 0;
    for (int ixy = 1; ixy <= 2; ixy++) {
        const int ni = ixy == 1 ? g.mx + 1 : g.mx, nj = ixy == 1 ? g.my : g.my + 1;
        for (int i = 0; i < ni; i++)
            for (int j = 0; j < nj; j++, f++) {
                const int di = ixy == 1 ? 1 : 0, dj = ixy == 1 ? 0 : 1;
                /* 1-based cells of the stencil: (i+1) + di*(s-3), (j+1) + dj*(s-3) */
                double Qs[6][MEQN_MAX], Fs[6][MEQN_MAX];
                for (int s = 0; s < 6; s++) {
                    const int I = i + 1 + di * (s - 3), J = j + 1 + dj * (s - 3);
                    const double* Qp = q + IDX(&g, I, J, 1);
                    double fx[MEQN_MAX], fy[MEQN_MAX];
                    euler_flux(p->gamma, Qp, fx, fy);
                    for (int m = 0; m < 5; m++) {
                        Qs[s][m] = Qp[m];
                        Fs[s][m] = ixy == 1 ? fx[m] : fy[m];
                    }
                }
                double Qavg[MEQN_MAX];
                for (int m = 0; m < 5; m++) Qavg[m] = 0.5 * (Qs[3][m] + Qs[2][m]);
                eig_t el = euler_eig(ixy, p->gamma, Qavg, 0);
                double W[6][MEQN_MAX], G[6][MEQN_MAX];
                for (int s = 0; s < 6; s++) {
                    euler_left(&el, Qs[s], W[s]);
                    euler_left(&el, Fs[s], G[s]);
                }
                const int fields[4] = {0, el.mu, el.mv, 4};
                for (int t = 0; t < 4; t++) {
                    double d[5], mm = 1e-3;
                    for (int s = 0; s < 5; s++) {
                        d[s] = W[s + 1][fields[t]] - W[s][fields[t]];
                        if (fabs(d[s]) > mm) mm = fabs(d[s]);
                    }
                    for (int s = 0; s < 5; s++) X[f * 20 + t * 5 + s] = d[s] / mm;
                }
                double s1, s2;
                if (ixy == 1) euler_wave_spd(p->gamma, 1.0, 0.0, Qs[2], Qs[3], &s1, &s2);
                else euler_wave_spd(p->gamma, 0.0, 1.0, Qs[2], Qs[3], &s1, &s2);
                const double alpha = Max(ixy == 1 ? alpha1 : alpha2, Max(fabs(s1), fabs(s2)));
                const double la = p->alpha_scaling * alpha;
                double dep = 0.0;
                for (int t = 0; t < 4; t++) {
                    const int k = fields[t];
                    double gp[5], gm[5], w[3];
                    for (int s = 0; s < 5; s++) {
                        gp[s] = 0.5 * (G[s][k] + la * W[s][k]);
                        gm[s] = 0.5 * (G[5 - s][k] - la * W[5 - s][k]);
                    }
                    static const double dl[3] = {0.1, 0.6, 0.3};
                    oracle_weno_js5_weights(p->epsilon, p->power_param, gp, w);
                    for (int r = 0; r < 3; r++) dep = Max(dep, fabs(w[r] - dl[r]) / dl[r]);
                    oracle_weno_js5_weights(p->epsilon, p->power_param, gm, w);
                    for (int r = 0; r < 3; r++) dep = Max(dep, fabs(w[r] - dl[r]) / dl[r]);
                }
                y[f] = dep > 0.1 ? 1 : 0;
            }
    }
}
