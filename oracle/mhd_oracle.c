/*
 * mhd_oracle.c -- CPU restatement (plain C, FP64) of the reference's 2D ideal
 * MHD path: ConstructL of lib/2d with the MHD callbacks of apps/2d/mhd/lib
 * (8 components, 8 x 8 eigenvector projections), the Hamilton-Jacobi
 * right-hand side of the magnetic potential A3, the stage update with the
 * auxiliary array, constrained transport, the MHD CFL number and the SSP-RK3
 * driver of apps/2d/mhd/lib/FinSolveRK.cpp, with the doubly periodic
 * boundaries of apps/2d/mhd/orszag_tang.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this library, and only as the checker.
 *
 * Expressions keep the reference's operation order (left-to-right
 * evaluation, divisions where it divides), so that, built without FMA
 * contraction, the results are bit-identical to the reference's own sources
 * compiled in place (oracle/_ref/libfinref_mhd.so); the tests pin that.
 *
 * Arrays use the reference's ghosted dTensorBC3 layout: q (mx, my, 8) and
 * aux (mx, my, 1), idx(i,j,m) = ((i+mbc-1)*(my+2*mbc) + (j+mbc-1))*meqn + (m-1).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "finess_oracle.h"

#define MQ 8

/* dog_math.h:18-22 */
static double Max(double a, double b) { return a > b ? a : b; }
static double Min(double a, double b) { return a < b ? a : b; }
/* std::max as ConstructHJ_L.cpp:478-489 uses it */
static double std_max(double a, double b) { return a < b ? b : a; }

typedef struct { int mx, my, mbc, meqn, sy; } mgrid_t;

static mgrid_t mgrid(const fin_params* p, int mx, int my, int meqn)
{
    mgrid_t g = {mx, my, p->mbc, meqn, my + 2 * p->mbc};
    return g;
}
static size_t MI(const mgrid_t* g, int i, int j, int m)
{
    return ((size_t)(i + g->mbc - 1) * g->sy + (size_t)(j + g->mbc - 1)) * g->meqn + (m - 1);
}
static size_t mnumel(const mgrid_t* g) { return (size_t)(g->mx + 2 * g->mbc) * g->sy * g->meqn; }
static double get_dx(const fin_params* p) { return (p->xhigh - p->xlow) / p->mx; }
static double get_dy(const fin_params* p) { return (p->yhigh - p->ylow) / p->my; }

/* ---------------------------------------------------------------------- */
/* Callbacks (apps/2d/mhd/lib)                                             */
/* ---------------------------------------------------------------------- */

/* FluxFunc.cpp:19-54, one point: f = flux(.,1), g = flux(.,2). */
static void mhd_flux(double gamma, const double* Q, double* f, double* g)
{
    const double rho = Q[0];
    const double u1 = Q[1] / rho, u2 = Q[2] / rho, u3 = Q[3] / rho;
    const double energy = Q[4];
    const double B1 = Q[5], B2 = Q[6], B3 = Q[7];
    const double press = (gamma - 1.0e0) * (energy - 0.5 * rho * (u1 * u1 + u2 * u2 + u3 * u3) -
                                            0.5 * (B1 * B1 + B2 * B2 + B3 * B3));
    const double Bm = 0.5 * (B1 * B1 + B2 * B2 + B3 * B3);
    const double Bu = u1 * B1 + u2 * B2 + u3 * B3;
    const double eb = energy + press + Bm;
    f[0] = rho * u1;
    f[1] = rho * u1 * u1 + press + Bm - B1 * B1;
    f[2] = rho * u1 * u2 - B1 * B2;
    f[3] = rho * u1 * u3 - B1 * B3;
    f[4] = u1 * eb - B1 * Bu;
    f[5] = 0.0;
    f[6] = u1 * B2 - u2 * B1;
    f[7] = u1 * B3 - u3 * B1;
    g[0] = rho * u2;
    g[1] = rho * u1 * u2 - B2 * B1;
    g[2] = rho * u2 * u2 + press + Bm - B2 * B2;
    g[3] = rho * u2 * u3 - B2 * B3;
    g[4] = u2 * eb - B2 * Bu;
    g[5] = u2 * B1 - u1 * B2;
    g[6] = 0.0;
    g[7] = u2 * B3 - u3 * B2;
}

/* Fast magnetosonic speed of SetWaveSpd.cpp:66-74 (pow(x,2) == x*x; the
 * first magnetic component enters for either normal). */
static double fast_speed(double a2, double Bm2, double rho, double B1)
{
    const double t = a2 + Bm2 / rho;
    return sqrt(0.5 * (a2 + Bm2 / rho + sqrt(fabs(t * t - 4.0 * a2 * B1 * B1 / rho))));
}

typedef struct { double rho, u1, u2, u3, press, B1, B2, B3, Bm2; } side_t;

static side_t side_of(double gamma, const double* Q)
{
    side_t s;
    s.rho = Q[0];
    s.u1 = Q[1] / s.rho;
    s.u2 = Q[2] / s.rho;
    s.u3 = Q[3] / s.rho;
    const double energy = Q[4];
    s.B1 = Q[5]; s.B2 = Q[6]; s.B3 = Q[7];
    s.Bm2 = s.B1 * s.B1 + s.B2 * s.B2 + s.B3 * s.B3;
    const double um2 = s.u1 * s.u1 + s.u2 * s.u2 + s.u3 * s.u3;
    s.press = (gamma - 1.0e0) * (energy - 0.5 * s.rho * um2 - 0.5 * s.Bm2);
    return s;
}

/* SetWaveSpd.cpp:11-90 (arithmetic-mean state). */
static void mhd_wave_spd(double gamma, double n1, double n2, const double* Ql, const double* Qr, double* s1,
                         double* s2)
{
    const side_t l = side_of(gamma, Ql), r = side_of(gamma, Qr);
    const double rho = 0.5e0 * (l.rho + r.rho);
    const double u1 = 0.5e0 * (l.u1 + r.u1);
    const double u2 = 0.5e0 * (l.u2 + r.u2);
    const double press = 0.5e0 * (l.press + r.press);
    const double B1 = 0.5e0 * (l.B1 + r.B1);
    const double B2 = 0.5e0 * (l.B2 + r.B2);
    const double B3 = 0.5e0 * (l.B3 + r.B3);
    const double Bm2 = B1 * B1 + B2 * B2 + B3 * B3;
    const double a2l = fabs(gamma * l.press / l.rho);
    const double a2r = fabs(gamma * r.press / r.rho);
    const double a2 = fabs(gamma * press / rho);
    const double nmag = sqrt(n1 * n1 + n2 * n2);
    const double cf_l = nmag * fast_speed(a2l, l.Bm2, l.rho, l.B1);
    const double cf_r = nmag * fast_speed(a2r, r.Bm2, r.rho, r.B1);
    const double cf = nmag * fast_speed(a2, Bm2, rho, B1);
    const double un = n1 * u1 + n2 * u2;
    const double unl = n1 * l.u1 + n2 * l.u2;
    const double unr = n1 * r.u1 + n2 * r.u2;
    *s1 = Min(unl - cf_l, un - cf);
    *s2 = Max(unr + cf_r, un + cf);
}

/* Left and right eigenvector matrices of ProjectLeftEig.cpp:13-192 and
 * ProjectRightEig.cpp:13-190 at the average state Q (0-based components). */
static void mhd_eig(int ixy, double gamma, const double* Q, double L[MQ][MQ], double Rm[MQ][MQ])
{
    const int mu1 = ixy == 1 ? 1 : 2, mu2 = ixy == 1 ? 2 : 1;
    const int mb1 = ixy == 1 ? 5 : 6, mb2 = ixy == 1 ? 6 : 5;
    const double rho = Q[0];
    const double u1 = Q[mu1] / rho, u2 = Q[mu2] / rho, u3 = Q[3] / rho;
    const double energy = Q[4];
    const double B1 = Q[mb1], B2 = Q[mb2], B3 = Q[7];
    const double um2 = 0.5 * (u1 * u1 + u2 * u2 + u3 * u3);
    const double Bm2 = 0.5 * (B1 * B1 + B2 * B2 + B3 * B3);
    const double press = (gamma - 1.0) * (energy - rho * um2 - Bm2);
    const double rhosq = sqrt(rho);
    const double twosq = sqrt(2.0);
    const double gm1 = gamma - 1.0;
    const double a2 = (gamma * press / rho);
    const double a = sqrt(a2);
    const double d = a2 + (B1 * B1 + B2 * B2 + B3 * B3) / rho;
    const double cf = sqrt(0.5 * (d + sqrt(d * d - 4.0 * a2 * B1 * B1 / rho)));
    const double cs = sqrt(0.5 * (d - sqrt(d * d - 4.0 * a2 * B1 * B1 / rho)));
    double beta1, beta2, beta3, alphaf, alphas;
    beta1 = B1 < 0.0 ? -1.0 : 1.0;
    if ((B2 * B2 + B3 * B3) <= 1.0e-12) {
        beta2 = 1.0 / twosq;
        beta3 = 1.0 / twosq;
    } else {
        beta2 = B2 / sqrt(B2 * B2 + B3 * B3);
        beta3 = B3 / sqrt(B2 * B2 + B3 * B3);
    }
    if ((B2 * B2 + B3 * B3) <= 1.0e-12 && fabs(a2 - B1 * B1 / rho) <= 1.0e-12) {
        alphaf = sin(atan(1.0) / 2.0);
        alphas = cos(atan(1.0) / 2.0);
    } else {
        alphaf = sqrt(fabs(a2 - cs * cs)) / sqrt(fabs(cf * cf - cs * cs));
        alphas = sqrt(fabs(cf * cf - a2)) / sqrt(fabs(cf * cf - cs * cs));
    }

    /* primitive left eigenvectors, one row per wave (ProjectLeftEig.cpp:92-174) */
    double ru[MQ][MQ];
    memset(ru, 0, sizeof(ru));
    ru[0][mu1] = -alphaf * cf / (2.0 * a2);
    ru[0][mu2] = alphas * cs * beta2 * beta1 / (2.0 * a2);
    ru[0][3] = alphas * cs * beta3 * beta1 / (2.0 * a2);
    ru[0][4] = alphaf / (2.0 * rho * a2);
    ru[0][mb2] = alphas * beta2 / (2.0 * rhosq * a);
    ru[0][7] = alphas * beta3 / (2.0 * rhosq * a);
    ru[1][mu2] = -beta3 / twosq;
    ru[1][3] = beta2 / twosq;
    ru[1][mb2] = -beta3 / (twosq * rhosq);
    ru[1][7] = beta2 / (twosq * rhosq);
    ru[2][mu1] = -alphas * cs / (2.0 * a2);
    ru[2][mu2] = -alphaf * cf * beta2 * beta1 / (2.0 * a2);
    ru[2][3] = -alphaf * cf * beta3 * beta1 / (2.0 * a2);
    ru[2][4] = alphas / (2.0 * rho * a2);
    ru[2][mb2] = -alphaf * beta2 / (2.0 * rhosq * a);
    ru[2][7] = -alphaf * beta3 / (2.0 * rhosq * a);
    ru[3][0] = 1.0;
    ru[3][4] = -1.0 / a2;
    ru[4][mb1] = 1.0;
    ru[5][mu1] = alphas * cs / (2.0 * a2);
    ru[5][mu2] = alphaf * cf * beta2 * beta1 / (2.0 * a2);
    ru[5][3] = alphaf * cf * beta3 * beta1 / (2.0 * a2);
    ru[5][4] = alphas / (2.0 * rho * a2);
    ru[5][mb2] = -alphaf * beta2 / (2.0 * rhosq * a);
    ru[5][7] = -alphaf * beta3 / (2.0 * rhosq * a);
    ru[6][mu2] = -beta3 / twosq;
    ru[6][3] = beta2 / twosq;
    ru[6][mb2] = beta3 / (twosq * rhosq);
    ru[6][7] = -beta2 / (twosq * rhosq);
    ru[7][mu1] = alphaf * cf / (2.0 * a2);
    ru[7][mu2] = -alphas * cs * beta2 * beta1 / (2.0 * a2);
    ru[7][3] = -alphas * cs * beta3 * beta1 / (2.0 * a2);
    ru[7][4] = alphaf / (2.0 * rho * a2);
    ru[7][mb2] = alphas * beta2 / (2.0 * rhosq * a);
    ru[7][7] = alphas * beta3 / (2.0 * rhosq * a);
    /* conservative rows (ProjectLeftEig.cpp:179-192) */
    for (int m = 0; m < MQ; m++) {
        const double* r = ru[m];
        L[m][0] = r[0] - r[mu1] * u1 / rho - r[mu2] * u2 / rho - r[3] * u3 / rho + r[4] * um2 * gm1;
        L[m][mu1] = r[mu1] / rho - r[4] * u1 * gm1;
        L[m][mu2] = r[mu2] / rho - r[4] * u2 * gm1;
        L[m][3] = r[3] / rho - r[4] * u3 * gm1;
        L[m][4] = r[4] * gm1;
        L[m][mb1] = -r[4] * B1 * gm1 + r[mb1];
        L[m][mb2] = -r[4] * B2 * gm1 + r[mb2];
        L[m][7] = -r[4] * B3 * gm1 + r[7];
    }

    /* primitive right eigenvectors, one column per wave (ProjectRightEig.cpp:89-171) */
    double rc[MQ][MQ];   /* rc[row][wave] */
    memset(rc, 0, sizeof(rc));
    rc[0][0] = rho * alphaf;
    rc[mu1][0] = -alphaf * cf;
    rc[mu2][0] = alphas * beta2 * cs * beta1;
    rc[3][0] = alphas * beta3 * cs * beta1;
    rc[4][0] = alphaf * gamma * press;
    rc[mb2][0] = alphas * beta2 * a * rhosq;
    rc[7][0] = alphas * beta3 * a * rhosq;
    rc[mu2][1] = -beta3 / twosq;
    rc[3][1] = beta2 / twosq;
    rc[mb2][1] = -beta3 * rhosq / twosq;
    rc[7][1] = beta2 * rhosq / twosq;
    rc[0][2] = rho * alphas;
    rc[mu1][2] = -alphas * cs;
    rc[mu2][2] = -alphaf * beta2 * cf * beta1;
    rc[3][2] = -alphaf * beta3 * cf * beta1;
    rc[4][2] = alphas * gamma * press;
    rc[mb2][2] = -alphaf * beta2 * a * rhosq;
    rc[7][2] = -alphaf * beta3 * a * rhosq;
    rc[0][3] = 1.0;
    rc[mb1][4] = 1.0;
    rc[0][5] = rho * alphas;
    rc[mu1][5] = alphas * cs;
    rc[mu2][5] = alphaf * beta2 * cf * beta1;
    rc[3][5] = alphaf * beta3 * cf * beta1;
    rc[4][5] = alphas * gamma * press;
    rc[mb2][5] = -alphaf * beta2 * a * rhosq;
    rc[7][5] = -alphaf * beta3 * a * rhosq;
    rc[mu2][6] = -beta3 / twosq;
    rc[3][6] = beta2 / twosq;
    rc[mb2][6] = beta3 * rhosq / twosq;
    rc[7][6] = -beta2 * rhosq / twosq;
    rc[0][7] = rho * alphaf;
    rc[mu1][7] = alphaf * cf;
    rc[mu2][7] = -alphas * beta2 * cs * beta1;
    rc[3][7] = -alphas * beta3 * cs * beta1;
    rc[4][7] = alphaf * gamma * press;
    rc[mb2][7] = alphas * beta2 * a * rhosq;
    rc[7][7] = alphas * beta3 * a * rhosq;
    /* conservative columns (ProjectRightEig.cpp:176-190) */
    for (int m = 0; m < MQ; m++) {
        Rm[0][m] = rc[0][m];
        Rm[mu1][m] = rc[mu1][m] * rho + rc[0][m] * u1;
        Rm[mu2][m] = rc[mu2][m] * rho + rc[0][m] * u2;
        Rm[3][m] = rc[3][m] * rho + rc[0][m] * u3;
        Rm[4][m] = um2 * rc[0][m] + rho * u1 * rc[mu1][m] + rho * u2 * rc[mu2][m] + rho * u3 * rc[3][m] +
                   rc[4][m] / gm1 + B1 * rc[mb1][m] + B2 * rc[mb2][m] + B3 * rc[7][m];
        Rm[mb1][m] = rc[mb1][m];
        Rm[mb2][m] = rc[mb2][m];
        Rm[7][m] = rc[7][m];
    }
}

/* Mat-vec of ProjectLeftEig.cpp:194-206 / ProjectRightEig.cpp:194-203. */
static void matvec8(double M[MQ][MQ], const double* x, double* y)
{
    for (int m = 0; m < MQ; m++) {
        double s = 0.0;
        for (int l = 0; l < MQ; l++) s = s + M[m][l] * x[l];
        y[m] = s;
    }
}

/* ---------------------------------------------------------------------- */
/* Boundary conditions, wave speeds, ConstructL                            */
/* ---------------------------------------------------------------------- */

static int wrap(int k, int n)
{
    while (k < 1) k += n;
    while (k > n) k -= n;
    return k;
}

/* apps/2d/mhd/orszag_tang/SetBndValues.cpp:44-230: every ghost cell of q
 * and aux (A3 unchanged: A3_original_to_periodic is the identity there)
 * takes the periodic image, corners included. */
void oracle_mhd_set_bnd(const fin_params* p, double* q, double* aux)
{
    const mgrid_t g = mgrid(p, p->mx, p->my, MQ), ga = mgrid(p, p->mx, p->my, 1);
    for (int i = 1 - g.mbc; i <= g.mx + g.mbc; i++)
        for (int j = 1 - g.mbc; j <= g.my + g.mbc; j++) {
            if (i >= 1 && i <= g.mx && j >= 1 && j <= g.my) continue;
            const int si = wrap(i, g.mx), sj = wrap(j, g.my);
            for (int m = 1; m <= MQ; m++) q[MI(&g, i, j, m)] = q[MI(&g, si, sj, m)];
            if (aux) aux[MI(&ga, i, j, 1)] = aux[MI(&ga, si, sj, 1)];
        }
}

/* lib/2d/GlobalWaveSpd.cpp:41-78 with the MHD SetWaveSpd. */
void oracle_mhd_global_wave_spd(const fin_params* p, const double* q, double* alpha1, double* alpha2)
{
    const mgrid_t g = mgrid(p, p->mx, p->my, MQ);
    double a1 = 0.0, a2 = 0.0, s1, s2;
    for (int i = 1; i <= g.mx; i++)
        for (int j = 1; j <= g.my; j++) {
            const double* Q = q + MI(&g, i, j, 1);
            mhd_wave_spd(p->gamma, 1.0, 0.0, Q, Q, &s1, &s2);
            a1 = Max(a1, Max(fabs(s1), fabs(s2)));
            mhd_wave_spd(p->gamma, 0.0, 1.0, Q, Q, &s1, &s2);
            a2 = Max(a2, Max(fabs(s1), fabs(s2)));
        }
    *alpha1 = a1;
    *alpha2 = a2;
}

/* lib/2d/ConstructL.cpp:13-408 with meqn = 8 and the MHD callbacks.  The
 * face loop body is ConstructL.cpp:72-206 (x) and 224-356 (y). */
int oracle_mhd_construct_l(const fin_params* p, const double* q, double* L, double* smax)
{
    if (p->space_order != 5 ||
        (p->weno_version != FIN_WENO_JS && p->weno_version != FIN_WENO_Z && p->weno_version != FIN_WENO_FD))
        return FIN_ERR_ARG;
    const mgrid_t g = mgrid(p, p->mx, p->my, MQ);
    const mgrid_t gF = mgrid(p, p->mx + 1, p->my, MQ), gG = mgrid(p, p->mx, p->my + 1, MQ);
    const mgrid_t gS = {p->mx + 1, p->my + 1, p->mbc, 2, p->my + 1 + 2 * p->mbc};
    const int mx = g.mx, my = g.my;
    const double dx = get_dx(p), dy = get_dy(p);
    double* Fhat = (double*)calloc(mnumel(&gF), sizeof(double));
    double* Ghat = (double*)calloc(mnumel(&gG), sizeof(double));
    double alpha1 = 0., alpha2 = 0.;
    if (p->global_alpha) oracle_mhd_global_wave_spd(p, q, &alpha1, &alpha2);

    for (int ixy = 1; ixy <= 2; ixy++) {
        const int imax = ixy == 1 ? mx + 1 : mx, jmax = ixy == 1 ? my : my + 1;
        const int di = ixy == 1 ? 1 : 0, dj = ixy == 1 ? 0 : 1;
        for (int i = 1; i <= imax; i++)
            for (int j = 1; j <= jmax; j++) {
                const double* Qr = q + MI(&g, i, j, 1);
                const double* Ql = q + MI(&g, i - di, j - dj, 1);
                double Qavg[MQ], w[6][MQ], gv[6][MQ], Lm[MQ][MQ], Rm[MQ][MQ];
                for (int m = 0; m < MQ; m++) Qavg[m] = 0.5 * (Qr[m] + Ql[m]);
                mhd_eig(ixy, p->gamma, Qavg, Lm, Rm);
                for (int s = 1; s <= 6; s++) {
                    const double* Qs = q + MI(&g, i + di * (s - 4), j + dj * (s - 4), 1);
                    double fx[MQ], fy[MQ];
                    mhd_flux(p->gamma, Qs, fx, fy);
                    matvec8(Lm, Qs, w[s - 1]);
                    matvec8(Lm, ixy == 1 ? fx : fy, gv[s - 1]);
                }
                double s1, s2;
                mhd_wave_spd(p->gamma, ixy == 1 ? 1.0 : 0.0, ixy == 1 ? 0.0 : 1.0, Ql, Qr, &s1, &s2);
                const double alpha = Max(ixy == 1 ? alpha1 : alpha2, Max(fabs(s1), fabs(s2)));
                double* sm = smax + MI(&gS, i, j, ixy);
                *sm = Max(*sm, alpha);
                const double l_alpha = p->alpha_scaling * alpha;
                double ghat[MQ], fhat[MQ];
                for (int m = 0; m < MQ; m++) {
                    double gp[5], gm[5];
                    for (int s = 1; s <= 5; s++) {
                        gp[s - 1] = 0.5 * (gv[s - 1][m] + l_alpha * w[s - 1][m]);
                        gm[s - 1] = 0.5 * (gv[5 - s + 1][m] - l_alpha * w[5 - s + 1][m]);
                    }
                    ghat[m] = oracle_weno5(p->weno_version, p->epsilon, p->power_param, gp) +
                              oracle_weno5(p->weno_version, p->epsilon, p->power_param, gm);
                }
                matvec8(Rm, ghat, fhat);
                double* out = ixy == 1 ? Fhat + MI(&gF, i, j, 1) : Ghat + MI(&gG, i, j, 1);
                for (int m = 0; m < MQ; m++) out[m] = fhat[m];
            }
    }
    /* ConstructL.cpp:390-401 */
    for (int i = 1; i <= mx; i++)
        for (int j = 1; j <= my; j++)
            for (int m = 1; m <= MQ; m++) {
                double tmp = -(Fhat[MI(&gF, i + 1, j, m)] - Fhat[MI(&gF, i, j, m)]) / dx;
                tmp = tmp - (Ghat[MI(&gG, i, j + 1, m)] - Ghat[MI(&gG, i, j, m)]) / dy;
                L[MI(&g, i, j, m)] = tmp;
            }
    free(Fhat);
    free(Ghat);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Magnetic potential, constrained transport, stepping                    */
/* ---------------------------------------------------------------------- */

/* max_speed_in_x_y_directions, ConstructHJ_L.cpp:472-497. */
static void hj_max_speeds(const fin_params* p, const double* q, double* sx, double* sy)
{
    const mgrid_t g = mgrid(p, p->mx, p->my, MQ);
    double mxs = 1e-15, mys = 1e-15;
    for (int i = 1; i <= g.mx; i++)
        for (int j = 1; j <= g.my; j++) {
            const double* Q = q + MI(&g, i, j, 1);
            mxs = std_max(mxs, fabs(Q[1] / Q[0]));
            mys = std_max(mys, fabs(Q[2] / Q[0]));
        }
    *sx = mxs;
    *sy = mys;
}

/* ConstructHJ_L_Order1 (ConstructHJ_L.cpp:29-113): Laux zero everywhere
 * except cells -1 .. mx+2, -1 .. my+2. */
int oracle_mhd_construct_hj_l(const fin_params* p, const double* q, const double* aux, double* Laux)
{
    const mgrid_t g = mgrid(p, p->mx, p->my, MQ), ga = mgrid(p, p->mx, p->my, 1);
    if (p->space_order != 5 || p->mbc < 5) return FIN_ERR_ARG;
    const int ws = 5, r = 3;
    const double dx = get_dx(p), dy = get_dy(p);
    double msx, msy;
    hj_max_speeds(p, q, &msx, &msy);
    memset(Laux, 0, mnumel(&ga) * sizeof(double));
    const int ver = p->weno_version;
    for (int i = 1 - 2; i <= g.mx + 2; i++)
        for (int j = 1 - 2; j <= g.my + 2; j++) {
            double in[5];
#define A(ii, jj) aux[MI(&ga, (ii), (jj), 1)]
            for (int k = 1; k <= ws; k++) in[k - 1] = (A(i - r + k, j) - A(i - r + k - 1, j)) / dx;
            const double A3xm = oracle_weno5(ver, p->epsilon, p->power_param, in);
            for (int k = 1; k <= ws; k++) in[k - 1] = (A(i + r - (k - 1), j) - A(i + r - k, j)) / dx;
            const double A3xp = oracle_weno5(ver, p->epsilon, p->power_param, in);
            for (int k = 1; k <= ws; k++) in[k - 1] = (A(i, j - r + k) - A(i, j - r + k - 1)) / dy;
            const double A3ym = oracle_weno5(ver, p->epsilon, p->power_param, in);
            for (int k = 1; k <= ws; k++) in[k - 1] = (A(i, j + r - (k - 1)) - A(i, j + r - k)) / dy;
            const double A3yp = oracle_weno5(ver, p->epsilon, p->power_param, in);
#undef A
            const double* Q = q + MI(&g, i, j, 1);
            const double u1 = Q[1] / Q[0];
            const double u2 = Q[2] / Q[0];
            Laux[MI(&ga, i, j, 1)] = -u1 * 0.5 * (A3xm + A3xp) - u2 * 0.5 * (A3ym + A3yp) +
                                     msx * 0.5 * (A3xp - A3xm) + msy * 0.5 * (A3yp - A3ym);
        }
    return 0;
}

/* AfterStep.cpp:13-60: B1 = dA3/dy, B2 = -dA3/dx by 4th-order central
 * differences of aux (ghosts as they are), when constrained transport is on
 * (the MPP branch is off: mpp_limiter defaults to false). */
void oracle_mhd_after_step(const fin_params* p, double* q, const double* aux)
{
    const mgrid_t g = mgrid(p, p->mx, p->my, MQ), ga = mgrid(p, p->mx, p->my, 1);
    if (!p->constrained_transport) return;
    const double dx = get_dx(p), dy = get_dy(p);
#define A(ii, jj) aux[MI(&ga, (ii), (jj), 1)]
    for (int i = 1; i <= g.mx; i++)
        for (int j = 1; j <= g.my; j++) {
            const double B1 = 1.0 / (12.0 * dy) * (A(i, j - 2) - 8 * A(i, j - 1) + 8 * A(i, j + 1) - A(i, j + 2));
            const double B2 = -1.0 / (12.0 * dx) * (A(i - 2, j) - 8 * A(i - 1, j) + 8 * A(i + 1, j) - A(i + 2, j));
            q[MI(&g, i, j, 6)] = B1;
            q[MI(&g, i, j, 7)] = B2;
        }
#undef A
}

/* UpdateSolnWithAux (apps/2d/mhd/lib/UpdateSoln.cpp:21-58) on the interior;
 * its closing SetBndValues rebuilds every ghost, so the ghost updates of the
 * reference are not needed. */
static void update_with_aux(const fin_params* p, double a1, double a2, double beta, double dt, const double* qs,
                            const double* auxs, const double* L, const double* Laux, double* qn, double* auxn)
{
    const mgrid_t g = mgrid(p, p->mx, p->my, MQ), ga = mgrid(p, p->mx, p->my, 1);
    for (int i = 1; i <= g.mx; i++)
        for (int j = 1; j <= g.my; j++) {
            const size_t k = MI(&ga, i, j, 1);
            auxn[k] = a1 * auxs[k] + a2 * auxn[k] + beta * dt * Laux[k];
            for (int m = 1; m <= MQ; m++) {
                const size_t kq = MI(&g, i, j, m);
                qn[kq] = a1 * qs[kq] + a2 * qn[kq] + beta * dt * L[kq];
            }
        }
    oracle_mhd_set_bnd(p, qn, auxn);
}

/* apps/2d/mhd/lib/GetCFL.cpp:31-73 (smax-array form). */
static int mhd_get_cfl(const fin_params* p, double dt, double dtmax, const double* smax, double* cfl_out)
{
    if (dt > dtmax) return FIN_ERR_DT_BOUNDS;
    const mgrid_t gS = {p->mx + 1, p->my + 1, p->mbc, 2, p->my + 1 + 2 * p->mbc};
    const double dx = get_dx(p), dy = get_dy(p);
    double cfl = -100.0;
    for (int i = 1; i <= p->mx; i++)
        for (int j = 1; j <= p->my; j++)
            cfl = std_max(cfl, dt * std_max(smax[MI(&gS, i, j, 1)], smax[MI(&gS, i, j, 2)]) * (1.0 / dx + 1.0 / dy));
    if (cfl > 1.0e8) return FIN_ERR_CFL_BOUNDS;
    *cfl_out = cfl;
    return FIN_OK;
}

typedef struct {
    mgrid_t g, ga, gS;
    size_t n, na, nS;
    double *qold, *auxold, *qstar, *auxstar, *L, *Laux, *smax;
} mwork_t;

static void mwork_init(mwork_t* w, const fin_params* p)
{
    w->g = mgrid(p, p->mx, p->my, MQ);
    w->ga = mgrid(p, p->mx, p->my, 1);
    mgrid_t gS = {p->mx + 1, p->my + 1, p->mbc, 2, p->my + 1 + 2 * p->mbc};
    w->gS = gS;
    w->n = mnumel(&w->g);
    w->na = mnumel(&w->ga);
    w->nS = mnumel(&w->gS);
    w->qold = (double*)calloc(w->n, sizeof(double));
    w->qstar = (double*)calloc(w->n, sizeof(double));
    w->L = (double*)calloc(w->n, sizeof(double));
    w->auxold = (double*)calloc(w->na, sizeof(double));
    w->auxstar = (double*)calloc(w->na, sizeof(double));
    w->Laux = (double*)calloc(w->na, sizeof(double));
    w->smax = (double*)calloc(w->nS, sizeof(double));
}
static void mwork_free(mwork_t* w)
{
    free(w->qold); free(w->qstar); free(w->L); free(w->auxold); free(w->auxstar); free(w->Laux); free(w->smax);
}

/* The three stages of apps/2d/mhd/lib/FinSolveRK.cpp:176-219 (time_order 3,
 * SetRKinfo.cpp:50-64) from (q, aux) into (q, aux), stage register
 * (qstar, auxstar). */
static int mhd_take_stages(const fin_params* p, mwork_t* w, double* q, double* aux, double* tnew, double* tstar,
                           double dt)
{
    static const double a1[3] = {1.0, 0.75, 2.0e0 / 3.0e0};
    static const double a2[3] = {0.0, 0.25, 1.0e0 / 3.0e0};
    static const double bt[3] = {1.0, 0.25, 2.0e0 / 3.0e0};
    int rc;
    /* stage 1: Qnew -> Qstar */
    oracle_mhd_set_bnd(p, q, aux);
    if ((rc = oracle_mhd_construct_l(p, q, w->L, w->smax))) return rc;
    if ((rc = oracle_mhd_construct_hj_l(p, q, aux, w->Laux))) return rc;
    update_with_aux(p, a1[0], a2[0], bt[0], dt, q, aux, w->L, w->Laux, w->qstar, w->auxstar);
    *tstar = a1[0] * *tnew + a2[0] * *tstar + bt[0] * dt;
    oracle_mhd_after_step(p, w->qstar, w->auxstar);
    /* stage 2: (Qnew, Qstar) -> Qstar */
    oracle_mhd_set_bnd(p, w->qstar, w->auxstar);
    if ((rc = oracle_mhd_construct_l(p, w->qstar, w->L, w->smax))) return rc;
    if ((rc = oracle_mhd_construct_hj_l(p, w->qstar, w->auxstar, w->Laux))) return rc;
    update_with_aux(p, a1[1], a2[1], bt[1], dt, q, aux, w->L, w->Laux, w->qstar, w->auxstar);
    *tstar = a1[1] * *tnew + a2[1] * *tstar + bt[1] * dt;
    oracle_mhd_after_step(p, w->qstar, w->auxstar);
    /* stage 3: (Qstar, Qnew) -> Qnew */
    oracle_mhd_set_bnd(p, w->qstar, w->auxstar);
    if ((rc = oracle_mhd_construct_l(p, w->qstar, w->L, w->smax))) return rc;
    if ((rc = oracle_mhd_construct_hj_l(p, w->qstar, w->auxstar, w->Laux))) return rc;
    update_with_aux(p, a1[2], a2[2], bt[2], dt, w->qstar, w->auxstar, w->L, w->Laux, q, aux);
    *tnew = a1[2] * *tstar + a2[2] * *tnew + bt[2] * dt;
    oracle_mhd_after_step(p, q, aux);
    return FIN_OK;
}

static int mhd_check(const fin_params* p)
{
    if (p->meqn != 8 || p->maux != 1 || p->time_order != 3 || p->mbc < 5) return FIN_ERR_ARG;
    return FIN_OK;
}

int oracle_mhd_step_fixed(const fin_params* p, double* q, double* aux, double dt, double* cfl)
{
    if (mhd_check(p)) return FIN_ERR_ARG;
    mwork_t w;
    mwork_init(&w, p);
    memcpy(w.qstar, q, w.n * sizeof(double));
    memcpy(w.auxstar, aux, w.na * sizeof(double));
    double tnew = 0.0, tstar = 0.0;
    int rc = mhd_take_stages(p, &w, q, aux, &tnew, &tstar, dt);
    if (rc == FIN_OK) rc = mhd_get_cfl(p, dt, 1e300, w.smax, cfl);
    mwork_free(&w);
    return rc;
}

/* apps/2d/mhd/lib/FinSolveRK.cpp:17-395 (time_order 3). */
int oracle_mhd_finsolve(const fin_params* p, double* q, double* aux, double* t_io, double tend, double* dtv,
                        int* nsteps)
{
    if (mhd_check(p)) return FIN_ERR_ARG;
    mwork_t w;
    mwork_init(&w, p);
    const double CFL_max = p->max_cfl, CFL_target = p->desired_cfl;
    double t = *t_io, tq = *t_io, told_q = *t_io, tstar = *t_io;
    double dt = dtv[1], cfl = 0.0;
    memcpy(w.qstar, q, w.n * sizeof(double));
    memcpy(w.auxstar, aux, w.na * sizeof(double));
    int n_step = 0, accepted = 0, rc = FIN_OK;
    while (t < tend) {
        int m_accept = 0;
        n_step = n_step + 1;
        if (n_step > p->nv) { rc = FIN_ERR_NSTEPS; break; }
        memcpy(w.qold, q, w.n * sizeof(double));
        memcpy(w.auxold, aux, w.na * sizeof(double));
        told_q = tq;
        while (m_accept == 0) {
            tq = t;
            const double told = t;
            if (told + dt > tend) dt = tend - told;
            t = told + dt;
            memset(w.smax, 0, w.nS * sizeof(double));
            if ((rc = mhd_take_stages(p, &w, q, aux, &tq, &tstar, dt))) goto done;
            if ((rc = mhd_get_cfl(p, dt, dtv[2], w.smax, &cfl))) goto done;
            if (cfl > 0.0) dt = Min(dtv[2], dt * CFL_target / cfl);
            else dt = dtv[2];
            if (cfl <= CFL_max) m_accept = 1;
            else {
                t = told;
                memcpy(q, w.qold, w.n * sizeof(double));
                memcpy(aux, w.auxold, w.na * sizeof(double));
                tq = told_q;
            }
        }
        accepted++;
    }
    dtv[1] = dt;
done:
    *t_io = tq;
    if (nsteps) *nsteps = accepted;
    mwork_free(&w);
    return rc;
}

/* Orszag-Tang initial state: QinitFunc (apps/2d/mhd/orszag_tang/
 * QinitFunc.cpp:10-52) at the cell centres lib/2d/SampleFunction.cpp:45-48
 * uses, and AfterQinit (AfterQinit.cpp:10-35) for A3 = 0.5 cos 2x + cos y;
 * interior cells, ghosts by the periodic images. */
void oracle_orszag_tang(const fin_params* p, double* q, double* aux)
{
    const mgrid_t g = mgrid(p, p->mx, p->my, MQ), ga = mgrid(p, p->mx, p->my, 1);
    const double dx = get_dx(p), dy = get_dy(p);
    const double gamma_gas = p->gamma, gamma1 = p->gamma - 1.0;
    for (int i = 1; i <= g.mx; i++)
        for (int j = 1; j <= g.my; j++) {
            const double x = p->xlow + ((double)i - 0.5) * dx;
            const double y = p->ylow + ((double)j - 0.5) * dy;
            const double rho = pow(gamma_gas, 2);
            const double u1 = -sin(y), u2 = sin(x), u3 = 0.0;
            const double press = gamma_gas;
            const double B1 = -sin(y), B2 = sin(2.0 * x), B3 = 0.0;
            const double energy =
                press / gamma1 + 0.5 * rho * (u1 * u1 + u2 * u2 + u3 * u3) + 0.5 * (B1 * B1 + B2 * B2 + B3 * B3);
            double* Q = q + MI(&g, i, j, 1);
            Q[0] = rho; Q[1] = rho * u1; Q[2] = rho * u2; Q[3] = rho * u3;
            Q[4] = energy; Q[5] = B1; Q[6] = B2; Q[7] = B3;
            const double xa = p->xlow + (i - 0.5) * dx, ya = p->ylow + (j - 0.5) * dy;
            aux[MI(&ga, i, j, 1)] = 0.5 * cos(2.0 * xa) + cos(ya);
        }
    oracle_mhd_set_bnd(p, q, aux);
}

/* ---------------------------------------------------------------------- */
/* Troubled-face samples of the MHD learned indicator                      */
/* ---------------------------------------------------------------------- */

/* Features and labels of every face (x faces, then y faces; (i, j) with j
 * fastest), for the face between cells i-1 and i (1-based i = f_i + 1) with
 * the 6-point stencil i-3 .. i+2:
 *   w = Lmat q at the six points, Lmat the left eigenvectors at the face
 *   average (ProjectLeftEig.cpp:179-192); for each of the eight fields, with
 *   D_s = w(s+1) - w(s) and M = max |D_s|: max |D_(s+1) - D_s| / max(M, 1e-3)
 *   and M / (M + 1e-3); 16 features, the last 4 of 20 zero;
 *   label: 1 when the WENO5-JS weights of gp or gm (ConstructL.cpp:179-192)
 *   of any of the eight fields depart from (0.1, 0.6, 0.3) by more than 10 %
 *   (lib/WenoReconstruct.cpp:104, 131-134). */
void oracle_mhd_face_samples(const fin_params* p, const double* q, double* X, unsigned char* y)
{
    const mgrid_t g = mgrid(p, p->mx, p->my, MQ);
    double alpha1 = 0., alpha2 = 0.;
    if (p->global_alpha) oracle_mhd_global_wave_spd(p, q, &alpha1, &alpha2);
    static const double dl[3] = {0.1, 0.6, 0.3};
    long long f = 0;
    for (int ixy = 1; ixy <= 2; ixy++) {
        const int ni = ixy == 1 ? g.mx + 1 : g.mx, nj = ixy == 1 ? g.my : g.my + 1;
        const int di = ixy == 1 ? 1 : 0, dj = ixy == 1 ? 0 : 1;
        for (int i = 0; i < ni; i++)
            for (int j = 0; j < nj; j++, f++) {
                double Qs[6][MQ], Fs[6][MQ];
                for (int s = 0; s < 6; s++) {
                    const double* Qp = q + MI(&g, i + 1 + di * (s - 3), j + 1 + dj * (s - 3), 1);
                    double fx[MQ], fy[MQ];
                    mhd_flux(p->gamma, Qp, fx, fy);
                    for (int m = 0; m < MQ; m++) {
                        Qs[s][m] = Qp[m];
                        Fs[s][m] = ixy == 1 ? fx[m] : fy[m];
                    }
                }
                double Qavg[MQ], Lm[MQ][MQ], Rm[MQ][MQ], W[6][MQ], G[6][MQ];
                for (int m = 0; m < MQ; m++) Qavg[m] = 0.5 * (Qs[3][m] + Qs[2][m]);
                mhd_eig(ixy, p->gamma, Qavg, Lm, Rm);
                for (int s = 0; s < 6; s++) {
                    matvec8(Lm, Qs[s], W[s]);
                    matvec8(Lm, Fs[s], G[s]);
                }
                for (int k = 0; k < MQ; k++) {
                    double d[5], M = 0.0, S = 0.0;
                    for (int s = 0; s < 5; s++) {
                        d[s] = W[s + 1][k] - W[s][k];
                        if (fabs(d[s]) > M) M = fabs(d[s]);
                    }
                    for (int s = 0; s < 4; s++)
                        if (fabs(d[s + 1] - d[s]) > S) S = fabs(d[s + 1] - d[s]);
                    X[f * 20 + 2 * k] = S / (M > 1e-3 ? M : 1e-3);
                    X[f * 20 + 2 * k + 1] = M / (M + 1e-3);
                }
                for (int k = 16; k < 20; k++) X[f * 20 + k] = 0.0;
                double s1, s2;
                mhd_wave_spd(p->gamma, ixy == 1 ? 1.0 : 0.0, ixy == 1 ? 0.0 : 1.0, Qs[2], Qs[3], &s1, &s2);
                const double alpha = Max(ixy == 1 ? alpha1 : alpha2, Max(fabs(s1), fabs(s2)));
                const double la = p->alpha_scaling * alpha;
                double dep = 0.0;
                for (int k = 0; k < MQ; k++) {
                    double gp[5], gm[5], w[3];
                    for (int s = 0; s < 5; s++) {
                        gp[s] = 0.5 * (G[s][k] + la * W[s][k]);
                        gm[s] = 0.5 * (G[5 - s][k] - la * W[5 - s][k]);
                    }
                    oracle_weno_js5_weights(p->epsilon, p->power_param, gp, w);
                    for (int r = 0; r < 3; r++) dep = Max(dep, fabs(w[r] - dl[r]) / dl[r]);
                    oracle_weno_js5_weights(p->epsilon, p->power_param, gm, w);
                    for (int r = 0; r < 3; r++) dep = Max(dep, fabs(w[r] - dl[r]) / dl[r]);
                }
                y[f] = dep > 0.1 ? 1 : 0;
            }
    }
}
