// The other spatial orders of ConstructL (space_order 1, 7, 9, 11; order 5
// is the fused stage kernel's): one thread per face gathers the 2r-point
// stencil (r = (space_order+1)/2, ConstructL.cpp:31-33, 94-113), forms the
// characteristic split values and reconstructs them with the reference's
// WENO of that order (lib/WenoReconstruct.cpp:151-375, 440-575, 618-690), the
// face fluxes go to two face arrays, and a second kernel differences them
// into L and applies the stage update.  FP64 only.  The reconstruction
// coefficients -- candidate-stencil weights, linear weights and the
// smoothness-indicator polynomials of Balsara & Shu (J. Comput. Phys. 160,
// 2000) -- are the reference's, restated value for value: the method is
// defined by them.
#pragma once
#include "fin_stage.cuh"

namespace fin {
namespace hi {

// (eps + beta)^-p and (tau / (eps + beta))^p, with p = 2 evaluated by products.
__device__ __forceinline__ double js_w(double g, double eps, double beta, double pw)
{
    const double x = eps + beta;
    return g * (pw == 2.0 ? 1.0 / (x * x) : pow(x, -pw));
}
__device__ __forceinline__ double z_w(double g, double eps, double beta, double tau, double pw)
{
    const double x = tau / (eps + beta);
    return g * (1. + (pw == 2.0 ? x * x : pow(x, pw)));
}

// u[0 .. 6] = u_{i-3} .. u_{i+3}: value at i+1/2 (WenoReconstruct.cpp:151-205,
// 440-495, 618-650).
template <int VER>
__device__ __forceinline__ double recon7(const double* u, double eps, double pw)
{
    const double uim3 = u[0], uim2 = u[1], uim1 = u[2], ui = u[3], uip1 = u[4], uip2 = u[5], uip3 = u[6];
    const double g0 = 1. / 35., g1 = 12. / 35., g2 = 18. / 35., g3 = 4. / 35.;
    const double u1 = (-1. / 4.) * uim3 + (13. / 12.) * uim2 - (23. / 12.) * uim1 + (25. / 12.) * ui;
    const double u2 = (1. / 12.) * uim2 - (5. / 12.) * uim1 + (13. / 12.) * ui + (1. / 4.) * uip1;
    const double u3 = (-1. / 12.) * uim1 + (7. / 12.) * ui + (7. / 12.) * uip1 - (1. / 12.) * uip2;
    const double u4 = (1. / 4.) * ui + (13. / 12.) * uip1 - (5. / 12.) * uip2 + (1. / 12.) * uip3;
    if (VER == FIN_WENO_FD) return g0 * u1 + g1 * u2 + g2 * u3 + g3 * u4;
    const double b0 = uim3 * (547. * uim3 - 3882. * uim2 + 4642. * uim1 - 1854. * ui) +
                      uim2 * (7043. * uim2 - 17246. * uim1 + 7042. * ui) + uim1 * (11003. * uim1 - 9402. * ui) +
                      2107. * (ui * ui);
    const double b1 = uim2 * (267. * uim2 - 1642. * uim1 + 1602. * ui - 494. * uip1) +
                      uim1 * (2843. * uim1 - 5966. * ui + 1922. * uip1) + ui * (3443. * ui - 2522. * uip1) +
                      547. * (uip1 * uip1);
    const double b2 = uim1 * (547. * uim1 - 2522. * ui + 1922. * uip1 - 494. * uip2) +
                      ui * (3443. * ui - 5966. * uip1 + 1602. * uip2) + uip1 * (2843. * uip1 - 1642. * uip2) +
                      267. * (uip2 * uip2);
    const double b3 = ui * (2107. * ui - 9402. * uip1 + 7042. * uip2 - 1854. * uip3) +
                      uip1 * (11003. * uip1 - 17246. * uip2 + 4642. * uip3) + uip2 * (7043. * uip2 - 3882. * uip3) +
                      547. * (uip3 * uip3);
    double o0, o1, o2, o3;
    if (VER == FIN_WENO_Z) {
        const double tau = fabs(b0 + 3. * (b1 - b2) - b3);
        o0 = z_w(g0, eps, b0, tau, pw); o1 = z_w(g1, eps, b1, tau, pw);
        o2 = z_w(g2, eps, b2, tau, pw); o3 = z_w(g3, eps, b3, tau, pw);
    } else {
        o0 = js_w(g0, eps, b0, pw); o1 = js_w(g1, eps, b1, pw);
        o2 = js_w(g2, eps, b2, pw); o3 = js_w(g3, eps, b3, pw);
    }
    return (o0 * u1 + o1 * u2 + o2 * u3 + o3 * u4) / (o0 + o1 + o2 + o3);
}

// u[0 .. 8] = u_{i-4} .. u_{i+4} (WenoReconstruct.cpp:207-280, 497-575, 652-684).
template <int VER>
__device__ __forceinline__ double recon9(const double* u, double eps, double pw)
{
    const double uim4 = u[0], uim3 = u[1], uim2 = u[2], uim1 = u[3], ui = u[4], uip1 = u[5], uip2 = u[6],
                 uip3 = u[7], uip4 = u[8];
    const double g0 = 1.0 / 126.0, g1 = 10. / 63., g2 = 10. / 21., g3 = 20. / 63., g4 = 5. / 126.;
    const double u1 = (1. / 5.) * uim4 + (-21. / 20.) * uim3 + (137. / 60.) * uim2 + (-163. / 60.) * uim1 +
                      (137. / 60.) * ui;
    const double u2 = (-1. / 20.) * uim3 + (17. / 60.) * uim2 + (-43. / 60.) * uim1 + (77. / 60.) * ui +
                      (1. / 5.) * uip1;
    const double u3 = (1. / 30.) * uim2 + (-13. / 60.) * uim1 + (47. / 60.) * ui + (9. / 20.) * uip1 +
                      (-1. / 20.) * uip2;
    const double u4 = (-1. / 20.) * uim1 + (9. / 20.) * ui + (47. / 60.) * uip1 + (-13. / 60.) * uip2 +
                      (1. / 30.) * uip3;
    const double u5 = (1. / 5.) * ui + (77. / 60.) * uip1 + (-43. / 60.) * uip2 + (17. / 60.) * uip3 +
                      (-1. / 20.) * uip4;
    if (VER == FIN_WENO_FD) return g0 * u1 + g1 * u2 + g2 * u3 + g3 * u4 + g4 * u5;
    const double b0 = uim4 * (22658. * uim4 - 208501. * uim3 + 364863. * uim2 - 288007. * uim1 + 86329. * ui) +
                      uim3 * (482963. * uim3 - 1704396. * uim2 + 1358458. * uim1 - 411487. * ui) +
                      uim2 * (1521393. * uim2 - 2462076. * uim1 + 758823. * ui) +
                      uim1 * (1020563. * uim1 - 649501. * ui) + 107918. * (ui * ui);
    const double b1 = uim3 * (6908. * uim3 - 60871. * uim2 + 99213. * uim1 - 70237. * ui + 18079. * uip1) +
                      uim2 * (138563. * uim2 - 464976. * uim1 + 337018. * ui - 88297. * uip1) +
                      uim1 * (406293. * uim1 - 611976. * ui + 165153. * uip1) +
                      ui * (242723. * ui - 140251. * uip1) + 22658. * (uip1 * uip1);
    const double b2 = uim2 * (6908. * uim2 - 51001. * uim1 + 67923. * ui - 38947. * uip1 + 8209. * uip2) +
                      uim1 * (104963. * uim1 - 299076. * ui + 179098. * uip1 - 38947. * uip2) +
                      ui * (231153. * ui - 299076. * uip1 + 67923. * uip2) +
                      uip1 * (104963. * uip1 - 51001. * uip2) + 6908. * (uip2 * uip2);
    const double b3 = uim1 * (22658. * uim1 - 140251. * ui + 165153. * uip1 - 88297. * uip2 + 18079. * uip3) +
                      ui * (242723. * ui - 611976. * uip1 + 337018. * uip2 - 70237. * uip3) +
                      uip1 * (406293. * uip1 - 464976. * uip2 + 99213. * uip3) +
                      uip2 * (138563. * uip2 - 60871. * uip3) + 6908. * (uip3 * uip3);
    const double b4 = ui * (107918. * ui - 649501. * uip1 + 758823. * uip2 - 411487. * uip3 + 86329. * uip4) +
                      uip1 * (1020563. * uip1 - 2462076. * uip2 + 1358458. * uip3 - 288007. * uip4) +
                      uip2 * (1521393. * uip2 - 1704396. * uip3 + 364863. * uip4) +
                      uip3 * (482963. * uip3 - 208501. * uip4) + 22658. * (uip4 * uip4);
    double o0, o1, o2, o3, o4;
    if (VER == FIN_WENO_Z) {
        const double tau = fabs(b4 - b0);
        o0 = z_w(g0, eps, b0, tau, pw); o1 = z_w(g1, eps, b1, tau, pw); o2 = z_w(g2, eps, b2, tau, pw);
        o3 = z_w(g3, eps, b3, tau, pw); o4 = z_w(g4, eps, b4, tau, pw);
    } else {
        o0 = js_w(g0, eps, b0, pw); o1 = js_w(g1, eps, b1, pw); o2 = js_w(g2, eps, b2, pw);
        o3 = js_w(g3, eps, b3, pw); o4 = js_w(g4, eps, b4, pw);
    }
    return (o0 * u1 + o1 * u2 + o2 * u3 + o3 * u4 + o4 * u5) / (o0 + o1 + o2 + o3 + o4);
}

// u[0 .. 10] = u_{i-5} .. u_{i+5}, Jiang-Shu weights (WenoReconstruct.cpp:283-375).
__device__ __forceinline__ double recon11(const double* u, double eps, double pw)
{
    const double uim5 = u[0], uim4 = u[1], uim3 = u[2], uim2 = u[3], uim1 = u[4], ui = u[5], uip1 = u[6],
                 uip2 = u[7], uip3 = u[8], uip4 = u[9], uip5 = u[10];
    const double g0 = 1.0 / 462., g1 = 5. / 77, g2 = 25. / 77., g3 = 100. / 231., g4 = 25. / 154., g5 = 1. / 77.;
    const double b0 =
        uim5 * (1152561. * uim5 - 12950184. * uim4 + 29442256. * uim3 - 33918804. * uim2 + 19834350. * uim1 -
                4712740. * ui) +
        uim4 * (36480687. * uim4 - 166461044. * uim3 + 192596472. * uim2 - 113206788. * uim1 + 27060170. * ui) +
        uim3 * (190757572. * uim3 - 444003904. * uim2 + 262901672. * uim1 - 63394124. * ui) +
        uim2 * (260445372. * uim2 - 311771244. * uim1 + 76206736. * ui) +
        uim1 * (94851237. * uim1 - 47460464. * ui) + 6150211. * ui * ui;
    const double b1 =
        uim4 * (271779. * uim4 - 3015728. * uim3 + 6694608. * uim2 - 7408908. * uim1 + 4067018. * ui - 880548. * uip1) +
        uim3 * (8449957. * uim3 - 37913324. * uim2 + 42405032. * uim1 - 23510468. * ui + 5134574. * uip1) +
        uim2 * (43093692. * uim2 - 97838784. * uim1 + 55053752. * ui - 12183636. * uip1) +
        uim1 * (56662212. * uim1 - 65224244. * ui + 14742480. * uip1) + ui * (19365967. * ui - 9117992. * uip1) +
        1152561. * uip1 * uip1;
    const double b2 =
        uim3 * (139633. * uim3 - 1429976. * uim2 + 2863984. * uim1 - 2792660. * ui + 1325006. * uip1 - 245620. * uip2) +
        uim2 * (3824847. * uim2 - 15880404. * uim1 + 15929912. * ui - 7727988. * uip1 + 1458762. * uip2) +
        uim1 * (17195652. * uim1 - 35817664. * ui + 17905032. * uip1 - 3462252. * uip2) +
        ui * (19510972. * ui - 20427884. * uip1 + 4086352. * uip2) + uip1 * (5653317. * uip1 - 2380800. * uip2) +
        271779. * uip2 * uip2;
    const double b3 =
        uim2 * (271779. * uim2 - 2380800. * uim1 + 4086352. * ui - 3462252. * uip1 + 1458762. * uip2 - 245620. * uip3) +
        uim1 * (5653317. * uim1 - 20427884. * ui + 17905032. * uip1 - 7727988. * uip2 + 1325006. * uip3) +
        ui * (19510972. * ui - 35817664. * uip1 + 15929912. * uip2 - 2792660. * uip3) +
        uip1 * (17195652. * uip1 - 15880404. * uip2 + 2863984. * uip3) + uip2 * (3824847. * uip2 - 1429976. * uip3) +
        139633. * uip3 * uip3;
    const double b4 =
        uim1 * (1152561. * uim1 - 9117992. * ui + 14742480. * uip1 - 12183636. * uip2 + 5134574. * uip3 - 880548. * uip4) +
        ui * (19365967. * ui - 65224244. * uip1 + 55053752. * uip2 - 23510468. * uip3 + 4067018. * uip4) +
        uip1 * (56662212. * uip1 - 97838784. * uip2 + 42405032. * uip3 - 7408908. * uip4) +
        uip2 * (43093692. * uip2 - 37913324. * uip3 + 6694608. * uip4) + uip3 * (8449957. * uip3 - 3015728. * uip4) +
        271779. * uip4 * uip4;
    const double b5 =
        ui * (6150211. * ui - 47460464. * uip1 + 76206736. * uip2 - 63394124. * uip3 + 27060170. * uip4 - 4712740. * uip5) +
        uip1 * (94851237. * uip1 - 311771244. * uip2 + 262901672. * uip3 - 113206788. * uip4 + 19834350. * uip5) +
        uip2 * (260445372. * uip2 - 444003904. * uip3 + 192596472. * uip4 - 33918804. * uip5) +
        uip3 * (190757572. * uip3 - 166461044. * uip4 + 29442256. * uip5) + uip4 * (36480687. * uip4 - 12950184. * uip5) +
        1152561. * uip5 * uip5;
    const double u1 = (-1. / 6.) * uim5 + (31. / 30.) * uim4 + (-163. / 60.) * uim3 + (79. / 20.) * uim2 +
                      (-71. / 20.) * uim1 + (49. / 20.) * ui;
    const double u2 = (1. / 30.) * uim4 + (-13. / 60.) * uim3 + (37. / 60.) * uim2 + (-21. / 20.) * uim1 +
                      (29. / 20.) * ui + (1. / 6.) * uip1;
    const double u3 = (-1. / 60.) * uim3 + (7. / 60.) * uim2 + (-23. / 60.) * uim1 + (19. / 20.) * ui +
                      (11. / 30.) * uip1 + (-1. / 30.) * uip2;
    const double u4 = (1. / 60.) * uim2 + (-2. / 15.) * uim1 + (37. / 60.) * ui + (37. / 60.) * uip1 +
                      (-2. / 15.) * uip2 + (1. / 60.) * uip3;
    const double u5 = (-1. / 30.) * uim1 + (11. / 30.) * ui + (19. / 20.) * uip1 + (-23. / 60.) * uip2 +
                      (7. / 60.) * uip3 + (-1. / 60.) * uip4;
    const double u6 = (1. / 6.) * ui + (29. / 20.) * uip1 + (-21. / 20.) * uip2 + (37. / 60.) * uip3 +
                      (-13. / 60.) * uip4 + (1. / 30.) * uip5;
    const double o0 = js_w(g0, eps, b0, pw), o1 = js_w(g1, eps, b1, pw), o2 = js_w(g2, eps, b2, pw),
                 o3 = js_w(g3, eps, b3, pw), o4 = js_w(g4, eps, b4, pw), o5 = js_w(g5, eps, b5, pw);
    return (o0 * u1 + o1 * u2 + o2 * u3 + o3 * u4 + o4 * u5 + o5 * u6) / (o0 + o1 + o2 + o3 + o4 + o5);
}

// The reconstruction of an order: ORDER - the stencil length (2r - 1).
template <int ORDER, int VER>
__device__ __forceinline__ double recon(const double* u, double eps, double pw)
{
    static_assert(ORDER == 1 || ORDER == 7 || ORDER == 9 || ORDER == 11, "orders 1, 7, 9, 11");
    if constexpr (ORDER == 1) return u[0];   // WenoReconstructLLF, :686-695
    else if constexpr (ORDER == 7) return recon7<VER>(u, eps, pw);
    else if constexpr (ORDER == 9) return recon9<VER>(u, eps, pw);
    else return recon11(u, eps, pw);
}

struct HiArgs {
    const double* q;      // stage input planes
    size_t plane;
    int mx, my;
    int bc[4];
    double gamma, eps, pw, alpha_scaling;
    const double* alpha_in;   // [2] global alpha of q (global_alpha), else null
    double* fx;           // [m][mx+1][my] x-face fluxes
    double* fy;           // [m][mx][my+1] y-face fluxes
    double* smax_out;     // [2] face-speed maxima over GetCFL's faces
    double* face_alpha_x; // optional per-face speeds (fin_construct_l's smax)
    double* face_alpha_y;
    unsigned int* status;
};

// One thread per face: x faces (i = 0 .. mx between cells i-1 and i, j < my),
// then y faces (i < mx, j = 0 .. my); ConstructL.cpp:62-208 / 214-358 for one
// face, with r = (ORDER + 1) / 2.
template <int ORDER, int VER>
__global__ void __launch_bounds__(128) k_hi_faces(const HiArgs a)
{
    constexpr int R = (ORDER + 1) / 2, NP = 2 * R, NW = ORDER;
    const int mx = a.mx, my = a.my;
    const long long nfx = (long long)(mx + 1) * my, nf = nfx + (long long)mx * (my + 1);
    const long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double sx = 0.0, sy = 0.0;
    bool neg = false, nonfinite = false;
    if (f < nf) {
        const bool isx = f < nfx;
        int i, j;
        if (isx) { i = int(f / my); j = int(f - (long long)i * my); }
        else { const long long g = f - nfx; i = int(g / (my + 1)); j = int(g - (long long)i * (my + 1)); }
        const int cn = isx ? 1 : 2, ct = isx ? 2 : 1;
        const int ml[MEQN] = {0, cn, ct, 3, 4};
        // stencil point s (0 .. NP-1) is cell i-r+s (x faces) or j-r+s (y
        // faces); values in the normal frame
        auto load = [&](int s, double* Qn) {
            const int ci = isx ? i - R + s : i, cj = isx ? j : j - R + s;
            const size_t g = size_t(bc_remap(ci, mx, a.bc[0], a.bc[1])) * my + bc_remap(cj, my, a.bc[2], a.bc[3]);
#pragma unroll
            for (int m = 0; m < MEQN; m++) Qn[m] = a.q[ml[m] * a.plane + g];
        };
        double Ql[MEQN], Qr[MEQN], Qa[MEQN];
        load(R - 1, Ql);
        load(R, Qr);
#pragma unroll
        for (int m = 0; m < MEQN; m++) Qa[m] = 0.5 * (Qr[m] + Ql[m]);
        const Euler::Eig<double> e = Euler::eig(a.gamma, Qa);
        const Euler::Cell<double> cl = Euler::cell(a.gamma, Ql), cr = Euler::cell(a.gamma, Qr);
        const double ag = a.alpha_in ? a.alpha_in[isx ? 0 : 1] : 0.0;
        const double alpha = Max(ag, Euler::speed(a.gamma, cl, cr, &neg));
        if (!(alpha <= 1e30)) nonfinite = true;
        const double lah = 0.5 * a.alpha_scaling * alpha;
        // gp = L (0.5 f + 0.5 l_alpha q) at points 0 .. NW-1, gm = L (0.5 f -
        // 0.5 l_alpha q) at points NP-1 .. 1 (ConstructL.cpp:179-185); the
        // flux in the normal frame is the x flux of the frame-swapped state
        double Wp[NP][MEQN], Wm[NP][MEQN];
        for (int s = 0; s < NP; s++) {
            double Qn[MEQN], fn[MEQN], gn[MEQN], vp[MEQN], vm[MEQN];
            load(s, Qn);
            Euler::flux(a.gamma, Qn, fn, gn);
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                vp[m] = 0.5 * fn[m] + lah * Qn[m];
                vm[m] = 0.5 * fn[m] - lah * Qn[m];
            }
            Euler::left(e, vp, Wp[s]);
            Euler::left(e, vm, Wm[s]);
        }
        double gh[MEQN];
        for (int k = 0; k < MEQN; k++) {
            double up[NW], um[NW];
            for (int s = 0; s < NW; s++) {
                up[s] = Wp[s][k];
                um[s] = Wm[NP - 1 - s][k];
            }
            gh[k] = recon<ORDER, VER>(up, a.eps, a.pw) + recon<ORDER, VER>(um, a.eps, a.pw);
        }
        double fh[MEQN];
        Euler::right(e, gh, fh);
        if (isx) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) a.fx[(size_t(m) * (mx + 1) + i) * my + j] = fh[m];
            if (i < mx && alpha <= 1e30) sx = alpha;
            if (a.face_alpha_x) a.face_alpha_x[size_t(i) * my + j] = alpha;
        } else {
            const double o[MEQN] = {fh[0], fh[2], fh[1], fh[3], fh[4]};
#pragma unroll
            for (int m = 0; m < MEQN; m++) a.fy[(size_t(m) * mx + i) * (my + 1) + j] = o[m];
            if (j < my && alpha <= 1e30) sy = alpha;
            if (a.face_alpha_y) a.face_alpha_y[size_t(i) * (my + 1) + j] = alpha;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sx = Max(sx, __shfl_xor_sync(0xffffffffu, sx, o));
        sy = Max(sy, __shfl_xor_sync(0xffffffffu, sy, o));
    }
    if ((threadIdx.x & 31) == 0 && a.smax_out) {
        if (sx > 0.0) atomic_max_nonneg(a.smax_out, sx);
        if (sy > 0.0) atomic_max_nonneg(a.smax_out + 1, sy);
    }
    if (neg) atomicOr(a.status, 2u);
    if (nonfinite) atomicOr(a.status, 1u);
}

// Per cell: L (ConstructL.cpp:396-398, as the fused kernel forms it), the
// stage update q_out = a1 A + a2 B + bdt L (UpdateSoln.cpp:29-35) and the
// new state's global wave speeds (GlobalWaveSpd.cpp:71-76).
__global__ void __launch_bounds__(256) k_hi_update(const double* __restrict__ fx, const double* __restrict__ fy,
                                                   const StageArgs a)
{
    __shared__ double red[2][8];
    const int mx = a.mx, my = a.my;
    const size_t n = size_t(mx) * my;
    double sx = 0.0, sy = 0.0;
    bool nonfinite = false;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const int i = int(g / my), j = int(g - size_t(i) * my);
        // operand loads ahead of the first store (qout may alias A or B as
        // far as the compiler knows)
        double va[MEQN], vb[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            va[m] = a.A ? a.A[m * a.plane + g] : 0.0;
            vb[m] = a.B ? a.B[m * a.plane + g] : 0.0;
        }
        double qn[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            const double f1 = fx[(size_t(m) * (mx + 1) + i + 1) * my + j], f0 = fx[(size_t(m) * (mx + 1) + i) * my + j];
            const double g1 = fy[(size_t(m) * mx + i) * (my + 1) + j + 1], g0 = fy[(size_t(m) * mx + i) * (my + 1) + j];
            double L = -(f1 - f0) * a.rdx;
            L = L - (g1 - g0) * a.rdy;
            double v = 0.0;
            if (a.A) v = a.a1 * va[m];
            if (a.B) v = v + a.a2 * vb[m];
            v = v + a.bdt * L;
            qn[m] = v;
            a.qout[m * a.plane + g] = v;
        }
        if (a.alpha_out) {
            const double qy[MEQN] = {qn[0], qn[2], qn[1], qn[3], qn[4]};
            const double ax = Euler::cell_speed(Euler::cell(a.gamma, qn));
            const double ay = Euler::cell_speed(Euler::cell(a.gamma, qy));
            if (!(ax <= 1e300) || !(ay <= 1e300)) nonfinite = true;
            else {
                sx = Max(sx, ax);
                sy = Max(sy, ay);
            }
        }
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
    if (threadIdx.x == 0 && a.alpha_out) {
        for (int w = 1; w < int(blockDim.x >> 5); w++) {
            sx = Max(sx, red[0][w]);
            sy = Max(sy, red[1][w]);
        }
        atomic_max_nonneg(a.alpha_out, sx);
        atomic_max_nonneg(a.alpha_out + 1, sy);
    }
    if (nonfinite) atomicOr(a.status, 1u);
}

}  // namespace hi
}  // namespace fin
