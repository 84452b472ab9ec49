// Initial data sampled on the device: SampleFunction (lib/2d/SampleFunction.cpp:
// 62-125, called with QinitFunc from lib/2d/RunFinpack.cpp:80) with the
// application's QinitFunc as a __device__ functor.
//
// An application supplies a functor with the QinitFunc signature of
// lib/2d/app_defined.h:7 at one point,
//     struct MyQinit { __device__ void operator()(double x, double y, double* q) const; };
// (q[0..meqn-1] written; the functor is passed by value, so its fields carry
// the problem's parameters), and samples it into the device state planes with
// launch_sample<MyQinit>: every interior cell (i, j), 1-based, gets
// Qinit(xlow + (i - 1/2) dx, ylow + (j - 1/2) dy), as SampleFunction.cpp:
// 66-71 places the points.  The ghost frame is not sampled: the device state
// has none (the stages remap the boundary conditions on load), and the
// reference's sampled ghost values are overwritten by SetBndValues before
// any stage reads them.
//
// The functors below are the initial data of this library's built-in
// problems, in the operation order of the code they restate, every product,
// quotient and sum rounded on its own (no contraction, as the reference's
// x86-64 build has none); exp, pow and sin are CUDA's, within an ulp or two
// of the host's.
#pragma once
#include <cuda_runtime.h>
#include "fin_device.cuh"

namespace fin {
namespace qinit {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dv(double a, double b) { return __ddiv_rn(a, b); }

// (rho, u, v, p) -> (rho, rho u, rho v, 0, p/(gamma-1) + 0.5 rho (u^2 + v^2))
__device__ __forceinline__ void conserved(double g, double rho, double u, double v, double pr, double* q)
{
    q[0] = rho;
    q[1] = mul(rho, u);
    q[2] = mul(rho, v);
    q[3] = 0.0;
    q[4] = add(dv(pr, sub(g, 1.0)), mul(mul(0.5, rho), add(mul(u, u), mul(v, v))));
}

// Isentropic vortex of strength eps centred at (xc, yc) on the background
// (rho, u, v, p) = (1, 1, 1, 1): du = -eps/(2 pi) e^{(1-r^2)/2} (y - yc),
// dv = eps/(2 pi) e^{(1-r^2)/2} (x - xc), T = 1 - (gamma-1) eps^2/(8 gamma
// pi^2) e^{1-r^2}, rho = T^{1/(gamma-1)}, p = rho^gamma (the benchmark's
// vortex on [0,10]^2, eps 5, centre (5, 5)).
struct Vortex {
    double gamma, eps, xc, yc;
    __device__ void operator()(double x, double y, double* q) const
    {
        const double g = gamma, pi = 3.141592653589793;
        const double dxv = sub(x, xc), dyv = sub(y, yc);
        const double r2 = add(mul(dxv, dxv), mul(dyv, dyv));
        const double ex = exp(dv(sub(1.0, r2), 2.0));
        const double c = dv(-eps, mul(2.0, pi));
        const double du = mul(mul(c, ex), dyv);
        const double dvv = mul(mul(dv(eps, mul(2.0, pi)), ex), dxv);
        const double k = dv(mul(mul(sub(g, 1.0), eps), eps), mul(mul(mul(8.0, g), pi), pi));
        const double T = sub(1.0, mul(k, exp(sub(1.0, r2))));
        const double rho = pow(T, dv(1.0, sub(g, 1.0)));
        const double pr = pow(rho, g);
        conserved(g, rho, add(1.0, du), add(1.0, dvv), pr, q);
    }
};

// Four-quadrant Riemann problem with the interface at (xc, yc): states
// s[k] = (rho, u, v, p) for k = upper-right, upper-left, lower-left,
// lower-right; x >= xc is right, y >= yc is upper.
struct Riemann4 {
    double gamma, xc, yc;
    double s[4][4];
    __device__ void operator()(double x, double y, double* q) const
    {
        const bool r = x >= xc, u = y >= yc;
        const int k = u ? (r ? 0 : 1) : (r ? 3 : 2);
        conserved(gamma, s[k][0], s[k][1], s[k][2], s[k][3], q);
    }
};

// Shock / entropy-wave interaction on [-5,5] x [0,1]: x < -4 the post-shock
// state (3.857143, 2.629369, 0, 10.33333), else rho = 1 + 0.2 sin(5x) +
// 0.1 sin(2 pi y), u = v = 0, p = 1.
struct ShockEntropy {
    double gamma;
    __device__ void operator()(double x, double y, double* q) const
    {
        const double pi = 3.141592653589793;
        if (x < -4.0) {
            conserved(gamma, 3.857143, 2.629369, 0.0, 10.33333, q);
        } else {
            const double rho = add(add(1.0, mul(0.2, sin(mul(5.0, x)))), mul(0.1, sin(mul(mul(2.0, pi), y))));
            conserved(gamma, rho, 0.0, 0.0, 1.0, q);
        }
    }
};

// The reference's own shock-tube application (apps/2d/euler/riemann_test/
// QinitFunc.cpp:26-84): opt 1 splits at x = 0.5, otherwise at y = 0.5;
// (1, 0, 0, 0, 1) beyond the split, (3, 0, 0, 0, 3) before it.
struct ShockTube {
    double gamma;
    int opt;
    __device__ void operator()(double x, double y, double* q) const
    {
        const bool hi = opt == 1 ? x > 0.5 : y > 0.5;
        const double rho = hi ? 1.0 : 3.0, press = hi ? 1.0 : 3.0;
        q[0] = rho;
        q[1] = mul(rho, 0.0);
        q[2] = mul(rho, 0.0);
        q[3] = mul(rho, 0.0);
        // QinitFunc.cpp:78-79: press/(gamma-1) + 0.5 rho (u1^2 + u2^2 + u3^2)
        q[4] = add(dv(press, sub(gamma, 1.0)), mul(mul(0.5, rho), 0.0));
    }
};

// The reference's own isentropic-vortex application (apps/2d/euler/
// test_exact2/QinitFunc.cpp:26-73, domain [-5,5]^2): epsilon 10.0828, the
// vortex built on the temperature tpr = p/rho and the entropy p/rho^gamma.
struct VortexExact2 {
    double gamma;
    __device__ void operator()(double xp, double yp, double* q) const
    {
        const double g = gamma, epsilon = 10.0828, pi = 3.1415926535897932385;
        double x = xp, y = yp;   // t0 = 0: x - t0*1.0 is x
        if (x < -5.0) x = add(x, 10.0);
        if (y < -5.0) y = add(y, 10.0);
        double rho = 1.0, u1 = 1.0, u2 = 1.0;
        const double u3 = 0.0;
        double press = 1.0;
        double tpr = dv(press, rho);
        const double entpy = dv(press, pow(rho, g));
        const double r2 = add(mul(x, x), mul(y, y));
        // -epsilon/2.e0/pi*exp((1.e0-r2)/2.e0)*y, left to right
        const double e1 = exp(dv(sub(1.0, r2), 2.0));
        const double du = mul(mul(dv(dv(-epsilon, 2.0), pi), e1), y);
        const double dvv = mul(mul(dv(dv(epsilon, 2.0), pi), e1), x);
        // (1.e0-gamma)/gamma * epsilon*epsilon/8.e0/pi/pi*exp(1.e0-r2)
        const double dtpr =
            mul(dv(dv(dv(mul(mul(dv(sub(1.0, g), g), epsilon), epsilon), 8.0), pi), pi), exp(sub(1.0, r2)));
        u1 = add(u1, du);
        u2 = add(u2, dvv);
        tpr = add(tpr, dtpr);
        press = dv(pow(tpr, dv(g, sub(g, 1.0))), pow(entpy, dv(1.0, sub(g, 1.0))));
        rho = dv(press, tpr);
        const double energy = add(dv(press, sub(g, 1.0)), mul(mul(0.5, rho), add(add(mul(u1, u1), mul(u2, u2)), mul(u3, u3))));
        q[0] = rho;
        q[1] = mul(rho, u1);
        q[2] = mul(rho, u2);
        q[3] = mul(rho, u3);
        q[4] = energy;
    }
};

}  // namespace qinit

// SampleFunction over the interior cells into planes q[m * plane + i * my + j].
template <class Qinit>
__global__ void k_sample(const Qinit f, double xlow, double ylow, double dx, double dy, int mx, int my, double* q,
                         size_t plane)
{
    const size_t n = size_t(mx) * my;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const int i = int(g / my), j = int(g - size_t(i) * my);
        // SampleFunction.cpp:66-71 with 1-based i, j: xlow + (double(i) - 0.5) dx
        const double xc = __dadd_rn(xlow, __dmul_rn(__dsub_rn(double(i + 1), 0.5), dx));
        const double yc = __dadd_rn(ylow, __dmul_rn(__dsub_rn(double(j + 1), 0.5), dy));
        double v[MEQN];
        f(xc, yc, v);
#pragma unroll
        for (int m = 0; m < MEQN; m++) q[m * plane + g] = v[m];
    }
}

template <class Qinit>
cudaError_t launch_sample(const Qinit& f, double xlow, double ylow, double dx, double dy, int mx, int my, double* q,
                          size_t plane, cudaStream_t stream)
{
    const size_t n = size_t(mx) * my;
    size_t blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    k_sample<Qinit><<<unsigned(blocks), 256, 0, stream>>>(f, xlow, ylow, dx, dy, mx, my, q, plane);
    return cudaGetLastError();
}

}  // namespace fin
