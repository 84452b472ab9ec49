// Device building blocks of the B200 WENO right-hand side: grid indexing with
// the boundary-condition remap, FP64 order-preserving atomics, the Euler
// callbacks as __device__ functors, and the WENO5 reconstructions.
//
// Precision: every function is templated on the arithmetic type R (double for
// the plain form, float for the FP32-bulk form).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "finess_b200.h"

namespace fin {

constexpr int MEQN = 5;   // Euler: rho, rho u, rho v, rho w, E

// ---------------------------------------------------------------------------
// Boundary conditions as an index remap on load.  Periodic: wrap (the pattern
// of apps/2d/euler/test_exact2/SetBndValues.cpp:28-197); transmissive:
// zeroth-order extrapolation, i.e. clamp (apps/2d/euler/riemann_test/
// SetBndValues.cpp:30-111).  Corners get both remaps.
// ---------------------------------------------------------------------------
// Any k maps into [0, n): cells of a partial tile beyond the domain (whose
// results are discarded) may lie more than one period away.
__device__ __forceinline__ int bc_remap(int k, int n, int bc_lo, int bc_hi)
{
    if (k < 0) {
        if (bc_lo != FIN_BC_PERIODIC) return 0;
        k %= n;
        return k < 0 ? k + n : k;
    }
    if (k >= n) return bc_hi == FIN_BC_PERIODIC ? k % n : n - 1;
    return k;
}

// Non-negative doubles order like their bit patterns, so an unsigned 64-bit
// atomicMax is an exact max (NaN with a clear sign bit compares above +Inf,
// so a NaN wave speed wins the max and is seen by the host).
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v)
{
    atomicMax(reinterpret_cast<unsigned long long*>(addr),
              static_cast<unsigned long long>(__double_as_longlong(v)));
}

// dog_math.h:18-22 (NaN behaviour included: Max(a, NaN) = NaN, Max(NaN, b) = b)
template <class R> __host__ __device__ __forceinline__ R Max(R a, R b) { return a > b ? a : b; }
template <class R> __host__ __device__ __forceinline__ R Min(R a, R b) { return a < b ? a : b; }

// Reciprocal by Newton-Raphson refinement of the hardware approximation
// (PTX rcp.approx.ftz): r <- r + r(1 - x r), which squares the relative error
// per step.  Two steps bring the FP64 approximation to within an ulp or two
// (the plain form's parity bar is 1e-12, four orders above); FP32 uses the
// approximation alone (~1 ulp).  x = 0 gives NaN instead of Inf; every use
// here divides by a density, pressure or WENO weight sum, where 0 is already
// a failed state that the non-finite check reports.
__device__ __forceinline__ double rcp(double x)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}
__device__ __forceinline__ float rcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// Packed pairs of FP32 values for sm_100's f32x2 arithmetic (PTX add / mul /
// fma .rn.f32x2): one instruction computes two independent lanes, each
// rounded exactly as the scalar operation would be, so code written on pairs
// gives the bits of the same scalar code with half the instructions.
struct f2 {
    unsigned long long v;
};
__device__ __forceinline__ f2 f2_make(float a, float b)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ f2 f2_of(float2 a) { return f2_make(a.x, a.y); }
__device__ __forceinline__ float f2_lo(f2 a)
{
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
    return lo;
}
__device__ __forceinline__ float f2_hi(f2 a)
{
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
    return hi;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c)   // a b + c per lane
{
    f2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b)
{
    f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b)
{
    f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}

__device__ __forceinline__ double fsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float fsqrt(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// ---------------------------------------------------------------------------
// Euler callbacks (apps/2d/euler/lib).  Component order inside a face is the
// "normal frame" (rho, m_n, m_t, m_w, E): for x faces (ixy=1) m_n = rho u,
// m_t = rho v; for y faces (ixy=2) m_n = rho v, m_t = rho u.  This is the
// mu/mv swap of ProjectLeftEig.cpp:20-32.  The characteristic fields are
// reconstructed one by one, so their order never matters.
// ---------------------------------------------------------------------------
struct Euler {
    // FluxFunc.cpp:19-42 for one point: both flux components.
    template <class R>
    __device__ __forceinline__ static void flux(R gamma, const R* Q, R* f, R* g)
    {
        const R rho = Q[0];
        const R ir = rcp(rho);
        const R u1 = Q[1] * ir, u2 = Q[2] * ir, u3 = Q[3] * ir;
        const R energy = Q[4];
        const R press = (gamma - R(1)) * (energy - R(0.5) * rho * (u1 * u1 + u2 * u2 + u3 * u3));
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

    // Average-state eigen data of ProjectLeftEig.cpp:34-44 / ProjectRightEig.cpp:33-43,
    // in the normal frame, with the two denominators of the left projection
    // inverted once per face.
    template <class R>
    struct Eig {
        R u1, u2, u3, umag2, c, cl, H, hu2;   // hu2 = umag2/2
        R inv_cd;    // 1/(c*(2H-umag2))   (left rows 1 and 5)
        R inv_d2;    // 2/(2H-umag2)       (left row mu)
    };

    template <class R>
    __device__ __forceinline__ static Eig<R> eig(R gamma, const R* Qn)
    {
        Eig<R> e;
        const R rho = Qn[0];
        const R ir = rcp(rho);
        e.u1 = Qn[1] * ir;
        e.u2 = Qn[2] * ir;
        e.u3 = Qn[3] * ir;
        const R energy = Qn[4];
        e.umag2 = (e.u1 * e.u1 + e.u2 * e.u2 + e.u3 * e.u3);
        const R press = (gamma - R(1)) * (energy - R(0.5) * rho * e.umag2);
        const R c2 = gamma * press * ir;
        // Right projection uses sqrt(fabs()) (ProjectRightEig.cpp:42), the
        // left one plain sqrt (ProjectLeftEig.cpp:43): identical unless the
        // pressure is negative, where the left one is NaN.
        e.c = fsqrt(fabs(c2));
        e.cl = c2 < R(0) ? R(NAN) : e.c;
        e.H = (energy + press) * ir;
        e.hu2 = e.umag2 / R(2);
        const R d = R(2) * e.H - e.umag2;
        e.inv_cd = rcp(e.cl * d);
        e.inv_d2 = R(2) * rcp(d);
        return e;
    }

    // Per-face coefficients of the three full rows of the left projection
    // (ProjectLeftEig.cpp:49-65): W0 = (a0 v1 + b0 v0 + c tail) inv_cd,
    // W4 = (a4 v1 + b4 v0 + c tail) inv_cd, W1 = (e1 v0 + u1 v1 + u2 v2 + u3 v3 - v4) inv_d2,
    // with tail = v4 - u2 v2 - u3 v3; rows 2 and 3 are v2 - u2 v0, v3 - u3 v0.
    template <class R>
    struct Rows { R a0, b0, a4, b4, e1; };

    template <class R>
    __device__ __forceinline__ static Rows<R> rows(const Eig<R>& e)
    {
        Rows<R> r;
        const R c = e.cl;
        r.a0 = e.hu2 - e.H - e.u1 * c;
        r.b0 = e.hu2 * (c - e.u1) + e.H * e.u1;
        r.a4 = e.H - e.hu2 - e.u1 * c;
        r.b4 = e.hu2 * (c + e.u1) - e.H * e.u1;
        r.e1 = e.H - e.umag2;
        return r;
    }

    // Rows 0 and 4 of the left projection of one vector (normal frame).
    template <class R>
    __device__ __forceinline__ static void left04(const Eig<R>& e, const Rows<R>& r, const R* v, R& w0, R& w4)
    {
        const R ct = e.cl * (v[4] - e.u2 * v[2] - e.u3 * v[3]);
        w0 = (r.a0 * v[1] + r.b0 * v[0] + ct) * e.inv_cd;
        w4 = (r.a4 * v[1] + r.b4 * v[0] + ct) * e.inv_cd;
    }
    // Row 1 of the left projection of one vector (normal frame).
    template <class R>
    __device__ __forceinline__ static R left1(const Eig<R>& e, const Rows<R>& r, const R* v)
    {
        return (r.e1 * v[0] + e.u1 * v[1] + e.u2 * v[2] + e.u3 * v[3] - v[4]) * e.inv_d2;
    }

    // Rows 0, 1 and 4 of the left projection of one vector (normal frame).
    template <class R>
    __device__ __forceinline__ static void left014(const Eig<R>& e, const Rows<R>& r, const R* v, R& w0, R& w1, R& w4)
    {
        const R tail = v[4] - e.u2 * v[2] - e.u3 * v[3];
        const R ct = e.cl * tail;
        w0 = (r.a0 * v[1] + r.b0 * v[0] + ct) * e.inv_cd;
        w4 = (r.a4 * v[1] + r.b4 * v[0] + ct) * e.inv_cd;
        w1 = (r.e1 * v[0] + e.u1 * v[1] + e.u2 * v[2] + e.u3 * v[3] - v[4]) * e.inv_d2;
    }

    // ProjectLeftEig.cpp:47-66 for one point (normal frame in and out).
    template <class R>
    __device__ __forceinline__ static void left(const Eig<R>& e, const R* Q, R* W)
    {
        const R c = e.cl;
        const R tail = c * (Q[4] - e.u2 * Q[2] - e.u3 * Q[3]);
        W[0] = ((e.hu2 - e.H - e.u1 * c) * Q[1] + (e.hu2 * (c - e.u1) + e.H * e.u1) * Q[0] + tail) * e.inv_cd;
        W[1] = ((e.H - e.umag2) * Q[0] + e.u1 * Q[1] + e.u2 * Q[2] + e.u3 * Q[3] - Q[4]) * e.inv_d2;
        W[2] = Q[2] - e.u2 * Q[0];
        W[3] = Q[3] - e.u3 * Q[0];
        W[4] = ((e.H - e.hu2 - e.u1 * c) * Q[1] + (e.hu2 * (c + e.u1) - e.H * e.u1) * Q[0] + tail) * e.inv_cd;
    }

    // ProjectRightEig.cpp:46-62 for one point (normal frame in and out).
    template <class R>
    __device__ __forceinline__ static void right(const Eig<R>& e, const R* W, R* Q)
    {
        const R c = e.c;
        const R s = W[0] + W[1] + W[4];
        Q[0] = s;
        Q[1] = (e.u1 - c) * W[0] + e.u1 * W[1] + (e.u1 + c) * W[4];
        Q[2] = e.u2 * s + W[2];
        Q[3] = e.u3 * s + W[3];
        Q[4] = (e.H - e.u1 * c) * W[0] + e.hu2 * W[1] + e.u2 * W[2] + e.u3 * W[3] + (e.H + e.u1 * c) * W[4];
    }

    // Per-cell quantities of SetWaveSpd.cpp:24-37 (normal frame, nmag = 1).
    template <class R>
    struct Cell { R rho, un, p, c; };

    template <class R>
    __device__ __forceinline__ static Cell<R> cell(R gamma, const R* Qn)
    {
        Cell<R> s;
        s.rho = Qn[0];
        const R ir = rcp(s.rho);
        const R u1 = Qn[1] * ir, u2 = Qn[2] * ir, u3 = Qn[3] * ir;
        s.un = u1;
        s.p = (gamma - R(1)) * (Qn[4] - R(0.5) * s.rho * (u1 * u1 + u2 * u2 + u3 * u3));
        s.c = fsqrt(fabs(gamma * s.p * ir));
        return s;
    }

    // SetWaveSpd.cpp:39-68 from two cells' data; returns max(|s1|, |s2|)
    // (ConstructL.cpp:172 before the Max with the global alpha).  *neg is
    // set when the average pressure or density is negative (the reference
    // prints a warning there, SetWaveSpd.cpp:52-57).
    template <class R>
    __device__ __forceinline__ static R speed(R gamma, const Cell<R>& l, const Cell<R>& r, bool* neg)
    {
        const R rho = R(0.5) * (l.rho + r.rho);
        const R un = R(0.5) * (l.un + r.un);
        const R press = R(0.5) * (l.p + r.p);
        const R c = fsqrt(fabs(gamma * press * rcp(rho)));
        if (press < R(0) || rho < R(0)) *neg = true;
        const R s1 = Min(l.un - l.c, un - c);
        const R s2 = Max(r.un + r.c, un + c);
        return Max(fabs(s1), fabs(s2));
    }

    // GlobalWaveSpd.cpp:71-76 for one cell (Ql = Qr): Max(|u_n - c|, |u_n + c|).
    template <class R>
    __device__ __forceinline__ static R cell_speed(const Cell<R>& s)
    {
        return Max(fabs(s.un - s.c), fabs(s.un + s.c));
    }
};

// ---------------------------------------------------------------------------
// WENO5 point-value reconstruction of u_{i+1/2} from {u_{i-2} .. u_{i+2}}
// (lib/WenoReconstruct.cpp: JS5 90-141, Z5 385-438, FD5 580-616).
//
// Smoothness indicators and candidate stencils follow :121-128 term by term.
// The nonlinear weights are evaluated with one division: with d_k = eps+beta_k
// and power 2, omt_k = g_k / d_k^2 (JS) or g_k (d_k^2 + tau^2)/d_k^2 (Z), and
// the normalised sum  sum(omt_k u_k)/sum(omt_k)  is unchanged when every omt_k
// is multiplied by D = d_0^2 d_1^2 d_2^2.  In FP32 the d_k^2 are first scaled
// by 1/max(d_k^2) so no product over- or underflows for any epsilon; this is
// the "epsilon rescaled to the FP32 range" form.  Other powers call pow().
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ void weno5_parts(const R* u, R& b0, R& b1, R& b2, R& c0, R& c1, R& c2)
{
    const R uim2 = u[0], uim1 = u[1], ui = u[2], uip1 = u[3], uip2 = u[4];
    R t, s;
    t = uim2 - R(2) * uim1 + ui;       s = uim2 - R(4) * uim1 + R(3) * ui;
    b0 = (R(13) / R(12)) * (t * t) + R(0.25) * (s * s);
    t = uim1 - R(2) * ui + uip1;       s = uim1 - uip1;
    b1 = (R(13) / R(12)) * (t * t) + R(0.25) * (s * s);
    t = ui - R(2) * uip1 + uip2;       s = R(3) * ui - R(4) * uip1 + uip2;
    b2 = (R(13) / R(12)) * (t * t) + R(0.25) * (s * s);
    c0 = (R(1) / R(3)) * uim2 - (R(7) / R(6)) * uim1 + (R(11) / R(6)) * ui;
    c1 = (R(-1) / R(6)) * uim1 + (R(5) / R(6)) * ui + (R(1) / R(3)) * uip1;
    c2 = (R(1) / R(3)) * ui + (R(5) / R(6)) * uip1 - (R(1) / R(6)) * uip2;
}

template <class R, int VER, bool P2>
__device__ __forceinline__ R weno5(const R* u, R eps, R pw)
{
    R b0, b1, b2, c0, c1, c2;
    weno5_parts(u, b0, b1, b2, c0, c1, c2);
    if (VER == FIN_WENO_FD) return R(0.1) * c0 + R(0.6) * c1 + R(0.3) * c2;
    R w0, w1, w2;
    if (P2) {
        const R d0 = eps + b0, d1 = eps + b1, d2 = eps + b2;
        R D0 = d0 * d0, D1 = d1 * d1, D2 = d2 * d2;
        R T = R(0);
        if (VER == FIN_WENO_Z) { const R tau = fabs(b0 - b2); T = tau * tau; }
        if (sizeof(R) == 4) {
            const R s = rcp(Max(D0, Max(D1, D2)));
            D0 *= s; D1 *= s; D2 *= s; T *= s;
        }
        if (VER == FIN_WENO_JS) {
            w0 = R(0.1) * (D1 * D2);
            w1 = R(0.6) * (D0 * D2);
            w2 = R(0.3) * (D0 * D1);
        } else {
            w0 = R(0.1) * ((D0 + T) * (D1 * D2));
            w1 = R(0.6) * ((D1 + T) * (D0 * D2));
            w2 = R(0.3) * ((D2 + T) * (D0 * D1));
        }
    } else {
        if (VER == FIN_WENO_JS) {
            w0 = R(0.1) * pow(eps + b0, -pw);
            w1 = R(0.6) * pow(eps + b1, -pw);
            w2 = R(0.3) * pow(eps + b2, -pw);
        } else {
            const R tau = fabs(b0 - b2);
            w0 = R(0.1) * (R(1) + pow(tau / (eps + b0), pw));
            w1 = R(0.6) * (R(1) + pow(tau / (eps + b1), pw));
            w2 = R(0.3) * (R(1) + pow(tau / (eps + b2), pw));
        }
    }
    return (w0 * c0 + w1 * c1 + w2 * c2) * rcp(w0 + w1 + w2);
}

// The two WENO5 reconstructions of a face's split (u = gp, the points of
// the + split; the pair's second lane gm) in FP32 as f32x2 pairs, with power
// 2 (or the linear FD5 weights): the operations of weno5<float, VER, true>,
// each product and sum written out (explicit fma where the scalar form
// contracts), both lanes in one instruction; the weight normalisation's
// maxima and reciprocals per lane.  Returns WENO(gp) + WENO(gm).
__device__ __forceinline__ f2 f2_splat(float a) { return f2_make(a, a); }
__device__ __forceinline__ f2 f2_abs(f2 a)
{
    f2 r;
    r.v = a.v & 0x7fffffff7fffffffull;
    return r;
}
template <int VER>
__device__ __forceinline__ float weno5_pair_x2(const float* up, const float* um, float eps)
{
    f2 u[5];
#pragma unroll
    for (int k = 0; k < 5; k++) u[k] = f2_make(up[k], um[k]);
    const f2 uim2 = u[0], uim1 = u[1], ui = u[2], uip1 = u[3], uip2 = u[4];
    const f2 k1312 = f2_splat(13.0f / 12.0f), k025 = f2_splat(0.25f);
    auto beta = [&](f2 t, f2 s) { return f2_fma(k1312, f2_mul(t, t), f2_mul(k025, f2_mul(s, s))); };
    const f2 b0 = beta(f2_add(f2_fma(f2_splat(-2.0f), uim1, uim2), ui),
                       f2_fma(f2_splat(3.0f), ui, f2_fma(f2_splat(-4.0f), uim1, uim2)));
    const f2 b1 = beta(f2_add(f2_fma(f2_splat(-2.0f), ui, uim1), uip1), f2_fma(f2_splat(-1.0f), uip1, uim1));
    const f2 b2 = beta(f2_add(f2_fma(f2_splat(-2.0f), uip1, ui), uip2),
                       f2_add(f2_fma(f2_splat(-4.0f), uip1, f2_mul(f2_splat(3.0f), ui)), uip2));
    const f2 c0 = f2_fma(f2_splat(11.0f / 6.0f), ui, f2_fma(f2_splat(-7.0f / 6.0f), uim1, f2_mul(f2_splat(1.0f / 3.0f), uim2)));
    const f2 c1 = f2_fma(f2_splat(1.0f / 3.0f), uip1, f2_fma(f2_splat(5.0f / 6.0f), ui, f2_mul(f2_splat(-1.0f / 6.0f), uim1)));
    const f2 c2 = f2_fma(f2_splat(-1.0f / 6.0f), uip2, f2_fma(f2_splat(5.0f / 6.0f), uip1, f2_mul(f2_splat(1.0f / 3.0f), ui)));
    f2 r;
    if (VER == FIN_WENO_FD) {
        r = f2_fma(f2_splat(0.3f), c2, f2_fma(f2_splat(0.6f), c1, f2_mul(f2_splat(0.1f), c0)));
    } else {
        const f2 e = f2_splat(eps);
        const f2 d0 = f2_add(e, b0), d1 = f2_add(e, b1), d2 = f2_add(e, b2);
        f2 D0 = f2_mul(d0, d0), D1 = f2_mul(d1, d1), D2 = f2_mul(d2, d2);
        const float sl = rcp(Max(f2_lo(D0), Max(f2_lo(D1), f2_lo(D2))));
        const float sh = rcp(Max(f2_hi(D0), Max(f2_hi(D1), f2_hi(D2))));
        const f2 sc = f2_make(sl, sh);
        D0 = f2_mul(D0, sc);
        D1 = f2_mul(D1, sc);
        D2 = f2_mul(D2, sc);
        f2 w0, w1, w2;
        if (VER == FIN_WENO_JS) {
            w0 = f2_mul(f2_splat(0.1f), f2_mul(D1, D2));
            w1 = f2_mul(f2_splat(0.6f), f2_mul(D0, D2));
            w2 = f2_mul(f2_splat(0.3f), f2_mul(D0, D1));
        } else {
            const f2 tau = f2_abs(f2_fma(f2_splat(-1.0f), b2, b0));
            const f2 T = f2_mul(f2_mul(tau, tau), sc);
            w0 = f2_mul(f2_splat(0.1f), f2_mul(f2_add(D0, T), f2_mul(D1, D2)));
            w1 = f2_mul(f2_splat(0.6f), f2_mul(f2_add(D1, T), f2_mul(D0, D2)));
            w2 = f2_mul(f2_splat(0.3f), f2_mul(f2_add(D2, T), f2_mul(D0, D1)));
        }
        const f2 num = f2_fma(w2, c2, f2_fma(w1, c1, f2_mul(w0, c0)));
        const f2 den = f2_add(f2_add(w0, w1), w2);
        r = f2_mul(num, f2_make(rcp(f2_lo(den)), rcp(f2_hi(den))));
    }
    return f2_lo(r) + f2_hi(r);
}

}  // namespace fin
