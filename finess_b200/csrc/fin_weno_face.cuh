// Full characteristic WENO flux of one face (ConstructL.cpp:62-208 for x
// faces, 214-358 for y faces) from its 6-point stencil, with the stencil
// access abstracted: pt(s, q, f) fills the normal-frame conserved values q[5]
// and half fluxes f[5] (0.5 f_n) of stencil point s = 0..5 (cells i-3 .. i+2
// of the face between i-1 and i).  The arithmetic is the stage kernel's:
//   gp_s = L (f_s + l q_s), s = 0..4;  gm_s = L (f_{5-s} - l q_{5-s})
//   (ConstructL.cpp:179-185, with l = 0.5 alpha_scaling alpha),
//   ghat_k = WENO(gp_k) + WENO(gm_k)  (ConstructL.cpp:191-199),
//   fh = R ghat accumulated field by field (ConstructL.cpp:202-206),
// in three passes over the fields (0 and 4; 1; 2 and 3) so that no more than
// two fields' stencils are live at once.
#pragma once
#include "fin_device.cuh"

namespace fin {

// Scheduling fences: an empty volatile asm that reads and writes x.  Volatile
// asm statements keep their order, so fencing the inputs and result of each
// pair of WENO reconstructions stops the scheduler from evaluating all ten of
// a face at once.
__device__ __forceinline__ void wfence(double& x) { asm volatile("" : "+d"(x)); }
__device__ __forceinline__ void wfence(float& x) { asm volatile("" : "+f"(x)); }

template <class R, int VER, bool P2>
__device__ __forceinline__ R weno_pair_f(R* up, R* um, R eps, R pw)
{
#pragma unroll
    for (int k = 0; k < 5; k++) { wfence(up[k]); wfence(um[k]); }
    R g;
    if constexpr (sizeof(R) == 4 && (P2 || VER == FIN_WENO_FD)) g = weno5_pair_x2<VER>(up, um, eps);   // f32x2 pairs
    else g = weno5<R, VER, P2>(up, eps, pw) + weno5<R, VER, P2>(um, eps, pw);
    wfence(g);
    return g;
}

// Right projection (ProjectRightEig.cpp:46-62) of field k with amplitude gk,
// added into the face flux f[0..4] (normal frame).
template <class R>
__device__ __forceinline__ void right_add_f(const typename Euler::Eig<R>& e, int k, R gk, R* f)
{
    if (k == 0) {
        f[0] += gk; f[1] += (e.u1 - e.c) * gk; f[2] += e.u2 * gk; f[3] += e.u3 * gk; f[4] += (e.H - e.u1 * e.c) * gk;
    } else if (k == 4) {
        f[0] += gk; f[1] += (e.u1 + e.c) * gk; f[2] += e.u2 * gk; f[3] += e.u3 * gk; f[4] += (e.H + e.u1 * e.c) * gk;
    } else if (k == 1) {
        f[0] += gk; f[1] += e.u1 * gk; f[2] += e.u2 * gk; f[3] += e.u3 * gk; f[4] += e.hu2 * gk;
    } else if (k == 2) {
        f[2] += gk; f[4] += e.u2 * gk;
    } else {
        f[3] += gk; f[4] += e.u3 * gk;
    }
}

template <class R, int VER, bool P2, class Pt>
__device__ __forceinline__ void weno_char_flux(const typename Euler::Eig<R>& ev, R lah, R eps, R pw, const Pt& pt,
                                               R* fh)
{
    const typename Euler::Rows<R> rw = Euler::rows(ev);
#pragma unroll
    for (int m = 0; m < MEQN; m++) fh[m] = R(0);
    {
        // pass 1: characteristic fields 0 and 4 (acoustic rows, shared tail)
        R p0[5], p4[5], m0[5], m4[5];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            // keep the compiler from hoisting every stencil point's loads
            // ahead of the arithmetic
            asm volatile("" ::: "memory");
            R q[MEQN], f[MEQN];
            pt(s, q, f);
            if (s < 5) {
                const R v[MEQN] = {f[0] + lah * q[0], f[1] + lah * q[1], f[2] + lah * q[2], f[3] + lah * q[3],
                                   f[4] + lah * q[4]};
                Euler::left04(ev, rw, v, p0[s], p4[s]);
            }
            if (s > 0) {
                const R v[MEQN] = {f[0] - lah * q[0], f[1] - lah * q[1], f[2] - lah * q[2], f[3] - lah * q[3],
                                   f[4] - lah * q[4]};
                Euler::left04(ev, rw, v, m0[5 - s], m4[5 - s]);
            }
        }
#pragma unroll 1
        for (int k = 0; k < 2; k++) {
            R up[5], um[5];
#pragma unroll
            for (int t = 0; t < 5; t++) {
                up[t] = k == 0 ? p0[t] : p4[t];
                um[t] = k == 0 ? m0[t] : m4[t];
            }
            right_add_f<R>(ev, k == 0 ? 0 : 4, weno_pair_f<R, VER, P2>(up, um, eps, pw), fh);
        }
    }
    {
        // pass 2: characteristic field 1 (the entropy-like row)
        R p1[5], m1[5];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            asm volatile("" ::: "memory");
            R q[MEQN], f[MEQN];
            pt(s, q, f);
            if (s < 5) {
                const R v[MEQN] = {f[0] + lah * q[0], f[1] + lah * q[1], f[2] + lah * q[2], f[3] + lah * q[3],
                                   f[4] + lah * q[4]};
                p1[s] = Euler::left1(ev, rw, v);
            }
            if (s > 0) {
                const R v[MEQN] = {f[0] - lah * q[0], f[1] - lah * q[1], f[2] - lah * q[2], f[3] - lah * q[3],
                                   f[4] - lah * q[4]};
                m1[5 - s] = Euler::left1(ev, rw, v);
            }
        }
        right_add_f<R>(ev, 1, weno_pair_f<R, VER, P2>(p1, m1, eps, pw), fh);
    }
    {
        // pass 3: fields 2 and 3 (rows v_t - u2 v0 and v_w - u3 v0)
        R p2[5], p3[5], m2[5], m3[5];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            asm volatile("" ::: "memory");
            R q[MEQN], f[MEQN];
            pt(s, q, f);
            if (s < 5) {
                const R v0 = f[0] + lah * q[0];
                p2[s] = (f[2] + lah * q[2]) - ev.u2 * v0;
                p3[s] = (f[3] + lah * q[3]) - ev.u3 * v0;
            }
            if (s > 0) {
                const R v0 = f[0] - lah * q[0];
                m2[5 - s] = (f[2] - lah * q[2]) - ev.u2 * v0;
                m3[5 - s] = (f[3] - lah * q[3]) - ev.u3 * v0;
            }
        }
#pragma unroll 1
        for (int k = 0; k < 2; k++) {
            R up[5], um[5];
#pragma unroll
            for (int t = 0; t < 5; t++) {
                up[t] = k == 0 ? p2[t] : p3[t];
                um[t] = k == 0 ? m2[t] : m3[t];
            }
            right_add_f<R>(ev, k == 0 ? 2 : 3, weno_pair_f<R, VER, P2>(up, um, eps, pw), fh);
        }
    }
}

// weno_char_flux in FP32 with f32x2 pairs: the + and - split values of a
// stencil point, v = f + l q and f - l q, are one pair, projected together
// (left04 / left1 lane by lane), and the two reconstructions of each field
// run as one paired WENO (weno5_pair_x2).  The field passes and their order
// are weno_char_flux's.
__device__ __forceinline__ void left04_x2(const Euler::Eig<float>& e, const Euler::Rows<float>& r, const f2* v, f2& w0,
                                          f2& w4)
{
    // ct = c (v4 - u2 v2 - u3 v3); w0 = (a0 v1 + b0 v0 + ct) inv_cd; w4 = (a4 v1 + b4 v0 + ct) inv_cd
    const f2 ct = f2_mul(f2_splat(e.cl),
                         f2_fma(f2_splat(-e.u3), v[3], f2_fma(f2_splat(-e.u2), v[2], v[4])));
    w0 = f2_mul(f2_add(f2_fma(f2_splat(r.a0), v[1], f2_mul(f2_splat(r.b0), v[0])), ct), f2_splat(e.inv_cd));
    w4 = f2_mul(f2_add(f2_fma(f2_splat(r.a4), v[1], f2_mul(f2_splat(r.b4), v[0])), ct), f2_splat(e.inv_cd));
}
__device__ __forceinline__ f2 left1_x2(const Euler::Eig<float>& e, const Euler::Rows<float>& r, const f2* v)
{
    // (e1 v0 + u1 v1 + u2 v2 + u3 v3 - v4) inv_d2
    f2 a = f2_mul(f2_splat(r.e1), v[0]);
    a = f2_fma(f2_splat(e.u1), v[1], a);
    a = f2_fma(f2_splat(e.u2), v[2], a);
    a = f2_fma(f2_splat(e.u3), v[3], a);
    a = f2_fma(f2_splat(-1.0f), v[4], a);
    return f2_mul(a, f2_splat(e.inv_d2));
}

// FIN_X2_MERGE: fields 0, 4 and 1 in one sweep of the stencil (one load of
// each point instead of two), at the price of six live reconstruction
// stencils instead of four.  Measured on B200 at 4096^2: the FP32 stage
// 2.28 -> 2.18 ms, the hybrid stage 1.24 -> 1.16 ms at mid-run; built.
#ifndef FIN_X2_MERGE
#define FIN_X2_MERGE 1
#endif
template <int VER, class Pt>
__device__ __forceinline__ void weno_char_flux_x2(const Euler::Eig<float>& ev, float lah, const Pt& pt, float eps,
                                                  float* fh)
{
    const Euler::Rows<float> rw = Euler::rows(ev);
    const f2 pmla = f2_make(lah, -lah);
#pragma unroll
    for (int m = 0; m < MEQN; m++) fh[m] = 0.0f;
    // the split pair of point s: (f + l q, f - l q) per component
    auto split = [&](int s, f2* v) {
        float q[MEQN], f[MEQN];
        pt(s, q, f);
#pragma unroll
        for (int m = 0; m < MEQN; m++) v[m] = f2_fma(pmla, f2_splat(q[m]), f2_splat(f[m]));
    };
#if FIN_X2_MERGE
    {
        // fields 0, 4 and 1 in one sweep; the right projections are added
        // in the order 0, 4, 1 as the separate passes add them
        float p0[5], p4[5], m0[5], m4[5], p1[5], m1[5];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            asm volatile("" ::: "memory");
            f2 v[MEQN], w0, w4;
            split(s, v);
            left04_x2(ev, rw, v, w0, w4);
            const f2 w1 = left1_x2(ev, rw, v);
            if (s < 5) { p0[s] = f2_lo(w0); p4[s] = f2_lo(w4); p1[s] = f2_lo(w1); }
            if (s > 0) { m0[5 - s] = f2_hi(w0); m4[5 - s] = f2_hi(w4); m1[5 - s] = f2_hi(w1); }
        }
#pragma unroll 1
        for (int k = 0; k < 3; k++) {
            float up[5], um[5];
#pragma unroll
            for (int t = 0; t < 5; t++) {
                up[t] = k == 0 ? p0[t] : (k == 1 ? p4[t] : p1[t]);
                um[t] = k == 0 ? m0[t] : (k == 1 ? m4[t] : m1[t]);
            }
            right_add_f<float>(ev, k == 0 ? 0 : (k == 1 ? 4 : 1), weno_pair_f<float, VER, true>(up, um, eps, 2.0f), fh);
        }
    }
#else
    {
        // pass 1: fields 0 and 4
        float p0[5], p4[5], m0[5], m4[5];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            asm volatile("" ::: "memory");
            f2 v[MEQN], w0, w4;
            split(s, v);
            left04_x2(ev, rw, v, w0, w4);
            if (s < 5) { p0[s] = f2_lo(w0); p4[s] = f2_lo(w4); }
            if (s > 0) { m0[5 - s] = f2_hi(w0); m4[5 - s] = f2_hi(w4); }
        }
#pragma unroll 1
        for (int k = 0; k < 2; k++) {
            float up[5], um[5];
#pragma unroll
            for (int t = 0; t < 5; t++) {
                up[t] = k == 0 ? p0[t] : p4[t];
                um[t] = k == 0 ? m0[t] : m4[t];
            }
            right_add_f<float>(ev, k == 0 ? 0 : 4, weno_pair_f<float, VER, true>(up, um, eps, 2.0f), fh);
        }
    }
    {
        // pass 2: field 1
        float p1[5], m1[5];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            asm volatile("" ::: "memory");
            f2 v[MEQN];
            split(s, v);
            const f2 w = left1_x2(ev, rw, v);
            if (s < 5) p1[s] = f2_lo(w);
            if (s > 0) m1[5 - s] = f2_hi(w);
        }
        right_add_f<float>(ev, 1, weno_pair_f<float, VER, true>(p1, m1, eps, 2.0f), fh);
    }
#endif
    {
        // pass 3: fields 2 and 3 (v_t - u2 v0, v_w - u3 v0)
        float p2[5], p3[5], m2[5], m3[5];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            asm volatile("" ::: "memory");
            f2 v[MEQN];
            split(s, v);
            const f2 w2 = f2_fma(f2_splat(-ev.u2), v[0], v[2]);
            const f2 w3 = f2_fma(f2_splat(-ev.u3), v[0], v[3]);
            if (s < 5) { p2[s] = f2_lo(w2); p3[s] = f2_lo(w3); }
            if (s > 0) { m2[5 - s] = f2_hi(w2); m3[5 - s] = f2_hi(w3); }
        }
#pragma unroll 1
        for (int k = 0; k < 2; k++) {
            float up[5], um[5];
#pragma unroll
            for (int t = 0; t < 5; t++) {
                up[t] = k == 0 ? p2[t] : p3[t];
                um[t] = k == 0 ? m2[t] : m3[t];
            }
            right_add_f<float>(ev, k == 0 ? 2 : 3, weno_pair_f<float, VER, true>(up, um, eps, 2.0f), fh);
        }
    }
}

}  // namespace fin
