// The hybrid-form stage kernel: FP32 bulk with the troubled-face flags of the
// step.  It computes what k_stage computes for one RK stage (ConstructL,
// UpdateSoln and the wave-speed maxima of the next stage and the CFL), with
//   * smooth faces (no flag in the 3 x 3 window of same-direction faces): the
//     linear FD5 flux in its component-wise 6-point form (linear_face), which
//     equals the reference's characteristic FD5 path (WenoReconstruct_FD5,
//     lib/WenoReconstruct.cpp:580-616) because the reconstruction is linear;
//   * troubled faces: the full characteristic WENO flux (weno_char_flux).
// Layout and schedule, for B200:
//   * one TI x TJ tile per CTA, three CTAs (24 warps) per SM;
//   * q_in's tile + halo arrives by one TMA copy (tiles clear of the domain
//     boundary) into an FP64 staging tile that the update reads again for
//     q_in's interior; the other stage operand's interior arrives by a second
//     TMA copy that lands while the faces are computed;
//   * per cell the half flux and the state are stored as (0.5 f, q) pairs
//     along each stencil direction, so one 8-byte load serves both terms of
//     the split; the cell primitives (u, v, p, c) are one 16-byte load;
//   * the flags are the indicator's bit masks, two words per window row.
#pragma once
#include "fin_stage.cuh"
#include "fin_weno_face.cuh"
#include <type_traits>

namespace fin {

using HybCfg = TileCfg<15, 16, 256>;

// Resident CTAs per SM the kernel is laid out for: 3 keeps the update's
// stage operands in shared memory (q_in's interior in the staging tile, the
// other operand by a second TMA copy); 4 shares the staging tile's space with
// the face fluxes and reads both operands from L2 (q_in's interior is there
// from the tile's own copy, the other operand is prefetched into L2 by TMA),
// within 64 registers a thread.
#ifndef FIN_HYB_CTAS
#define FIN_HYB_CTAS 4
#endif

// Shared-memory layout (byte offsets) of k_stage_hyb.
template <class Cfg>
struct HybSmem {
    static constexpr int TI = Cfg::TI, TJ = Cfg::TJ, RI = Cfg::RI, RJ = Cfg::RJ, NT = Cfg::NT;
    static constexpr bool SHARE = FIN_HYB_CTAS >= 4;
    static constexpr size_t PRIM = 0;                                                    // float4 [RI][RJ]
    static constexpr size_t FQX = PRIM + size_t(RI) * RJ * 16;                          // float2 [M][RI][TJ]
    static constexpr size_t FQY = FQX + size_t(MEQN) * RI * TJ * 8;                     // float2 [M][TI][RJ]
    // face-flux rows of FP = TJ + 2 floats: the warps take face rows (and
    // the update cell rows) 8 apart, 8 x 18 = 144 words, 16 modulo 32, so a
    // warp's two rows fall in opposite halves of the banks
    static constexpr int FP = TJ + 2;
    static constexpr size_t FHGH = size_t(MEQN) * ((TI + 1) + TI) * FP * 4;             // Fh, Gh bytes
    static constexpr size_t STG = Cfg::pad128(FQY + size_t(MEQN) * TI * RJ * 8);        // double [M][RI][SJ]
    static constexpr size_t FH = SHARE ? STG : STG + Cfg::pad128(Cfg::STG_BYTES);       // float [M][TI+1][FP]
    static constexpr size_t GH = FH + size_t(MEQN) * (TI + 1) * FP * 4;                 // float [M][TI][FP]
    static constexpr size_t EBUF = Cfg::pad128(SHARE ? STG + Cfg::STG_BYTES : FH + FHGH);   // double [M][TI][TJ]
    static constexpr size_t RED = SHARE ? EBUF : EBUF + Cfg::ABUF_BYTES;               // double [NT/32][4]
    static constexpr size_t MASK = RED + size_t(NT / 32) * 4 * 8;                       // unsigned [FXR + FYR]
    static constexpr size_t NTRB = MASK + 4 * size_t(Cfg::FXR + Cfg::FYR);              // int
    static constexpr size_t TLIST = NTRB + 4;                                            // short [NFX + NFY]
    static constexpr size_t MBAR = (TLIST + 2 * size_t(Cfg::NFX + Cfg::NFY) + 7) / 8 * 8;   // uint64
    static constexpr size_t BYTES = MBAR + 8;
    static_assert(!SHARE || FHGH <= Cfg::STG_BYTES, "the face fluxes fit the staging tile");
};

// linear_face on (0.5 f, q) pairs: P points at stencil point 3.  The f sums
// and q differences run as f32x2 pairs, lane by lane the operations of
//   sf = 37 (f2 + f3) + (-8 (f1 + f4) + (f0 + f5)),
//   sq = 10 (q2 - q3) + (-5 (q1 - q4) + (q0 - q5)),
// (x + y and x - y as fma(y, +-1, x): the same rounding).
// The f32x2 form measured 1 % slower than the scalar one (B200, 4096^2,
// mid-run state), so the scalar form is built.
#ifndef FIN_X2_LINEAR
#define FIN_X2_LINEAR 0
#endif
__device__ __forceinline__ float linear_face2(const float2* P, int str, float lah)
{
#if FIN_X2_LINEAR
    const f2 pm = f2_make(1.0f, -1.0f), k1 = f2_make(-8.0f, -5.0f), k2 = f2_make(37.0f, 10.0f);
    const f2 s05 = f2_fma(f2_of(P[2 * str]), pm, f2_of(P[-3 * str]));
    const f2 s14 = f2_fma(f2_of(P[str]), pm, f2_of(P[-2 * str]));
    const f2 s23 = f2_fma(f2_of(P[0]), pm, f2_of(P[-str]));
    const f2 t = f2_fma(k2, s23, f2_fma(k1, s14, s05));
    return fmaf(lah, f2_hi(t), f2_lo(t)) * float(1.0 / 30.0);
#else
    const float2 a0 = P[-3 * str], a1 = P[-2 * str], a2 = P[-str], a3 = P[0], a4 = P[str], a5 = P[2 * str];
    const float sf = fmaf(37.0f, a2.x + a3.x, fmaf(-8.0f, a1.x + a4.x, a0.x + a5.x));
    const float sq = fmaf(10.0f, a2.y - a3.y, fmaf(-5.0f, a1.y - a4.y, a0.y - a5.y));
    return fmaf(lah, sq, sf) * float(1.0 / 30.0);
#endif
}

// Pass B of k_stage_hyb for one troubled face w (work-list index): the
// LLF speed again, the face-average eigensystem and the full characteristic
// WENO flux, stored into Fh / Gh.
template <int VER, bool P2, class Cfg>
__device__ __forceinline__ void hyb_troubled_face(int w, const float2* fqx, const float2* fqy, const float4* prim4,
                                               float* Fh, float* Gh, float gam, float eps, float pw, float ash,
                                               float ag1, float ag2)
{
    constexpr int TI = Cfg::TI, TJ = Cfg::TJ, H = Cfg::H, RI = Cfg::RI, RJ = Cfg::RJ;
    constexpr int XPL = RI * TJ, YPL = TI * RJ, FP = HybSmem<Cfg>::FP;
    const bool isx = w < Cfg::NFX;
    int fi, fj;
    if (isx) { fi = w / TJ; fj = w - fi * TJ; }
    else { const int v = w - Cfg::NFX; fi = v / (TJ + 1); fj = v - fi * (TJ + 1); }
    const int cn = isx ? 1 : 2, ct = isx ? 2 : 1;
    const float2* P0 = isx ? fqx + fi * TJ + fj : fqy + fi * RJ + fj;   // stencil point 0
    const int str = isx ? TJ : 1, pl = isx ? XPL : YPL;
    auto pt = [&](int s, float* q, float* f) {
        const float2* P = P0 + s * str;
        const float2 v0 = P[0], vn = P[cn * pl], vt = P[ct * pl], vw = P[3 * pl], ve = P[4 * pl];
        q[0] = v0.y; q[1] = vn.y; q[2] = vt.y; q[3] = vw.y; q[4] = ve.y;
        f[0] = v0.x; f[1] = vn.x; f[2] = vt.x; f[3] = vw.x; f[4] = ve.x;
    };
    // face average (ConstructL.cpp:72-77), normal frame
    float Qa[MEQN];
    {
        float q2[MEQN], q3[MEQN], f2[MEQN], f3[MEQN];
        pt(2, q2, f2);
        pt(3, q3, f3);
#pragma unroll
        for (int m = 0; m < MEQN; m++) Qa[m] = 0.5f * (q3[m] + q2[m]);
    }
    const typename Euler::Eig<float> ev = Euler::eig(gam, Qa);
    const int qb = (H + fi) * RJ + (H + fj), ql = qb - (isx ? RJ : 1);
    const float4 PL = prim4[ql], PR = prim4[qb];
    const float unl = isx ? PL.x : PL.y, unr = isx ? PR.x : PR.y;
    const float ua = 0.5f * (unl + unr), pa = 0.5f * (PL.z + PR.z);
    const float ca = fsqrt(fabsf(gam * pa * rcp(Qa[0])));
    const float s1 = Min(unl - PL.w, ua - ca), s2 = Max(unr + PR.w, ua + ca);
    const float alpha = Max(isx ? ag1 : ag2, Max(fabsf(s1), fabsf(s2)));
    float fh[MEQN];
    if constexpr (P2 || VER == FIN_WENO_FD) weno_char_flux_x2<VER>(ev, ash * alpha, pt, eps, fh);   // f32x2 pairs
    else weno_char_flux<float, VER, P2>(ev, ash * alpha, eps, pw, pt, fh);
    if (isx) {
#pragma unroll
        for (int m = 0; m < MEQN; m++) Fh[m * (TI + 1) * FP + fi * FP + fj] = fh[m];
    } else {
        const float o[MEQN] = {fh[0], fh[2], fh[1], fh[3], fh[4]};
#pragma unroll
        for (int m = 0; m < MEQN; m++) Gh[m * TI * FP + fi * FP + fj] = o[m];
    }
}

// One stage on the cell tile (i0, j0) of the state a describes.  With a.tma
// the tile's copies run on an mbarrier initialised here, so a CTA calls this
// once (k_stage_hyb); a persistent caller that walks several tiles passes
// a.tma = 0 and separates the calls by a barrier.
template <int VER, bool P2, class Cfg>
__device__ __forceinline__ void stage_hyb_tile(const StageArgs& a, const int i0, const int j0)
{
    using R = float;
    using L = HybSmem<Cfg>;
    static_assert(Cfg::MASKS_FIT, "flag row masks are 32-bit words");
    constexpr int TI = Cfg::TI, TJ = Cfg::TJ, NT = Cfg::NT, H = Cfg::H, RI = Cfg::RI, RJ = Cfg::RJ;
    constexpr int XPL = RI * TJ, YPL = TI * RJ, TT = TI * TJ;   // component planes of fqx, fqy, ebuf
    constexpr int FP = L::FP;                                    // face-flux row pitch
    static_assert(TI == 15 && TJ == 16 && NT == 256 && NT >= TT, "one face / cell per thread, rows 8 apart");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float4* prim4 = reinterpret_cast<float4*>(smem_raw + L::PRIM);
    float2* fqx = reinterpret_cast<float2*>(smem_raw + L::FQX);
    float2* fqy = reinterpret_cast<float2*>(smem_raw + L::FQY);
    float* Fh = reinterpret_cast<float*>(smem_raw + L::FH);
    float* Gh = reinterpret_cast<float*>(smem_raw + L::GH);
    double* red = reinterpret_cast<double*>(smem_raw + L::RED);
    unsigned* fxm = reinterpret_cast<unsigned*>(smem_raw + L::MASK);
    unsigned* fym = fxm + Cfg::FXR;
    int* ntrb = reinterpret_cast<int*>(smem_raw + L::NTRB);
    short* tlist = reinterpret_cast<short*>(smem_raw + L::TLIST);
    double* stg = reinterpret_cast<double*>(smem_raw + L::STG);
    double* ebuf = reinterpret_cast<double*>(smem_raw + L::EBUF);   // the other operand's interior
    uint64_t* mbq = reinterpret_cast<uint64_t*>(smem_raw + L::MBAR);

    const int tid = threadIdx.x, lane = tid & 31;
    const int mx = a.mx, my = a.my;
    const float gam = a.gamma_f, eps = a.eps_f, pw = a.pw_f, ash = 0.5f * a.alpha_scaling_f;
    const float ag1 = a.alpha_in ? float(a.alpha_in[0]) : 0.0f;
    const float ag2 = a.alpha_in ? float(a.alpha_in[1]) : 0.0f;
    const double* ext = (a.A && a.A != a.qin) ? a.A : ((a.B && a.B != a.qin) ? a.B : nullptr);
    const bool aligned = ((tc::smem_addr(stg) | (L::SHARE ? 0u : tc::smem_addr(ebuf))) & 127u) == 0;
    if (a.tma && !aligned && tid == 0) atomicOr(a.status, 16u);
    const bool tt = a.tma && aligned && tma_interior<Cfg>(i0, j0, mx, my);
    float smax_x = 0.0f, smax_y = 0.0f, csx = 0.0f, csy = 0.0f;
    bool neg = false, nonfinite = false;
    // ---- phase 0: q_in's tile + halo and the other operand's interior by
    // TMA (or q_in through the boundary remap); the flag masks ----
    if (tt && tid == 0) {
        const CUtensorMap* tmi = a.gtm_in ? a.gtm_in : &a.tm_in;
        const CUtensorMap* tme = a.gtm_A ? a.gtm_A : &a.tm_A;
        if (a.gtm_in) tc::tensormap_acquire(a.gtm_in);
        if (ext && a.gtm_A) tc::tensormap_acquire(a.gtm_A);
        tc::mbar_init(mbq, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        tc::mbar_expect_tx(mbq, uint32_t(Cfg::STG_BYTES + (ext && !L::SHARE ? Cfg::ABUF_BYTES : 0)));
        tc::tma_load_3d(stg, tmi, j0 - 4, i0 - H, 0, mbq);
        if (ext && !L::SHARE) tc::tma_load_3d(ebuf, tme, j0, i0, 0, mbq);
        if (ext && L::SHARE) tc::tma_prefetch_3d(tme, j0, i0, 0);
    }
    {
        const int wx = flag_wx(my), wy = flag_wy(my);
        unsigned fw_lo = 0, fw_hi = 0;
        const int k = (j0 - 1) >> 5;
        const unsigned* row = nullptr;
        int nw = 0;
        if (tid < Cfg::FXR) {
            const int a1 = i0 - 1 + tid;
            if (a1 >= 0 && a1 <= mx) { row = a.flags + size_t(a1) * wx; nw = wx; }
        } else if (tid >= 32 && tid < 32 + Cfg::FYR) {
            const int a1 = i0 - 1 + (tid - 32);
            if (a1 >= 0 && a1 < mx) { row = a.flags + size_t(mx + 1) * wx + size_t(a1) * wy; nw = wy; }
        }
        if (row) {
            if (k >= 0 && k < nw) fw_lo = __ldg(row + k);
            if (k + 1 < nw) fw_hi = __ldg(row + k + 1);
        }
        if (!tt) stage_remap<Cfg>(stg, a.qin, a.plane, i0, j0, mx, my, a.bc, tid);
        if (tid < Cfg::FXR) {
            const unsigned msk = row_bits(fw_lo, fw_hi, j0 - 1) & ((1u << Cfg::FXC) - 1u);
            fxm[tid] = msk | (msk >> 1) | (msk >> 2);
        } else if (tid >= 32 && tid < 32 + Cfg::FYR) {
            const unsigned msk = row_bits(fw_lo, fw_hi, j0 - 1) & ((1u << Cfg::FYC) - 1u);
            fym[tid - 32] = msk | (msk >> 1) | (msk >> 2);
        }
    }
    if (tid == 0) *ntrb = 0;
    __syncthreads();
    if (tt && !tc::mbar_wait(mbq, 0, 1u << 24)) {
        // the copy did not land in time: report it, and give it one more
        // bounded wait before the shared memory is read or released
        atomicOr(a.status, 8u);
        tc::mbar_wait(mbq, 0, 1u << 24);
    }
    {
        // ---- phase 1: per cell of the cross region: narrow to FP32,
        // FluxFunc (FluxFunc.cpp:19-42) halved for the split, primitives.
        // The region is walked as the x-stencil block (all RI rows of the
        // TJ interior columns) and then the 3 + 3 halo columns of the
        // interior rows, so the cell coordinates are shifts and adds ----
        auto cell1 = [&](int ii, int jj, bool xin, bool yin) {
            const double* sp = stg + ii * Cfg::SJ + jj + 1;
            const float rho = float(sp[0]), m1 = float(sp[RI * Cfg::SJ]), m2 = float(sp[2 * RI * Cfg::SJ]),
                        m3 = float(sp[3 * RI * Cfg::SJ]), en = float(sp[4 * RI * Cfg::SJ]);
            const float ir = rcp(rho);
            const float u1 = m1 * ir, u2 = m2 * ir, u3 = m3 * ir;
            const float press = (gam - 1.0f) * (en - 0.5f * rho * (u1 * u1 + u2 * u2 + u3 * u3));
            prim4[ii * RJ + jj] = make_float4(u1, u2, press, fsqrt(fabsf(gam * press * ir)));
            const float hr = 0.5f * rho, hep = 0.5f * (en + press);
            if (yin) {
                float2* d = fqx + ii * TJ + (jj - H);
                d[0] = make_float2(hr * u1, rho);
                d[XPL] = make_float2(hr * u1 * u1 + 0.5f * press, m1);
                d[2 * XPL] = make_float2(hr * u1 * u2, m2);
                d[3 * XPL] = make_float2(hr * u1 * u3, m3);
                d[4 * XPL] = make_float2(u1 * hep, en);
            }
            if (xin) {
                float2* d = fqy + (ii - H) * RJ + jj;
                d[0] = make_float2(hr * u2, rho);
                d[YPL] = make_float2(hr * u2 * u1, m1);
                d[2 * YPL] = make_float2(hr * u2 * u2 + 0.5f * press, m2);
                d[3 * YPL] = make_float2(hr * u2 * u3, m3);
                d[4 * YPL] = make_float2(u2 * hep, en);
            }
        };
        constexpr int NC1 = RI * TJ, NC2 = TI * 2 * H;
        for (int e = tid; e < NC1 + NC2; e += NT) {
            if (e < NC1) {
                const int ii = e / TJ, jj = H + (e - (e / TJ) * TJ);
                cell1(ii, jj, ii >= H && ii < H + TI, true);
            } else {
                const int h = e - NC1, ii = H + h / (2 * H), jh = h - (h / (2 * H)) * (2 * H);
                cell1(ii, jh < H ? jh : jh + TJ, true, false);
            }
        }
        __syncthreads();
        // ---- phase 2, pass A, every face: LLF speed (SetWaveSpd.cpp:39-68,
        // ConstructL.cpp:172-174) with the CFL / status bookkeeping, the
        // dilated flag, the linear flux of smooth faces; troubled faces to
        // the list.  x faces, then y faces, each with compile-time strides ----
        auto face_a = [&](auto isx_c, int fi, int fj) -> bool {
            constexpr bool isx = decltype(isx_c)::value;
            constexpr int str = isx ? TJ : 1, pl = isx ? XPL : YPL;
            const int qb = (H + fi) * RJ + (H + fj), ql = qb - (isx ? RJ : 1);
            const float2* P = isx ? fqx + (fi + 3) * TJ + fj : fqy + fi * RJ + fj + 3;   // stencil point 3
            const float4 PL = prim4[ql], PR = prim4[qb];
            const float unl = isx ? PL.x : PL.y, unr = isx ? PR.x : PR.y;
            const float rho = 0.5f * (P[-str].y + P[0].y);
            const float ua = 0.5f * (unl + unr), pa = 0.5f * (PL.z + PR.z);
            const float ca = fsqrt(fabsf(gam * pa * rcp(rho)));
            if (pa < 0.0f || rho < 0.0f) neg = true;
            const float s1 = Min(unl - PL.w, ua - ca), s2 = Max(unr + PR.w, ua + ca);
            const float alpha = Max(isx ? ag1 : ag2, Max(fabsf(s1), fabsf(s2)));
            if (!(alpha <= 1e30f)) nonfinite = true;
            const unsigned* fm = isx ? fxm : fym;
            const bool trb = (((fm[fi] | fm[fi + 1] | fm[fi + 2]) >> fj) & 1u) != 0;
            if (i0 + fi < mx && j0 + fj < my && alpha <= 1e30f) {
                if (isx) smax_x = Max(smax_x, alpha);
                else smax_y = Max(smax_y, alpha);
            }
            if (!trb) {
                const float lah = ash * alpha;
                float* dst = (isx ? Fh : Gh) + fi * FP + fj;
                constexpr int dplane = isx ? (TI + 1) * FP : TI * FP;
#pragma unroll
                for (int m = 0; m < MEQN; m++) dst[m * dplane] = linear_face2(P + m * pl, str, lah);
            }
            return trb;
        };
        auto append = [&](bool push, int w) {
            const unsigned bal = __ballot_sync(0xffffffffu, push);
            if (bal) {
                int base = 0;
                if (lane == __ffs(bal) - 1) base = atomicAdd(ntrb, __popc(bal));
                base = __shfl_sync(0xffffffffu, base, __ffs(bal) - 1);
                if (push) tlist[base + __popc(bal & ((1u << lane) - 1u))] = short(w);
            }
        };
        // One face per thread, x faces then y faces: a half-warp takes 16
        // faces of one row (it reads one row of the pairs and primitives),
        // the two half-warps of a warp rows 8 apart (the flux stores fall in
        // opposite bank halves); the last warp of y faces takes row 7 and
        // the last column.  The list holds face indices (fi (TJ+1) + fj for
        // y faces after the NFX x faces, fi TJ + fj for x faces).
        {
            const int w = tid, fi = (w >> 5) + ((w >> 1) & 8), fj = w & 15;
            const bool push = face_a(std::true_type{}, fi, fj);
            append(push, fi * TJ + fj);
        }
        {
            const int v = tid, wv = v >> 5, ln = v & 31;
            int fi, fj;
            if (wv < 7) { fi = wv + (ln & 16 ? 8 : 0); fj = ln & 15; }
            else if (ln < 16) { fi = 7; fj = ln; }
            else { fi = ln - 16; fj = TJ; }
            bool push = false;
            if (v < Cfg::NFY) push = face_a(std::false_type{}, fi, fj);
            append(push, Cfg::NFX + fi * (TJ + 1) + fj);
        }
        __syncthreads();
        // ---- phase 2, pass B: full characteristic WENO on the listed faces ----
        {
            const int nt = *ntrb;
            const float agx[2] = {ag1, ag2};
#pragma unroll 1
            for (int k = tid; k < nt; k += NT)
                hyb_troubled_face<VER, P2, Cfg>(tlist[k], fqx, fqy, prim4, Fh, Gh, gam, eps, pw, ash, agx[0], agx[1]);
        }
        __syncthreads();
        // ---- phase 3: flux difference (ConstructL.cpp:396-398), update
        // (UpdateSoln.cpp:29-35), next-stage wave speed (GlobalWaveSpd.cpp:71-76) ----
        {
            // operand selection and constants hoisted out of the cell loop
            const bool hasA = a.A != nullptr, hasB = a.B != nullptr;
            const bool Aq = a.A == a.qin, Bq = a.B == a.qin;
            const double a1 = a.a1, a2 = a.a2, bdt = a.bdt;
            const float rdx = float(a.rdx), rdy = float(a.rdy);
            const size_t plane = a.plane;
            // one cell per thread (NT >= TT), half-warps on cell rows 8
            // apart (warp 7: row 7)
            for (int c = tid; c < TT; c += NT) {
                const int wv = c >> 5, ln = c & 31;
                const int ci = wv < 7 ? wv + (ln & 16 ? 8 : 0) : 7, cj = ln & 15;
                const int gi = i0 + ci, gj = j0 + cj;
                if (gi >= mx || gj >= my) continue;
                const size_t g = size_t(gi) * my + gj;
                const float* fh = Fh + ci * FP + cj;
                const float* gh = Gh + ci * FP + cj;
                const double* si = stg + (H + ci) * Cfg::SJ + H + cj + 1;
                const double* se = ebuf + ci * TJ + cj;
                const double* ge = ext ? ext + g : nullptr;
                double* out = a.qout + g;
                // every operand load ahead of the first store: out may alias
                // them as far as the compiler knows, and loads interleaved
                // with the stores would wait one L2 round trip per component
                double qiv[MEQN], qev[MEQN];
#pragma unroll
                for (int m = 0; m < MEQN; m++) {
                    qiv[m] = L::SHARE ? a.qin[m * plane + g] : si[m * RI * Cfg::SJ];
                    qev[m] = (tt && !L::SHARE) ? se[m * TT] : (ge ? ge[m * plane] : 0.0);
                }
                float qf[MEQN];
#pragma unroll
                for (int m = 0; m < MEQN; m++) {
                    const float f1 = fh[m * (TI + 1) * FP + FP], f0 = fh[m * (TI + 1) * FP];
                    const float g1 = gh[m * TI * FP + 1], g0 = gh[m * TI * FP];
                    const float Lr = -(f1 - f0) * rdx - (g1 - g0) * rdy;
                    const double qi = qiv[m], qe = qev[m];
                    double v = hasA ? a1 * (Aq ? qi : qe) : 0.0;
                    if (hasB) v = v + a2 * (Bq ? qi : qe);
                    v = v + bdt * double(Lr);
                    out[m * plane] = v;
                    qf[m] = float(v);
                }
                if (a.alpha_out) {
                    // GlobalWaveSpd.cpp:71-76 in both directions; with Ql = Qr
                    // max(|u_n - c|, |u_n + c|) is |u_n| + c, and p, c are
                    // the same for both directions
                    const float ir = rcp(qf[0]);
                    const float u1 = qf[1] * ir, u2 = qf[2] * ir, u3 = qf[3] * ir;
                    const float press = (gam - 1.0f) * (qf[4] - 0.5f * qf[0] * (u1 * u1 + u2 * u2 + u3 * u3));
                    const float cc = fsqrt(fabsf(gam * press * ir));
                    const float sx = fabsf(u1) + cc, sy = fabsf(u2) + cc;
                    if (!(sx <= 1e30f) || !(sy <= 1e30f)) nonfinite = true;
                    if (sx <= 1e30f) csx = Max(csx, sx);
                    if (sy <= 1e30f) csy = Max(csy, sy);
                }
            }
        }
    }

    // ---- block reductions of the four maxima (FP32 values, reduced in
    // FP32), one atomic each ----
    float v4[4] = {smax_x, smax_y, csx, csy};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float v = v4[k] <= 1e30f ? v4[k] : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = Max(v, __shfl_xor_sync(0xffffffffu, v, o));
        v4[k] = v;
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) red[(tid >> 5) * 4 + k] = double(v4[k]);
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

// One CTA per tile of the state.
template <int VER, bool P2, class Cfg>
__global__ void __launch_bounds__(Cfg::NT, FIN_HYB_CTAS) k_stage_hyb(const __grid_constant__ StageArgs a)
{
    const int ntj = (a.my + Cfg::TJ - 1) / Cfg::TJ;
    const int t = blockIdx.x;
    stage_hyb_tile<VER, P2, Cfg>(a, (t / ntj) * Cfg::TI, (t % ntj) * Cfg::TJ);
}

}  // namespace fin
