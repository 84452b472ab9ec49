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
//   prim [4][TI+6][TJ+6]  u, v, p, c of the cells
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
#include "fin_tc.cuh"
#include "fin_weno_face.cuh"

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
    float gamma_f, eps_f, pw_f, alpha_scaling_f;   // the same in FP32 (set by the launcher)
    const double* alpha_in;   // [2] global alpha of q_in (x, y); nullptr = local LLF
    double* alpha_out;        // [2] max cell speed of q_out; nullptr = skip
    double* smax_out;         // [2] max face speed over GetCFL's faces; nullptr = skip
    double* face_alpha_x;     // optional per-face alpha, (mx+1)*my, face-major i then j
    double* face_alpha_y;     // optional per-face alpha, mx*(my+1)
    unsigned int* status;     // bit 0: non-finite speed, bit 1: negative p or rho, bit 3: TMA wait ran out,
                              // bit 4: misaligned TMA destination (remap path taken)
    int bc[4];                // xlow, xhigh, ylow, yhigh
    // Lax-Wendroff / multiderivative stages (ConstructLxWL): the split fluxes
    // are the time-integrated F, G (ghosted (mx+6) x (my+6) planes) instead of
    // FluxFunc of q_in (lib/2d/ConstructLxWL.cpp:150-155).
    const double* Fg;
    const double* Gg;
    size_t gplane;
    // Lax-Wendroff with the MPP limiter (FinSolveLxW.cpp:126-151): the stage
    // writes its face fluxes (flux_x [m][mx+1][my], flux_y [m][mx][my+1],
    // ConstructLxWL's Fhat / Ghat) and no update (flux_only), and leaves the
    // first face of each direction out of the face-speed maximum, whose smax
    // entry ConstructLFL.cpp:62-65 overwrites with the global wave speed.
    double* flux_x;
    double* flux_y;
    int flux_only;
    // Hybrid form: troubled-face flags of the step as bit masks (layout of
    // flag_wx / flag_wy below, written by the indicator).  A face takes full
    // WENO when any flag in the 3 x 3 window of same-direction faces around
    // it is set, else the linear FD5 weights (lib/WenoReconstruct.cpp:580-616).
    const unsigned* flags;
    // Hybrid form on grids whose row pitch suits TMA (my even): tensor maps
    // of q_in (box (TJ+8) x (TI+6) x 5, the tile with its halo) and of the
    // stage operand that is not q_in (box TJ x TI x 5); tiles clear of the
    // domain boundary stage both with one TMA transaction each.
    int tma;
    CUtensorMap tm_in;
    CUtensorMap tm_A;
    CUtensorMap tm_qi;   // q_in with the interior-tile box (TJ x TI x 5)
    // The same two maps held in global memory (batches, whose stage
    // arguments live in global memory): used instead of tm_in / tm_A when
    // set, after a tensormap-proxy acquire fence.
    const CUtensorMap* gtm_in;
    const CUtensorMap* gtm_A;
};

// Troubled-face flags, one bit per face: x faces (rows 0 .. mx) take
// flag_wx words per row, bit b of word k being column 32 k + b; the y faces
// (rows 0 .. mx-1, columns 0 .. my) follow with flag_wy words per row.
__host__ __device__ __forceinline__ int flag_wx(int my) { return (my + 31) >> 5; }
__host__ __device__ __forceinline__ int flag_wy(int my) { return (my + 32) >> 5; }
__host__ __device__ __forceinline__ size_t flag_words(int mx, int my)
{
    return size_t(mx + 1) * flag_wx(my) + size_t(mx) * flag_wy(my);
}
// Bits of columns b0 .. b0+31 of one mask row from the words holding them
// (k = b0 >> 5 and k + 1; columns outside the row read as 0).
__device__ __forceinline__ unsigned row_bits(unsigned lo, unsigned hi, int b0)
{
    return unsigned(((unsigned long long)hi << 32 | lo) >> (b0 & 31));
}

template <int TI_, int TJ_, int NT_>
struct TileCfg {
    static constexpr int TI = TI_, TJ = TJ_, NT = NT_, H = 3;
    static constexpr int RI = TI + 2 * H, RJ = TJ + 2 * H;
    static constexpr int NFX = (TI + 1) * TJ, NFY = TI * (TJ + 1);
    static constexpr int NPRIM = 4;   // per-cell u, v, p, c of the cross region
    // FP32 faces of a 15 x 16 tile go to threads so that the two half-warps
    // of a warp take face rows 8 apart (XROW8): 8 rows of RJ = 22 words are
    // 176 words, 16 modulo 32, so the two rows' words fall in opposite
    // halves of the banks; the x-direction flux rows get a pitch of 18 for
    // the same reason (8 x 18 = 144).  FP64 (a half-warp reads one row of
    // 8-byte words) keeps the row-by-row order.
    template <class R>
    __host__ __device__ static constexpr bool XROW8() { return sizeof(R) == 4 && TI == 15 && TJ == 16; }
    template <class R>
    __host__ __device__ static constexpr int FSJ() { return XROW8<R>() ? TJ + 2 : TJ; }
    // byte offset of the reduction scratch (after the arrays, 16-B aligned)
    template <class R>
    __host__ __device__ static constexpr size_t red_offset()
    {
        return (sizeof(R) * (size_t(MEQN) * (size_t(RI) * RJ + size_t(RI) * FSJ<R>() + size_t(TI) * RJ +
                                             size_t(TI + 1) * TJ + size_t(TI) * (TJ + 1)) +
                             size_t(NPRIM) * RI * RJ) + 15) / 16 * 16;
    }
    template <class R>
    __host__ __device__ static constexpr size_t smem_bytes() { return red_offset<R>() + 4 * (NT / 32) * sizeof(double); }
    // Hybrid form (k_stage_hyb): the flag windows of the 3 x 3 dilation as
    // one bit mask per face row (x faces: rows i0-1 .. i0+TI+1, bit c =
    // column j0-1+c, c < TJ+2; y faces: rows i0-1 .. i0+TI, c < TJ+3).
    static constexpr int FXR = TI + 3, FXC = TJ + 2, FYR = TI + 2, FYC = TJ + 3;
    static constexpr bool MASKS_FIT = FYC <= 32;   // flag row masks are 32-bit words
    // The FP64 staging tile of q_in (rows i0-3 .. i0+TI+2, columns j0-4 ..
    // j0+TJ+3, so the TMA box starts on a 16-byte boundary) and the interior
    // tile of a stage operand; a TMA destination starts on a 128-byte
    // boundary, so buffers are padded to multiples of 128 bytes.
    static constexpr int SJ = TJ + 8;
    static constexpr size_t STG_BYTES = size_t(MEQN) * RI * SJ * 8;
    static constexpr size_t ABUF_BYTES = size_t(MEQN) * TI * TJ * 8;
    __host__ __device__ static constexpr size_t pad128(size_t b) { return (b + 127) / 128 * 128; }
};

// Staging of q_in's tile + 3-cell halo (the cross region: rows i0-3 ..
// i0+TI+2 at columns j0 .. j0+TJ-1, columns j0-3 .. j0+TJ+2 at rows i0 ..
// i0+TI-1) as FP64 in stg [M][RI][SJ], column jj of the tile frame at jj+1.
// A tile whose box (rows i0-3 .. i0+TI+2, columns j0-4 .. j0+TJ+3) lies in
// the domain is staged by one TMA copy; any other by loads through the
// boundary remap.
template <class Cfg>
__device__ __forceinline__ bool tma_interior(int i0, int j0, int mx, int my)
{
    return i0 >= Cfg::H && i0 + Cfg::TI + Cfg::H <= mx && j0 >= 4 && j0 + Cfg::TJ + 4 <= my;
}

template <class Cfg>
__device__ __forceinline__ void stage_remap(double* stg, const double* q, size_t plane, int i0, int j0, int mx, int my,
                                            const int* bc, int tid)
{
    constexpr int H = Cfg::H, TI = Cfg::TI, TJ = Cfg::TJ, RI = Cfg::RI, RJ = Cfg::RJ;
    for (int e = tid; e < RI * RJ; e += Cfg::NT) {
        const int ii = e / RJ, jj = e - ii * RJ;
        const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
        if (!xin && !yin) continue;
        const int gi = bc_remap(i0 + ii - H, mx, bc[0], bc[1]);
        const int gj = bc_remap(j0 + jj - H, my, bc[2], bc[3]);
        const size_t g = size_t(gi) * my + gj;
#pragma unroll
        for (int m = 0; m < MEQN; m++) stg[(m * RI + ii) * Cfg::SJ + jj + 1] = __ldg(q + m * plane + g);
    }
}

template <class Cfg, class R>
__device__ __forceinline__ void stage_convert(const double* stg, R* qs, int tid)
{
    constexpr int H = Cfg::H, TI = Cfg::TI, TJ = Cfg::TJ, RI = Cfg::RI, RJ = Cfg::RJ;
    for (int e = tid; e < RI * RJ; e += Cfg::NT) {
        const int ii = e / RJ, jj = e - ii * RJ;
        const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
        if (!xin && !yin) continue;
#pragma unroll
        for (int m = 0; m < MEQN; m++) qs[m * RI * RJ + e] = R(stg[(m * RI + ii) * Cfg::SJ + jj + 1]);
    }
}

// 6-point flux of a face that takes the linear FD5 weights: with v+- =
// 0.5 f +- l q, the reference's characteristic form R FD5(L v+) + R FD5'(L v-)
// (ConstructL.cpp:179-250 with WenoReconstruct_FD5, WenoReconstruct.cpp:
// 580-616) equals FD5(v+) + FD5'(v-) component by component, because the
// reconstruction is linear and R L = I.  FD5 has the weights (2, -13, 47, 27,
// -3)/60 on points 0..4 and FD5' the same on points 5..1, so the face flux is
//   (1/30) [ (f0+f5) - 8 (f1+f4) + 37 (f2+f3)                      (0.5 f terms)
//          + l ((q0-q5) - 5 (q1-q4) + 10 (q2-q3)) ]                  (l = lah)
// with f the half fluxes held in shared memory: 12 operations per component
// instead of a projection, two reconstructions and a back projection.
template <class R>
__device__ __forceinline__ R linear_face(const R* f, int fstr, const R* q, int qstr, R lah)
{
    const R sf = fma(R(37), f[-1 * fstr] + f[0], fma(R(-8), f[-2 * fstr] + f[fstr], f[-3 * fstr] + f[2 * fstr]));
    const R sq = fma(R(10), q[-1 * qstr] - q[0], fma(R(-5), q[-2 * qstr] - q[qstr], q[-3 * qstr] - q[2 * qstr]));
    return fma(lah, sq, sf) * R(1.0 / 30.0);
}

// Resident blocks per SM the register budget is sized for: FP64 faces need
// about 110 registers a thread, FP32 about 70.
// Measured on B200 at 4096^2 (stage-kernel ms, FP64 / FP32): one block per
// SM 5.81 / 2.71; two FP64 blocks (128 registers, ~200 B spilled to L1) and
// three FP32 blocks 4.07 / 2.44.  More resident warps beat the spills, up to
// a point: four FP32 blocks (64 registers, 236 B spilled) took 2.14 ms where
// three took 2.06 (the current kernel).
#ifndef FIN_MINB_F64
#define FIN_MINB_F64 2
#endif
#ifndef FIN_MINB_F32
#define FIN_MINB_F32 3
#endif
template <class R> struct MinBlocks { static constexpr int value = FIN_MINB_F64; };
// FP64 face body: fields 0, 4 and 1 in one sweep of the stencil (1: one
// load and split of each stencil point instead of two; measured 4 % faster
// on B200 at 4096^2) or the three passes of the register-lean form (0).
#ifndef FIN_F64_MERGE
#define FIN_F64_MERGE 1
#endif
template <> struct MinBlocks<float> { static constexpr int value = FIN_MINB_F32; };

// Scalar parameters read from kernel-parameter space where they are used
// (keeps them out of the register budget of the face loop).
template <class R> struct Par;
template <> struct Par<double> {
    __device__ static double gamma(const StageArgs& a) { return a.gamma; }
    __device__ static double eps(const StageArgs& a) { return a.eps; }
    __device__ static double pw(const StageArgs& a) { return a.pw; }
    __device__ static double ascale(const StageArgs& a) { return a.alpha_scaling; }
};
template <> struct Par<float> {
    __device__ static float gamma(const StageArgs& a) { return a.gamma_f; }
    __device__ static float eps(const StageArgs& a) { return a.eps_f; }
    __device__ static float pw(const StageArgs& a) { return a.pw_f; }
    __device__ static float ascale(const StageArgs& a) { return a.alpha_scaling_f; }
};

// Scheduling fences: an empty volatile asm that reads and writes x.  Volatile
// asm statements keep their order, so fencing the inputs and result of each
// pair of WENO reconstructions stops the scheduler from evaluating all ten of
// a face at once (which wants ~230 registers in FP64).
__device__ __forceinline__ void fence(double& x) { asm volatile("" : "+d"(x)); }
__device__ __forceinline__ void fence(float& x) { asm volatile("" : "+f"(x)); }
template <class R>
__device__ __forceinline__ void fence5(R* u)
{
#pragma unroll
    for (int k = 0; k < 5; k++) fence(u[k]);
}

// gp and gm reconstructions of one characteristic field, fenced as a unit.
template <class R, int VER, bool P2>
__device__ __forceinline__ R weno_pair(R* up, R* um, R eps, R pw)
{
    fence5(up);
    fence5(um);
    R g;
    if constexpr (sizeof(R) == 4 && (P2 || VER == FIN_WENO_FD)) g = weno5_pair_x2<VER>(up, um, eps);   // f32x2 pairs
    else g = weno5<R, VER, P2>(up, eps, pw) + weno5<R, VER, P2>(um, eps, pw);
    fence(g);
    return g;
}

// Right projection (ProjectRightEig.cpp:46-62) of one characteristic field k
// with amplitude gk, added into the face flux f[0..4] (normal frame).  The
// projection is linear, so the face flux is accumulated field by field.
template <class R>
__device__ __forceinline__ void right_add(const typename Euler::Eig<R>& e, int k, R gk, R* f)
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

// One tile (rows i0 .., columns j0 ..) of a stage; the whole CTA takes part.
template <class R, int VER, bool P2, class Cfg, bool FG = false>
__device__ __forceinline__ void stage_tile(const StageArgs& a, const int i0, const int j0)
{
    constexpr int TI = Cfg::TI, TJ = Cfg::TJ, NT = Cfg::NT, H = Cfg::H;
    constexpr int RI = Cfg::RI, RJ = Cfg::RJ;
    constexpr int PQ = RI * RJ;                    // plane size of qs and prim
    extern __shared__ __align__(128) unsigned char smem_raw[];
    R* prim = reinterpret_cast<R*>(smem_raw);      // [4][RI][RJ]   u, v, p, c
    R* qs = prim + Cfg::NPRIM * PQ;                // [M][RI][RJ]
    constexpr int FS = Cfg::template FSJ<R>();
    R* fs = qs + MEQN * PQ;                        // [M][RI][FS]   0.5 * f
    R* gs = fs + MEQN * RI * FS;                   // [M][TI][RJ]   0.5 * g
    R* Fh = gs + MEQN * TI * RJ;                   // [M][TI+1][TJ]
    R* Gh = Fh + MEQN * (TI + 1) * TJ;             // [M][TI][TJ+1]
    double* red = reinterpret_cast<double*>(smem_raw + Cfg::template red_offset<R>());

    const int tid = threadIdx.x;
    const int mx = a.mx, my = a.my;
#define gamma (Par<R>::gamma(a))

    // ---- phase 0: load the tile + halo, boundary conditions by remap ----
    // FP64: all of a thread's loads are issued before its stores (one memory
    // round trip per tile, not one per pass over the region; 1-3 % faster at
    // 2 CTAs per SM).  FP32 (3 CTAs per SM, whose register budget it tightens)
    // keeps one pass at a time.
    if constexpr (sizeof(R) == 4) {
        for (int e = tid; e < PQ; e += NT) {
            const int ii = e / RJ, jj = e - ii * RJ;
            const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
            if (!xin && !yin) continue;
            const int gi = bc_remap(i0 + ii - H, mx, a.bc[0], a.bc[1]);
            const int gj = bc_remap(j0 + jj - H, my, a.bc[2], a.bc[3]);
            const size_t g = size_t(gi) * my + gj;
#pragma unroll
            for (int m = 0; m < MEQN; m++) qs[m * PQ + e] = R(__ldg(a.qin + m * a.plane + g));
        }
        __syncthreads();
    } else {
        constexpr int NIT = (PQ + NT - 1) / NT;
        double v[NIT][MEQN];
#pragma unroll
        for (int it = 0; it < NIT; it++) {
            const int e = tid + it * NT;
            const int ii = e / RJ, jj = e - ii * RJ;
            const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
            if (e < PQ && (xin || yin)) {
                const int gi = bc_remap(i0 + ii - H, mx, a.bc[0], a.bc[1]);
                const int gj = bc_remap(j0 + jj - H, my, a.bc[2], a.bc[3]);
                const size_t g = size_t(gi) * my + gj;
#pragma unroll
                for (int m = 0; m < MEQN; m++) v[it][m] = __ldg(a.qin + m * a.plane + g);
            }
        }
#pragma unroll
        for (int it = 0; it < NIT; it++) {
            const int e = tid + it * NT;
            const int ii = e / RJ, jj = e - ii * RJ;
            const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
            if (e < PQ && (xin || yin)) {
#pragma unroll
                for (int m = 0; m < MEQN; m++) qs[m * PQ + e] = R(v[it][m]);
            }
        }
        __syncthreads();
    }

    // ---- phase 1: per cell of the cross region: FluxFunc (FluxFunc.cpp:19-42,
    // once per cell instead of once per stencil point of every face), halved
    // for the LLF split, and the cell's u, v, p, c for SetWaveSpd.cpp:24-50 ----
    for (int e = tid; e < PQ; e += NT) {
        const int ii = e / RJ, jj = e - ii * RJ;
        const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
        if (!xin && !yin) continue;
        R rho, m1, m2, m3, en;
        {
            rho = qs[e]; m1 = qs[PQ + e]; m2 = qs[2 * PQ + e]; m3 = qs[3 * PQ + e]; en = qs[4 * PQ + e];
        }
        const R ir = rcp(rho);
        const R u1 = m1 * ir, u2 = m2 * ir, u3 = m3 * ir;
        const R press = (gamma - R(1)) * (en - R(0.5) * rho * (u1 * u1 + u2 * u2 + u3 * u3));
        {
            prim[e] = u1;
            prim[PQ + e] = u2;
            prim[2 * PQ + e] = press;
            prim[3 * PQ + e] = fsqrt(fabs(gamma * press * ir));
        }
        if (FG) {
            // 0.5 * F, 0.5 * G of the integrated-flux kernel, unremapped: it
            // covers the 3-cell ghost frame; cells of a partial tile beyond it
            // only feed discarded faces, so their index is clamped.
            int ci = i0 + ii - H, cj = j0 + jj - H;
            ci = ci < -3 ? -3 : (ci > mx + 2 ? mx + 2 : ci);
            cj = cj < -3 ? -3 : (cj > my + 2 ? my + 2 : cj);
            const size_t o = size_t(ci + 3) * (my + 6) + (cj + 3);
            if (yin) {
                const int d = ii * FS + (jj - H);
#pragma unroll
                for (int m = 0; m < MEQN; m++) fs[m * RI * FS + d] = R(0.5 * __ldg(a.Fg + m * a.gplane + o));
            }
            if (xin) {
                const int d = (ii - H) * RJ + jj;
#pragma unroll
                for (int m = 0; m < MEQN; m++) gs[m * TI * RJ + d] = R(0.5 * __ldg(a.Gg + m * a.gplane + o));
            }
            continue;
        }
        const R hr = R(0.5) * rho, hep = R(0.5) * (en + press);
        if (yin) {
            const int o = ii * FS + (jj - H);
            fs[o] = hr * u1;
            fs[RI * FS + o] = hr * u1 * u1 + R(0.5) * press;
            fs[2 * RI * FS + o] = hr * u1 * u2;
            fs[3 * RI * FS + o] = hr * u1 * u3;
            fs[4 * RI * FS + o] = u1 * hep;
        }
        if (xin) {
            const int o = (ii - H) * RJ + jj;
            gs[o] = hr * u2;
            gs[TI * RJ + o] = hr * u2 * u1;
            gs[2 * TI * RJ + o] = hr * u2 * u2 + R(0.5) * press;
            gs[3 * TI * RJ + o] = hr * u2 * u3;
            gs[4 * TI * RJ + o] = u2 * hep;
        }
    }
    __syncthreads();

    // ---- phase 2: one thread per face (x faces then y faces) ----
#define eps (Par<R>::eps(a))
#define pw (Par<R>::pw(a))
    const R ag1 = a.alpha_in ? R(a.alpha_in[0]) : R(0);
    const R ag2 = a.alpha_in ? R(a.alpha_in[1]) : R(0);
    R smax_x = R(0), smax_y = R(0);
    bool neg = false, nonfinite = false;
    const int nwork = Cfg::NFX + Cfg::NFY;
#pragma unroll 1
    for (int k = tid; k < nwork; k += NT) {
        const int w = k;
        const bool isx = w < Cfg::NFX;
        int fi, fj, qbase, qstr, fbase, fstr, fplane;
        const R* fl;
        if (isx) {
            // face between rows fi-1, fi of the tile
            if constexpr (Cfg::template XROW8<R>()) {
                fi = (w >> 5) + ((w >> 1) & 8); fj = w & 15;   // half-warps on rows r and r + 8
            } else {
                fi = w / TJ; fj = w - fi * TJ;
            }
            qbase = (H + fi) * RJ + (H + fj); qstr = RJ;
            fl = fs; fbase = (H + fi) * FS + fj; fstr = FS; fplane = RI * FS;
        } else {
            // face between cols fj-1, fj; taken by rows of TJ, then the last
            // column, so a half-warp reads one row of the staged tile (FP32:
            // half-warps on rows r and r + 8; the last warp takes row 7 and
            // the last column)
            const int v = w - Cfg::NFX;
            if constexpr (Cfg::template XROW8<R>()) {
                const int wv = v >> 5, ln = v & 31;
                if (wv < 7) { fi = wv + (ln & 16 ? 8 : 0); fj = ln & 15; }
                else if (ln < 16) { fi = 7; fj = ln; }
                else { fi = ln - 16; fj = TJ; }
            } else {
                fi = v < TI * TJ ? v / TJ : v - TI * TJ;
                fj = v < TI * TJ ? v - fi * TJ : TJ;
            }
            qbase = (H + fi) * RJ + (H + fj); qstr = 1;
            fl = gs; fbase = fi * RJ + (H + fj); fstr = 1; fplane = TI * RJ;
        }
        const int cn = isx ? 1 : 2, ct = isx ? 2 : 1;   // normal / tangential momentum
        const int ql = qbase - qstr;
        // Face average (ConstructL.cpp:72-77) in the normal frame.
        R Qa[MEQN];
        Qa[0] = R(0.5) * (qs[qbase] + qs[ql]);
        Qa[1] = R(0.5) * (qs[cn * PQ + qbase] + qs[cn * PQ + ql]);
        Qa[2] = R(0.5) * (qs[ct * PQ + qbase] + qs[ct * PQ + ql]);
        Qa[3] = R(0.5) * (qs[3 * PQ + qbase] + qs[3 * PQ + ql]);
        Qa[4] = R(0.5) * (qs[4 * PQ + qbase] + qs[4 * PQ + ql]);
        const typename Euler::Eig<R> ev = Euler::eig(gamma, Qa);
        // SetWaveSpd.cpp:39-68 from the two cells' u_n, p, c (nmag = 1) and
        // the LLF alpha of ConstructL.cpp:172-174.
        R alpha;
        {
            const int un = isx ? 0 : 1;
            R unl, unr, pl, pr, cl, cr;
            {
                unl = prim[un * PQ + ql]; unr = prim[un * PQ + qbase];
                pl = prim[2 * PQ + ql]; pr = prim[2 * PQ + qbase];
                cl = prim[3 * PQ + ql]; cr = prim[3 * PQ + qbase];
            }
            const R rho = Qa[0];
            const R ua = R(0.5) * (unl + unr);
            const R pa = R(0.5) * (pl + pr);
            const R ca = fsqrt(fabs(gamma * pa * rcp(rho)));
            if (pa < R(0) || rho < R(0)) neg = true;
            const R s1 = Min(unl - cl, ua - ca);
            const R s2 = Max(unr + cr, ua + ca);
            alpha = Max(isx ? ag1 : ag2, Max(fabs(s1), fabs(s2)));
        }
        if (!(alpha <= R(1e30))) nonfinite = true;
        // gp = 0.5 (L f + l_alpha L q) = L (0.5 f + 0.5 l_alpha q), points
        // 0..4; gm the same with -l_alpha, points 5..1 (ConstructL.cpp:179-185).
        const R lah = R(0.5) * Par<R>::ascale(a) * alpha;
        const typename Euler::Rows<R> rw = Euler::rows(ev);
        R fh[MEQN] = {R(0), R(0), R(0), R(0), R(0)};
        if constexpr (sizeof(R) == 4 && (P2 || VER == FIN_WENO_FD)) {
            // FP32: the split pairs and the paired reconstructions of
            // weno_char_flux_x2 (f32x2), the same passes over the fields
            auto pt = [&](int s, float* q, float* f) {
                const int oq = qbase + (s - 3) * qstr, of = fbase + (s - 3) * fstr;
                q[0] = qs[oq]; q[1] = qs[cn * PQ + oq]; q[2] = qs[ct * PQ + oq]; q[3] = qs[3 * PQ + oq];
                q[4] = qs[4 * PQ + oq];
                f[0] = fl[of]; f[1] = fl[cn * fplane + of]; f[2] = fl[ct * fplane + of]; f[3] = fl[3 * fplane + of];
                f[4] = fl[4 * fplane + of];
            };
            weno_char_flux_x2<VER>(ev, lah, pt, eps, fh);
        } else if (FIN_F64_MERGE && sizeof(R) == 8) {
            // fields 0, 4 and 1 in one sweep of the stencil (left014 shares
            // the acoustic rows' tail), then fields 2 and 3; the right
            // projections are added in the same order as the three passes below
            R p0[5], p4[5], m0[5], m4[5], p1[5], m1[5];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                asm volatile("" ::: "memory");
                const int oq = qbase + (s - 3) * qstr, of = fbase + (s - 3) * fstr;
                const R q0 = qs[oq], qn = qs[cn * PQ + oq], qt = qs[ct * PQ + oq], qw = qs[3 * PQ + oq], qe = qs[4 * PQ + oq];
                const R f0 = fl[of], fn = fl[cn * fplane + of], ft = fl[ct * fplane + of], fw = fl[3 * fplane + of],
                        fe = fl[4 * fplane + of];
                if (s < 5) {
                    const R v[MEQN] = {f0 + lah * q0, fn + lah * qn, ft + lah * qt, fw + lah * qw, fe + lah * qe};
                    Euler::left014(ev, rw, v, p0[s], p1[s], p4[s]);
                }
                if (s > 0) {
                    const R v[MEQN] = {f0 - lah * q0, fn - lah * qn, ft - lah * qt, fw - lah * qw, fe - lah * qe};
                    Euler::left014(ev, rw, v, m0[5 - s], m1[5 - s], m4[5 - s]);
                }
            }
#pragma unroll 1
            for (int k = 0; k < 3; k++) {
                R up[5], um[5];
#pragma unroll
                for (int t = 0; t < 5; t++) {
                    up[t] = k == 0 ? p0[t] : (k == 1 ? p4[t] : p1[t]);
                    um[t] = k == 0 ? m0[t] : (k == 1 ? m4[t] : m1[t]);
                }
                right_add<R>(ev, k == 0 ? 0 : (k == 1 ? 4 : 1), weno_pair<R, VER, P2>(up, um, eps, pw), fh);
            }
            {
                // fields 2 and 3 (rows v_t - u2 v0 and v_w - u3 v0)
                R p2[5], p3[5], m2[5], m3[5];
#pragma unroll
                for (int s = 0; s < 6; s++) {
                    asm volatile("" ::: "memory");
                    const int oq = qbase + (s - 3) * qstr, of = fbase + (s - 3) * fstr;
                    const R q0 = qs[oq], qt = qs[ct * PQ + oq], qw = qs[3 * PQ + oq];
                    const R f0 = fl[of], ft = fl[ct * fplane + of], fw = fl[3 * fplane + of];
                    if (s < 5) {
                        const R v0 = f0 + lah * q0;
                        p2[s] = (ft + lah * qt) - ev.u2 * v0;
                        p3[s] = (fw + lah * qw) - ev.u3 * v0;
                    }
                    if (s > 0) {
                        const R v0 = f0 - lah * q0;
                        m2[5 - s] = (ft - lah * qt) - ev.u2 * v0;
                        m3[5 - s] = (fw - lah * qw) - ev.u3 * v0;
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
                    right_add<R>(ev, k == 0 ? 2 : 3, weno_pair<R, VER, P2>(up, um, eps, pw), fh);
                }
            }
        } else {
        {
            // pass 1: characteristic fields 0 and 4 (acoustic rows, shared tail)
            R p0[5], p4[5], m0[5], m4[5];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                // keep the compiler from hoisting every stencil point's loads
                // ahead of the arithmetic (that would hold ~60 values live)
                asm volatile("" ::: "memory");
                const int oq = qbase + (s - 3) * qstr, of = fbase + (s - 3) * fstr;
                const R q0 = qs[oq], qn = qs[cn * PQ + oq], qt = qs[ct * PQ + oq], qw = qs[3 * PQ + oq], qe = qs[4 * PQ + oq];
                const R f0 = fl[of], fn = fl[cn * fplane + of], ft = fl[ct * fplane + of], fw = fl[3 * fplane + of],
                        fe = fl[4 * fplane + of];
                if (s < 5) {
                    const R v[MEQN] = {f0 + lah * q0, fn + lah * qn, ft + lah * qt, fw + lah * qw, fe + lah * qe};
                    Euler::left04(ev, rw, v, p0[s], p4[s]);
                }
                if (s > 0) {
                    const R v[MEQN] = {f0 - lah * q0, fn - lah * qn, ft - lah * qt, fw - lah * qw, fe - lah * qe};
                    Euler::left04(ev, rw, v, m0[5 - s], m4[5 - s]);
                }
            }
            // one reconstruction pair per iteration; the loop is not unrolled,
            // which keeps the scheduler from overlapping the two pairs
#pragma unroll 1
            for (int k = 0; k < 2; k++) {
                R up[5], um[5];
#pragma unroll
                for (int t = 0; t < 5; t++) {
                    up[t] = k == 0 ? p0[t] : p4[t];
                    um[t] = k == 0 ? m0[t] : m4[t];
                }
                right_add<R>(ev, k == 0 ? 0 : 4, weno_pair<R, VER, P2>(up, um, eps, pw), fh);
            }
        }
        {
            // pass 2: characteristic field 1 (the entropy-like row)
            R p1[5], m1[5];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                // keep the compiler from hoisting every stencil point's loads
                // ahead of the arithmetic (that would hold ~60 values live)
                asm volatile("" ::: "memory");
                const int oq = qbase + (s - 3) * qstr, of = fbase + (s - 3) * fstr;
                const R q0 = qs[oq], qn = qs[cn * PQ + oq], qt = qs[ct * PQ + oq], qw = qs[3 * PQ + oq], qe = qs[4 * PQ + oq];
                const R f0 = fl[of], fn = fl[cn * fplane + of], ft = fl[ct * fplane + of], fw = fl[3 * fplane + of],
                        fe = fl[4 * fplane + of];
                if (s < 5) {
                    const R v[MEQN] = {f0 + lah * q0, fn + lah * qn, ft + lah * qt, fw + lah * qw, fe + lah * qe};
                    p1[s] = Euler::left1(ev, rw, v);
                }
                if (s > 0) {
                    const R v[MEQN] = {f0 - lah * q0, fn - lah * qn, ft - lah * qt, fw - lah * qw, fe - lah * qe};
                    m1[5 - s] = Euler::left1(ev, rw, v);
                }
            }
            right_add<R>(ev, 1, weno_pair<R, VER, P2>(p1, m1, eps, pw), fh);
        }
        {
            // pass 3: fields 2 and 3 (rows v_t - u2 v0 and v_w - u3 v0)
            R p2[5], p3[5], m2[5], m3[5];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                // keep the compiler from hoisting every stencil point's loads
                // ahead of the arithmetic (that would hold ~60 values live)
                asm volatile("" ::: "memory");
                const int oq = qbase + (s - 3) * qstr, of = fbase + (s - 3) * fstr;
                const R q0 = qs[oq], qt = qs[ct * PQ + oq], qw = qs[3 * PQ + oq];
                const R f0 = fl[of], ft = fl[ct * fplane + of], fw = fl[3 * fplane + of];
                if (s < 5) {
                    const R v0 = f0 + lah * q0;
                    p2[s] = (ft + lah * qt) - ev.u2 * v0;
                    p3[s] = (fw + lah * qw) - ev.u3 * v0;
                }
                if (s > 0) {
                    const R v0 = f0 - lah * q0;
                    m2[5 - s] = (ft - lah * qt) - ev.u2 * v0;
                    m3[5 - s] = (fw - lah * qw) - ev.u3 * v0;
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
                right_add<R>(ev, k == 0 ? 2 : 3, weno_pair<R, VER, P2>(up, um, eps, pw), fh);
            }
        }
        }
        // Back to (rho, rho u, rho v, rho w, E) and store.
        if (isx) {
            const R o[MEQN] = {fh[0], fh[1], fh[2], fh[3], fh[4]};
#pragma unroll
            for (int m = 0; m < MEQN; m++) Fh[m * (TI + 1) * TJ + fi * TJ + fj] = o[m];
            const int gfi = i0 + fi, gj = j0 + fj;
            if (FG && a.flux_x && gfi <= mx && gj < my) {
#pragma unroll
                for (int m = 0; m < MEQN; m++) a.flux_x[(size_t(m) * (mx + 1) + gfi) * my + gj] = double(o[m]);
            }
            // GetCFL's Max skips NaN entries (Max(NaN, c) = c), so only
            // finite face speeds enter the CFL maximum.
            if (gfi < mx && gj < my && alpha <= R(1e30) && !(FG && a.flux_only && gfi == 0 && gj == 0))
                smax_x = Max(smax_x, alpha);
            if (a.face_alpha_x && gfi <= mx && gj < my) a.face_alpha_x[size_t(gfi) * my + gj] = double(alpha);
        } else {
            const R o[MEQN] = {fh[0], fh[2], fh[1], fh[3], fh[4]};
#pragma unroll
            for (int m = 0; m < MEQN; m++) Gh[m * TI * (TJ + 1) + fi * (TJ + 1) + fj] = o[m];
            const int gi = i0 + fi, gfj = j0 + fj;
            if (FG && a.flux_y && gi < mx && gfj <= my) {
#pragma unroll
                for (int m = 0; m < MEQN; m++) a.flux_y[(size_t(m) * mx + gi) * (my + 1) + gfj] = double(o[m]);
            }
            if (gi < mx && gfj < my && alpha <= R(1e30) && !(FG && a.flux_only && gi == 0 && gfj == 0))
                smax_y = Max(smax_y, alpha);
            if (a.face_alpha_y && gi < mx && gfj <= my) a.face_alpha_y[size_t(gi) * (my + 1) + gfj] = double(alpha);
        }
    }
    __syncthreads();
#undef gamma
#undef eps
#undef pw

    // ---- phase 3: flux difference, stage update, next-stage wave speed ----
    double cs_x = 0.0, cs_y = 0.0;
    const double gam = a.gamma;
    for (int c = tid; c < ((FG && a.flux_only) ? 0 : TI * TJ); c += NT) {
        const int ci = c / TJ, cj = c - ci * TJ;
        const int gi = i0 + ci, gj = j0 + cj;
        if (gi >= mx || gj >= my) continue;
        const size_t g = size_t(gi) * my + gj;
        // every operand load ahead of the first store: qout may alias A or
        // B as far as the compiler knows, so loads interleaved with the
        // stores would wait one memory round trip per component
        double va[MEQN], vb[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            va[m] = a.A ? a.A[m * a.plane + g] : 0.0;
            vb[m] = a.B ? a.B[m * a.plane + g] : 0.0;
        }
        double qn[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            // ConstructL.cpp:396-398
            // (the FP32 forms difference their FP32 fluxes in FP32 and widen
            // the result once)
            const R f1 = Fh[m * (TI + 1) * TJ + (ci + 1) * TJ + cj], f0 = Fh[m * (TI + 1) * TJ + ci * TJ + cj];
            const R g1 = Gh[m * TI * (TJ + 1) + ci * (TJ + 1) + cj + 1], g0 = Gh[m * TI * (TJ + 1) + ci * (TJ + 1) + cj];
            R Lr = -(f1 - f0) * R(a.rdx);
            Lr = Lr - (g1 - g0) * R(a.rdy);
            const double L = double(Lr);
            double v = 0.0;
            {
                if (a.A) v = a.a1 * va[m];
                if (a.B) v = v + a.a2 * vb[m];
            }
            v = v + a.bdt * L;
            qn[m] = v;
            a.qout[m * a.plane + g] = v;
        }
        if (a.alpha_out) {
            // GlobalWaveSpd.cpp:71-76 on the new state, both directions.
            // The FP32 forms use it only as the FP32 LLF speed of the next
            // stage, so they evaluate it in FP32.
            const R qx[MEQN] = {R(qn[0]), R(qn[1]), R(qn[2]), R(qn[3]), R(qn[4])};
            const R qy[MEQN] = {qx[0], qx[2], qx[1], qx[3], qx[4]};
            const double sx = double(Euler::cell_speed(Euler::cell(R(gam), qx)));
            const double sy = double(Euler::cell_speed(Euler::cell(R(gam), qy)));
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

template <class R, int VER, bool P2, class Cfg, bool FG = false>
__global__ void __launch_bounds__(Cfg::NT, MinBlocks<R>::value) k_stage(const __grid_constant__ StageArgs a)
{
    stage_tile<R, VER, P2, Cfg, FG>(a, blockIdx.y * Cfg::TI, blockIdx.x * Cfg::TJ);
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
