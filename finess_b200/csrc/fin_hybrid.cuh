// The hybrid form's per-step troubled-face indicator: features -> network on
// tcgen05 tensor cores -> a bit mask of troubled faces.  (The training-sample
// extractor and the judge step's state comparison are in finess_b200.cu.)
#pragma once
#include <cmath>
#include <cstring>
#include "fin_indicator.cuh"
#include "fin_mlp.cuh"
#include "fin_stage.cuh"

namespace fin {

struct IndicatorArgs {
    const double* q;
    size_t plane;
    int mx, my;
    int bc[4];
    float gamma;
    const float* P;            // network parameters (FP32, mlp::NPARAM)
    float zthr;                // a face is troubled when its logit exceeds zthr
    unsigned* flags;           // bit masks (flag_wx / flag_wy layout), zeroed before the launch
    unsigned int* status;
    unsigned long long* count; // troubled faces (accumulated)
    int tma;                   // tm maps q (box (TJ+8) x (TI+6) x 5, as the stage kernel's)
    CUtensorMap tm;
    int skip_const;            // the network's output for an all-zero feature row is known to be
                               // "not troubled" (ind::zero_row_logit): constant stencils skip it
};

namespace ind {

// The network as the indicator kernel holds it: W1 with the layer-1 bias in
// its input column NIN (the feature row carries a 1 there, so the tensor
// core adds the BF16 bias), and W2 and w3 halved, because the kernel stores
// 2 gelu(x) = x (1 + tanh(...)) -- one FMA after the tanh -- and a factor 2
// is exact in BF16 and FP32.  The results equal the plain network's.
struct IndWeights {
    alignas(128) __nv_bfloat16 W1[mlp::NH * mlp::KIN];
    alignas(128) __nv_bfloat16 W2[mlp::NH * mlp::NH];
    float b2[mlp::NH], w3h[mlp::NH], b3;
};

__device__ __forceinline__ void load_ind_weights(IndWeights& w, const float* P, int tid, int nthreads)
{
    using namespace mlp;
    for (int e = tid; e < NH * KIN; e += nthreads) {
        const int o = e / KIN, i = e - o * KIN;
        const float v = i < NIN ? P[OFF_W1 + o * NIN + i] : (i == NIN ? P[OFF_B1 + o] : 0.0f);
        w.W1[tc::kmaj(o, i, KIN)] = __float2bfloat16_rn(v);
    }
    for (int e = tid; e < NH * NH; e += nthreads) {
        const int o = e / NH, i = e - o * NH;
        w.W2[tc::kmaj(o, i, NH)] = __float2bfloat16_rn(0.5f * bf16r(P[OFF_W2 + o * NH + i]));
    }
    for (int e = tid; e < NH; e += nthreads) {
        w.b2[e] = P[OFF_B2 + e];
        w.w3h[e] = 0.5f * bf16r(P[OFF_W3 + e]);
    }
    if (tid == 0) w.b3 = P[OFF_B3];
}

// 2 gelu(x) in the tanh form (the constants of mlp::gelu).
__device__ __forceinline__ float gelu2(float x)
{
    return fmaf(x, mlp::tanh_approx(x * fmaf(mlp::GK1, x * x, mlp::GK0)), x);
}
// gelu2 of two values as f32x2 pairs: lane by lane the same operations (5 %
// faster than two scalar calls in the indicator, B200, 4096^2, mid-run).
#ifndef FIN_X2_GELU
#define FIN_X2_GELU 1
#endif
__device__ __forceinline__ f2 gelu2_x2(f2 x)
{
#if !FIN_X2_GELU
    return f2_make(gelu2(f2_lo(x)), gelu2(f2_hi(x)));
#else
    const f2 a = f2_mul(x, f2_fma(f2_make(mlp::GK1, mlp::GK1), f2_mul(x, x), f2_make(mlp::GK0, mlp::GK0)));
    return f2_fma(x, f2_make(mlp::tanh_approx(f2_lo(a)), mlp::tanh_approx(f2_hi(a))), x);
#endif
}

// D (TMEM columns at tmem_d) = A (128 x 32, K-major) * B (32 x 32, K-major)^T,
// issued by one thread, no commit.
__device__ __forceinline__ void mma_128x32x32(uint32_t tmem_d, const __nv_bfloat16* A, const __nv_bfloat16* B)
{
    constexpr uint32_t idesc = tc::idesc_bf16(128, mlp::NH);
    const uint32_t a0 = tc::smem_addr(A), b0 = tc::smem_addr(B);
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
        const uint64_t ad = tc::smem_desc(a0 + kk * 256, 128, (mlp::KIN / 8) * 128);
        const uint64_t bd = tc::smem_desc(b0 + kk * 256, 128, (mlp::KIN / 8) * 128);
        tc::mma_bf16(tmem_d, ad, bd, idesc, kk > 0 ? 1u : 0u);
    }
}

// The network's logit for an all-zero feature row (the features of a face
// whose six stencil states are equal: every undivided difference is exactly
// 0), restated on the host with the kernel's roundings: layer 1 is the BF16
// bias alone, 2 gelu in BF16, layer 2 with the halved BF16 W2 in FP32, + b2,
// 2 gelu, the halved output weights.  The host's tanh and the tensor core's
// summation order differ from the device's by far less than the margin the
// caller demands.
inline float bf16_host(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}
inline double zero_row_logit(const float* P)
{
    using namespace mlp;
    auto g2 = [](double x) { return x * (1.0 + std::tanh(x * (double(GK0) + double(GK1) * x * x))); };
    double a1[NH];
    for (int o = 0; o < NH; o++) a1[o] = bf16_host(float(g2(bf16_host(P[OFF_B1 + o]))));
    double z = P[OFF_B3];
    for (int o = 0; o < NH; o++) {
        double h = 0.0;
        for (int i = 0; i < NH; i++) h += double(bf16_host(0.5f * bf16_host(P[OFF_W2 + o * NH + i]))) * a1[i];
        z += double(0.5f * bf16_host(P[OFF_W3 + o])) * g2(h + P[OFF_B2 + o]);
    }
    return z;
}

}  // namespace ind

// Shared memory of the indicator kernel for the stage kernel's tile shape.
// The four 128-row feature matrices X are overwritten by the layer-1
// activations once the layer-1 products have completed.
template <class Cfg>
struct IndTile {
    ind::IndWeights w;
    alignas(128) __nv_bfloat16 X[4 * 128 * mlp::KIN];
    alignas(128) double stg[MEQN * Cfg::RI * Cfg::SJ];
    float qs[MEQN * Cfg::RI * Cfg::RJ];
    uint64_t mbar_tma, mbar_mma;
    uint32_t tmem;
    int abort;
    unsigned int cnt;
};

// Steps 2-5 of the indicator for the cell tile (i0, j0) whose FP32 state
// (tile + halo) is in S.qs: the features of the tile's faces, the network on
// tcgen05 and the flags.  Per tile the CTA owns the x faces of rows i0 ..
// i0+TI-1 and the y faces of columns j0 .. j0+TJ-1 (the last tile row /
// column also the domain's last face row / column): at most 511 faces, laid
// out as four 128-row matrices (slots 0..255 x faces, slots 256..510 y
// faces, each warp's half-warps on face rows 8 apart).
//   2. each thread: the features of its two slots from shared memory;
//   3. layer 1 on tcgen05 (4 x two K=16 steps into TMEM columns 0..127);
//   4. 2 gelu, BF16, back into the X matrices; layer 2 into the same columns;
//   5. 2 gelu + b2 -> output layer in FP32 -> flag.
// TMEM lane quarter q = warp % 4 holds rows 32q .. 32q+31 of every matrix;
// warps 0-3 take matrices 0 and 1, warps 4-7 matrices 2 and 3.  Flagged
// faces set their bits (the words are cleared before the run).  Sets S.abort
// when a tensor-core wait ran out (uniform across the CTA on return).
//
// With skip_const, a warp whose 32 faces of a matrix all have six equal
// stencil states (or are not owned) skips their features, activations and
// output: their features are exactly 0, and the network's output for a zero
// row is known to be "not troubled" (the caller checked
// ind::zero_row_logit against the threshold with a margin), so the flags
// are the same as with the network evaluated.
template <class Cfg>
__device__ __forceinline__ void indicator_tile(IndTile<Cfg>& S, const int mx, const int my, const float gamma,
                                               const float zthr, unsigned* flags, const int i0, const int j0,
                                               const uint32_t tmem, uint32_t& mma_phase, const bool skip_const = false)
{
    using namespace mlp;
    constexpr int TI = Cfg::TI, TJ = Cfg::TJ, H = Cfg::H, RJ = Cfg::RJ, PQ = Cfg::RI * Cfg::RJ;
    static_assert(Cfg::NT == 256 && TI == 15 && TJ == 16, "face slots: 256 x faces, 255 y faces, rows 8 apart");
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t lane_base = uint32_t((warp & 3) * 32) << 16;
    // ---- 2. features of the thread's two slots ----
    long long fword[2];   // flag word of the slot's face (-1: not owned)
    unsigned fbit[2];
    bool wconst[2];       // the warp's 32 slots of matrix h are all constant stencils (or unowned)
    const int wx = flag_wx(my), wy = flag_wy(my);
#pragma unroll 1
    for (int h = 0; h < 2; h++) {
        const int mt = 2 * (warp >> 2) + h, row = 32 * (warp & 3) + lane, sl = 128 * mt + row;
        float xr[KIN];
#pragma unroll
        for (int k = 0; k < KIN; k++) xr[k] = 0.0f;
        fword[h] = -1;
        fbit[h] = 0;
        bool isx = sl < 256;
        int fi, fj;
        // half-warps on face rows r and r + 8: 8 rows of RJ = 22 words are
        // 176 words, 16 modulo 32, so the two rows' stencil loads fall in
        // opposite halves of the banks (the last warp of y slots takes row
        // 7 and the last column)
        if (isx) { fi = (sl >> 5) + ((sl >> 1) & 8); fj = sl & 15; }
        else {
            const int v = sl - 256, wv = v >> 5, ln = v & 31;
            if (wv < 7) { fi = wv + (ln & 16 ? 8 : 0); fj = ln & 15; }
            else if (ln < 16) { fi = 7; fj = ln; }
            else { fi = ln - 16; fj = TJ; }
        }
        const int gi = i0 + fi, gj = j0 + fj;
        bool own;
        if (isx) own = gj < my && gi <= mx && (fi < TI || gi == mx);
        else own = sl < 511 && gi < mx && gj <= my && (fj < TJ || gj == my);
        float Q[6][MEQN];
        bool cst = skip_const;   // an unowned slot counts as constant
        if (own) {
            fword[h] = isx ? (long long)gi * wx + (gj >> 5) : (long long)(mx + 1) * wx + (long long)gi * wy + (gj >> 5);
            fbit[h] = 1u << (gj & 31);
            const int cn = isx ? 1 : 2, ct = isx ? 2 : 1;
            const int base = isx ? (H + fi - 3) * RJ + (H + fj) : (H + fi) * RJ + (H + fj - 3);
            const int str = isx ? RJ : 1;
#pragma unroll
            for (int st = 0; st < 6; st++) {
                const int o = base + st * str;
                Q[st][0] = S.qs[o];
                Q[st][1] = S.qs[cn * PQ + o];
                Q[st][2] = S.qs[ct * PQ + o];
                Q[st][3] = S.qs[3 * PQ + o];
                Q[st][4] = S.qs[4 * PQ + o];
            }
#pragma unroll
            for (int st = 1; st < 6; st++)
#pragma unroll
                for (int m = 0; m < MEQN; m++) cst = cst && Q[st][m] == Q[0][m];
        }
        wconst[h] = __all_sync(0xffffffffu, cst);   // every lane takes part
        if (own) {
            if (!wconst[h]) ind::stencil_features<float>(Q, gamma, xr);
            xr[NIN] = 1.0f;   // the layer-1 bias input
        }
        store_row32(S.X + mt * 128 * KIN, row, xr);
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    // ---- 3. layer 1 ----
    if (tid == 0) {
        tc::fence_after_sync();
#pragma unroll
        for (int mt = 0; mt < 4; mt++) ind::mma_128x32x32(tmem + 32 * mt, S.X + mt * 128 * KIN, S.w.W1);
        tc::commit(&S.mbar_mma);
    }
    if (!tc::mbar_wait(&S.mbar_mma, mma_phase)) S.abort = 1;
    mma_phase ^= 1;
    tc::fence_after_sync();
    // ---- 4. 2 gelu of layer 1 into the X matrices; layer 2 ----
#pragma unroll 1
    for (int h = 0; h < 2; h++) {
        const int mt = 2 * (warp >> 2) + h, row = 32 * (warp & 3) + lane;
        if (wconst[h]) continue;   // rows whose output is known: layer 2 sees their zero features
        float v[32];
        tc::tmem_ld32(tmem + lane_base + 32 * mt, v);
#pragma unroll
        for (int o = 0; o < NH; o += 2) {
            const f2 g = ind::gelu2_x2(f2_make(v[o], v[o + 1]));
            v[o] = f2_lo(g);
            v[o + 1] = f2_hi(g);
        }
        store_row32(S.X + mt * 128 * KIN, row, v);
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    if (S.abort) return;
    if (tid == 0) {
        tc::fence_after_sync();
#pragma unroll
        for (int mt = 0; mt < 4; mt++) ind::mma_128x32x32(tmem + 32 * mt, S.X + mt * 128 * KIN, S.w.W2);
        tc::commit(&S.mbar_mma);
    }
    if (!tc::mbar_wait(&S.mbar_mma, mma_phase)) S.abort = 1;
    mma_phase ^= 1;
    tc::fence_after_sync();
    // ---- 5. output layer and flags ----
#pragma unroll 1
    for (int h = 0; h < 2; h++) {
        const int mt = 2 * (warp >> 2) + h;
        if (wconst[h]) continue;   // not troubled (the zero row's known output)
        float v[32];
        tc::tmem_ld32(tmem + lane_base + 32 * mt, v);
        float zz = S.w.b3;
#pragma unroll
        for (int o = 0; o < NH; o += 2) {
            const f2 g = ind::gelu2_x2(f2_add(f2_make(v[o], v[o + 1]), f2_make(S.w.b2[o], S.w.b2[o + 1])));
            zz = fmaf(S.w.w3h[o], f2_lo(g), zz);
            zz = fmaf(S.w.w3h[o + 1], f2_hi(g), zz);
        }
        const bool fl = fword[h] >= 0 && zz > zthr;
        if (fl) atomicOr(flags + fword[h], fbit[h]);
        const unsigned bal = __ballot_sync(0xffffffffu, fl);
        if (lane == 0 && bal) atomicAdd(&S.cnt, unsigned(__popc(bal)));
    }
    tc::fence_before_sync();
    __syncthreads();
}

// One flag per face of the state a.q.  Persistent CTAs walk the stage
// kernel's TI x TJ cell tiles; per tile
//   1. q's tile + halo: TMA (prefetched during the previous tile) or remap
//      loads, FP64 -> FP32 in shared memory;
//   2-5. indicator_tile.
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT, 3) k_indicator(const __grid_constant__ IndicatorArgs a)
{
    constexpr int TI = Cfg::TI, TJ = Cfg::TJ, H = Cfg::H;
    static_assert(Cfg::NT == 256 && TI == 15 && TJ == 16, "face slots: 256 x faces, 255 y faces, rows 8 apart");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    IndTile<Cfg>& S = *reinterpret_cast<IndTile<Cfg>*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    ind::load_ind_weights(S.w, a.P, tid, Cfg::NT);
    if (warp == 0) tc::tmem_alloc(&S.tmem, 128);
    if (tid == 0) {
        tc::mbar_init(&S.mbar_tma, 1);
        tc::mbar_init(&S.mbar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        S.abort = 0;
        S.cnt = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem;
    const int mx = a.mx, my = a.my;
    const int ntj = (my + TJ - 1) / TJ;
    const long long ntiles = (long long)((mx + TI - 1) / TI) * ntj;
    const bool aligned = (tc::smem_addr(S.stg) & 127u) == 0;
    if (a.tma && !aligned && tid == 0) atomicOr(a.status, 16u);
    uint32_t tma_phase = 0, mma_phase = 0;
    // TMA of tile t's box into stg when the tile qualifies (one thread issues)
    auto issue = [&](long long t) -> bool {
        const int ti0 = int(t / ntj) * TI, tj0 = int(t % ntj) * TJ;
        if (!(a.tma && aligned && tma_interior<Cfg>(ti0, tj0, mx, my))) return false;
        if (tid == 0) {
            tc::mbar_expect_tx(&S.mbar_tma, uint32_t(Cfg::STG_BYTES));
            tc::tma_load_3d(S.stg, &a.tm, tj0 - 4, ti0 - H, 0, &S.mbar_tma);
        }
        return true;
    };
    bool pending = (long long)blockIdx.x < ntiles ? issue(blockIdx.x) : false;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i0 = int(t / ntj) * TI, j0 = int(t % ntj) * TJ;
        // ---- 1. stage the tile ----
        if (pending) {
            if (!tc::mbar_wait(&S.mbar_tma, tma_phase, 1u << 24)) {
                atomicOr(a.status, 8u);
                tc::mbar_wait(&S.mbar_tma, tma_phase, 1u << 24);
                S.abort = 1;
            }
            tma_phase ^= 1;
        } else {
            stage_remap<Cfg>(S.stg, a.q, a.plane, i0, j0, mx, my, a.bc, tid);
            __syncthreads();
        }
        stage_convert<Cfg, float>(S.stg, S.qs, tid);
        tc::fence_smem_to_async();     // the reads of stg precede the next TMA write into it
        __syncthreads();
        if (S.abort) { pending = false; break; }
        pending = t + gridDim.x < ntiles ? issue(t + gridDim.x) : false;
        indicator_tile<Cfg>(S, mx, my, a.gamma, a.zthr, a.flags, i0, j0, tmem, mma_phase, a.skip_const != 0);
        if (S.abort) break;
    }
    // a copy still in flight lands before the shared memory is released
    if (pending && !tc::mbar_wait(&S.mbar_tma, tma_phase, 1u << 24)) atomicOr(a.status, 8u);
    __syncthreads();
    if (tid == 0) {
        if (S.abort) atomicOr(a.status, 4u);
        atomicAdd(a.count, (unsigned long long)S.cnt);
    }
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tmem, 128);
}

}  // namespace fin
