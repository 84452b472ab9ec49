// The learned troubled-face indicator of the ideal-MHD path: face features,
// the labels the method generates itself, the training-sample extractor and
// the indicator kernel (features -> network on tcgen05 tensor cores -> bit
// mask of troubled faces).
//
// For the face between cells i-1 and i (x faces; y faces alike along j) with
// the 6-point WENO stencil i-3 .. i+2 and the left eigenvectors at the face
// average (ProjectLeftEig.cpp:179-192, in the structured form of
// fin_mhd.cuh):
//   features: w = L q at the six points; for each of the eight fields k,
//     with D_s = w_k(s+1) - w_k(s) and M = max_s |D_s|: the relative second
//     difference max_s |D_(s+1) - D_s| / max(M, 1e-3) (in [0, 2]; large where
//     the field is not smooth on the stencil) and the magnitude M / (M + 1e-3)
//     (small where the field varies too little to move the WENO weights, beta
//     ~ D^2 against epsilon = 1e-6); 16 values, the last 4 inputs zero.  One
//     number pair per field keeps every field visible to the network, which
//     the labels need: any of the eight can trigger;
//   label: 1 when the WENO5-JS weights of gp or gm (ConstructL.cpp:179-192)
//     of any of the eight fields depart from the linear weights (0.1, 0.6,
//     0.3) by more than 10 % (lib/WenoReconstruct.cpp:104, 131-134).
// The network (20 -> 32 -> 32 -> 1, BF16 weights, FP32 accumulation) and its
// tensor-core evaluation are the Euler indicator's (fin_hybrid.cuh).
#pragma once
#include "fin_hybrid.cuh"
#include "fin_mhd.cuh"

namespace fin {
namespace mind {

constexpr float FEAT_FLOOR = 1e-3f;

// Features of one face from its stencil Qn[s][c] (normal-frame components).
template <class R>
__device__ __forceinline__ void features(const MhdArgs& a, R gamma, const R (&Qn)[6][MHD_NQ], float* x)
{
    R Qa[MHD_NQ];
#pragma unroll
    for (int c = 0; c < MHD_NQ; c++) Qa[c] = R(0.5) * (Qn[3][c] + Qn[2][c]);
    MhdFace<R> f;
    bool neg = false;
    mhd_face_setup<R>(a, gamma, Qa, f, nullptr, 0, neg);
    R w[MHD_NQ][6];
#pragma unroll
    for (int s = 0; s < 6; s++) {
        R r0, r7, r2, r5, r1, r6, r3, r4;
        mhd_left_fs4<R>(f, Qn[s], r0, r7, r2, r5);
        mhd_left_alf<R>(f, Qn[s], r1, r6);
        mhd_left_ent<R>(f, Qn[s], r3, r4);
        w[0][s] = r0; w[7][s] = r7; w[2][s] = r2; w[5][s] = r5;
        w[1][s] = r1; w[6][s] = r6; w[3][s] = r3; w[4][s] = r4;
    }
#pragma unroll
    for (int k = 0; k < MHD_NQ; k++) {
        R d[5], M = R(0), S = R(0);
#pragma unroll
        for (int s = 0; s < 5; s++) {
            d[s] = w[k][s + 1] - w[k][s];
            M = Max(M, R(fabs(d[s])));
        }
#pragma unroll
        for (int s = 0; s < 4; s++) S = Max(S, R(fabs(d[s + 1] - d[s])));
        x[2 * k] = float(S / Max(M, R(FEAT_FLOOR)));
        x[2 * k + 1] = float(M / (M + R(FEAT_FLOOR)));
    }
#pragma unroll
    for (int k = 2 * MHD_NQ; k < ind::NFEAT; k++) x[k] = 0.0f;
}

// Stencil cell s (0..5) of face (isx, i, j) under the periodic remap.
__device__ __forceinline__ size_t stencil_cell(bool isx, int i, int j, int s, int mx, int my)
{
    const int ci = isx ? i + s - 3 : i, cj = isx ? j : j + s - 3;
    return size_t(pwrap(ci, mx)) * my +
           pwrap(cj, my);
}

// Label of one face (FP64): the reference's split (SetWaveSpd with the two
// adjacent cells, ConstructL.cpp:170-185) and WENO5-JS weights of all fields.
__device__ __forceinline__ unsigned char label(const MhdArgs& a, const double* q, double alpha_g, bool isx, int i,
                                               int j)
{
    const int mx = a.mx, my = a.my;
    const int cn = isx ? 1 : 2, ct = isx ? 2 : 1, bn = isx ? 5 : 6, bt = isx ? 6 : 5;
    const int perm[MHD_NQ] = {0, cn, ct, 3, 4, bn, bt, 7};
    const double gamma = a.gamma;
    double Q[6][MHD_NQ], F[6][MHD_NQ];
    double u1l = 0, u2l = 0, pl = 0, cfl = 0, u1r = 0, u2r = 0, pr = 0, cfr = 0;
#pragma unroll
    for (int s = 0; s < 6; s++) {
        const size_t c = stencil_cell(isx, i, j, s, mx, my);
        double P[MHD_NQ];
#pragma unroll
        for (int m = 0; m < MHD_NQ; m++) P[m] = q[m * a.plane + c];
        const double ir = 1.0 / P[0];
        const double u1 = P[1] * ir, u2 = P[2] * ir, u3 = P[3] * ir;
        const double Bsq = P[5] * P[5] + P[6] * P[6] + P[7] * P[7];
        const double press = (gamma - 1.0) * (P[4] - 0.5 * P[0] * (u1 * u1 + u2 * u2 + u3 * u3) - 0.5 * Bsq);
        const double Bm = 0.5 * Bsq, Bu = u1 * P[5] + u2 * P[6] + u3 * P[7], eb = P[4] + press + Bm;
        double fl[MHD_NQ];
        if (isx) {
            fl[0] = P[0] * u1; fl[1] = P[0] * u1 * u1 + press + Bm - P[5] * P[5]; fl[2] = P[0] * u1 * u2 - P[5] * P[6];
            fl[3] = P[0] * u1 * u3 - P[5] * P[7]; fl[4] = u1 * eb - P[5] * Bu; fl[5] = 0.0;
            fl[6] = u1 * P[6] - u2 * P[5]; fl[7] = u1 * P[7] - u3 * P[5];
        } else {
            fl[0] = P[0] * u2; fl[1] = P[0] * u1 * u2 - P[6] * P[5]; fl[2] = P[0] * u2 * u2 + press + Bm - P[6] * P[6];
            fl[3] = P[0] * u2 * u3 - P[6] * P[7]; fl[4] = u2 * eb - P[6] * Bu; fl[5] = u2 * P[5] - u1 * P[6];
            fl[6] = 0.0; fl[7] = u2 * P[7] - u3 * P[6];
        }
#pragma unroll
        for (int m = 0; m < MHD_NQ; m++) {
            Q[s][m] = P[perm[m]];
            F[s][m] = fl[perm[m]];
        }
        if (s == 2 || s == 3) {
            const double a2c = fabs(gamma * press * ir), t = a2c + Bsq * ir;
            const double cf = sqrt(0.5 * (t + sqrt(fabs(t * t - 4.0 * a2c * (P[5] * P[5]) * ir))));
            if (s == 2) { u1l = u1; u2l = u2; pl = press; cfl = cf; }
            else { u1r = u1; u2r = u2; pr = press; cfr = cf; }
        }
    }
    double Qa[MHD_NQ];
#pragma unroll
    for (int m = 0; m < MHD_NQ; m++) Qa[m] = 0.5 * (Q[3][m] + Q[2][m]);
    double alpha;
    {
        const double unl = isx ? u1l : u2l, unr = isx ? u1r : u2r;
        const double rho = Qa[0], B1x = isx ? Qa[5] : Qa[6];
        const double Bm2 = Qa[5] * Qa[5] + Qa[6] * Qa[6] + Qa[7] * Qa[7];
        const double a2 = fabs(gamma * (0.5 * (pl + pr)) / rho), t = a2 + Bm2 / rho;
        const double cf = sqrt(0.5 * (t + sqrt(fabs(t * t - 4.0 * a2 * B1x * B1x / rho))));
        const double ua = 0.5 * (unl + unr);
        const double s1 = Min(unl - cfl, ua - cf), s2 = Max(unr + cfr, ua + cf);
        alpha = Max(alpha_g, Max(fabs(s1), fabs(s2)));
    }
    const double la = a.alpha_scaling * alpha;
    MhdFace<double> f;
    bool neg = false;
    mhd_face_setup<double>(a, gamma, Qa, f, nullptr, 0, neg);
    double W[6][MHD_NQ], G[6][MHD_NQ];
#pragma unroll
    for (int s = 0; s < 6; s++) {
        mhd_left_fs4<double>(f, Q[s], W[s][0], W[s][7], W[s][2], W[s][5]);
        mhd_left_alf<double>(f, Q[s], W[s][1], W[s][6]);
        mhd_left_ent<double>(f, Q[s], W[s][3], W[s][4]);
        mhd_left_fs4<double>(f, F[s], G[s][0], G[s][7], G[s][2], G[s][5]);
        mhd_left_alf<double>(f, F[s], G[s][1], G[s][6]);
        mhd_left_ent<double>(f, F[s], G[s][3], G[s][4]);
    }
    double dep = 0.0;
#pragma unroll 1
    for (int k = 0; k < MHD_NQ; k++) {
        double gp[5], gm[5];
#pragma unroll
        for (int s = 0; s < 5; s++) {
            gp[s] = 0.5 * (G[s][k] + la * W[s][k]);
            gm[s] = 0.5 * (G[5 - s][k] - la * W[5 - s][k]);
        }
        dep = Max(dep, Max(ind::js5_departure(gp, a.eps, a.pw), ind::js5_departure(gm, a.eps, a.pw)));
    }
    return dep > 0.1 ? 1 : 0;
}

}  // namespace mind

// Training samples of the MHD state q: features and labels of faces f0,
// f0 + stride, ... (x faces, then y faces).
__global__ void k_mhd_face_samples(const MhdArgs a, const double* q, const double* alpha_g, long long f0,
                                   long long stride, long long n, float* X, unsigned char* y)
{
    const int mx = a.mx, my = a.my;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const long long f = f0 + s * stride;
        bool isx;
        int i, j;
        ind::face_of(f, mx, my, isx, i, j);
        const int cn = isx ? 1 : 2, ct = isx ? 2 : 1, bn = isx ? 5 : 6, bt = isx ? 6 : 5;
        const int perm[MHD_NQ] = {0, cn, ct, 3, 4, bn, bt, 7};
        float Qn[6][MHD_NQ];
#pragma unroll
        for (int st = 0; st < 6; st++) {
            const size_t c = mind::stencil_cell(isx, i, j, st, mx, my);
#pragma unroll
            for (int m = 0; m < MHD_NQ; m++) Qn[st][m] = float(q[perm[m] * a.plane + c]);
        }
        float x[ind::NFEAT];
        mind::features<float>(a, a.gamma_f, Qn, x);
#pragma unroll
        for (int k = 0; k < ind::NFEAT; k++) X[s * ind::NFEAT + k] = x[k];
        y[s] = mind::label(a, q, alpha_g ? alpha_g[isx ? 0 : 1] : 0.0, isx, i, j);
    }
}

// Shared memory of the MHD indicator: weights, the four 128-row feature /
// activation matrices, and q's tile + 3-cell cross halo in FP32.
template <class Cfg>
struct MhdIndTile {
    ind::IndWeights w;
    alignas(128) __nv_bfloat16 X[4 * 128 * mlp::KIN];
    float qs[MHD_NQ * Cfg::RI * Cfg::RJ];
    uint64_t mbar_mma;
    uint32_t tmem;
    int abort;
    unsigned int cnt;
};

struct MhdIndArgs {
    MhdArgs m;                 // grid, state planes (m.qin), parameters
    const float* P;            // network parameters (FP32, mlp::NPARAM)
    float zthr;                // a face is troubled when its logit exceeds zthr
    unsigned* flags;           // bit masks (flag_wx / flag_wy layout), zeroed before the launch
    unsigned long long* count; // troubled faces (accumulated)
};

// One flag per face of the state a.m.qin, in the tile walk and face-slot
// layout of k_indicator (fin_hybrid.cuh): persistent CTAs over 15 x 16 cell
// tiles; per tile the x faces of rows i0 .. i0+14 and the y faces of columns
// j0 .. j0+15 (the domain's last face row / column with the last tiles),
// at most 511 faces in four 128-row matrices; layer 1 and layer 2 on
// tcgen05 with the accumulator in TMEM, every wait bounded.
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT, 3) k_mhd_indicator(const __grid_constant__ MhdIndArgs ia)
{
    using namespace mlp;
    const MhdArgs& a = ia.m;
    constexpr int TI = Cfg::TI, TJ = Cfg::TJ, H = Cfg::H, RI = Cfg::RI, RJ = Cfg::RJ, PQ = RI * RJ;
    static_assert(Cfg::NT == 256 && (TI + 1) * TJ <= 256 && TI * (TJ + 1) <= 255 && TJ == 16, "face slots");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    MhdIndTile<Cfg>& S = *reinterpret_cast<MhdIndTile<Cfg>*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    ind::load_ind_weights(S.w, ia.P, tid, Cfg::NT);
    if (warp == 0) tc::tmem_alloc(&S.tmem, 128);
    if (tid == 0) {
        tc::mbar_init(&S.mbar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        S.abort = 0;
        S.cnt = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem;
    const uint32_t lane_base = uint32_t((warp & 3) * 32) << 16;
    const int mx = a.mx, my = a.my;
    const int ntj = (my + TJ - 1) / TJ;
    const long long ntiles = (long long)((mx + TI - 1) / TI) * ntj;
    uint32_t mma_phase = 0;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i0 = int(t / ntj) * TI, j0 = int(t % ntj) * TJ;
        // ---- 1. the tile + 3-cell cross halo, FP32 ----
        for (int e = tid; e < PQ; e += Cfg::NT) {
            const int ii = e / RJ, jj = e - ii * RJ;
            const bool xin = ii >= H && ii < H + TI, yin = jj >= H && jj < H + TJ;
            if (!xin && !yin) continue;
            const int gi = pwrap(i0 + ii - H, mx);
            const int gj = pwrap(j0 + jj - H, my);
            const size_t g = size_t(gi) * my + gj;
#pragma unroll
            for (int m = 0; m < MHD_NQ; m++) S.qs[m * PQ + e] = float(__ldg(a.qin + m * a.plane + g));
        }
        __syncthreads();
        // ---- 2. features of the thread's two slots ----
        long long fword[2];
        unsigned fbit[2];
        const int wx = flag_wx(my), wy = flag_wy(my);
#pragma unroll 1
        for (int h = 0; h < 2; h++) {
            const int mt = 2 * (warp >> 2) + h, row = 32 * (warp & 3) + lane, sl = 128 * mt + row;
            float xr[KIN];
#pragma unroll
            for (int k = 0; k < KIN; k++) xr[k] = 0.0f;
            fword[h] = -1;
            fbit[h] = 0;
            const bool isx = sl < 256;
            int fi, fj;
            if (isx) { fi = sl >> 4; fj = sl & 15; }
            else { const int v = sl - 256; fi = v / (TJ + 1); fj = v - fi * (TJ + 1); }
            const int gi = i0 + fi, gj = j0 + fj;
            bool own;
            if (isx) own = gj < my && gi <= mx && (fi < TI || gi == mx);
            else own = sl < 511 && gi < mx && gj <= my && (fj < TJ || gj == my);
            if (own) {
                fword[h] = isx ? (long long)gi * wx + (gj >> 5) : (long long)(mx + 1) * wx + (long long)gi * wy + (gj >> 5);
                fbit[h] = 1u << (gj & 31);
                const int cn = isx ? 1 : 2, ct = isx ? 2 : 1, bn = isx ? 5 : 6, bt = isx ? 6 : 5;
                const int perm[MHD_NQ] = {0, cn, ct, 3, 4, bn, bt, 7};
                const int base = isx ? (H + fi - 3) * RJ + (H + fj) : (H + fi) * RJ + (H + fj - 3);
                const int str = isx ? RJ : 1;
                float Qn[6][MHD_NQ];
#pragma unroll
                for (int st = 0; st < 6; st++)
#pragma unroll
                    for (int m = 0; m < MHD_NQ; m++) Qn[st][m] = S.qs[perm[m] * PQ + base + st * str];
                mind::features<float>(a, a.gamma_f, Qn, xr);
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
        if (S.abort) break;
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
            float v[32];
            tc::tmem_ld32(tmem + lane_base + 32 * mt, v);
            float zz = S.w.b3;
#pragma unroll
            for (int o = 0; o < NH; o += 2) {
                const f2 g = ind::gelu2_x2(f2_add(f2_make(v[o], v[o + 1]), f2_make(S.w.b2[o], S.w.b2[o + 1])));
                zz = fmaf(S.w.w3h[o], f2_lo(g), zz);
                zz = fmaf(S.w.w3h[o + 1], f2_hi(g), zz);
            }
            const bool fl = fword[h] >= 0 && zz > ia.zthr;
            if (fl) atomicOr(ia.flags + fword[h], fbit[h]);
            const unsigned bal = __ballot_sync(0xffffffffu, fl);
            if (lane == 0 && bal) atomicAdd(&S.cnt, unsigned(__popc(bal)));
        }
        tc::fence_before_sync();
        __syncthreads();
        if (S.abort) break;
    }
    __syncthreads();
    if (tid == 0) {
        if (S.abort) atomicOr(a.status, 4u);
        atomicAdd(ia.count, (unsigned long long)S.cnt);
    }
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tmem, 128);
}

}  // namespace fin
