// Kernels of the hybrid form: the per-step troubled-face indicator (features
// -> network on tcgen05 tensor cores -> one flag byte per face), the
// training-sample extractor, and the judge step's state comparison.
#pragma once
#include "fin_indicator.cuh"
#include "fin_mlp.cuh"

namespace fin {

struct IndicatorArgs {
    const double* q;
    size_t plane;
    int mx, my;
    int bc[4];
    float gamma;
    const float* P;            // network parameters (FP32, mlp::NPARAM)
    float zthr;                // a face is troubled when its logit exceeds zthr
    unsigned char* flags;      // x faces then y faces
    unsigned int* status;
    unsigned long long* count; // troubled faces (accumulated)
};

struct IndSmem {
    alignas(128) mlp::Weights w;
    alignas(128) __nv_bfloat16 Xs[mlp::TILE * mlp::KIN];
    alignas(128) __nv_bfloat16 G1s[mlp::TILE * mlp::NH];
    uint64_t mbar;
    uint32_t tmem;
    int abort;
    unsigned int cnt;
};

// One flag per face of the state a.q: 128 faces per tile, one per thread.
__global__ void __launch_bounds__(mlp::TILE) k_indicator(const IndicatorArgs a)
{
    using namespace mlp;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    IndSmem& S = *reinterpret_cast<IndSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    load_weights(S.w, a.P, tid, TILE);
    if (warp == 0) tc::tmem_alloc(&S.tmem, 64);
    if (tid == 0) {
        tc::mbar_init(&S.mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        S.abort = 0;
        S.cnt = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem;
    const uint32_t lane_base = uint32_t(warp * 32) << 16;
    uint32_t phase = 0;
    const long long nf = (long long)(a.mx + 1) * a.my + (long long)a.mx * (a.my + 1);
    const long long ntiles = (nf + TILE - 1) / TILE;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long f = t * TILE + tid;
        float x[ind::NFEAT];
        if (f < nf) {
            bool isx;
            int i, j;
            ind::face_of(f, a.mx, a.my, isx, i, j);
            ind::face_features<float>(a.q, a.plane, a.mx, a.my, a.bc, a.gamma, isx, i, j, x);
        } else {
#pragma unroll
            for (int k = 0; k < ind::NFEAT; k++) x[k] = 0.0f;
        }
#pragma unroll
        for (int k = 0; k < KIN; k++) S.Xs[tc::kmaj(tid, k, KIN)] = __float2bfloat16_rn(k < NIN ? x[k] : 0.0f);
        tc::fence_smem_to_async();
        __syncthreads();
        if (tid == 0) gemm_tile_k32(tmem, S.Xs, S.w.W1, &S.mbar);
        if (!tc::mbar_wait(&S.mbar, phase)) S.abort = 1;
        phase ^= 1;
        tc::fence_after_sync();
        float h[32];
        tc::tmem_ld32(tmem + lane_base, h);
#pragma unroll
        for (int o = 0; o < NH; o++) S.G1s[tc::kmaj(tid, o, NH)] = __float2bfloat16_rn(gelu(h[o] + S.w.b1[o]));
        tc::fence_smem_to_async();
        tc::fence_before_sync();
        __syncthreads();
        if (S.abort) break;
        if (tid == 0) gemm_tile_k32(tmem + 32, S.G1s, S.w.W2, &S.mbar);
        if (!tc::mbar_wait(&S.mbar, phase)) S.abort = 1;
        phase ^= 1;
        tc::fence_after_sync();
        tc::tmem_ld32(tmem + lane_base + 32, h);
        float zz = S.w.b3;
#pragma unroll
        for (int o = 0; o < NH; o++) zz += S.w.w3[o] * bf16r(gelu(h[o] + S.w.b2[o]));
        if (f < nf) {
            const unsigned char fl = zz > a.zthr ? 1 : 0;
            a.flags[f] = fl;
            if (fl) atomicAdd(&S.cnt, 1u);
        }
        tc::fence_before_sync();
        __syncthreads();
        if (S.abort) break;
    }
    __syncthreads();
    if (tid == 0) {
        if (S.abort) atomicOr(a.status, 4u);
        atomicAdd(a.count, (unsigned long long)S.cnt);
    }
    if (warp == 0) tc::tmem_free(tmem, 64);
}

// Training samples: features and labels of faces f0, f0 + stride, ...
__global__ void k_face_samples(const double* q, size_t plane, int mx, int my, int bc0, int bc1, int bc2, int bc3,
                               double gamma, double eps, double pw, double ascale, const double* alpha_g,
                               long long f0, long long stride, long long n, float* X, unsigned char* y)
{
    const int bc[4] = {bc0, bc1, bc2, bc3};
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const long long f = f0 + s * stride;
        bool isx;
        int i, j;
        ind::face_of(f, mx, my, isx, i, j);
        float x[ind::NFEAT];
        ind::face_features<float>(q, plane, mx, my, bc, float(gamma), isx, i, j, x);
#pragma unroll
        for (int k = 0; k < ind::NFEAT; k++) X[s * ind::NFEAT + k] = x[k];
        const double ag = alpha_g ? alpha_g[isx ? 0 : 1] : 0.0;
        y[s] = ind::face_label(q, plane, mx, my, bc, gamma, eps, pw, ascale, ag, isx, i, j);
    }
}

// max |a - b| and max |b| over all planes' interior values (judge step).
__global__ void k_max_diff(const double* a, const double* b, size_t plane, size_t n, double* out)
{
    __shared__ double red[2][32];
    double d = 0.0, m = 0.0;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
#pragma unroll
        for (int c = 0; c < MEQN; c++) {
            const double va = a[c * plane + g], vb = b[c * plane + g];
            const double dd = fabs(va - vb);
            d = dd > d || dd != dd ? dd : d;     // NaN wins
            m = Max(m, fabs(vb));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double od = __shfl_xor_sync(0xffffffffu, d, o);
        d = od > d || od != od ? od : d;
        m = Max(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = d; red[1][w] = m; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < nw; k++) {
            d = red[0][k] > d || red[0][k] != red[0][k] ? red[0][k] : d;
            m = Max(m, red[1][k]);
        }
        atomic_max_nonneg(out, d != d ? __longlong_as_double(0x7ff0000000000000ll) : d);
        atomic_max_nonneg(out + 1, m);
    }
}

}  // namespace fin
