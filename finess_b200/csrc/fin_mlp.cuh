// The troubled-cell indicator network: 20 inputs -> 32 -> 32 -> 1, GELU,
// BF16 weights (the layer-1 bias included) and BF16 activations at both
// hidden-layer matrix products, FP32 accumulation; the 32 -> 1 output layer
// takes the layer-2 activations in FP32.
// Parameters (FP32 master copy, length MLP_NPARAM):
//   W1[32][20], b1[32], W2[32][32], b2[32], w3[32], b3.
// The layer-1 and layer-2 products, the back-propagated activation gradient
// and both weight gradients run on tcgen05 tensor cores (fin_tc.cuh); the
// 32 -> 1 output layer and the element-wise work run on CUDA cores in FP32.
#pragma once
#include <cuda_bf16.h>
#include "fin_tc.cuh"

namespace fin {
namespace mlp {

constexpr int NIN = 20, KIN = 32, NH = 32, TILE = 128;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NIN, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
              OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NH, NPARAM = OFF_B3 + 1;

// GELU in its tanh form (Hendrycks & Gimpel, arXiv:1606.08415):
//   gelu(x) = x/2 (1 + tanh(k0 x + k1 x^3)),  k0 = sqrt(2/pi), k1 = 0.044715 k0,
// with tanh from the hardware approximation (PTX tanh.approx.f32, one
// special-function op; its error, below 2^-10 absolute, is under half a BF16
// step of the activations it feeds).  The derivative uses the same t.
constexpr float GK0 = 0.79788456080286536f, GK1 = 0.79788456080286536f * 0.044715f;
__device__ __forceinline__ float tanh_approx(float x)
{
    float r;
    asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float gelu(float x)
{
    const float t = tanh_approx(x * fmaf(GK1, x * x, GK0));
    const float h = 0.5f * x;
    return fmaf(h, t, h);
}
__device__ __forceinline__ float gelu_grad(float x)
{
    const float x2 = x * x;
    const float t = tanh_approx(x * fmaf(GK1, x2, GK0));
    return fmaf(0.5f * x * fmaf(-t, t, 1.0f), fmaf(3.0f * GK1, x2, GK0), 0.5f + 0.5f * t);
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Row r of an R x 32 K-major bf16 tile from 32 FP32 values: four 16-byte
// stores, one per core-matrix row (8 consecutive threads fill one 128-byte
// core matrix, so the stores are free of bank conflicts).
__device__ __forceinline__ void store_row32(__nv_bfloat16* tile, int r, const float* v)
{
#pragma unroll
    for (int c = 0; c < 4; c++) {
        uint4 u;
        uint32_t* w = reinterpret_cast<uint32_t*>(&u);
#pragma unroll
        for (int h = 0; h < 4; h++) {
            const __nv_bfloat162 b = __floats2bfloat162_rn(v[c * 8 + 2 * h], v[c * 8 + 2 * h + 1]);
            w[h] = *reinterpret_cast<const uint32_t*>(&b);
        }
        *reinterpret_cast<uint4*>(tile + tc::kmaj(r, c * 8, 32)) = u;
    }
}

// Shared-memory image of the network for one CTA: the three matrices as
// tcgen05 B operands (K-major, [N][K]) plus biases and the output layer.
struct Weights {
    alignas(128) __nv_bfloat16 W1[NH * KIN];      // B of layer 1: [out][in], in padded 20 -> 32 with zeros
    alignas(128) __nv_bfloat16 W2[NH * NH];       // B of layer 2: [out][in]
    alignas(128) __nv_bfloat16 W2T[NH * NH];      // B of the activation-gradient product: [in][out]
    float b1[NH], b2[NH], w3[NH], b3;
};

__device__ __forceinline__ void load_weights(Weights& w, const float* P, int tid, int nthreads)
{
    for (int e = tid; e < NH * KIN; e += nthreads) {
        const int o = e / KIN, i = e - o * KIN;
        w.W1[tc::kmaj(o, i, KIN)] = __float2bfloat16_rn(i < NIN ? P[OFF_W1 + o * NIN + i] : 0.0f);
    }
    for (int e = tid; e < NH * NH; e += nthreads) {
        const int o = e / NH, i = e - o * NH;
        const __nv_bfloat16 v = __float2bfloat16_rn(P[OFF_W2 + o * NH + i]);
        w.W2[tc::kmaj(o, i, NH)] = v;
        w.W2T[tc::kmaj(i, o, NH)] = v;
    }
    for (int e = tid; e < NH; e += nthreads) {
        w.b1[e] = bf16r(P[OFF_B1 + e]);
        w.b2[e] = P[OFF_B2 + e];
        w.w3[e] = bf16r(P[OFF_W3 + e]);
    }
    if (tid == 0) w.b3 = P[OFF_B3];
}

// D (TMEM columns at tmem_d) = A (TILE x 32, K-major) * B (32 x 32, K-major)^T:
// two K=16 steps, issued by one thread, completion signalled on mbar.
__device__ __forceinline__ void gemm_tile_k32(uint32_t tmem_d, const __nv_bfloat16* A, const __nv_bfloat16* B,
                                              uint64_t* mbar)
{
    constexpr uint32_t idesc = tc::idesc_bf16(TILE, NH);
    const uint32_t a0 = tc::smem_addr(A), b0 = tc::smem_addr(B);
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
        const uint64_t ad = tc::smem_desc(a0 + kk * 256, 128, (KIN / 8) * 128);
        const uint64_t bd = tc::smem_desc(b0 + kk * 256, 128, (KIN / 8) * 128);
        tc::mma_bf16(tmem_d, ad, bd, idesc, kk > 0 ? 1u : 0u);
    }
    tc::commit(mbar);
}

}  // namespace mlp
}  // namespace fin
