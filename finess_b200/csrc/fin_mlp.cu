// Troubled-cell indicator network: inference and training kernels on tcgen05
// tensor cores, an Adam update, and the C ABI around them (fin_mlp_*).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>
#include "finess_b200.h"
#include "fin_mlp.cuh"

using namespace fin;
using namespace fin::mlp;

namespace {

thread_local std::string g_mlp_err;
int mlp_fail(int code, const std::string& m)
{
    g_mlp_err = m;
    return code;
}
#define MCK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return mlp_fail(FIN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

__device__ __forceinline__ void mbar_setup(uint64_t* mbar)
{
    tc::mbar_init(mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Inference: z = network(X) for n rows of NIN features.  128 threads, one row
// each; CTAs stride over 128-row tiles.
// ---------------------------------------------------------------------------
struct FwdSmem {
    alignas(128) Weights w;
    alignas(128) __nv_bfloat16 Xs[TILE * KIN];
    alignas(128) __nv_bfloat16 G1s[TILE * NH];
    uint64_t mbar;
    uint32_t tmem;
    int abort;
};

__global__ void __launch_bounds__(TILE) k_mlp_forward(const float* X, long long n, const float* P, float* z,
                                                     unsigned int* status)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    FwdSmem& S = *reinterpret_cast<FwdSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    load_weights(S.w, P, tid, TILE);
    if (warp == 0) tc::tmem_alloc(&S.tmem, 64);
    if (tid == 0) {
        mbar_setup(&S.mbar);
        S.abort = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem;
    const uint32_t lane_base = uint32_t(warp * 32) << 16;
    uint32_t phase = 0;
    const long long ntiles = (n + TILE - 1) / TILE;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long row = t * TILE + tid;
        float xr[KIN];
#pragma unroll
        for (int k = 0; k < KIN; k++) xr[k] = (row < n && k < NIN) ? X[row * NIN + k] : 0.0f;
        store_row32(S.Xs, tid, xr);
        tc::fence_smem_to_async();
        __syncthreads();
        if (tid == 0) gemm_tile_k32(tmem, S.Xs, S.w.W1, &S.mbar);
        if (!tc::mbar_wait(&S.mbar, phase)) S.abort = 1;
        phase ^= 1;
        tc::fence_after_sync();
        float h[32];
        tc::tmem_ld32(tmem + lane_base, h);
#pragma unroll
        for (int o = 0; o < NH; o++) h[o] = gelu(h[o] + S.w.b1[o]);
        store_row32(S.G1s, tid, h);
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
        for (int o = 0; o < NH; o++) zz += S.w.w3[o] * gelu(h[o] + S.w.b2[o]);
        if (row < n) z[row] = zz;
        tc::fence_before_sync();
        __syncthreads();
        if (S.abort) break;
    }
    if (S.abort && tid == 0) atomicOr(status, 4u);
    __syncthreads();
    if (warp == 0) tc::tmem_free(tmem, 64);
}

// ---------------------------------------------------------------------------
// Training: forward + backward for one 128-row tile per CTA, gradients added
// into grad[NPARAM] (mean over the batch), loss sum into *loss.
// Products on tensor cores:
//   layer 1  D1[b][o] = X[b][:] . W1[o][:]
//   layer 2  D2[b][o] = G1[b][:] . W2[o][:]
//   dG1      D3[b][i] = dH2[b][:] . W2T[i][:]
//   weights  D4[r][c] = A4[r][:] . B4[c][:] over the 128 rows b, with
//            A4 = [dH2^T; dH1^T; 0] and B4 = [G1^T; X^T]: the (dH2, G1) block
//            is dW2 and the (dH1, X) block dW1.
// ---------------------------------------------------------------------------
struct TrainSmem {
    alignas(128) Weights w;
    alignas(128) __nv_bfloat16 Xs[TILE * KIN];
    alignas(128) __nv_bfloat16 G1s[TILE * NH];
    alignas(128) __nv_bfloat16 dH2s[TILE * NH];
    alignas(128) __nv_bfloat16 A4[128 * TILE];
    alignas(128) __nv_bfloat16 B4[64 * TILE];
    float red[NH * 3 + 2];
    uint64_t mbar;
    uint32_t tmem;
    int abort;
};

__global__ void __launch_bounds__(TILE) k_mlp_train(const float* X, const unsigned char* y, const int* idx, int nb,
                                                   const float* P, float* grad, float* loss, float pos_weight,
                                                   unsigned int* status)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    load_weights(S.w, P, tid, TILE);
    for (int e = tid; e < 128 * TILE; e += TILE) S.A4[e] = __float2bfloat16_rn(0.0f);
    for (int e = tid; e < NH * 3 + 2; e += TILE) S.red[e] = 0.0f;
    if (warp == 0) tc::tmem_alloc(&S.tmem, 256);
    if (tid == 0) {
        mbar_setup(&S.mbar);
        S.abort = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem;
    const uint32_t lane_base = uint32_t(warp * 32) << 16;
    uint32_t phase = 0;

    const int r = blockIdx.x * TILE + tid;
    const bool valid = r < nb;
    const int sample = valid ? idx[r] : 0;
    float x[KIN];
#pragma unroll
    for (int k = 0; k < KIN; k++) {
        x[k] = (valid && k < NIN) ? bf16r(X[size_t(sample) * NIN + k]) : 0.0f;
        const __nv_bfloat16 xb = __float2bfloat16_rn(x[k]);
        S.Xs[tc::kmaj(tid, k, KIN)] = xb;
        S.B4[tc::kmaj(32 + k, tid, TILE)] = xb;
    }
    tc::fence_smem_to_async();
    __syncthreads();
    // ---- forward ----
    if (tid == 0) gemm_tile_k32(tmem, S.Xs, S.w.W1, &S.mbar);
    if (!tc::mbar_wait(&S.mbar, phase)) S.abort = 1;
    phase ^= 1;
    tc::fence_after_sync();
    float a1[NH], g[NH];
    tc::tmem_ld32(tmem + lane_base, a1);
#pragma unroll
    for (int o = 0; o < NH; o++) {
        a1[o] += S.w.b1[o];
        const __nv_bfloat16 gb = __float2bfloat16_rn(gelu(a1[o]));
        S.G1s[tc::kmaj(tid, o, NH)] = gb;
        S.B4[tc::kmaj(o, tid, TILE)] = gb;
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    if (!S.abort && tid == 0) gemm_tile_k32(tmem + 32, S.G1s, S.w.W2, &S.mbar);
    if (!S.abort && !tc::mbar_wait(&S.mbar, phase)) S.abort = 1;
    phase ^= 1;
    tc::fence_after_sync();
    float a2[NH];
    tc::tmem_ld32(tmem + lane_base + 32, a2);
    float zz = S.w.b3;
#pragma unroll
    for (int o = 0; o < NH; o++) {
        a2[o] += S.w.b2[o];
        g[o] = gelu(a2[o]);
        zz += S.w.w3[o] * g[o];
    }
    // ---- loss: weighted binary cross-entropy on the logit, mean over the batch ----
    const float yy = valid ? float(y[sample]) : 0.0f;
    const float wgt = yy > 0.5f ? pos_weight : 1.0f;
    const float sp = fmaxf(zz, 0.0f) + log1pf(__expf(-fabsf(zz)));   // softplus(z)
    const float li = valid ? wgt * (sp - yy * zz) : 0.0f;
    const float pz = 1.0f / (1.0f + __expf(-zz));
    const float dz = valid ? wgt * (pz - yy) / float(nb) : 0.0f;
    // ---- backward through the output layer and layer 2 ----
    float dh2[NH];
#pragma unroll
    for (int o = 0; o < NH; o++) {
        dh2[o] = dz * S.w.w3[o] * gelu_grad(a2[o]);
        const __nv_bfloat16 db = __float2bfloat16_rn(dh2[o]);
        S.dH2s[tc::kmaj(tid, o, NH)] = db;
        S.A4[tc::kmaj(o, tid, TILE)] = db;
    }
    // per-CTA sums: dw3 = sum dz g2, db2 = sum dh2, db3 = sum dz, loss
#pragma unroll
    for (int o = 0; o < NH; o++) {
        float v1 = dz * g[o], v2 = dh2[o];
        for (int s = 16; s > 0; s >>= 1) {
            v1 += __shfl_xor_sync(0xffffffffu, v1, s);
            v2 += __shfl_xor_sync(0xffffffffu, v2, s);
        }
        if (lane == 0) {
            atomicAdd(&S.red[o], v1);
            atomicAdd(&S.red[NH + o], v2);
        }
    }
    {
        float v1 = dz, v2 = li;
        for (int s = 16; s > 0; s >>= 1) {
            v1 += __shfl_xor_sync(0xffffffffu, v1, s);
            v2 += __shfl_xor_sync(0xffffffffu, v2, s);
        }
        if (lane == 0) {
            atomicAdd(&S.red[3 * NH], v1);
            atomicAdd(&S.red[3 * NH + 1], v2);
        }
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    // ---- dG1 = dH2 W2 ----
    if (!S.abort && tid == 0) gemm_tile_k32(tmem + 64, S.dH2s, S.w.W2T, &S.mbar);
    if (!S.abort && !tc::mbar_wait(&S.mbar, phase)) S.abort = 1;
    phase ^= 1;
    tc::fence_after_sync();
    float dg1[NH];
    tc::tmem_ld32(tmem + lane_base + 64, dg1);
#pragma unroll
    for (int o = 0; o < NH; o++) {
        const float dh1 = dg1[o] * gelu_grad(a1[o]);
        S.A4[tc::kmaj(32 + o, tid, TILE)] = __float2bfloat16_rn(dh1);
        float v = dh1;
        for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
        if (lane == 0) atomicAdd(&S.red[2 * NH + o], v);
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    // ---- weight gradients: D4 = A4 B4^T over K = 128 rows ----
    if (!S.abort && tid == 0) {
        constexpr uint32_t idesc = tc::idesc_bf16(128, 64);
        const uint32_t a0 = tc::smem_addr(S.A4), b0 = tc::smem_addr(S.B4);
#pragma unroll
        for (int kk = 0; kk < TILE / 16; kk++) {
            const uint64_t ad = tc::smem_desc(a0 + kk * 256, 128, (TILE / 8) * 128);
            const uint64_t bd = tc::smem_desc(b0 + kk * 256, 128, (TILE / 8) * 128);
            tc::mma_bf16(tmem + 128, ad, bd, idesc, kk > 0 ? 1u : 0u);
        }
        tc::commit(&S.mbar);
    }
    if (!S.abort && !tc::mbar_wait(&S.mbar, phase)) S.abort = 1;
    phase ^= 1;
    tc::fence_after_sync();
    if (!S.abort && warp < 2) {
        float d[32];
        // warp 0: rows dH2^T (o), columns 0..31 = G1^T -> dW2[o][i]
        // warp 1: rows dH1^T (o), columns 32..63 = X^T -> dW1[o][k]
        tc::tmem_ld32(tmem + lane_base + 128 + (warp == 0 ? 0 : 32), d);
        if (warp == 0) {
#pragma unroll
            for (int i = 0; i < NH; i++) atomicAdd(&grad[OFF_W2 + lane * NH + i], d[i]);
        } else {
#pragma unroll
            for (int k = 0; k < NIN; k++) atomicAdd(&grad[OFF_W1 + lane * NIN + k], d[k]);
        }
    }
    __syncthreads();
    if (tid < NH) {
        atomicAdd(&grad[OFF_W3 + tid], S.red[tid]);
        atomicAdd(&grad[OFF_B2 + tid], S.red[NH + tid]);
        atomicAdd(&grad[OFF_B1 + tid], S.red[2 * NH + tid]);
    }
    if (tid == 0) {
        atomicAdd(&grad[OFF_B3], S.red[3 * NH]);
        atomicAdd(loss, S.red[3 * NH + 1]);
        if (S.abort) atomicOr(status, 4u);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tmem, 256);
}

// Adam (Kingma & Ba) on the FP32 master parameters.
__global__ void k_adam(float* P, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    m[i] = b1 * m[i] + (1.0f - b1) * g[i];
    v[i] = b2 * v[i] + (1.0f - b2) * g[i] * g[i];
    P[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

}  // namespace

struct fin_mlp {
    float* P;        // device parameters (FP32 master)
    float* grad;
    float* m;
    float* v;
    float* loss;
    unsigned int* status;
    cudaStream_t stream;
    long long step;
};

namespace {
int check_mlp_status(fin_mlp* h)
{
    unsigned int st = 0;
    MCK(cudaMemcpyAsync(&st, h->status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    if (st & 4u) return mlp_fail(FIN_ERR_CUDA, "tensor-core wait ran out of iterations");
    return FIN_OK;
}
// At least 29 KB per inference CTA: at most 8 CTAs share an SM, so their
// 64-column TMEM allocations (512 columns per SM) never have to wait.
size_t fwd_smem() { return std::max(sizeof(FwdSmem), size_t(29 * 1024)); }
size_t train_smem() { return sizeof(TrainSmem); }
}  // namespace

extern "C" {

int fin_mlp_nparam(void) { return NPARAM; }
const char* fin_mlp_last_error(void) { return g_mlp_err.c_str(); }

int fin_mlp_create(const float* params, unsigned long long seed, fin_mlp** out)
{
    if (!out) return mlp_fail(FIN_ERR_ARG, "null out");
    *out = nullptr;
    std::vector<float> p0(NPARAM, 0.0f);
    if (params) {
        memcpy(p0.data(), params, NPARAM * sizeof(float));
    } else {
        // He-style uniform initialisation, biases zero.
        std::mt19937_64 rng(seed);
        auto fill = [&](int off, int n, int fan_in) {
            std::uniform_real_distribution<float> U(-std::sqrt(6.0f / fan_in), std::sqrt(6.0f / fan_in));
            for (int i = 0; i < n; i++) p0[off + i] = U(rng);
        };
        fill(OFF_W1, NH * NIN, NIN);
        fill(OFF_W2, NH * NH, NH);
        fill(OFF_W3, NH, NH);
    }
    fin_mlp* h = new fin_mlp();
    memset(h, 0, sizeof(*h));
    auto fail = [&](cudaError_t e) {
        cudaFree(h->P); cudaFree(h->grad); cudaFree(h->m); cudaFree(h->v); cudaFree(h->loss);
        if (h->stream) cudaStreamDestroy(h->stream);
        delete h;
        return mlp_fail(FIN_ERR_CUDA, cudaGetErrorString(e));
    };
    cudaError_t e;
    if ((e = cudaMalloc(&h->P, NPARAM * sizeof(float))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&h->grad, NPARAM * sizeof(float))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&h->m, NPARAM * sizeof(float))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&h->v, NPARAM * sizeof(float))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&h->loss, 64)) != cudaSuccess) return fail(e);
    h->status = reinterpret_cast<unsigned int*>(h->loss + 8);
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(h->P, p0.data(), NPARAM * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(h->m, 0, NPARAM * sizeof(float))) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(h->v, 0, NPARAM * sizeof(float))) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(h->loss, 0, 64)) != cudaSuccess) return fail(e);
    if ((e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, int(fwd_smem()))) != cudaSuccess) return fail(e);
    if ((e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(train_smem()))) != cudaSuccess) return fail(e);
    *out = h;
    return FIN_OK;
}

int fin_mlp_destroy(fin_mlp* h)
{
    if (!h) return FIN_OK;
    cudaStreamSynchronize(h->stream);
    cudaFree(h->P); cudaFree(h->grad); cudaFree(h->m); cudaFree(h->v); cudaFree(h->loss);
    cudaStreamDestroy(h->stream);
    delete h;
    return FIN_OK;
}

int fin_mlp_get_params(fin_mlp* h, float* out)
{
    if (!h || !out) return mlp_fail(FIN_ERR_ARG, "null argument");
    MCK(cudaMemcpyAsync(out, h->P, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    return FIN_OK;
}

int fin_mlp_set_params(fin_mlp* h, const float* in)
{
    if (!h || !in) return mlp_fail(FIN_ERR_ARG, "null argument");
    MCK(cudaMemcpyAsync(h->P, in, NPARAM * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    return FIN_OK;
}

// Device parameter pointer (FP32, NPARAM) for kernels that run the network.
int fin_mlp_device_params(fin_mlp* h, const float** P)
{
    if (!h || !P) return mlp_fail(FIN_ERR_ARG, "null argument");
    *P = h->P;
    return FIN_OK;
}

int fin_mlp_forward(fin_mlp* h, const float* X_host, long long n, float* z_host)
{
    if (!h || !X_host || !z_host || n < 0) return mlp_fail(FIN_ERR_ARG, "bad argument");
    if (n == 0) return FIN_OK;
    float *dX = nullptr, *dz = nullptr;
    MCK(cudaMallocAsync(&dX, size_t(n) * NIN * sizeof(float), h->stream));
    MCK(cudaMallocAsync(&dz, size_t(n) * sizeof(float), h->stream));
    MCK(cudaMemcpyAsync(dX, X_host, size_t(n) * NIN * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemsetAsync(h->status, 0, sizeof(unsigned int), h->stream));
    const long long tiles = (n + TILE - 1) / TILE;
    const int grid = int(std::min<long long>(tiles, 148 * 4));
    k_mlp_forward<<<grid, TILE, fwd_smem(), h->stream>>>(dX, n, h->P, dz, h->status);
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(z_host, dz, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaFreeAsync(dX, h->stream));
    MCK(cudaFreeAsync(dz, h->stream));
    return check_mlp_status(h);
}

static int train_batches(fin_mlp* h, const float* dX, const unsigned char* dy, const int* didx, long long n,
                         int batch, float pos_weight, bool update, float lr, float* loss_sum)
{
    for (long long b0 = 0; b0 < n; b0 += batch) {
        const int nb = int(std::min<long long>(batch, n - b0));
        MCK(cudaMemsetAsync(h->grad, 0, NPARAM * sizeof(float), h->stream));
        k_mlp_train<<<(nb + TILE - 1) / TILE, TILE, train_smem(), h->stream>>>(dX, dy, didx + b0, nb, h->P, h->grad,
                                                                                 h->loss, pos_weight, h->status);
        MCK(cudaGetLastError());
        if (update) {
            h->step++;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.0f - std::pow(b1, float(h->step)), c2 = 1.0f - std::pow(b2, float(h->step));
            k_adam<<<(NPARAM + 255) / 256, 256, 0, h->stream>>>(h->P, h->grad, h->m, h->v, NPARAM, lr, b1, b2, 1e-8f, c1, c2);
            MCK(cudaGetLastError());
        }
    }
    (void)loss_sum;
    return FIN_OK;
}

int fin_mlp_gradients(fin_mlp* h, const float* X_host, const unsigned char* y_host, long long n, float pos_weight,
                      float* grad_host, float* loss)
{
    if (!h || !X_host || !y_host || !grad_host || n <= 0 || n > (1ll << 30)) return mlp_fail(FIN_ERR_ARG, "bad argument");
    float* dX = nullptr;
    unsigned char* dy = nullptr;
    int* didx = nullptr;
    std::vector<int> idx(n);
    for (long long i = 0; i < n; i++) idx[i] = int(i);
    MCK(cudaMallocAsync(&dX, size_t(n) * NIN * sizeof(float), h->stream));
    MCK(cudaMallocAsync(&dy, size_t(n), h->stream));
    MCK(cudaMallocAsync(&didx, size_t(n) * sizeof(int), h->stream));
    MCK(cudaMemcpyAsync(dX, X_host, size_t(n) * NIN * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemcpyAsync(dy, y_host, size_t(n), cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemcpyAsync(didx, idx.data(), size_t(n) * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemsetAsync(h->loss, 0, sizeof(float), h->stream));
    MCK(cudaMemsetAsync(h->status, 0, sizeof(unsigned int), h->stream));
    int rc = train_batches(h, dX, dy, didx, n, int(n), pos_weight, false, 0.0f, nullptr);
    if (rc) return rc;
    MCK(cudaMemcpyAsync(grad_host, h->grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    if (loss) MCK(cudaMemcpyAsync(loss, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaFreeAsync(dX, h->stream));
    MCK(cudaFreeAsync(dy, h->stream));
    MCK(cudaFreeAsync(didx, h->stream));
    return check_mlp_status(h);
}

int fin_mlp_train(fin_mlp* h, const float* X_host, const unsigned char* y_host, long long n, int epochs, int batch,
                  float lr, float pos_weight, unsigned long long seed, float* epoch_loss)
{
    if (!h || !X_host || !y_host || n <= 0 || epochs < 1 || batch < TILE || n > (1ll << 30))
        return mlp_fail(FIN_ERR_ARG, "bad argument");
    float* dX = nullptr;
    unsigned char* dy = nullptr;
    int* didx = nullptr;
    MCK(cudaMallocAsync(&dX, size_t(n) * NIN * sizeof(float), h->stream));
    MCK(cudaMallocAsync(&dy, size_t(n), h->stream));
    MCK(cudaMallocAsync(&didx, size_t(n) * sizeof(int), h->stream));
    MCK(cudaMemcpyAsync(dX, X_host, size_t(n) * NIN * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemcpyAsync(dy, y_host, size_t(n), cudaMemcpyHostToDevice, h->stream));
    std::vector<int> idx(n);
    for (long long i = 0; i < n; i++) idx[i] = int(i);
    std::mt19937_64 rng(seed);
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(idx.begin(), idx.end(), rng);
        MCK(cudaMemcpyAsync(didx, idx.data(), size_t(n) * sizeof(int), cudaMemcpyHostToDevice, h->stream));
        MCK(cudaMemsetAsync(h->loss, 0, sizeof(float), h->stream));
        MCK(cudaMemsetAsync(h->status, 0, sizeof(unsigned int), h->stream));
        int rc = train_batches(h, dX, dy, didx, n, batch, pos_weight, true, lr, nullptr);
        if (rc) return rc;
        float l = 0.0f;
        MCK(cudaMemcpyAsync(&l, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        if ((rc = check_mlp_status(h))) return rc;
        if (epoch_loss) epoch_loss[ep] = l / float(n);
    }
    MCK(cudaFreeAsync(dX, h->stream));
    MCK(cudaFreeAsync(dy, h->stream));
    MCK(cudaFreeAsync(didx, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    return FIN_OK;
}

}  // extern "C"
