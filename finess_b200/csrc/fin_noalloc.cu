// ConstructL for callers that cannot allocate device memory.
//
// Some callers of this library must not call cudaMalloc: code that runs
// while the application's own allocator owns the device (a host framework
// with a fixed memory pool, or a real-time loop that forbids allocation once
// it is running), or code that only receives device pointers from another
// component and may not create a fin_solver, which allocates its state
// buffers.  fin_construct_l_noalloc serves them: it computes the same
// right-hand side as fin_construct_l, but the caller passes the input state
// and the output L as device memory, and every scratch buffer the
// computation needs lives in one file-scope device array below.  Nothing is
// allocated: no cudaMalloc, no cudaFree, no allocating library call.
//
// Scratch layout (doubles): input planes [5][NA_MAX_CELLS], output planes
// [5][NA_MAX_CELLS], then NA_SLOTS reduction slots (global wave speeds of
// the input, the status word).  Every GPU that loads this library holds the
// array (about 21 MB) until the process exits.
#include <cuda_runtime.h>
#include <cstring>
#include <mutex>
#include "finess_b200.h"
#include "fin_stage.cuh"

namespace {

using namespace fin;
// A type of this file's own, so the stage-kernel instantiations below are
// distinct (internal-linkage) kernels, not a second copy of the main ones.
struct NaCfg : TileCfg<15, 16, 256> {};

constexpr size_t NA_MAX_CELLS = size_t(1) << 18;   // 262,144 interior cells (e.g. 512 x 512)
constexpr size_t NA_SLOTS = 8;                      // [0..1] alpha x/y, [2..3] smax x/y, [4] status
constexpr size_t NA_SCRATCH_DOUBLES = 2 * MEQN * NA_MAX_CELLS + NA_SLOTS;

}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[NA_SCRATCH_DOUBLES];

namespace {

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
double* g_na_ptr[NA_MAX_DEVICES] = {};

// Reference ghosted AoS (i, j, m) on the device -> interior planes.
__global__ void k_na_aos_to_planes(const double* aos, double* planes, int mx, int my, int mbc, size_t plane)
{
    const size_t n = size_t(mx) * my;
    const int sy = my + 2 * mbc;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const int i = int(g / my), j = int(g - size_t(i) * my);
        const size_t src = (size_t(i + mbc) * sy + (j + mbc)) * MEQN;
#pragma unroll
        for (int m = 0; m < MEQN; m++) planes[m * plane + g] = aos[src + m];
    }
}

// Interior planes -> interior of the ghosted AoS output (ghosts untouched,
// as the reference leaves Lstar's ghost entries).
__global__ void k_na_planes_to_aos(const double* planes, double* aos, int mx, int my, int mbc, size_t plane)
{
    const size_t n = size_t(mx) * my;
    const int sy = my + 2 * mbc;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const int i = int(g / my), j = int(g - size_t(i) * my);
        const size_t dst = (size_t(i + mbc) * sy + (j + mbc)) * MEQN;
#pragma unroll
        for (int m = 0; m < MEQN; m++) aos[dst + m] = planes[m * plane + g];
    }
}

// GlobalWaveSpd (lib/2d/GlobalWaveSpd.cpp:52-78): block max, one atomic per
// block; a non-finite speed sets bit 0 of the status word, as in the main
// library's k_wave_spd_max.
__global__ void k_na_wave_spd_max(const double* q, int mx, int my, size_t plane, double gamma, double* alpha_out,
                                  unsigned int* status)
{
    __shared__ double red[2][32];
    double ax = 0.0, ay = 0.0;
    bool nonfinite = false;
    const size_t n = size_t(mx) * my;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        double Q[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) Q[m] = q[m * plane + g];
        const double Qy[MEQN] = {Q[0], Q[2], Q[1], Q[3], Q[4]};
        const double sx = Euler::cell_speed(Euler::cell(gamma, Q));
        const double sy = Euler::cell_speed(Euler::cell(gamma, Qy));
        if (!(sx <= 1e300) || !(sy <= 1e300)) nonfinite = true;
        if (sx <= 1e300) ax = Max(ax, sx);
        if (sy <= 1e300) ay = Max(ay, sy);
    }
    if (nonfinite) atomicOr(status, 1u);
    for (int o = 16; o > 0; o >>= 1) {
        ax = Max(ax, __shfl_xor_sync(0xffffffffu, ax, o));
        ay = Max(ay, __shfl_xor_sync(0xffffffffu, ay, o));
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = ax; red[1][w] = ay; }
    __syncthreads();
    if (threadIdx.x < 2) {
        double v = 0.0;
        for (int k = 0; k < nw; k++) v = Max(v, red[threadIdx.x][k]);
        atomic_max_nonneg(alpha_out + threadIdx.x, v);
    }
}

template <int VER, bool P2>
cudaError_t na_set_smem_attr()
{
    return cudaFuncSetAttribute(k_stage<double, VER, P2, NaCfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(NaCfg::smem_bytes<double>()));
}

// Once per device, with that device current: the device address of the
// scratch array (its host-side name is only a stand-in, not a device
// address) and the stage kernels' shared-memory attribute.
int na_setup(double** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return FIN_ERR_CUDA;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return FIN_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
        double* ptr = nullptr;
        if (cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return FIN_ERR_CUDA;
        if (na_set_smem_attr<FIN_WENO_JS, true>() != cudaSuccess ||
            na_set_smem_attr<FIN_WENO_JS, false>() != cudaSuccess ||
            na_set_smem_attr<FIN_WENO_Z, true>() != cudaSuccess ||
            na_set_smem_attr<FIN_WENO_Z, false>() != cudaSuccess ||
            na_set_smem_attr<FIN_WENO_FD, true>() != cudaSuccess)
            return FIN_ERR_CUDA;
        g_na_ptr[dev] = ptr;
    }
    *out = g_na_ptr[dev];
    return FIN_OK;
}

template <int VER, bool P2>
void na_launch_stage(const StageArgs& a, cudaStream_t st)
{
    dim3 grid((a.my + NaCfg::TJ - 1) / NaCfg::TJ, (a.mx + NaCfg::TI - 1) / NaCfg::TI);
    k_stage<double, VER, P2, NaCfg><<<grid, NaCfg::NT, NaCfg::smem_bytes<double>(), st>>>(a);
}

}  // namespace

extern "C" int fin_construct_l_noalloc(const fin_params* p, const double* q_dev, double* L_dev, void* stream,
                                       int check)
{
    if (!p || !q_dev || !L_dev) return FIN_ERR_ARG;
    if (p->physics != FIN_PHYS_EULER || p->meqn != 5 || p->space_order != 5) return FIN_ERR_UNSUPPORTED;
    if (p->weno_version != FIN_WENO_JS && p->weno_version != FIN_WENO_Z && p->weno_version != FIN_WENO_FD)
        return FIN_ERR_ARG;
    if (p->mx < 1 || p->my < 1 || p->mbc < 3 || p->source_term) return FIN_ERR_ARG;
    if (!(p->xhigh > p->xlow) || !(p->yhigh > p->ylow)) return FIN_ERR_ARG;
    for (int b : {p->bc_xlow, p->bc_xhigh, p->bc_ylow, p->bc_yhigh})
        if (b != FIN_BC_PERIODIC && b != FIN_BC_TRANSMISSIVE) return FIN_ERR_ARG;
    if ((p->bc_xlow == FIN_BC_PERIODIC) != (p->bc_xhigh == FIN_BC_PERIODIC) ||
        (p->bc_ylow == FIN_BC_PERIODIC) != (p->bc_yhigh == FIN_BC_PERIODIC))
        return FIN_ERR_ARG;
    if ((p->bc_xlow == FIN_BC_PERIODIC && p->mx < 3) || (p->bc_ylow == FIN_BC_PERIODIC && p->my < 3))
        return FIN_ERR_ARG;
    if (p->precision != FIN_PREC_FP64) return FIN_ERR_UNSUPPORTED;
    const size_t n = size_t(p->mx) * size_t(p->my);
    if (n > NA_MAX_CELLS) return FIN_ERR_SIZE;

    // An error left pending by the caller's earlier CUDA work stays where it
    // is (peeked, not cleared) and this call launches nothing.
    if (cudaPeekAtLastError() != cudaSuccess) return FIN_ERR_CUDA;
    double* scratch = nullptr;
    int rc = na_setup(&scratch);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* in_planes = scratch;
    double* out_planes = scratch + MEQN * NA_MAX_CELLS;
    double* slots = scratch + 2 * MEQN * NA_MAX_CELLS;
    const size_t plane = NA_MAX_CELLS;

    // The slots keep the previous call's values: the maxima must start at 0.
    if (cudaMemsetAsync(slots, 0, NA_SLOTS * sizeof(double), st) != cudaSuccess) return FIN_ERR_CUDA;
    int blocks = int((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    unsigned int* status = reinterpret_cast<unsigned int*>(slots + 4);
    k_na_aos_to_planes<<<blocks, 256, 0, st>>>(q_dev, in_planes, p->mx, p->my, p->mbc, plane);
    if (cudaGetLastError() != cudaSuccess) return FIN_ERR_CUDA;
    if (p->global_alpha) {
        k_na_wave_spd_max<<<blocks, 256, 0, st>>>(in_planes, p->mx, p->my, plane, p->gamma, slots, status);
        if (cudaGetLastError() != cudaSuccess) return FIN_ERR_CUDA;
    }

    StageArgs a;
    memset(&a, 0, sizeof(a));
    a.qin = in_planes;
    a.A = nullptr; a.B = nullptr;
    a.qout = out_planes;
    a.a1 = 0.0; a.a2 = 0.0; a.bdt = 1.0;
    a.mx = p->mx; a.my = p->my;
    a.plane = plane;
    a.rdx = 1.0 / ((p->xhigh - p->xlow) / p->mx);
    a.rdy = 1.0 / ((p->yhigh - p->ylow) / p->my);
    a.gamma = p->gamma;
    a.eps = p->epsilon;
    a.pw = p->power_param;
    a.alpha_scaling = p->alpha_scaling;
    a.gamma_f = float(a.gamma);
    a.eps_f = float(a.eps);
    a.pw_f = float(a.pw);
    a.alpha_scaling_f = float(a.alpha_scaling);
    a.alpha_in = p->global_alpha ? slots : nullptr;
    a.status = status;
    a.bc[0] = p->bc_xlow; a.bc[1] = p->bc_xhigh; a.bc[2] = p->bc_ylow; a.bc[3] = p->bc_yhigh;
    const bool p2 = p->power_param == 2.0;
    if (p->weno_version == FIN_WENO_JS) {
        if (p2) na_launch_stage<FIN_WENO_JS, true>(a, st); else na_launch_stage<FIN_WENO_JS, false>(a, st);
    } else if (p->weno_version == FIN_WENO_Z) {
        if (p2) na_launch_stage<FIN_WENO_Z, true>(a, st); else na_launch_stage<FIN_WENO_Z, false>(a, st);
    } else {
        na_launch_stage<FIN_WENO_FD, true>(a, st);
    }
    if (cudaGetLastError() != cudaSuccess) return FIN_ERR_CUDA;
    k_na_planes_to_aos<<<blocks, 256, 0, st>>>(out_planes, L_dev, p->mx, p->my, p->mbc, plane);
    if (cudaGetLastError() != cudaSuccess) return FIN_ERR_CUDA;
    if (!check) return FIN_OK;
    // The caller asked for the status: wait for the stream and read the
    // status word (a 4-byte copy into this stack variable; the driver stages
    // it, nothing is allocated).
    unsigned int hst = 0;
    if (cudaMemcpyAsync(&hst, status, sizeof(hst), cudaMemcpyDeviceToHost, st) != cudaSuccess) return FIN_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return FIN_ERR_CUDA;
    if (hst & 1u) return FIN_ERR_NONFINITE;
    return FIN_OK;
}
