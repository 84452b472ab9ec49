// Host driver and C ABI of the ideal-MHD path (the reference's apps/2d/mhd
// application: lib/2d/ConstructL.cpp with the MHD callbacks, the A3
// Hamilton-Jacobi update, constrained transport, apps/2d/mhd/lib/
// FinSolveRK.cpp's SSP-RK3 with GetCFL.cpp's CFL number).
//
// One fin_mhd owns one problem on the current CUDA device: four 9-plane FP64
// state buffers (q^n, two stage registers, q^{n+1}: the accept/reject logic of
// FinSolveRK.cpp:86-357 keeps q^n intact until the CFL check), reduction
// slots and a stream.  Each stage is one launch of k_mhd_stage (fin_mhd.cuh);
// per step the host reads back the face-speed maxima and the status word.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>
#include "finess_b200.h"
#include "fin_weno_face.cuh"
#include "fin_mhd.cuh"
#include "fin_mhd_hyb.cuh"

using namespace fin;

namespace {

thread_local std::string g_mhd_err = "";

int merr(int code, const std::string& msg)
{
    g_mhd_err = msg;
    return code;
}

#define MCK(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return merr(FIN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

// Tile of the stage kernel: 15 x 16 cells, 511 faces.  Threads per block,
// measured on B200 at 2048^2 (stage ms, fast and slow pairs merged): FP64
// 256 threads with up to 255 registers and no spills 2.58, 512 threads at
// 128 registers (~500 B spilled, missing L1 beside 160 KB of shared memory)
// 2.71.  FP32 and the hybrid form: 256 threads at 128 registers, two blocks
// per SM, so that one block's loads and barriers overlap the other's
// arithmetic (1024^2, stage ms: FP32 0.268 against 0.323 for one 512-thread
// block per SM; hybrid with no troubled face 0.186 against 0.246).
#ifndef FIN_MHD_NT64
#define FIN_MHD_NT64 256
#endif
#ifndef FIN_MHD_NT32
#define FIN_MHD_NT32 256
#endif
#ifndef FIN_MHD_MINB32
#define FIN_MHD_MINB32 2
#endif
#ifndef FIN_MHD_NTH
#define FIN_MHD_NTH 256
#endif
#ifndef FIN_MHD_MINBH
#define FIN_MHD_MINBH 2
#endif
template <class R, bool HYB> struct MCfgOf { using T = MhdCfg<15, 16, FIN_MHD_NT64>; };
template <> struct MCfgOf<float, false> { using T = MhdCfg<15, 16, FIN_MHD_NT32, FIN_MHD_MINB32>; };
template <> struct MCfgOf<float, true> { using T = MhdCfg<15, 16, FIN_MHD_NTH, FIN_MHD_MINBH>; };

// Reduction slots (doubles): face-speed maxima of the step, then per state
// buffer its GlobalWaveSpd maxima and its HJ speeds, the status word, and the
// divergence diagnostic.
// Buffer 4 is the hybrid form's judge buffer.  SMAX_ALT keeps the hybrid
// attempt's face-speed maxima while a judge step recomputes with full WENO;
// DIFF receives the judge's max |q_hybrid - q_full| and max |q_full|.
enum { MNBUF = 5, MS_SMAX = 0, MS_ALPHA = 2, MS_HJ = MS_ALPHA + 2 * MNBUF, MS_STATUS = MS_HJ + 2 * MNBUF,
       MS_DIV = MS_STATUS + 1, MS_SMAX_ALT = MS_DIV + 1, MS_DIFF = MS_SMAX_ALT + 2, MS_N = MS_DIFF + 2 };
// The indicator's tile (the stage kernel's 15 x 16, 256 threads).
using ICfg = MhdCfg<15, 16, 256>;

int grid_blocks(size_t n)
{
    size_t b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return int(b);
}

}  // namespace

struct fin_mhd {
    fin_params p;
    double dx, dy;
    size_t plane;
    double* q[MNBUF];       // 9-plane state buffers; q[cur] holds q^n
    int cur;
    double* slots;
    unsigned int* status;
    double* h_slots;        // pinned mirror
    double* d_aos;          // staging for the reference ghosted layout (q then aux)
    double* d_face_x;
    double* d_face_y;
    cudaStream_t stream;
    cudaEvent_t ev0, ev1, kev[6];
    bool time_kernels;
    double kernel_ms;
    long long kernel_launches;
    double last_ms;
    double t;
    bool max_valid;         // slots hold the maxima of q[cur]
    long long launches;
    // hybrid form
    float* mlpP;            // network parameters on the device
    unsigned* flags;        // troubled-face bit masks of the current indicator pass
    unsigned long long* ind_count;
    float zthr;
    int judge_every;
    double judge_tol;
    int ind_every, ind_since, hyb_off;
    bool judge_pending;
    long long hstep, judges, reverts, troubled_last, faces;
    cudaEvent_t iev[2];
    bool ind_timed;
    double ind_ms;
    long long ind_launches;
};

namespace fin {

__global__ void k_mhd_state_max(const double* q, int mx, int my, size_t plane, double gamma, double* alpha_out,
                                double* hj_out, unsigned int* status)
{
    __shared__ double red[4][32];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    bool nonfinite = false;
    const size_t n = size_t(mx) * my;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        double Q[MHD_NQ];
#pragma unroll
        for (int m = 0; m < MHD_NQ; m++) Q[m] = q[m * plane + g];
        const double ir = 1.0 / Q[0];
        const double u1 = Q[1] * ir, u2 = Q[2] * ir, u3 = Q[3] * ir;
        const double Bsq = Q[5] * Q[5] + Q[6] * Q[6] + Q[7] * Q[7];
        const double press = (gamma - 1.0) * (Q[4] - 0.5 * Q[0] * (u1 * u1 + u2 * u2 + u3 * u3) - 0.5 * Bsq);
        const double a2 = fabs(gamma * press * ir);
        const double t = a2 + Bsq * ir;
        const double cf = sqrt(0.5 * (t + sqrt(fabs(t * t - 4.0 * a2 * (Q[5] * Q[5]) * ir))));
        const double s[4] = {Max(fabs(u1 - cf), fabs(u1 + cf)), Max(fabs(u2 - cf), fabs(u2 + cf)), fabs(u1),
                             fabs(u2)};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (s[k] <= 1e300) v[k] = Max(v[k], s[k]);
            else nonfinite = true;
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] = Max(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 4; k++) red[k][w] = v[k];
    if (nonfinite) atomicOr(status, 1u);
    __syncthreads();
    if (threadIdx.x < 4) {
        double r = 0.0;
        for (int k = 0; k < nw; k++) r = Max(r, red[threadIdx.x][k]);
        atomic_max_nonneg((threadIdx.x < 2 ? alpha_out : hj_out) + (threadIdx.x & 1), r);
    }
}

__global__ void k_mhd_after_step(double* q, int mx, int my, size_t plane, double ct_y, double ct_x)
{
    const size_t n = size_t(mx) * my;
    const double* A = q + 8 * plane;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const int i = int(g / my), j = int(g - size_t(i) * my);
        auto at = [&](int ii, int jj) {
            return A[size_t(bc_remap(ii, mx, FIN_BC_PERIODIC, FIN_BC_PERIODIC)) * my +
                     bc_remap(jj, my, FIN_BC_PERIODIC, FIN_BC_PERIODIC)];
        };
        q[5 * plane + g] = ct_y * (at(i, j - 2) - 8 * at(i, j - 1) + 8 * at(i, j + 1) - at(i, j + 2));
        q[6 * plane + g] = ct_x * (at(i - 2, j) - 8 * at(i - 1, j) + 8 * at(i + 1, j) - at(i + 2, j));
    }
}

__global__ void k_mhd_div_b(const double* q, int mx, int my, size_t plane, double rdx, double rdy, double* out)
{
    __shared__ double red[32];
    double v = 0.0;
    const size_t n = size_t(mx) * my;
    const double* B1 = q + 5 * plane;
    const double* B2 = q + 6 * plane;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const int i = int(g / my), j = int(g - size_t(i) * my);
        auto at = [&](const double* P, int ii, int jj) {
            return P[size_t(bc_remap(ii, mx, FIN_BC_PERIODIC, FIN_BC_PERIODIC)) * my +
                     bc_remap(jj, my, FIN_BC_PERIODIC, FIN_BC_PERIODIC)];
        };
        const double dB1 = (at(B1, i - 2, j) - 8 * at(B1, i - 1, j) + 8 * at(B1, i + 1, j) - at(B1, i + 2, j)) *
                           (rdx / 12.0);
        const double dB2 = (at(B2, i, j - 2) - 8 * at(B2, i, j - 1) + 8 * at(B2, i, j + 1) - at(B2, i, j + 2)) *
                           (rdy / 12.0);
        const double d = fabs(dB1 + dB2);
        v = d <= 1e300 ? Max(v, d) : v;
    }
    for (int o = 16; o > 0; o >>= 1) v = Max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int k = 0; k < int(blockDim.x >> 5); k++) r = Max(r, red[k]);
        atomic_max_nonneg(out, r);
    }
}

// max |a - b| and max |b| over the 9 planes (judge step); a NaN difference wins.
__global__ void k_mhd_max_diff(const double* a, const double* b, size_t plane, size_t n, double* out)
{
    __shared__ double red[2][32];
    double d = 0.0, m = 0.0;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
#pragma unroll
        for (int c = 0; c < MHD_NP; c++) {
            const double va = a[c * plane + g], vb = b[c * plane + g];
            const double dd = fabs(va - vb);
            d = dd > d || dd != dd ? dd : d;
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

// Reference ghosted AoS q (8 components) and aux (1) -> the 9 interior planes.
__global__ void k_mhd_aos_to_planes(const double* q, const double* aux, double* planes, int mx, int my, int mbc,
                                    size_t plane)
{
    const size_t n = size_t(mx) * my;
    const int sy = my + 2 * mbc;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const int i = int(g / my), j = int(g - size_t(i) * my);
        const size_t c = size_t(i + mbc) * sy + (j + mbc);
#pragma unroll
        for (int m = 0; m < MHD_NQ; m++) planes[m * plane + g] = q[c * MHD_NQ + m];
        planes[8 * plane + g] = aux[c];
    }
}

// 9 planes -> ghosted AoS q and aux with every ghost the periodic image (what
// the Orszag-Tang SetBndValues leaves); planes with fewer than 9 components
// (nplanes = 8) leave aux untouched.
__global__ void k_mhd_planes_to_aos(const double* planes, double* q, double* aux, int mx, int my, int mbc,
                                    size_t plane, int interior_only)
{
    const int sx = mx + 2 * mbc, sy = my + 2 * mbc;
    const size_t n = size_t(sx) * sy;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
        const int ii = int(e / sy), jj = int(e - size_t(ii) * sy);
        const bool in = ii >= mbc && ii < mbc + mx && jj >= mbc && jj < mbc + my;
        if (interior_only && !in) continue;
        const int gi = bc_remap(ii - mbc, mx, FIN_BC_PERIODIC, FIN_BC_PERIODIC);
        const int gj = bc_remap(jj - mbc, my, FIN_BC_PERIODIC, FIN_BC_PERIODIC);
        const size_t g = size_t(gi) * my + gj;
#pragma unroll
        for (int m = 0; m < MHD_NQ; m++) q[e * MHD_NQ + m] = planes[m * plane + g];
        if (aux) aux[e] = planes[8 * plane + g];
    }
}

}  // namespace fin

namespace {

double* alpha_slot(fin_mhd* s, int b) { return s->slots + MS_ALPHA + 2 * b; }
double* hj_slot(fin_mhd* s, int b) { return s->slots + MS_HJ + 2 * b; }

MhdArgs base_args(fin_mhd* s)
{
    MhdArgs a;
    memset(&a, 0, sizeof(a));
    const fin_params& p = s->p;
    a.mx = p.mx;
    a.my = p.my;
    a.plane = s->plane;
    a.rdx = 1.0 / s->dx;
    a.rdy = 1.0 / s->dy;
    a.ct_y = 1.0 / (12.0 * s->dy);
    a.ct_x = -1.0 / (12.0 * s->dx);
    a.ct = p.constrained_transport != 0;
    a.gamma = p.gamma;
    a.eps = p.epsilon;
    a.pw = p.power_param;
    a.alpha_scaling = p.alpha_scaling;
    a.gamma_f = float(p.gamma);
    a.eps_f = float(p.epsilon);
    a.pw_f = float(p.power_param);
    a.alpha_scaling_f = float(p.alpha_scaling);
    a.r_sqrt2 = 1.0 / sqrt(2.0);
    a.alf_deg = sin(atan(1.0) / 2.0);
    a.als_deg = cos(atan(1.0) / 2.0);
    a.status = s->status;
    return a;
}

template <class R, int VER, bool P2, bool HYB>
int launch_t(fin_mhd* s, const MhdArgs& a)
{
    using MCfg = typename MCfgOf<R, HYB>::T;
    constexpr size_t smem = HYB ? MCfg::template smem_bytes_hyb<R>() : MCfg::template smem_bytes<R>();
    static bool attr = false;
    if (!attr) {
        MCK(cudaFuncSetAttribute(k_mhd_stage<R, VER, P2, MCfg, HYB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem)));
        attr = true;
    }
    dim3 grid((s->p.my + MCfg::TJ - 1) / MCfg::TJ, (s->p.mx + MCfg::TI - 1) / MCfg::TI);
    k_mhd_stage<R, VER, P2, MCfg, HYB><<<grid, MCfg::NT, smem, s->stream>>>(a);
    s->launches++;
    MCK(cudaGetLastError());
    return FIN_OK;
}

template <class R, bool HYB>
int launch_r(fin_mhd* s, const MhdArgs& a)
{
    const bool p2 = s->p.power_param == 2.0;
    switch (s->p.weno_version) {
        case FIN_WENO_JS:
            return p2 ? launch_t<R, FIN_WENO_JS, true, HYB>(s, a) : launch_t<R, FIN_WENO_JS, false, HYB>(s, a);
        case FIN_WENO_Z:
            return p2 ? launch_t<R, FIN_WENO_Z, true, HYB>(s, a) : launch_t<R, FIN_WENO_Z, false, HYB>(s, a);
        default: return launch_t<R, FIN_WENO_FD, true, HYB>(s, a);
    }
}

// A stage in the solver's form: FP64, FP32, or (hybrid) FP32 with the
// per-face choice when a.flags is set and full FP32 WENO otherwise.
int launch_stage(fin_mhd* s, const MhdArgs& a, int k)
{
    if (s->time_kernels) MCK(cudaEventRecord(s->kev[2 * k], s->stream));
    int rc;
    if (s->p.precision == FIN_PREC_FP64) rc = launch_r<double, false>(s, a);
    else if (a.flags) rc = launch_r<float, true>(s, a);
    else rc = launch_r<float, false>(s, a);
    if (rc) return rc;
    if (s->time_kernels) MCK(cudaEventRecord(s->kev[2 * k + 1], s->stream));
    return FIN_OK;
}

int collect_times(fin_mhd* s, int nk)
{
    if (s->ind_timed) {
        float ms = 0.f;
        MCK(cudaEventSynchronize(s->iev[1]));
        MCK(cudaEventElapsedTime(&ms, s->iev[0], s->iev[1]));
        s->ind_ms += ms;
        s->ind_launches++;
        s->ind_timed = false;
    }
    if (!s->time_kernels) return FIN_OK;
    MCK(cudaEventSynchronize(s->kev[2 * nk - 1]));
    for (int k = 0; k < nk; k++) {
        float ms = 0.f;
        MCK(cudaEventElapsedTime(&ms, s->kev[2 * k], s->kev[2 * k + 1]));
        s->kernel_ms += ms;
        s->kernel_launches++;
    }
    return FIN_OK;
}

int compute_max(fin_mhd* s, int buf)
{
    MCK(cudaMemsetAsync(alpha_slot(s, buf), 0, 2 * sizeof(double), s->stream));
    MCK(cudaMemsetAsync(hj_slot(s, buf), 0, 2 * sizeof(double), s->stream));
    const size_t n = size_t(s->p.mx) * s->p.my;
    k_mhd_state_max<<<grid_blocks(n), 256, 0, s->stream>>>(s->q[buf], s->p.mx, s->p.my, s->plane, s->p.gamma,
                                                            alpha_slot(s, buf), hj_slot(s, buf), s->status);
    s->launches++;
    MCK(cudaGetLastError());
    return FIN_OK;
}

int read_status(fin_mhd* s, unsigned* st)
{
    MCK(cudaMemcpyAsync(s->h_slots, s->slots, MS_N * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MCK(cudaStreamSynchronize(s->stream));
    memcpy(st, s->h_slots + MS_STATUS, sizeof(*st));
    return FIN_OK;
}

int check_status(fin_mhd* s)
{
    unsigned st = 0;
    int rc = read_status(s, &st);
    if (rc) return rc;
    if (st & 1u) {
        MCK(cudaMemsetAsync(s->slots + MS_STATUS, 0, sizeof(double), s->stream));
        return merr(FIN_ERR_NONFINITE, "non-finite wave speed or state");
    }
    return FIN_OK;
}

size_t aos_q_elems(const fin_params& p) { return size_t(p.mx + 2 * p.mbc) * (p.my + 2 * p.mbc) * MHD_NQ; }
size_t aos_a_elems(const fin_params& p) { return size_t(p.mx + 2 * p.mbc) * (p.my + 2 * p.mbc); }

int ensure_aos(fin_mhd* s)
{
    if (!s->d_aos) MCK(cudaMalloc(&s->d_aos, (aos_q_elems(s->p) + aos_a_elems(s->p)) * sizeof(double)));
    return FIN_OK;
}

int upload(fin_mhd* s, const double* q_host, const double* aux_host, int buf)
{
    int rc = ensure_aos(s);
    if (rc) return rc;
    const size_t nq = aos_q_elems(s->p), na = aos_a_elems(s->p);
    MCK(cudaMemcpyAsync(s->d_aos, q_host, nq * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    MCK(cudaMemcpyAsync(s->d_aos + nq, aux_host, na * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    const size_t n = size_t(s->p.mx) * s->p.my;
    k_mhd_aos_to_planes<<<grid_blocks(n), 256, 0, s->stream>>>(s->d_aos, s->d_aos + nq, s->q[buf], s->p.mx,
                                                                s->p.my, s->p.mbc, s->plane);
    s->launches++;
    MCK(cudaGetLastError());
    return FIN_OK;
}

// The three stages of one step of size dt from q[cur] into q[out] through
// the stage registers q1, q2 (FinSolveRK.cpp:176-219 of the MHD application
// with SetRKinfo.cpp:50-64); flags: the hybrid form's troubled-face masks
// (nullptr: full WENO).
int stages(fin_mhd* s, double dt, int q1, int q2, int out, const unsigned* flags)
{
    const int qn = s->cur;
    MCK(cudaMemsetAsync(s->slots + MS_SMAX, 0, 2 * sizeof(double), s->stream));
    for (int b : {q1, q2, out}) {
        MCK(cudaMemsetAsync(alpha_slot(s, b), 0, 2 * sizeof(double), s->stream));
        MCK(cudaMemsetAsync(hj_slot(s, b), 0, 2 * sizeof(double), s->stream));
    }
    const bool ga = s->p.global_alpha != 0;
    int rc;
    MhdArgs a = base_args(s);
    a.smax_out = s->slots + MS_SMAX;
    a.flags = flags;
    // stage 1: Qstar = 1*Qnew + 0*Qstar + (1*dt) (L, Laux)(Qnew), then AfterStep
    a.qin = s->q[qn]; a.A = s->q[qn]; a.B = nullptr; a.qout = s->q[q1];
    a.a1 = 1.0; a.a2 = 0.0; a.bdt = 1.0 * dt;
    a.alpha_in = ga ? alpha_slot(s, qn) : nullptr; a.hj_in = hj_slot(s, qn);
    a.alpha_out = alpha_slot(s, q1); a.hj_out = hj_slot(s, q1);
    if ((rc = launch_stage(s, a, 0))) return rc;
    // stage 2: Qstar = 0.75 Qnew + 0.25 Qstar + (0.25 dt) (L, Laux)(Qstar)
    a.qin = s->q[q1]; a.A = s->q[qn]; a.B = s->q[q1]; a.qout = s->q[q2];
    a.a1 = 0.75; a.a2 = 0.25; a.bdt = 0.25 * dt;
    a.alpha_in = ga ? alpha_slot(s, q1) : nullptr; a.hj_in = hj_slot(s, q1);
    a.alpha_out = alpha_slot(s, q2); a.hj_out = hj_slot(s, q2);
    if ((rc = launch_stage(s, a, 1))) return rc;
    // stage 3: Qnew = (2/3) Qstar + (1/3) Qnew + ((2/3) dt) (L, Laux)(Qstar)
    a.qin = s->q[q2]; a.A = s->q[q2]; a.B = s->q[qn]; a.qout = s->q[out];
    a.a1 = 2.0e0 / 3.0e0; a.a2 = 1.0e0 / 3.0e0; a.bdt = (2.0e0 / 3.0e0) * dt;
    a.alpha_in = ga ? alpha_slot(s, q2) : nullptr; a.hj_in = hj_slot(s, q2);
    a.alpha_out = alpha_slot(s, out); a.hj_out = hj_slot(s, out);
    return launch_stage(s, a, 2);
}

// Troubled-face flags of q[buf] (fin_mhd_hyb.cuh).
int launch_indicator(fin_mhd* s, int buf)
{
    MhdIndArgs ia;
    memset(&ia, 0, sizeof(ia));
    ia.m = base_args(s);
    ia.m.qin = s->q[buf];
    ia.P = s->mlpP;
    ia.zthr = s->zthr;
    ia.flags = s->flags;
    ia.count = s->ind_count;
    static bool configured = false;
    const size_t smem = sizeof(MhdIndTile<ICfg>);
    if (!configured) {
        MCK(cudaFuncSetAttribute(k_mhd_indicator<ICfg>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        configured = true;
    }
    MCK(cudaMemsetAsync(s->ind_count, 0, sizeof(unsigned long long), s->stream));
    MCK(cudaMemsetAsync(s->flags, 0, flag_words(s->p.mx, s->p.my) * sizeof(unsigned), s->stream));
    const long long tiles = (long long)((s->p.mx + ICfg::TI - 1) / ICfg::TI) * ((s->p.my + ICfg::TJ - 1) / ICfg::TJ);
    const int grid = int(tiles < 148 * 3 ? tiles : 148 * 3);
    k_mhd_indicator<ICfg><<<grid, ICfg::NT, smem, s->stream>>>(ia);
    s->launches++;
    s->faces = (long long)(s->p.mx + 1) * s->p.my + (long long)s->p.mx * (s->p.my + 1);
    MCK(cudaGetLastError());
    return FIN_OK;
}

// One step from q[cur] into q[nxt].  Hybrid form with a network: flags from
// the indicator on q^n when due, FP32 stages with the per-face choice; every
// judge_every-th such step also the full-WENO FP32 step from the same q^n
// into q[4], compared on the device (settled by settle_judge).
int take_stages(fin_mhd* s, double dt, int nxt)
{
    const int q1 = (s->cur + 1) % 4, q2 = (s->cur + 2) % 4;
    s->judge_pending = false;
    MCK(cudaMemsetAsync(s->slots + MS_STATUS, 0, sizeof(double), s->stream));
    if (s->p.precision != FIN_PREC_HYBRID || !s->mlpP) return stages(s, dt, q1, q2, nxt, nullptr);
    if (s->hyb_off > 0) {
        s->hyb_off--;
        return stages(s, dt, q1, q2, nxt, nullptr);
    }
    int rc;
    if (s->ind_since < 0 || s->ind_since >= s->ind_every) {
        if (s->time_kernels) MCK(cudaEventRecord(s->iev[0], s->stream));
        if ((rc = launch_indicator(s, s->cur))) return rc;
        if (s->time_kernels) {
            MCK(cudaEventRecord(s->iev[1], s->stream));
            s->ind_timed = true;
        }
        s->ind_since = 0;
    }
    if ((rc = stages(s, dt, q1, q2, nxt, s->flags))) return rc;
    s->hstep++;
    if (s->judge_every > 0 && s->hstep % s->judge_every == 0) {
        MCK(cudaMemcpyAsync(s->slots + MS_SMAX_ALT, s->slots + MS_SMAX, 2 * sizeof(double), cudaMemcpyDeviceToDevice,
                            s->stream));
        const bool tk = s->time_kernels;   // the step's stage times stay those of the hybrid stages
        s->time_kernels = false;
        rc = stages(s, dt, q1, q2, 4, nullptr);
        s->time_kernels = tk;
        if (rc) return rc;
        MCK(cudaMemsetAsync(s->slots + MS_DIFF, 0, 2 * sizeof(double), s->stream));
        const size_t n = size_t(s->p.mx) * s->p.my;
        k_mhd_max_diff<<<grid_blocks(n), 256, 0, s->stream>>>(s->q[nxt], s->q[4], s->plane, n, s->slots + MS_DIFF);
        s->launches++;
        MCK(cudaGetLastError());
        s->judge_pending = true;
    }
    return FIN_OK;
}

// After get_cfl brought the slots to the host: settle a judge step.  The
// hybrid result stays (with its face-speed maxima) unless it differs from
// the full-WENO result by more than judge_tol (relative L-infinity); then
// the full result takes its place, its maxima give the CFL, and the
// indicator stays off for judge_every steps.
void settle_judge(fin_mhd* s, int nxt, double dt, double* cfl)
{
    if (!s->judge_pending) return;
    s->judges++;
    const double d = s->h_slots[MS_DIFF], m = s->h_slots[MS_DIFF + 1];
    const bool revert = !(d <= s->judge_tol * (m > 0 ? m : 1.0));
    double sm;
    if (revert) {
        s->reverts++;
        s->hyb_off = s->judge_every;
        s->ind_since = -1;
        std::swap(s->q[4], s->q[nxt]);
        cudaMemcpyAsync(alpha_slot(s, nxt), alpha_slot(s, 4), 2 * sizeof(double), cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(hj_slot(s, nxt), hj_slot(s, 4), 2 * sizeof(double), cudaMemcpyDeviceToDevice, s->stream);
        sm = Max(s->h_slots[MS_SMAX], s->h_slots[MS_SMAX + 1]);
    } else {
        sm = Max(s->h_slots[MS_SMAX_ALT], s->h_slots[MS_SMAX_ALT + 1]);
    }
    double c = -100.0;
    c = Max(c, dt * sm * (1.0 / s->dx + 1.0 / s->dy));
    *cfl = c;
}

// GetCFL of the MHD application (GetCFL.cpp:31-73): the largest
// dt*max(smax1, smax2)*(1/dx + 1/dy) over the cells equals that expression
// at the largest face speed, the rounded products being monotone.
int get_cfl(fin_mhd* s, double dt, double dtmax, double* cfl, bool* nonfinite)
{
    unsigned st = 0;
    int rc = read_status(s, &st);
    if (rc) return rc;
    *nonfinite = (st & 1u) != 0;
    if (st & 4u) return merr(FIN_ERR_CUDA, "a bounded tensor-core wait of the indicator ran out");
    if (dt > dtmax) return merr(FIN_ERR_DT_BOUNDS, "dt is out of bounds");
    const double sm = Max(s->h_slots[MS_SMAX], s->h_slots[MS_SMAX + 1]);
    double c = -100.0;
    c = Max(c, dt * sm * (1.0 / s->dx + 1.0 / s->dy));
    if (c > 1.0e8) return merr(FIN_ERR_CFL_BOUNDS, "CFL number is out of bounds");
    *cfl = c;
    return FIN_OK;
}

int validate(const fin_params* p)
{
    if (!p) return merr(FIN_ERR_ARG, "null params");
    if (p->physics != FIN_PHYS_MHD || p->meqn != 8 || p->maux != 1)
        return merr(FIN_ERR_ARG, "the MHD path needs physics FIN_PHYS_MHD, meqn 8 and maux 1");
    if (p->space_order != 5) return merr(FIN_ERR_UNSUPPORTED, "space_order must be 5");
    if (p->weno_version != FIN_WENO_JS && p->weno_version != FIN_WENO_Z && p->weno_version != FIN_WENO_FD)
        return merr(FIN_ERR_ARG, "Requested WENO Reconstruction not implemented.");
    if (p->time_stepping_method != FIN_TS_RK || p->time_order != 3)
        return merr(FIN_ERR_UNSUPPORTED, "the MHD path is built for SSP-RK3 (Runge-Kutta, time_order 3)");
    // ConstructHJ_L.cpp:70 asserts mbc >= 2 + r
    if (p->mbc < 5) return merr(FIN_ERR_ARG, "the MHD path needs mbc >= 5");
    if (p->mx < 5 || p->my < 5) return merr(FIN_ERR_ARG, "periodic directions shorter than the A3 halo");
    for (int b : {p->bc_xlow, p->bc_xhigh, p->bc_ylow, p->bc_yhigh})
        if (b != FIN_BC_PERIODIC) return merr(FIN_ERR_UNSUPPORTED, "the MHD path has doubly periodic boundaries");
    if (p->source_term) return merr(FIN_ERR_UNSUPPORTED, "source terms are not built");
    if (!(p->xhigh > p->xlow) || !(p->yhigh > p->ylow)) return merr(FIN_ERR_ARG, "empty domain");
    if (p->precision != FIN_PREC_FP64 && p->precision != FIN_PREC_FP32 && p->precision != FIN_PREC_HYBRID)
        return merr(FIN_ERR_ARG, "unknown precision form");
    return FIN_OK;
}

}  // namespace

extern "C" {

const char* fin_mhd_last_error(void) { return g_mhd_err.c_str(); }

int fin_mhd_destroy(fin_mhd* s)
{
    if (!s) return FIN_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (int b = 0; b < MNBUF; b++) cudaFree(s->q[b]);
    cudaFree(s->slots);
    cudaFree(s->d_aos);
    cudaFree(s->d_face_x);
    cudaFree(s->d_face_y);
    cudaFree(s->mlpP);
    cudaFree(s->flags);
    cudaFree(s->ind_count);
    if (s->h_slots) cudaFreeHost(s->h_slots);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    for (int k = 0; k < 6; k++)
        if (s->kev[k]) cudaEventDestroy(s->kev[k]);
    for (int k = 0; k < 2; k++)
        if (s->iev[k]) cudaEventDestroy(s->iev[k]);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return FIN_OK;
}

int fin_mhd_create(const fin_params* p, fin_mhd** out)
{
    if (!out) return merr(FIN_ERR_ARG, "null out");
    *out = nullptr;
    int rc = validate(p);
    if (rc) return rc;
    int dev = 0, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return merr(FIN_ERR_NO_DEVICE, "no CUDA device");
    MCK(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    MCK(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) return merr(FIN_ERR_NO_DEVICE, "libfinb200 is compiled for sm_100a (B200)");
    fin_mhd* s = new fin_mhd();
    memset(s, 0, sizeof(*s));
    s->p = *p;
    s->dx = (p->xhigh - p->xlow) / p->mx;
    s->dy = (p->yhigh - p->ylow) / p->my;
    s->plane = (size_t(p->mx) * p->my + 31) / 32 * 32;
    auto fail = [&](cudaError_t e, const char* what) {
        fin_mhd_destroy(s);
        return merr(FIN_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    cudaError_t e;
    const int nbuf = p->precision == FIN_PREC_HYBRID ? 5 : 4;
    for (int b = 0; b < nbuf; b++)
        if ((e = cudaMalloc(&s->q[b], MHD_NP * s->plane * sizeof(double))) != cudaSuccess)
            return fail(e, "cudaMalloc state");
    if (p->precision == FIN_PREC_HYBRID) {
        if ((e = cudaMalloc(&s->flags, flag_words(p->mx, p->my) * sizeof(unsigned))) != cudaSuccess)
            return fail(e, "cudaMalloc flags");
        if ((e = cudaMalloc(&s->ind_count, 16)) != cudaSuccess) return fail(e, "cudaMalloc counter");
        if ((e = cudaMemset(s->ind_count, 0, 16)) != cudaSuccess) return fail(e, "memset");
        s->judge_every = 50;
        s->judge_tol = 1e-3;
        s->ind_every = 1;
        s->ind_since = -1;
    }
    if ((e = cudaMalloc(&s->slots, MS_N * sizeof(double))) != cudaSuccess) return fail(e, "cudaMalloc slots");
    s->status = reinterpret_cast<unsigned int*>(s->slots + MS_STATUS);
    if ((e = cudaMallocHost(&s->h_slots, MS_N * sizeof(double))) != cudaSuccess) return fail(e, "cudaMallocHost");
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaEventCreate(&s->ev0)) != cudaSuccess) return fail(e, "event");
    if ((e = cudaEventCreate(&s->ev1)) != cudaSuccess) return fail(e, "event");
    for (int k = 0; k < 6; k++)
        if ((e = cudaEventCreate(&s->kev[k])) != cudaSuccess) return fail(e, "event");
    for (int k = 0; k < 2; k++)
        if ((e = cudaEventCreate(&s->iev[k])) != cudaSuccess) return fail(e, "event");
    if ((e = cudaMemsetAsync(s->slots, 0, MS_N * sizeof(double), s->stream)) != cudaSuccess) return fail(e, "memset");
    for (int b = 0; b < nbuf; b++)
        if ((e = cudaMemsetAsync(s->q[b], 0, MHD_NP * s->plane * sizeof(double), s->stream)) != cudaSuccess)
            return fail(e, "memset");
    if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return fail(e, "sync");
    *out = s;
    return FIN_OK;
}

int fin_mhd_set_state(fin_mhd* s, const double* q_host, const double* aux_host, double t)
{
    if (!s || !q_host || !aux_host) return merr(FIN_ERR_ARG, "null argument");
    MCK(cudaMemsetAsync(s->slots + MS_STATUS, 0, sizeof(double), s->stream));
    int rc = upload(s, q_host, aux_host, s->cur);
    if (rc) return rc;
    s->t = t;
    if ((rc = compute_max(s, s->cur))) return rc;
    s->max_valid = true;
    return check_status(s);
}

int fin_mhd_get_state(fin_mhd* s, double* q_host, double* aux_host, double* t)
{
    if (!s || !q_host) return merr(FIN_ERR_ARG, "null argument");
    int rc = ensure_aos(s);
    if (rc) return rc;
    const size_t nq = aos_q_elems(s->p), na = aos_a_elems(s->p);
    k_mhd_planes_to_aos<<<grid_blocks(na), 256, 0, s->stream>>>(s->q[s->cur], s->d_aos, s->d_aos + nq, s->p.mx,
                                                                s->p.my, s->p.mbc, s->plane, 0);
    s->launches++;
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(q_host, s->d_aos, nq * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    if (aux_host) MCK(cudaMemcpyAsync(aux_host, s->d_aos + nq, na * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MCK(cudaStreamSynchronize(s->stream));
    if (t) *t = s->t;
    return FIN_OK;
}

// One right-hand-side evaluation of (q_host, aux_host) with no update:
// outb receives L (8 planes) and Laux (plane 8).
static int rhs_eval(fin_mhd* s, const double* q_host, const double* aux_host, bool faces, int* outb_out)
{
    const fin_params& p = s->p;
    const int buf = (s->cur + 3) % 4, outb = (s->cur + 2) % 4;
    MCK(cudaMemsetAsync(s->slots + MS_STATUS, 0, sizeof(double), s->stream));
    int rc = upload(s, q_host, aux_host, buf);
    if (rc) return rc;
    if ((rc = compute_max(s, buf))) return rc;
    if (faces) {
        if (!s->d_face_x) MCK(cudaMalloc(&s->d_face_x, size_t(p.mx + 1) * p.my * sizeof(double)));
        if (!s->d_face_y) MCK(cudaMalloc(&s->d_face_y, size_t(p.mx) * (p.my + 1) * sizeof(double)));
    }
    MCK(cudaMemsetAsync(s->slots + MS_SMAX, 0, 2 * sizeof(double), s->stream));
    MhdArgs a = base_args(s);
    a.qin = s->q[buf];
    a.A = nullptr; a.B = nullptr; a.qout = s->q[outb];
    a.a1 = 0.0; a.a2 = 0.0; a.bdt = 1.0;
    a.ct = 0;
    a.alpha_in = p.global_alpha ? alpha_slot(s, buf) : nullptr;
    a.hj_in = hj_slot(s, buf);
    a.smax_out = s->slots + MS_SMAX;
    a.face_alpha_x = faces ? s->d_face_x : nullptr;
    a.face_alpha_y = faces ? s->d_face_y : nullptr;
    if ((rc = launch_stage(s, a, 0))) return rc;
    *outb_out = outb;
    return FIN_OK;
}

int fin_mhd_construct_l(fin_mhd* s, const double* q_host, const double* aux_host, double* L_host, double* smax_host)
{
    if (!s || !q_host || !aux_host || !L_host) return merr(FIN_ERR_ARG, "null argument");
    const fin_params& p = s->p;
    int outb, rc;
    if ((rc = rhs_eval(s, q_host, aux_host, smax_host != nullptr, &outb))) return rc;
    // L: interior of the ghosted output, ghosts untouched
    const size_t nq = aos_q_elems(p), na = aos_a_elems(p);
    MCK(cudaMemcpyAsync(s->d_aos, L_host, nq * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    k_mhd_planes_to_aos<<<grid_blocks(na), 256, 0, s->stream>>>(s->q[outb], s->d_aos, nullptr, p.mx, p.my, p.mbc,
                                                                s->plane, 1);
    s->launches++;
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(L_host, s->d_aos, nq * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MCK(cudaStreamSynchronize(s->stream));
    if (smax_host) {
        std::vector<double> fx(size_t(p.mx + 1) * p.my), fy(size_t(p.mx) * (p.my + 1));
        MCK(cudaMemcpyAsync(fx.data(), s->d_face_x, fx.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        MCK(cudaMemcpyAsync(fy.data(), s->d_face_y, fy.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        MCK(cudaStreamSynchronize(s->stream));
        // smax is dTensorBC3(mx+1, my+1, 2, mbc), max-accumulated (ConstructL.cpp:173,324)
        const int sy = p.my + 1 + 2 * p.mbc;
        auto at = [&](int i, int j, int m) -> double& {
            return smax_host[(size_t(i + p.mbc - 1) * sy + (j + p.mbc - 1)) * 2 + (m - 1)];
        };
        for (int i = 1; i <= p.mx + 1; i++)
            for (int j = 1; j <= p.my; j++) {
                double& d = at(i, j, 1);
                d = Max(d, fx[size_t(i - 1) * p.my + (j - 1)]);
            }
        for (int i = 1; i <= p.mx; i++)
            for (int j = 1; j <= p.my + 1; j++) {
                double& d = at(i, j, 2);
                d = Max(d, fy[size_t(i - 1) * (p.my + 1) + (j - 1)]);
            }
    }
    return check_status(s);
}

int fin_mhd_construct_hj_l(fin_mhd* s, const double* q_host, const double* aux_host, double* Laux_host)
{
    if (!s || !q_host || !aux_host || !Laux_host) return merr(FIN_ERR_ARG, "null argument");
    const fin_params& p = s->p;
    int outb, rc;
    if ((rc = rhs_eval(s, q_host, aux_host, false, &outb))) return rc;
    const size_t n = size_t(p.mx) * p.my;
    std::vector<double> h(n);
    MCK(cudaMemcpyAsync(h.data(), s->q[outb] + 8 * s->plane, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MCK(cudaStreamSynchronize(s->stream));
    const int sy = p.my + 2 * p.mbc;
    for (int i = 0; i < p.mx; i++)
        for (int j = 0; j < p.my; j++) Laux_host[size_t(i + p.mbc) * sy + (j + p.mbc)] = h[size_t(i) * p.my + j];
    return check_status(s);
}

int fin_mhd_after_step(fin_mhd* s, double* q_host, const double* aux_host)
{
    if (!s || !q_host || !aux_host) return merr(FIN_ERR_ARG, "null argument");
    const fin_params& p = s->p;
    if (!p.constrained_transport) return FIN_OK;
    const int buf = (s->cur + 3) % 4;
    int rc = upload(s, q_host, aux_host, buf);
    if (rc) return rc;
    const size_t n = size_t(p.mx) * p.my, nq = aos_q_elems(p), na = aos_a_elems(p);
    k_mhd_after_step<<<grid_blocks(n), 256, 0, s->stream>>>(s->q[buf], p.mx, p.my, s->plane, 1.0 / (12.0 * s->dy),
                                                             -1.0 / (12.0 * s->dx));
    MCK(cudaMemcpyAsync(s->d_aos, q_host, nq * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    k_mhd_planes_to_aos<<<grid_blocks(na), 256, 0, s->stream>>>(s->q[buf], s->d_aos, nullptr, p.mx, p.my, p.mbc,
                                                                s->plane, 1);
    s->launches += 2;
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(q_host, s->d_aos, nq * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MCK(cudaStreamSynchronize(s->stream));
    return FIN_OK;
}

int fin_mhd_step_fixed(fin_mhd* s, double dt, double* cfl_out)
{
    if (!s) return merr(FIN_ERR_ARG, "null solver");
    int rc;
    if (!s->max_valid && (rc = compute_max(s, s->cur))) return rc;
    const int nxt = (s->cur + 3) % 4;
    MCK(cudaEventRecord(s->ev0, s->stream));
    if ((rc = take_stages(s, dt, nxt))) return rc;
    MCK(cudaEventRecord(s->ev1, s->stream));
    double cfl = 0.0;
    bool nonfinite = false;
    if ((rc = get_cfl(s, dt, 1e300, &cfl, &nonfinite))) return rc;
    if ((rc = collect_times(s, 3))) return rc;
    settle_judge(s, nxt, dt, &cfl);
    if (nonfinite) return merr(FIN_ERR_NONFINITE, "non-finite wave speed or state");
    float ms = 0.f;
    MCK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    s->last_ms = ms;
    s->cur = nxt;
    if (s->ind_since >= 0) s->ind_since++;
    s->max_valid = true;
    s->t = s->t + dt;
    if (cfl_out) *cfl_out = cfl;
    return FIN_OK;
}

// apps/2d/mhd/lib/FinSolveRK.cpp:17-395 (time_order 3), stopping early after
// max_steps accepted steps.
int fin_mhd_advance(fin_mhd* s, double tend, double* dtv, int max_steps, int* nsteps_out)
{
    if (!s || !dtv) return merr(FIN_ERR_ARG, "null argument");
    const fin_params& p = s->p;
    const double CFL_max = p.max_cfl, CFL_target = p.desired_cfl;
    double t = s->t, dt = dtv[1], cfl = 0.0;
    double t_star = s->t;
    int n_step = 0, accepted = 0, rc = FIN_OK;
    if (!s->max_valid && (rc = compute_max(s, s->cur))) return rc;
    MCK(cudaEventRecord(s->ev0, s->stream));
    while (t < tend && accepted < max_steps) {
        int m_accept = 0;
        n_step = n_step + 1;
        if (n_step > p.nv) { rc = merr(FIN_ERR_NSTEPS, "Exceeded allowed # of time steps"); break; }
        const double t_old_q = s->t;
        while (m_accept == 0) {
            s->t = t;
            const double told = t;
            if (told + dt > tend) dt = tend - told;
            t = told + dt;
            const int nxt = (s->cur + 3) % 4;
            if ((rc = take_stages(s, dt, nxt))) goto done;
            bool nonfinite = false;
            if ((rc = get_cfl(s, dt, dtv[2], &cfl, &nonfinite))) goto done;
            if ((rc = collect_times(s, 3))) goto done;
            settle_judge(s, nxt, dt, &cfl);
            // Qnew.t after the stages (UpdateSoln.cpp:27 of the MHD application)
            t_star = 1.0 * s->t + 0.0 * t_star + 1.0 * dt;
            t_star = 0.75 * s->t + 0.25 * t_star + 0.25 * dt;
            const double t_new = (2.0e0 / 3.0e0) * t_star + (1.0e0 / 3.0e0) * s->t + (2.0e0 / 3.0e0) * dt;
            if (cfl > 0.0) dt = Min(dtv[2], dt * CFL_target / cfl);
            else dt = dtv[2];
            if (p.verbosity)
                printf("FinSolveRK2D ... Step%5d   CFL =%6.3f   dt =%11.3e   t =%11.3e\n", n_step, cfl, dt, t);
            if (cfl <= CFL_max && nonfinite) {
                rc = merr(FIN_ERR_NONFINITE, "non-finite wave speed or state in an accepted step");
                goto done;
            }
            if (cfl <= CFL_max) {
                m_accept = 1;
                s->cur = nxt;
                if (s->ind_since >= 0) s->ind_since++;
                s->t = t_new;
            } else {
                t = told;
                s->t = t_old_q;
                if (p.verbosity) printf("FinSolveRK2D rejecting step...CFL number too large\n");
            }
        }
        accepted++;
    }
    dtv[1] = dt;
done:
    {
        cudaError_t e1 = cudaEventRecord(s->ev1, s->stream);
        if (e1 == cudaSuccess) e1 = cudaEventSynchronize(s->ev1);
        float ms = 0.f;
        if (e1 == cudaSuccess) e1 = cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        s->last_ms = e1 == cudaSuccess ? ms : 0.0;
    }
    if (nsteps_out) *nsteps_out = accepted;
    return rc;
}

int fin_mhd_solve(fin_mhd* s, double tend, double* dtv, int* nsteps_out)
{
    return fin_mhd_advance(s, tend, dtv, 0x7fffffff, nsteps_out);
}

int fin_mhd_div_b(fin_mhd* s, double* max_div)
{
    if (!s || !max_div) return merr(FIN_ERR_ARG, "null argument");
    MCK(cudaMemsetAsync(s->slots + MS_DIV, 0, sizeof(double), s->stream));
    const size_t n = size_t(s->p.mx) * s->p.my;
    k_mhd_div_b<<<grid_blocks(n), 256, 0, s->stream>>>(s->q[s->cur], s->p.mx, s->p.my, s->plane, 1.0 / s->dx,
                                                        1.0 / s->dy, s->slots + MS_DIV);
    s->launches++;
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(max_div, s->slots + MS_DIV, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MCK(cudaStreamSynchronize(s->stream));
    return FIN_OK;
}

int fin_mhd_set_indicator(fin_mhd* s, const float* params, float z_threshold, int judge_every, double judge_tol)
{
    if (!s || !params) return merr(FIN_ERR_ARG, "null argument");
    if (s->p.precision != FIN_PREC_HYBRID) return merr(FIN_ERR_ARG, "the solver was not created in the hybrid form");
    if (judge_every < 0) return merr(FIN_ERR_ARG, "judge_every must be >= 0");
    if (!s->mlpP) MCK(cudaMalloc(&s->mlpP, mlp::NPARAM * sizeof(float)));
    MCK(cudaMemcpyAsync(s->mlpP, params, mlp::NPARAM * sizeof(float), cudaMemcpyHostToDevice, s->stream));
    MCK(cudaStreamSynchronize(s->stream));
    s->zthr = z_threshold;
    s->judge_every = judge_every;
    s->judge_tol = judge_tol;
    s->hyb_off = 0;
    s->ind_since = -1;
    return FIN_OK;
}

int fin_mhd_set_indicator_every(fin_mhd* s, int every)
{
    if (!s) return merr(FIN_ERR_ARG, "null argument");
    if (every < 1) return merr(FIN_ERR_ARG, "the indicator period must be at least one step");
    s->ind_every = every;
    s->ind_since = -1;
    return FIN_OK;
}

int fin_mhd_hybrid_stats(fin_mhd* s, long long* troubled_faces, long long* faces, long long* judges,
                         long long* reverts)
{
    if (!s) return merr(FIN_ERR_ARG, "null solver");
    if (s->ind_count) {
        unsigned long long c = 0;
        MCK(cudaMemcpyAsync(&c, s->ind_count, sizeof(c), cudaMemcpyDeviceToHost, s->stream));
        MCK(cudaStreamSynchronize(s->stream));
        s->troubled_last = (long long)c;
    }
    if (troubled_faces) *troubled_faces = s->troubled_last;
    if (faces) *faces = s->faces;
    if (judges) *judges = s->judges;
    if (reverts) *reverts = s->reverts;
    return FIN_OK;
}

int fin_mhd_indicator_time(fin_mhd* s, double* ms, long long* launches)
{
    if (!s || !ms || !launches) return merr(FIN_ERR_ARG, "null argument");
    *ms = s->ind_ms;
    *launches = s->ind_launches;
    return FIN_OK;
}

int fin_mhd_face_samples(fin_mhd* s, long long offset, long long stride, long long max_n, float* X_host,
                         unsigned char* y_host, long long* n_out)
{
    if (!s || !X_host || !y_host || !n_out || stride < 1 || offset < 0) return merr(FIN_ERR_ARG, "bad argument");
    const fin_params& p = s->p;
    const long long nf = (long long)(p.mx + 1) * p.my + (long long)p.mx * (p.my + 1);
    long long n = offset < nf ? (nf - offset + stride - 1) / stride : 0;
    if (n > max_n) n = max_n;
    *n_out = n;
    if (n == 0) return FIN_OK;
    int rc;
    if (!s->max_valid && (rc = compute_max(s, s->cur))) return rc;
    float* dX = nullptr;
    unsigned char* dy = nullptr;
    MCK(cudaMallocAsync(&dX, size_t(n) * ind::NFEAT * sizeof(float), s->stream));
    MCK(cudaMallocAsync(&dy, size_t(n), s->stream));
    const MhdArgs a = base_args(s);
    k_mhd_face_samples<<<grid_blocks(size_t(n)), 256, 0, s->stream>>>(
        a, s->q[s->cur], p.global_alpha ? alpha_slot(s, s->cur) : nullptr, offset, stride, n, dX, dy);
    s->launches++;
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(X_host, dX, size_t(n) * ind::NFEAT * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    MCK(cudaMemcpyAsync(y_host, dy, size_t(n), cudaMemcpyDeviceToHost, s->stream));
    MCK(cudaFreeAsync(dX, s->stream));
    MCK(cudaFreeAsync(dy, s->stream));
    MCK(cudaStreamSynchronize(s->stream));
    return FIN_OK;
}

int fin_mhd_last_kernel_ms(fin_mhd* s, double* ms)
{
    if (!s || !ms) return merr(FIN_ERR_ARG, "null argument");
    *ms = s->last_ms;
    return FIN_OK;
}

int fin_mhd_set_kernel_timing(fin_mhd* s, int on)
{
    if (!s) return merr(FIN_ERR_ARG, "null solver");
    s->time_kernels = on != 0;
    s->kernel_ms = 0.0;
    s->kernel_launches = 0;
    return FIN_OK;
}

int fin_mhd_kernel_time(fin_mhd* s, double* ms, long long* launches)
{
    if (!s || !ms || !launches) return merr(FIN_ERR_ARG, "null argument");
    *ms = s->kernel_ms;
    *launches = s->kernel_launches;
    return FIN_OK;
}

int fin_mhd_launch_count(fin_mhd* s, long long* launches)
{
    if (!s || !launches) return merr(FIN_ERR_ARG, "null argument");
    *launches = s->launches;
    return FIN_OK;
}

int fin_mhd_device_state(fin_mhd* s, double** q_dev, size_t* plane_stride)
{
    if (!s || !q_dev) return merr(FIN_ERR_ARG, "null argument");
    *q_dev = s->q[s->cur];
    if (plane_stride) *plane_stride = s->plane;
    return FIN_OK;
}

}  // extern "C"
