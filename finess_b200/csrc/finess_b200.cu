// Host driver and C ABI of the B200 WENO right-hand side and time steppers.
//
// One fin_solver owns one problem on the current CUDA device: four FP64 state
// buffers (q^n, two stage registers, q^{n+1}; the accept/reject logic of
// lib/2d/FinSolveRK.cpp:98-357 needs q^n intact until the CFL check), a
// small block of reduction slots, and a stream.  The time-step control stays
// on the host and copies the reference exactly; per step the host reads back
// 16 bytes (the face-speed maxima) to evaluate GetCFL.
#include <cuda_runtime.h>
#include <sys/stat.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <algorithm>
#include "finess_b200.h"
#include "fin_stage.cuh"
#include "fin_stage_hyb.cuh"
#include "fin_intflux.cuh"
#include "fin_hybrid.cuh"
#include "fin_tmap.h"
#include "fin_output.h"
#include "fin_mpp.cuh"
#include "fin_rk.cuh"
#include "fin_weno_hi.cuh"
#include "fin_sample.cuh"

using namespace fin;

namespace {

thread_local std::string g_err = "";

int set_err(int code, const std::string& msg)
{
    g_err = msg;
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return set_err(FIN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Tile shape of the stage kernel: 16 x 16 cells, 544 faces over 288 threads
// (two rounds of the face loop, the second 89% full).
#ifndef FIN_TILE_TI
#define FIN_TILE_TI 15
#define FIN_TILE_TJ 16
#define FIN_TILE_NT 256
#endif
using Cfg = TileCfg<FIN_TILE_TI, FIN_TILE_TJ, FIN_TILE_NT>;

// Reduction slots (doubles) in one device block, reset by one memset per step.
// The status word (bit 0: non-finite speed or state, bit 1: negative p or rho,
// bit 2: a tensor-core wait ran out, bit 3: a TMA copy wait ran out, bit 4: a TMA
// destination was misaligned) sits in slot STATUS so one copy returns it
// with the maxima.  SMAX_ALT keeps the face-speed maxima of the hybrid attempt
// while a judge step recomputes with full WENO; DIFF receives the judge's
// max |q_hybrid - q_full| and max |q_full|.
enum { NBUF = 5, SLOT_SMAX = 0, SLOT_ALPHA = 2, SLOT_STATUS = SLOT_ALPHA + 2 * NBUF, SLOT_SMAX_ALT = SLOT_STATUS + 1,
       SLOT_DIFF = SLOT_SMAX_ALT + 2, NSLOTS = SLOT_DIFF + 2 };

}  // namespace

struct fin_solver {
    fin_params p;
    double dx, dy;
    size_t plane;           // elements per component plane
    double* q[NBUF];        // state buffers (planes); q[cur] holds q^n; q[4] only in the hybrid form
    int cur;                // index of q^n
    double* slots;          // NSLOTS doubles (+ status word after them)
    unsigned int* status;
    double* h_slots;        // pinned mirror
    double* d_aos;          // staging buffer for the reference ghosted layout
    size_t aos_elems;
    double* d_aux;          // second staging / L output buffer (planes)
    double* Fg;             // integrated fluxes F, G (Lax-Wendroff / multiderivative)
    double* Gg;
    size_t gplane;          // their ghosted plane stride
    double* d_face_x;       // per-face alpha buffers (only for fin_construct_l)
    double* d_face_y;
    cudaStream_t stream;
    cudaEvent_t ev0, ev1;
    cudaEvent_t kev[6];     // start/stop of the three stage kernels of the last step
    cudaEvent_t iev[2];     // start/stop of the indicator launch of the last step
    bool time_kernels;      // record kev around each stage launch (and iev)
    bool ind_timed;         // the last step launched the indicator under timing
    double ind_ms;          // accumulated indicator-kernel time
    long long ind_launches;
    double kernel_ms;       // accumulated stage-kernel time since the last reset
    long long kernel_launches;
    double t;               // Qnew.get_t()
    double step_ms;
    // hybrid form
    float* mlpP;            // network parameters on the device
    unsigned* flags;        // troubled-face flag masks of the current step
    unsigned long long* ind_count;
    float zthr;
    bool ind_skip_const;    // the network's zero-row output is "not troubled": constant stencils skip it
    int judge_every;
    double judge_tol;
    long long hstep, judges, reverts, troubled_last, faces;
    int hyb_off;            // steps left with the indicator switched off after a revert
    int ind_every;          // the indicator runs every ind_every accepted steps (>= 1)
    int ind_since;          // accepted steps since its last run; -1: flags not valid for q[cur]
    bool judge_pending;     // the last take_stages ran a judge (results in q[nxt] and q[4])
    bool alpha_valid;       // slots hold alpha of q[cur]
    double last_ms;
    long long launches;
    // TMA tensor maps of the state buffers for the hybrid stages (tile with
    // halo / interior tile boxes); tma_ok when all were encoded
    CUtensorMap tm_q[NBUF];
    CUtensorMap tm_a[NBUF];
    bool tma_ok;
    // output files (fin_output.cu); pointers, since the struct is memset
    fin::io::FrameWriter* writer;   // asynchronous q%04d.dat / a%04d.dat writer (made on first use)
    std::string* cons_path;         // conservation.dat appended after every accepted step (null: off)
    double* d_cons;                 // device totals (MEQN doubles) then the partial sums
    double* h_cons;                 // pinned copy of the totals
    bool cons_pending;              // h_cons holds the totals at cons_t, not yet written
    double cons_t;
    // Lax-Wendroff with the MPP limiter (fin_mpp.cuh): high-order face
    // fluxes and the cells' limiting factors
    double* mpp_fx;                 // [m][mx+1][my]
    double* mpp_fy;                 // [m][mx][my+1]
    double* mpp_amin;               // [4][mx][my]
    int timed_stages;               // stage launches timed in the current step (at most 3)
    double* d_upd;                  // fin_update_soln(5)'s four ghosted arrays (made on first use)
};

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------
namespace fin {

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

// UpdateSoln.cpp:29-35 element by element: ((a1 q*) + (a2 q)) + (b L) with
// b = beta*dt, every product and sum rounded on its own (no contraction).
__global__ void k_update_soln(const double* qstar, const double* L, double* qnew, size_t n, double a1, double a2,
                              double b)
{
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
        qnew[k] = __dadd_rn(__dadd_rn(__dmul_rn(a1, qstar[k]), __dmul_rn(a2, qnew[k])), __dmul_rn(b, L[k]));
}

// UpdateSoln.cpp:43-80 (the fifth-order stepper's form) element by element:
// q2 = q2 + delta q1, then q1 = ((g1 q1 + g2 q2) + g3 qold) + b L with
// b = beta*dt, every operation rounded on its own.
__global__ void k_update_soln5(const double* qold, const double* L, double* q1, double* q2, size_t n, double g1,
                               double g2, double g3, double delta, double b)
{
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        const double s1 = q1[k];
        const double s2 = __dadd_rn(q2[k], __dmul_rn(delta, s1));
        q2[k] = s2;
        const double s3 = qold[k];
        q1[k] = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(g1, s1), __dmul_rn(g2, s2)), __dmul_rn(g3, s3)),
                          __dmul_rn(b, L[k]));
    }
}

// GetCFL.cpp:54-59's maxima: smax(i, j, 1) and smax(i, j, 2) over i <= mx,
// j <= my of a ghosted (mx+1, my+1, 2) array; NaN entries skipped.
__global__ void k_smax_max(const double* smax, int mx, int my, int mbc, double* out)
{
    __shared__ double red[2][32];
    double a = 0.0, b = 0.0;
    const size_t n = size_t(mx) * my;
    const int sy = my + 1 + 2 * mbc;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const int i = int(g / my), j = int(g - size_t(i) * my);
        const size_t e = (size_t(i + mbc) * sy + (j + mbc)) * 2;
        const double v1 = smax[e], v2 = smax[e + 1];
        if (v1 == v1) a = v1 > a ? v1 : a;
        if (v2 == v2) b = v2 > b ? v2 : b;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a = Max(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = Max(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = a; red[1][w] = b; }
    __syncthreads();
    if (threadIdx.x < 2) {
        double v = 0.0;
        for (int k = 0; k < nw; k++) v = Max(v, red[threadIdx.x][k]);
        atomic_max_nonneg(out + threadIdx.x, v);
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


__global__ void k_wave_spd_max(const double* q, int mx, int my, size_t plane, double gamma,
                               double* alpha_out, unsigned int* status)
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
    if (!(ax <= 1e300)) ax = 0.0;
    if (!(ay <= 1e300)) ay = 0.0;
    for (int o = 16; o > 0; o >>= 1) {
        ax = Max(ax, __shfl_xor_sync(0xffffffffu, ax, o));
        ay = Max(ay, __shfl_xor_sync(0xffffffffu, ay, o));
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = ax; red[1][w] = ay; }
    if (nonfinite) atomicOr(status, 1u);
    __syncthreads();
    if (threadIdx.x < 2) {
        double v = 0.0;
        for (int k = 0; k < nw; k++) v = Max(v, red[threadIdx.x][k]);
        atomic_max_nonneg(alpha_out + threadIdx.x, v);
    }
}

// Ghosted AoS (i, j, m), m fastest, i slowest -> interior planes.
__global__ void k_aos_to_planes(const double* aos, double* planes, int mx, int my, int mbc, size_t plane)
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

// Interior planes -> ghosted AoS with the ghost frame filled by the BC remap
// (what SetBndValues leaves in the reference's arrays).
__global__ void k_planes_to_aos(const double* planes, double* aos, int mx, int my, int mbc, size_t plane,
                                int bc0, int bc1, int bc2, int bc3)
{
    const int sx = mx + 2 * mbc, sy = my + 2 * mbc;
    const size_t n = size_t(sx) * sy;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
        const int ii = int(e / sy), jj = int(e - size_t(ii) * sy);
        const int gi = bc_remap(ii - mbc, mx, bc0, bc1), gj = bc_remap(jj - mbc, my, bc2, bc3);
        const size_t g = size_t(gi) * my + gj;
#pragma unroll
        for (int m = 0; m < MEQN; m++) aos[e * MEQN + m] = planes[m * plane + g];
    }
}

// Interior planes -> interior of a ghosted AoS array, ghosts untouched.
__global__ void k_planes_to_aos_interior(const double* planes, double* aos, int mx, int my, int mbc, size_t plane)
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

// FMA throughput probe: 8 independent FMA chains per thread, no memory traffic
// inside the loop.  Used to measure the FP64 and FP32 pipe peaks that the
// stage kernel's pipe utilisation is quoted against.
template <class R>
__global__ void k_fma_peak(R* out, int iters, R a, R b)
{
    R x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = R(threadIdx.x + k);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = x[k] * a + b;
    }
    R s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == R(-1.2345)) out[0] = s;   // keeps the loop live; never true in practice
}

}  // namespace fin

// ---------------------------------------------------------------------------
// kernel dispatch
// ---------------------------------------------------------------------------
namespace {

int buffer_of(const fin_solver* s, const double* ptr)
{
    for (int b = 0; b < NBUF; b++)
        if (ptr && s->q[b] == ptr) return b;
    return -1;
}

template <class R, int VER, bool P2, bool FG = false>
int launch_stage_t(fin_solver* s, const StageArgs& a)
{
    const size_t smem = Cfg::template smem_bytes<R>();
    auto kern = k_stage<R, VER, P2, Cfg, FG>;
    static bool configured = false;   // per instantiation; attribute is per device function
    if (!configured) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        configured = true;
    }
    dim3 grid((a.my + Cfg::TJ - 1) / Cfg::TJ, (a.mx + Cfg::TI - 1) / Cfg::TI);
    kern<<<grid, Cfg::NT, smem, s->stream>>>(a);
    s->launches++;
    CK(cudaGetLastError());
    return FIN_OK;
}

template <class R>
int launch_stage_r(fin_solver* s, const StageArgs& a)
{
    const bool p2 = s->p.power_param == 2.0;
    switch (s->p.weno_version) {
    case FIN_WENO_JS: return p2 ? launch_stage_t<R, FIN_WENO_JS, true>(s, a) : launch_stage_t<R, FIN_WENO_JS, false>(s, a);
    case FIN_WENO_Z: return p2 ? launch_stage_t<R, FIN_WENO_Z, true>(s, a) : launch_stage_t<R, FIN_WENO_Z, false>(s, a);
    case FIN_WENO_FD: return launch_stage_t<R, FIN_WENO_FD, true>(s, a);
    }
    return set_err(FIN_ERR_ARG, "weno_version");
}

// Stages that split the time-integrated fluxes (ConstructLxWL): FP64 only.
int launch_stage_fg(fin_solver* s, const StageArgs& a)
{
    const bool p2 = s->p.power_param == 2.0;
    switch (s->p.weno_version) {
    case FIN_WENO_JS:
        return p2 ? launch_stage_t<double, FIN_WENO_JS, true, true>(s, a)
                  : launch_stage_t<double, FIN_WENO_JS, false, true>(s, a);
    case FIN_WENO_Z:
        return p2 ? launch_stage_t<double, FIN_WENO_Z, true, true>(s, a)
                  : launch_stage_t<double, FIN_WENO_Z, false, true>(s, a);
    case FIN_WENO_FD: return launch_stage_t<double, FIN_WENO_FD, true, true>(s, a);
    }
    return set_err(FIN_ERR_ARG, "weno_version");
}

// Hybrid stages (fin_stage_hyb.cuh): persistent CTAs, two per SM.
template <int VER, bool P2>
int launch_stage_hyb_t(fin_solver* s, const StageArgs& a)
{
    using Lh = HybSmem<HybCfg>;
    auto kern = k_stage_hyb<VER, P2, HybCfg>;
    static bool configured = false;   // per instantiation
    if (!configured) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(Lh::BYTES)));
        configured = true;
    }
    StageArgs b = a;
    b.tma = 0;
    const double* ext = (a.A && a.A != a.qin) ? a.A : ((a.B && a.B != a.qin) ? a.B : nullptr);
    const int iq = buffer_of(s, a.qin), ie = buffer_of(s, ext);
    if (s->tma_ok && iq >= 0 && (!ext || ie >= 0)) {
        b.tma = 1;
        b.tm_in = s->tm_q[iq];
        if (ext) b.tm_A = s->tm_a[ie];
    }
    const long long tiles = (long long)((a.mx + HybCfg::TI - 1) / HybCfg::TI) * ((a.my + HybCfg::TJ - 1) / HybCfg::TJ);
    kern<<<unsigned(tiles), HybCfg::NT, Lh::BYTES, s->stream>>>(b);
    s->launches++;
    CK(cudaGetLastError());
    return FIN_OK;
}

// Hybrid stages: FP32 with per-face choice between full WENO and FD5.
int launch_stage_hyb(fin_solver* s, const StageArgs& a)
{
    const bool p2 = s->p.power_param == 2.0;
    switch (s->p.weno_version) {
    case FIN_WENO_JS: return p2 ? launch_stage_hyb_t<FIN_WENO_JS, true>(s, a) : launch_stage_hyb_t<FIN_WENO_JS, false>(s, a);
    case FIN_WENO_Z: return p2 ? launch_stage_hyb_t<FIN_WENO_Z, true>(s, a) : launch_stage_hyb_t<FIN_WENO_Z, false>(s, a);
    case FIN_WENO_FD: return launch_stage_t<float, FIN_WENO_FD, true, false>(s, a);
    }
    return set_err(FIN_ERR_ARG, "weno_version");
}

int grid_blocks(size_t n);

// Spatial orders other than 5 (fin_weno_hi.cuh, FP64): one thread per face
// into the face-flux arrays, then the flux difference and stage update.
template <int ORDER, int VER>
int launch_stage_hi_t(fin_solver* s, const StageArgs& a)
{
    const size_t nx = size_t(a.mx + 1) * a.my, ny = size_t(a.mx) * (a.my + 1);
    if (!s->mpp_fx) CK(cudaMalloc(&s->mpp_fx, MEQN * nx * sizeof(double)));
    if (!s->mpp_fy) CK(cudaMalloc(&s->mpp_fy, MEQN * ny * sizeof(double)));
    hi::HiArgs h;
    memset(&h, 0, sizeof(h));
    h.q = a.qin;
    h.plane = a.plane;
    h.mx = a.mx;
    h.my = a.my;
    for (int k = 0; k < 4; k++) h.bc[k] = a.bc[k];
    h.gamma = a.gamma;
    h.eps = a.eps;
    h.pw = a.pw;
    h.alpha_scaling = a.alpha_scaling;
    h.alpha_in = a.alpha_in;
    h.fx = s->mpp_fx;
    h.fy = s->mpp_fy;
    h.smax_out = a.smax_out;
    h.face_alpha_x = a.face_alpha_x;
    h.face_alpha_y = a.face_alpha_y;
    h.status = a.status;
    const size_t nf = nx + ny;
    hi::k_hi_faces<ORDER, VER><<<unsigned((nf + 127) / 128), 128, 0, s->stream>>>(h);
    CK(cudaGetLastError());
    hi::k_hi_update<<<grid_blocks(size_t(a.mx) * a.my), 256, 0, s->stream>>>(s->mpp_fx, s->mpp_fy, a);
    CK(cudaGetLastError());
    s->launches += 2;
    return FIN_OK;
}

int launch_stage_hi(fin_solver* s, const StageArgs& a)
{
    const int v = s->p.weno_version;
    switch (s->p.space_order) {
    case 1: return launch_stage_hi_t<1, FIN_WENO_JS>(s, a);
    case 7:
        return v == FIN_WENO_Z ? launch_stage_hi_t<7, FIN_WENO_Z>(s, a)
             : v == FIN_WENO_FD ? launch_stage_hi_t<7, FIN_WENO_FD>(s, a) : launch_stage_hi_t<7, FIN_WENO_JS>(s, a);
    case 9:
        return v == FIN_WENO_Z ? launch_stage_hi_t<9, FIN_WENO_Z>(s, a)
             : v == FIN_WENO_FD ? launch_stage_hi_t<9, FIN_WENO_FD>(s, a) : launch_stage_hi_t<9, FIN_WENO_JS>(s, a);
    case 11: return launch_stage_hi_t<11, FIN_WENO_JS>(s, a);
    }
    return set_err(FIN_ERR_ARG, "Requested WENO Reconstruction not implemented.");
}

int launch_stage(fin_solver* s, const StageArgs& a)
{
    if (s->p.space_order != 5) return launch_stage_hi(s, a);
    if (a.Fg) return launch_stage_fg(s, a);
    if (a.flags) return launch_stage_hyb(s, a);
    if (s->p.precision == FIN_PREC_HYBRID) return launch_stage_r<float>(s, a);
    if (s->p.precision == FIN_PREC_FP64) return launch_stage_r<double>(s, a);
    if (s->p.precision == FIN_PREC_FP32) return launch_stage_r<float>(s, a);
    return set_err(FIN_ERR_UNSUPPORTED, "precision form not built");
}

// A stage launch bracketed by events when kernel timing is on (stage k of 3).
int launch_stage_timed(fin_solver* s, const StageArgs& a, int k)
{
    const bool timed = s->time_kernels && k < 3;   // three event pairs; later stages of a step run untimed
    if (timed) CK(cudaEventRecord(s->kev[2 * k], s->stream));
    int rc = launch_stage(s, a);
    if (rc) return rc;
    if (timed) {
        CK(cudaEventRecord(s->kev[2 * k + 1], s->stream));
        s->timed_stages = std::max(s->timed_stages, k + 1);
    }
    return FIN_OK;
}

// After the stream is synchronised: add the last step's stage-kernel times.
int collect_kernel_times(fin_solver* s)
{
    if (!s->time_kernels) return FIN_OK;
    const int nst = s->timed_stages;
    s->timed_stages = 0;
    for (int k = 0; k < nst; k++) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, s->kev[2 * k], s->kev[2 * k + 1]));
        s->kernel_ms += ms;
        s->kernel_launches++;
    }
    if (s->ind_timed) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, s->iev[0], s->iev[1]));
        s->ind_ms += ms;
        s->ind_launches++;
        s->ind_timed = false;
    }
    return FIN_OK;
}

StageArgs base_args(fin_solver* s)
{
    StageArgs a;
    memset(&a, 0, sizeof(a));
    a.mx = s->p.mx;
    a.my = s->p.my;
    a.plane = s->plane;
    a.rdx = 1.0 / s->dx;
    a.rdy = 1.0 / s->dy;
    a.gamma = s->p.gamma;
    a.eps = s->p.epsilon;
    a.pw = s->p.power_param;
    a.alpha_scaling = s->p.alpha_scaling;
    a.gamma_f = float(a.gamma);
    a.eps_f = float(a.eps);
    a.pw_f = float(a.pw);
    a.alpha_scaling_f = float(a.alpha_scaling);
    a.status = s->status;
    a.bc[0] = s->p.bc_xlow; a.bc[1] = s->p.bc_xhigh;
    a.bc[2] = s->p.bc_ylow; a.bc[3] = s->p.bc_yhigh;
    return a;
}

int grid_blocks(size_t n)
{
    size_t b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return int(b);
}

double* alpha_slot(fin_solver* s, int buf) { return s->slots + SLOT_ALPHA + 2 * buf; }

// Global alpha of buffer buf into its slot (used when no stage epilogue has
// produced it: after set_state, or when global_alpha is off it is unused).
int compute_alpha(fin_solver* s, int buf)
{
    CK(cudaMemsetAsync(alpha_slot(s, buf), 0, 2 * sizeof(double), s->stream));
    const size_t n = size_t(s->p.mx) * s->p.my;
    k_wave_spd_max<<<grid_blocks(n), 256, 0, s->stream>>>(s->q[buf], s->p.mx, s->p.my, s->plane, s->p.gamma,
                                                           alpha_slot(s, buf), s->status);
    s->launches++;
    CK(cudaGetLastError());
    return FIN_OK;
}

int check_status(fin_solver* s)
{
    unsigned int st = 0;
    CK(cudaMemcpyAsync(&st, s->status, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (st & 1u) {
        CK(cudaMemsetAsync(s->status, 0, sizeof(unsigned int), s->stream));
        return set_err(FIN_ERR_NONFINITE, "non-finite wave speed or state");
    }
    return FIN_OK;
}

// ConstructIntegratedR into s->Fg, s->Gg: mode 0/1 = 1-state without/with
// the f_tt terms, 2 = 2-state.
constexpr int IF_TI = 16, IF_TJ = 16;
int launch_intflux(fin_solver* s, int mode, const double* q1, const double* q2, double dt, double a1,
                   double b1, double a2, double b2, double c1 = 0.0, double c2 = 0.0)
{
    IntFluxArgs f;
    memset(&f, 0, sizeof(f));
    f.q1 = q1; f.q2 = q2; f.F = s->Fg; f.G = s->Gg;
    f.plane = s->plane; f.gplane = s->gplane;
    f.mx = s->p.mx; f.my = s->p.my;
    f.dx = s->dx; f.dy = s->dy; f.gamma = s->p.gamma; f.dt = dt;
    f.a1 = a1; f.b1 = b1; f.a2 = a2; f.b2 = b2;
    f.c1 = c1; f.c2 = c2;
    f.bc[0] = s->p.bc_xlow; f.bc[1] = s->p.bc_xhigh; f.bc[2] = s->p.bc_ylow; f.bc[3] = s->p.bc_yhigh;
    constexpr size_t smem = 3 * MEQN * (IF_TI + 4) * (IF_TJ + 4) * sizeof(double);
    dim3 grid((s->p.my + 6 + IF_TJ - 1) / IF_TJ, (s->p.mx + 6 + IF_TI - 1) / IF_TI);
    if (mode == 0) k_intflux<0, IF_TI, IF_TJ><<<grid, IF_TI * IF_TJ, smem, s->stream>>>(f);
    else if (mode == 1) k_intflux<1, IF_TI, IF_TJ><<<grid, IF_TI * IF_TJ, smem, s->stream>>>(f);
    else if (mode == 2) k_intflux<2, IF_TI, IF_TJ><<<grid, IF_TI * IF_TJ, smem, s->stream>>>(f);
    else k_intflux<3, IF_TI, IF_TJ><<<grid, IF_TI * IF_TJ, smem, s->stream>>>(f);
    s->launches++;
    CK(cudaGetLastError());
    return FIN_OK;
}

int take_stages_rk(fin_solver* s, double dt, int nxt, const unsigned* flags, int q1, int q2);

// Troubled-face flags of q[buf] (fin_hybrid.cuh).
int launch_indicator(fin_solver* s, int buf)
{
    IndicatorArgs ia;
    memset(&ia, 0, sizeof(ia));
    ia.q = s->q[buf];
    ia.plane = s->plane;
    ia.mx = s->p.mx;
    ia.my = s->p.my;
    ia.bc[0] = s->p.bc_xlow; ia.bc[1] = s->p.bc_xhigh; ia.bc[2] = s->p.bc_ylow; ia.bc[3] = s->p.bc_yhigh;
    ia.gamma = float(s->p.gamma);
    ia.P = s->mlpP;
    ia.zthr = s->zthr;
    ia.flags = s->flags;
    ia.status = s->status;
    ia.count = s->ind_count;
    ia.skip_const = s->ind_skip_const ? 1 : 0;
    ia.tma = 0;
    if (s->tma_ok) {
        ia.tma = 1;
        ia.tm = s->tm_q[buf];
    }
    static bool configured = false;
    const size_t smem = sizeof(IndTile<Cfg>);
    if (!configured) {
        CK(cudaFuncSetAttribute(k_indicator<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        configured = true;
    }
    CK(cudaMemsetAsync(s->ind_count, 0, sizeof(unsigned long long), s->stream));
    CK(cudaMemsetAsync(s->flags, 0, flag_words(s->p.mx, s->p.my) * sizeof(unsigned), s->stream));
    const long long nf = (long long)(s->p.mx + 1) * s->p.my + (long long)s->p.mx * (s->p.my + 1);
    const long long tiles = (long long)((s->p.mx + Cfg::TI - 1) / Cfg::TI) * ((s->p.my + Cfg::TJ - 1) / Cfg::TJ);
    const int grid = int(std::min<long long>(tiles, 148 * 3));
    k_indicator<Cfg><<<grid, Cfg::NT, smem, s->stream>>>(ia);
    s->launches++;
    s->faces = nf;
    CK(cudaGetLastError());
    return FIN_OK;
}

// The Lax-Wendroff step with the MPP limiter (FinSolveLxW.cpp:120-151):
// ConstructIntegratedR, the stage kernel in its flux-only mode (ConstructLxWL's
// Fhat / Ghat and the face-speed maxima without the first face of each
// direction, whose smax entry ConstructLFL.cpp:62-65 replaces by the global
// wave speed; get_cfl puts it back), then k_mpp_limit and k_mpp_update
// (ConstructLFL's fluxes, ApplyMPPLimiter2D and the update, fin_mpp.cuh).
int take_stage_lxw_mpp(fin_solver* s, double dt, int nxt)
{
    const fin_params& p = s->p;
    const int qn = s->cur;
    const size_t nx = size_t(p.mx + 1) * p.my, ny = size_t(p.mx) * (p.my + 1), nc = size_t(p.mx) * p.my;
    if (!s->mpp_fx) CK(cudaMalloc(&s->mpp_fx, MEQN * nx * sizeof(double)));
    if (!s->mpp_fy) CK(cudaMalloc(&s->mpp_fy, MEQN * ny * sizeof(double)));
    if (!s->mpp_amin) CK(cudaMalloc(&s->mpp_amin, 4 * nc * sizeof(double)));
    CK(cudaMemsetAsync(s->slots + SLOT_SMAX, 0, 2 * sizeof(double), s->stream));
    CK(cudaMemsetAsync(s->slots + SLOT_STATUS, 0, sizeof(double), s->stream));
    CK(cudaMemsetAsync(alpha_slot(s, nxt), 0, 2 * sizeof(double), s->stream));
    int rc;
    if ((rc = launch_intflux(s, p.time_order > 2 ? 1 : 0, s->q[qn], nullptr, dt, 0, 0, 0, 0))) return rc;
    StageArgs a = base_args(s);
    a.smax_out = s->slots + SLOT_SMAX;
    a.Fg = s->Fg; a.Gg = s->Gg; a.gplane = s->gplane;
    a.qin = s->q[qn]; a.A = s->q[qn]; a.B = nullptr; a.qout = s->q[nxt];
    a.a1 = 1.0; a.a2 = 0.0; a.bdt = dt;
    a.alpha_in = p.global_alpha ? alpha_slot(s, qn) : nullptr;
    a.alpha_out = nullptr;
    a.flux_x = s->mpp_fx;
    a.flux_y = s->mpp_fy;
    a.flux_only = 1;
    if ((rc = launch_stage_timed(s, a, 0))) return rc;
    mpp::MppArgs m;
    memset(&m, 0, sizeof(m));
    m.q = s->q[qn];
    m.qout = s->q[nxt];
    m.plane = s->plane;
    m.mx = p.mx;
    m.my = p.my;
    m.bc[0] = p.bc_xlow; m.bc[1] = p.bc_xhigh; m.bc[2] = p.bc_ylow; m.bc[3] = p.bc_yhigh;
    m.fhat = s->mpp_fx;
    m.ghat = s->mpp_fy;
    m.amin = s->mpp_amin;
    m.alpha = alpha_slot(s, qn);
    m.dt = dt;
    m.dx = s->dx;
    m.dy = s->dy;
    m.gamma = p.gamma;
    m.alpha_out = alpha_slot(s, nxt);
    m.status = s->status;
    const unsigned blocks = unsigned((nc + 127) / 128);
    mpp::k_mpp_limit<<<blocks, 128, 0, s->stream>>>(m);
    mpp::k_mpp_update<<<blocks, 128, 0, s->stream>>>(m);
    s->launches += 2;
    CK(cudaGetLastError());
    return FIN_OK;
}

// Lax-Wendroff (FinSolveLxW.cpp:120-176) and two-stage multiderivative
// (FinSolveMD.cpp:116-170, time_order 4) steps from q[cur] into q[nxt].
int take_stages_lw(fin_solver* s, double dt, int nxt)
{
    const fin_params& p = s->p;
    const int qn = s->cur;
    int q1 = 0;
    while (q1 == qn || q1 == nxt) q1++;
    CK(cudaMemsetAsync(s->slots + SLOT_SMAX, 0, 2 * sizeof(double), s->stream));
    CK(cudaMemsetAsync(s->slots + SLOT_STATUS, 0, sizeof(double), s->stream));
    CK(cudaMemsetAsync(alpha_slot(s, q1), 0, 2 * sizeof(double), s->stream));
    CK(cudaMemsetAsync(alpha_slot(s, nxt), 0, 2 * sizeof(double), s->stream));
    const bool ga = p.global_alpha != 0;
    int rc;
    StageArgs a = base_args(s);
    a.smax_out = s->slots + SLOT_SMAX;
    a.Fg = s->Fg; a.Gg = s->Gg; a.gplane = s->gplane;
    if (p.time_stepping_method == FIN_TS_LXW && p.mpp_limiter) return take_stage_lxw_mpp(s, dt, nxt);
    if (p.time_stepping_method == FIN_TS_LXW) {
        // F = ConstructIntegratedR(dt, q); q^{n+1} = q + dt L
        if ((rc = launch_intflux(s, p.time_order > 2 ? 1 : 0, s->q[qn], nullptr, dt, 0, 0, 0, 0))) return rc;
        a.qin = s->q[qn]; a.A = s->q[qn]; a.B = nullptr; a.qout = s->q[nxt];
        a.a1 = 1.0; a.a2 = 0.0; a.bdt = dt;
        a.alpha_in = ga ? alpha_slot(s, qn) : nullptr;
        a.alpha_out = alpha_slot(s, nxt);
        return launch_stage_timed(s, a, 0);
    }
    if (p.time_order == 5) {
        // FinSolveMD.cpp:172-226 (coefficients tuned for stability along the
        // imaginary axis, rho = 8.209945182837015e-02), the three-coefficient
        // ConstructIntegratedR of ConstructIntegratedR.cpp:608-700:
        // stage 1: F = CIR((2/5) dt; 1, 1/2, (125/8) rho; q^n | 0, 0, 0; q*),
        //          q* = q^n + ((2/5) dt) L(q^n)
        const double d1 = 2.0 / 5.0 * dt;
        if ((rc = launch_intflux(s, 3, s->q[qn], nullptr, d1, 1.0, 0.5, 0.0, 0.0, 125. / 8. * 8.209945182837015e-02,
                                 0.0)))
            return rc;
        a.qin = s->q[qn]; a.A = s->q[qn]; a.B = nullptr; a.qout = s->q[q1];
        a.a1 = 1.0; a.a2 = 0.0; a.bdt = d1;
        a.alpha_in = ga ? alpha_slot(s, qn) : nullptr;
        a.alpha_out = alpha_slot(s, q1);
        if ((rc = launch_stage_timed(s, a, 0))) return rc;
        // stage 2: F = CIR(dt; 1, 1/2, 1/16; q^n | 0, 0, 5/48; q*); q^{n+1} = q^n + dt L(q*)
        if ((rc = launch_intflux(s, 3, s->q[qn], s->q[q1], dt, 1.0, 0.5, 0.0, 0.0, (1.0 / 16.0), (5.0 / 48.0))))
            return rc;
        a.qin = s->q[q1]; a.A = s->q[qn]; a.B = nullptr; a.qout = s->q[nxt];
        a.a1 = 1.0; a.a2 = 0.0; a.bdt = dt;
        a.alpha_in = ga ? alpha_slot(s, q1) : nullptr;
        a.alpha_out = alpha_slot(s, nxt);
        return launch_stage_timed(s, a, 1);
    }
    // stage 1: F = ConstructIntegratedR(dt/2, q^n) (f_tt included: time_order 4 > 2);
    //          q* = q^n + (dt/2) L
    if ((rc = launch_intflux(s, 1, s->q[qn], nullptr, 0.5 * dt, 0, 0, 0, 0))) return rc;
    a.qin = s->q[qn]; a.A = s->q[qn]; a.B = nullptr; a.qout = s->q[q1];
    a.a1 = 1.0; a.a2 = 0.0; a.bdt = 0.5 * dt;
    a.alpha_in = ga ? alpha_slot(s, qn) : nullptr;
    a.alpha_out = alpha_slot(s, q1);
    if ((rc = launch_stage_timed(s, a, 0))) return rc;
    // stage 2: F = ConstructIntegratedR(dt, 1, 1/6, q^n, 0, 1/3, q*); q^{n+1} = q^n + dt L(q*)
    if ((rc = launch_intflux(s, 2, s->q[qn], s->q[q1], dt, 1.0, (1.0 / 6.0), 0.0, (1.0 / 3.0)))) return rc;
    a.qin = s->q[q1]; a.A = s->q[qn]; a.B = nullptr; a.qout = s->q[nxt];
    a.a1 = 1.0; a.a2 = 0.0; a.bdt = dt;
    a.alpha_in = ga ? alpha_slot(s, q1) : nullptr;
    a.alpha_out = alpha_slot(s, nxt);
    return launch_stage_timed(s, a, 1);
}

int launch_indicator(fin_solver* s, int buf);

// The two stage registers of a step from q[cur] into q[nxt]: the first two
// buffers that are neither (buffer 4 is reserved for the judge step).
void stage_registers(fin_solver* s, int nxt, int* q1, int* q2)
{
    int reg[2], k = 0;
    for (int b = 0; b < 4 && k < 2; b++)
        if (b != s->cur && b != nxt) reg[k++] = b;
    *q1 = reg[0];
    *q2 = reg[1];
}

int take_stages(fin_solver* s, double dt, int nxt)
{
    s->judge_pending = false;
    if (s->p.time_stepping_method != FIN_TS_RK) return take_stages_lw(s, dt, nxt);
    int q1, q2, rc;
    stage_registers(s, nxt, &q1, &q2);
    if (s->p.precision != FIN_PREC_HYBRID || !s->mlpP) return take_stages_rk(s, dt, nxt, nullptr, q1, q2);
    // Hybrid form: flags from the indicator on q^n, FP32 stages with the
    // per-face choice; every judge_every-th step also a full-WENO FP32 step
    // from the same q^n into q[4], compared on the device.
    const bool active = s->hyb_off == 0;
    if (!active) {
        s->hyb_off--;
        return take_stages_rk(s, dt, nxt, nullptr, q1, q2);
    }
    if (s->ind_since < 0 || s->ind_since >= s->ind_every) {
        if (s->time_kernels) CK(cudaEventRecord(s->iev[0], s->stream));
        if ((rc = launch_indicator(s, s->cur))) return rc;
        if (s->time_kernels) {
            CK(cudaEventRecord(s->iev[1], s->stream));
            s->ind_timed = true;
        }
        s->ind_since = 0;
    }
    if ((rc = take_stages_rk(s, dt, nxt, s->flags, q1, q2))) return rc;
    s->hstep++;
    if (s->judge_every > 0 && s->hstep % s->judge_every == 0) {
        CK(cudaMemcpyAsync(s->slots + SLOT_SMAX_ALT, s->slots + SLOT_SMAX, 2 * sizeof(double), cudaMemcpyDeviceToDevice,
                           s->stream));
        const bool tk = s->time_kernels;   // the step's stage times stay those of the hybrid stages
        s->time_kernels = false;
        rc = take_stages_rk(s, dt, 4, nullptr, q1, q2);
        s->time_kernels = tk;
        if (rc) return rc;
        CK(cudaMemsetAsync(s->slots + SLOT_DIFF, 0, 2 * sizeof(double), s->stream));
        const size_t n = size_t(s->p.mx) * s->p.my;
        k_max_diff<<<grid_blocks(n), 256, 0, s->stream>>>(s->q[nxt], s->q[4], s->plane, n, s->slots + SLOT_DIFF);
        s->launches++;
        CK(cudaGetLastError());
        s->judge_pending = true;
    }
    return FIN_OK;
}

// After get_cfl brought the slots to the host: settle a judge step.  Keeps
// the hybrid result (and its face-speed maxima) unless it differs from the
// full-WENO result by more than judge_tol (relative L-infinity); then the
// full result is taken (moved into q[nxt]), its maxima give the CFL, and the
// indicator stays off for judge_every steps.
void settle_judge(fin_solver* s, int nxt, double dt, double* cfl)
{
    if (!s->judge_pending) return;
    s->judges++;
    const double d = s->h_slots[SLOT_DIFF], m = s->h_slots[SLOT_DIFF + 1];
    const bool revert = !(d <= s->judge_tol * (m > 0 ? m : 1.0));
    double sx, sy;
    if (revert) {
        // q[nxt] <- the full-WENO result (pointer swap), with its alpha slot
        s->reverts++;
        s->hyb_off = s->judge_every;
        s->ind_since = -1;
        // the buffers trade places, and their tensor maps with them
        std::swap(s->q[4], s->q[nxt]);
        std::swap(s->tm_q[4], s->tm_q[nxt]);
        std::swap(s->tm_a[4], s->tm_a[nxt]);
        cudaMemcpyAsync(alpha_slot(s, nxt), alpha_slot(s, 4), 2 * sizeof(double), cudaMemcpyDeviceToDevice, s->stream);
        sx = s->h_slots[SLOT_SMAX];
        sy = s->h_slots[SLOT_SMAX + 1];
    } else {
        sx = s->h_slots[SLOT_SMAX_ALT];
        sy = s->h_slots[SLOT_SMAX_ALT + 1];
    }
    double c = -100.0;
    c = Max(dt * sx / s->dx, c);
    c = Max(dt * sy / s->dy, c);
    *cfl = c;
}

// The stages of one step of size dt from q[cur] into q[nxt] (RK3:
// FinSolveRK.cpp:158-211 with SetRKinfo.cpp:50-64).  Leaves the face-speed
// maxima of the step in slots SMAX and alpha(q[nxt]) in its slot.
// FinSolveRK's other orders (FinSolveRK.cpp:117-156, 213-299; coefficients
// of SetRKinfo.cpp:27-126): forward Euler, SSP-RK2, the ten-stage SSP-RK4 of
// Ketcheson (2008) and the eight-stage fifth-order method, each stage
// q_out = a1 A + a2 B + (beta dt) L(q_in) through the stage kernel (the
// in-place stages of the reference alternate between two registers here),
// with the element-wise parts of orders 4 and 5 in fin_rk.cuh.  A stage whose
// reference coefficient multiplies a register by 0 drops that term (0 x
// finite = 0).
int take_stages_rk_other(fin_solver* s, double dt, int nxt)
{
    const fin_params& p = s->p;
    const int qn = s->cur;
    int r1, r2;
    stage_registers(s, nxt, &r1, &r2);
    CK(cudaMemsetAsync(s->slots + SLOT_SMAX, 0, 2 * sizeof(double), s->stream));
    CK(cudaMemsetAsync(s->slots + SLOT_STATUS, 0, sizeof(double), s->stream));
    const bool ga = p.global_alpha != 0;
    StageArgs a = base_args(s);
    a.smax_out = s->slots + SLOT_SMAX;
    int k = 0;
    // q[out] = a1 q[A] + a2 q[B] + bdt L(q[in]); A, B < 0: term absent
    auto stage = [&](int in, int A, double a1, int B, double a2, double bdt, int out) -> int {
        if (out >= 0) CK(cudaMemsetAsync(alpha_slot(s, out), 0, 2 * sizeof(double), s->stream));
        a.qin = s->q[in];
        a.A = A >= 0 ? s->q[A] : nullptr;
        a.a1 = a1;
        a.B = B >= 0 ? s->q[B] : nullptr;
        a.a2 = a2;
        a.bdt = bdt;
        a.qout = s->q[out >= 0 ? out : r2];
        a.alpha_in = ga ? alpha_slot(s, in) : nullptr;
        a.alpha_out = out >= 0 ? alpha_slot(s, out) : nullptr;
        return launch_stage_timed(s, a, k++);
    };
    const size_t n = size_t(p.mx) * p.my;
    const int eb = grid_blocks(n);
    int rc;
    switch (p.time_order) {
    case 1:   // :123-130
        return stage(qn, qn, 1.0, -1, 0.0, 1.0 * dt, nxt);
    case 2:   // :136-157
        if ((rc = stage(qn, qn, 1.0, -1, 0.0, 1.0 * dt, r1))) return rc;
        return stage(r1, r1, 0.5, qn, 0.5, 0.5 * dt, nxt);
    case 4: {  // :213-265, stages 1-9 with (1, 0, 1/6), stage 10 with (1, 3/5, 1/10)
        const double b = (1.0 / 6.0) * dt;
        int in = qn, out = r1;
        for (int st = 1; st <= 5; st++) {
            if ((rc = stage(in, in, 1.0, -1, 0.0, b, out))) return rc;
            in = out;
            out = out == r1 ? r2 : r1;
        }
        // q1 in `in`; q2 = q^n until the swap: q2 <- (q2 + 9 q1)/25 into nxt,
        // q1 <- 15 q2 - 5 q1 in place
        CK(cudaMemsetAsync(alpha_slot(s, in), 0, 2 * sizeof(double), s->stream));
        rk::k_rk4_swap<<<eb, 256, 0, s->stream>>>(s->q[qn], s->q[nxt], s->q[in], s->plane, n, p.gamma,
                                                  alpha_slot(s, in), s->status);
        s->launches++;
        CK(cudaGetLastError());
        out = in == r1 ? r2 : r1;
        for (int st = 6; st <= 9; st++) {
            if ((rc = stage(in, in, 1.0, -1, 0.0, b, out))) return rc;
            in = out;
            out = out == r1 ? r2 : r1;
        }
        // q^{n+1} = 1 q2 + (3/5) q1 + ((1/10) dt) L(q1), written over q2
        return stage(in, nxt, 1.0, in, 3.0 / 5.0, (1.0 / 10.0) * dt, nxt);
    }
    case 5: {  // :267-288: per stage L(q1) into r2, then the update of q1 (nxt) and q2 (r1)
        const rk::Rk5Coef c = rk::rk5_coefficients();
        for (int st = 0; st < 8; st++) {
            const int in = st == 0 ? qn : nxt;
            if ((rc = stage(in, -1, 0.0, -1, 0.0, 1.0, -1))) return rc;
            CK(cudaMemsetAsync(alpha_slot(s, nxt), 0, 2 * sizeof(double), s->stream));
            rk::k_rk5_update<<<eb, 256, 0, s->stream>>>(s->q[in], s->q[nxt], st == 0 ? nullptr : s->q[r1], s->q[r1],
                                                        s->q[qn], s->q[r2], s->plane, n, c.g1[st], c.g2[st],
                                                        c.g3[st], c.delta[st], c.beta[st] * dt, p.gamma,
                                                        alpha_slot(s, nxt), s->status);
            s->launches++;
            CK(cudaGetLastError());
        }
        return FIN_OK;
    }
    default:
        return set_err(FIN_ERR_UNSUPPORTED, "Runge-Kutta time_order must be 1 to 5");
    }
}

int take_stages_rk(fin_solver* s, double dt, int nxt, const unsigned* flags, int q1, int q2)
{
    const fin_params& p = s->p;
    if (p.time_order != 3) return take_stages_rk_other(s, dt, nxt);
    const int qn = s->cur;
    // reset smax, the status word and the alpha slots of the three buffers
    // written this step
    CK(cudaMemsetAsync(s->slots + SLOT_SMAX, 0, 2 * sizeof(double), s->stream));
    CK(cudaMemsetAsync(s->slots + SLOT_STATUS, 0, sizeof(double), s->stream));
    CK(cudaMemsetAsync(alpha_slot(s, q1), 0, 2 * sizeof(double), s->stream));
    CK(cudaMemsetAsync(alpha_slot(s, q2), 0, 2 * sizeof(double), s->stream));
    CK(cudaMemsetAsync(alpha_slot(s, nxt), 0, 2 * sizeof(double), s->stream));
    const bool ga = p.global_alpha != 0;
    int rc;
    StageArgs a = base_args(s);
    a.smax_out = s->slots + SLOT_SMAX;
    a.flags = flags;
    // stage 1: q1 = 1*q^n + 0*q* + (1*dt) L(q^n)
    a.qin = s->q[qn]; a.A = s->q[qn]; a.B = nullptr; a.qout = s->q[q1];
    a.a1 = 1.0; a.a2 = 0.0; a.bdt = 1.0 * dt;
    a.alpha_in = ga ? alpha_slot(s, qn) : nullptr;
    a.alpha_out = alpha_slot(s, q1);
    if ((rc = launch_stage_timed(s, a, 0))) return rc;
    // stage 2: q2 = 0.75 q^n + 0.25 q1 + (0.25 dt) L(q1)
    a.qin = s->q[q1]; a.A = s->q[qn]; a.B = s->q[q1]; a.qout = s->q[q2];
    a.a1 = 0.75; a.a2 = 0.25; a.bdt = 0.25 * dt;
    a.alpha_in = ga ? alpha_slot(s, q1) : nullptr;
    a.alpha_out = alpha_slot(s, q2);
    if ((rc = launch_stage_timed(s, a, 1))) return rc;
    // stage 3: q^{n+1} = (2/3) q2 + (1/3) q^n + ((2/3) dt) L(q2)
    a.qin = s->q[q2]; a.A = s->q[q2]; a.B = s->q[qn]; a.qout = s->q[nxt];
    a.a1 = 2.0e0 / 3.0e0; a.a2 = 1.0e0 / 3.0e0; a.bdt = (2.0e0 / 3.0e0) * dt;
    a.alpha_in = ga ? alpha_slot(s, q2) : nullptr;
    a.alpha_out = alpha_slot(s, nxt);
    if ((rc = launch_stage_timed(s, a, 2))) return rc;
    return FIN_OK;
}

// GetCFL (lib/2d/GetCFL.cpp:31-73) from the step's face-speed maxima: the
// maximum of dt*smax/dx over faces equals dt*max(smax)/dx because the
// rounded product and quotient are monotone in smax.
// *nonfinite reports NaN/Inf met during the step: like the reference, such a
// step is judged by the CFL of its finite face speeds (a rejected step is
// simply retried); the caller refuses to accept it.
int get_cfl(fin_solver* s, double dt, double dtmax, double* cfl, bool* nonfinite)
{
    CK(cudaMemcpyAsync(s->h_slots, s->slots, NSLOTS * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    unsigned int st;
    memcpy(&st, s->h_slots + SLOT_STATUS, sizeof(st));
    *nonfinite = (st & 1u) != 0;
    if (st & 12u) return set_err(FIN_ERR_CUDA, "a bounded device wait (tensor-core or TMA copy) ran out");
    if (st & 16u) return set_err(FIN_ERR_CUDA, "a TMA destination in shared memory was not 128-byte aligned");
    if (dt > dtmax) return set_err(FIN_ERR_DT_BOUNDS, "dt is out of bounds");
    double sx = s->h_slots[SLOT_SMAX], sy = s->h_slots[SLOT_SMAX + 1];
    if (s->p.time_stepping_method == FIN_TS_LXW && s->p.mpp_limiter) {
        // ConstructLFL.cpp:64-65 set smax(1,1,.) to q^n's global wave speeds
        sx = Max(sx, s->h_slots[SLOT_ALPHA + 2 * s->cur]);
        sy = Max(sy, s->h_slots[SLOT_ALPHA + 2 * s->cur + 1]);
    }
    double c = -100.0;
    c = Max(dt * sx / s->dx, c);
    c = Max(dt * sy / s->dy, c);
    if (c > 1.0e8) return set_err(FIN_ERR_CFL_BOUNDS, "CFL number is out of bounds");
    *cfl = c;
    return FIN_OK;
}

int validate(const fin_params* p)
{
    if (!p) return set_err(FIN_ERR_ARG, "null params");
    if (p->physics != FIN_PHYS_EULER || p->meqn != 5) return set_err(FIN_ERR_UNSUPPORTED, "only 2D Euler (meqn 5)");
    if (p->weno_version != FIN_WENO_JS && p->weno_version != FIN_WENO_Z && p->weno_version != FIN_WENO_FD)
        return set_err(FIN_ERR_ARG, "Requested WENO Reconstruction not implemented.");
    // GetWenoReconstruct (lib/WenoReconstruct.cpp:40-71): JS 5/7/9/11, FD 5/7/9,
    // Z 5/7/9, and order 1 (LLF) for every version; anything else throws there
    {
        const int so = p->space_order, v = p->weno_version;
        const bool built = so == 1 || so == 5 || so == 7 || so == 9 || (so == 11 && v == FIN_WENO_JS);
        if (!built) return set_err(FIN_ERR_ARG, "Requested WENO Reconstruction not implemented.");
    }
    if (p->mx < 1 || p->my < 1) return set_err(FIN_ERR_ARG, "mx, my must be positive");
    if (p->mbc < 3) return set_err(FIN_ERR_ARG, "mbc must be >= 3 for WENO5");
    if (p->space_order != 5) {
        // ConstructL.cpp:31-33: the stencil reaches r = (space_order + 1) / 2 cells out
        if (p->mbc < (p->space_order + 1) / 2) return set_err(FIN_ERR_ARG, "mbc must be >= (space_order + 1) / 2");
        if (p->time_stepping_method != FIN_TS_RK || p->precision != FIN_PREC_FP64)
            return set_err(FIN_ERR_UNSUPPORTED, "space orders other than 5 are built for FP64 Runge-Kutta stepping");
    }
    if (p->time_stepping_method == FIN_TS_RK && (p->time_order < 1 || p->time_order > 5))
        return set_err(FIN_ERR_UNSUPPORTED, "Runge-Kutta: time_order 1 to 5 (FinSolveRK.cpp:117-299)");
    if (p->time_stepping_method == FIN_TS_RK && p->time_order != 3 && p->precision == FIN_PREC_HYBRID)
        return set_err(FIN_ERR_UNSUPPORTED, "the hybrid form is built for SSP-RK3 (time_order 3)");
    if (p->time_stepping_method == FIN_TS_MD && p->time_order != 4 && p->time_order != 5)
        return set_err(FIN_ERR_UNSUPPORTED, "Multiderivative: time_order 4 or 5 (two-stage, FinSolveMD.cpp:116-226)");
    if (p->time_stepping_method != FIN_TS_RK && p->time_stepping_method != FIN_TS_MD &&
        p->time_stepping_method != FIN_TS_LXW)
        return set_err(FIN_ERR_ARG, "time_stepping_method");
    if (p->time_stepping_method != FIN_TS_RK) {
        // the integrated fluxes reach 5 cells out (ConstructIntegratedR.cpp:565 asserts it)
        if (p->mbc < 5) return set_err(FIN_ERR_ARG, "Lax-Wendroff / multiderivative stepping needs mbc >= 5");
        if (p->precision != FIN_PREC_FP64)
            return set_err(FIN_ERR_UNSUPPORTED, "Lax-Wendroff / multiderivative stepping is built in FP64 only");
    }
    if (p->source_term) return set_err(FIN_ERR_UNSUPPORTED, "source terms are not built");
    if (!(p->xhigh > p->xlow) || !(p->yhigh > p->ylow)) return set_err(FIN_ERR_ARG, "empty domain");
    for (int b : {p->bc_xlow, p->bc_xhigh, p->bc_ylow, p->bc_yhigh})
        if (b != FIN_BC_PERIODIC && b != FIN_BC_TRANSMISSIVE) return set_err(FIN_ERR_ARG, "bad boundary condition");
    if ((p->bc_xlow == FIN_BC_PERIODIC) != (p->bc_xhigh == FIN_BC_PERIODIC) ||
        (p->bc_ylow == FIN_BC_PERIODIC) != (p->bc_yhigh == FIN_BC_PERIODIC))
        return set_err(FIN_ERR_ARG, "periodic boundaries come in pairs");
    const int H = std::max(3, (p->space_order + 1) / 2);
    if ((p->bc_xlow == FIN_BC_PERIODIC && p->mx < H) || (p->bc_ylow == FIN_BC_PERIODIC && p->my < H))
        return set_err(FIN_ERR_ARG, "periodic direction shorter than the stencil halo");
    if (p->precision != FIN_PREC_FP64 && p->precision != FIN_PREC_FP32 && p->precision != FIN_PREC_HYBRID)
        return set_err(FIN_ERR_ARG, "unknown precision form");
    if (p->precision == FIN_PREC_HYBRID && p->time_stepping_method != FIN_TS_RK)
        return set_err(FIN_ERR_UNSUPPORTED, "the hybrid form is built for SSP-RK3");
    return FIN_OK;
}

size_t aos_elems_of(const fin_params& p)
{
    return size_t(p.mx + 2 * p.mbc) * (p.my + 2 * p.mbc) * p.meqn;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void fin_params_default(fin_params* p)
{
    memset(p, 0, sizeof(*p));
    p->meqn = 5; p->maux = 0;
    p->space_order = 5; p->time_order = 3;
    p->time_stepping_method = FIN_TS_RK;
    p->global_alpha = 0; p->source_term = 0;
    p->nv = 500000; p->verbosity = 0;
    p->initial_dt = 1e-3; p->max_dt = 1e10; p->max_cfl = 0.45; p->desired_cfl = 0.4;
    p->mx = 10; p->my = 10; p->mbc = 3;
    p->xlow = 0; p->xhigh = 1; p->ylow = 0; p->yhigh = 1;
    p->weno_version = FIN_WENO_JS;
    p->epsilon = 1e-6; p->power_param = 2.0; p->alpha_scaling = 1.1;
    p->gamma = 1.4;
    p->bc_xlow = p->bc_xhigh = p->bc_ylow = p->bc_yhigh = FIN_BC_PERIODIC;
    p->physics = FIN_PHYS_EULER;
    p->precision = FIN_PREC_FP64;
    p->tfinal = 0.0;
    p->nout = 1;
    p->constrained_transport = 1;
    p->mpp_limiter = 0;
}

const char* fin_last_error(void) { return g_err.c_str(); }

int fin_abi_version(void) { return FIN_ABI_VERSION; }

int fin_create(const fin_params* p, fin_solver** out)
{
    if (!out) return set_err(FIN_ERR_ARG, "null out");
    *out = nullptr;
    int rc = validate(p);
    if (rc) return rc;
    int dev = 0, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_err(FIN_ERR_NO_DEVICE, "no CUDA device");
    CK(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) return set_err(FIN_ERR_NO_DEVICE, "libfinb200 is compiled for sm_100a (B200)");

    fin_solver* s = new fin_solver();
    memset(s, 0, sizeof(*s));
    s->p = *p;
    s->dx = (p->xhigh - p->xlow) / p->mx;
    s->dy = (p->yhigh - p->ylow) / p->my;
    // planes padded to 32 elements (256 B) so every plane starts aligned
    s->plane = (size_t(p->mx) * p->my + 31) / 32 * 32;
    s->aos_elems = aos_elems_of(*p);
    auto fail = [&](cudaError_t e, const char* what) {
        fin_destroy(s);
        return set_err(FIN_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    cudaError_t e;
    const int nbuf = p->precision == FIN_PREC_HYBRID ? 5 : 4;
    for (int b = 0; b < nbuf; b++)
        if ((e = cudaMalloc(&s->q[b], MEQN * s->plane * sizeof(double))) != cudaSuccess) return fail(e, "cudaMalloc state");
    if (p->precision == FIN_PREC_HYBRID) {
        if ((e = cudaMalloc(&s->flags, flag_words(p->mx, p->my) * sizeof(unsigned))) != cudaSuccess)
            return fail(e, "cudaMalloc flags");
        if ((e = cudaMalloc(&s->ind_count, 16)) != cudaSuccess) return fail(e, "cudaMalloc counter");
        if ((e = cudaMemset(s->ind_count, 0, 16)) != cudaSuccess) return fail(e, "memset");
        s->zthr = 0.0f;
        s->judge_every = 20;
        s->judge_tol = 1e-3;
        s->ind_every = 1;
        s->ind_since = -1;
        bool ok = true;
        for (int b = 0; b < nbuf && ok; b++)
            ok = make_state_map(&s->tm_q[b], s->q[b], p->mx, p->my, s->plane, Cfg::SJ, Cfg::RI) &&
                 make_state_map(&s->tm_a[b], s->q[b], p->mx, p->my, s->plane, Cfg::TJ, Cfg::TI);
        s->tma_ok = ok;
    }
    if (p->time_stepping_method != FIN_TS_RK) {
        s->gplane = (size_t(p->mx + 6) * (p->my + 6) + 31) / 32 * 32;
        if ((e = cudaMalloc(&s->Fg, MEQN * s->gplane * sizeof(double))) != cudaSuccess) return fail(e, "cudaMalloc F");
        if ((e = cudaMalloc(&s->Gg, MEQN * s->gplane * sizeof(double))) != cudaSuccess) return fail(e, "cudaMalloc G");
    }
    if ((e = cudaMalloc(&s->slots, NSLOTS * sizeof(double))) != cudaSuccess) return fail(e, "cudaMalloc slots");
    s->status = reinterpret_cast<unsigned int*>(s->slots + SLOT_STATUS);
    if ((e = cudaMallocHost(&s->h_slots, NSLOTS * sizeof(double))) != cudaSuccess) return fail(e, "cudaMallocHost");
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaEventCreate(&s->ev0)) != cudaSuccess) return fail(e, "event");
    if ((e = cudaEventCreate(&s->ev1)) != cudaSuccess) return fail(e, "event");
    for (int k = 0; k < 6; k++)
        if ((e = cudaEventCreate(&s->kev[k])) != cudaSuccess) return fail(e, "event");
    for (int k = 0; k < 2; k++)
        if ((e = cudaEventCreate(&s->iev[k])) != cudaSuccess) return fail(e, "event");
    if ((e = cudaMemsetAsync(s->slots, 0, NSLOTS * sizeof(double), s->stream)) != cudaSuccess) return fail(e, "memset");
    for (int b = 0; b < nbuf; b++)
        if ((e = cudaMemsetAsync(s->q[b], 0, MEQN * s->plane * sizeof(double), s->stream)) != cudaSuccess) return fail(e, "memset");
    if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return fail(e, "sync");
    s->t = 0.0;
    *out = s;
    return FIN_OK;
}

int fin_destroy(fin_solver* s)
{
    if (!s) return FIN_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    delete s->writer;   // waits for a frame still being written
    delete s->cons_path;
    cudaFree(s->d_cons);
    if (s->h_cons) cudaFreeHost(s->h_cons);
    cudaFree(s->mpp_fx);
    cudaFree(s->mpp_fy);
    cudaFree(s->mpp_amin);
    for (int b = 0; b < NBUF; b++) cudaFree(s->q[b]);
    cudaFree(s->mlpP);
    cudaFree(s->flags);
    cudaFree(s->ind_count);
    cudaFree(s->slots);
    cudaFree(s->d_aos);
    cudaFree(s->d_aux);
    cudaFree(s->Fg);
    cudaFree(s->Gg);
    cudaFree(s->d_face_x);
    cudaFree(s->d_face_y);
    cudaFree(s->d_upd);
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

static int ensure_aos(fin_solver* s)
{
    if (!s->d_aos) CK(cudaMalloc(&s->d_aos, s->aos_elems * sizeof(double)));
    return FIN_OK;
}

static int upload(fin_solver* s, const double* q_host, int buf)
{
    int rc = ensure_aos(s);
    if (rc) return rc;
    CK(cudaMemsetAsync(s->slots + SLOT_STATUS, 0, sizeof(double), s->stream));
    CK(cudaMemcpyAsync(s->d_aos, q_host, s->aos_elems * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    const size_t n = size_t(s->p.mx) * s->p.my;
    k_aos_to_planes<<<grid_blocks(n), 256, 0, s->stream>>>(s->d_aos, s->q[buf], s->p.mx, s->p.my, s->p.mbc, s->plane);
    s->launches++;
    CK(cudaGetLastError());
    return FIN_OK;
}

int fin_set_state(fin_solver* s, const double* q_host, double t)
{
    if (!s || !q_host) return set_err(FIN_ERR_ARG, "null argument");
    int rc = upload(s, q_host, s->cur);
    if (rc) return rc;
    s->t = t;
    s->ind_since = -1;
    CK(cudaMemsetAsync(s->slots + SLOT_STATUS, 0, sizeof(double), s->stream));
    if ((rc = compute_alpha(s, s->cur))) return rc;
    s->alpha_valid = true;
    return check_status(s);
}

// Initial data sampled on the device (SampleFunction with a QinitFunc
// functor, fin_sample.cuh) straight into q^n: no host array, no upload.
int fin_set_state_qinit(fin_solver* s, int problem, const double* prm, int nprm, double t)
{
    if (!s) return set_err(FIN_ERR_ARG, "null solver");
    if (nprm > 0 && !prm) return set_err(FIN_ERR_ARG, "null parameters");
    const fin_params& p = s->p;
    double* q = s->q[s->cur];
    const double g = p.gamma;
    cudaError_t e = cudaSuccess;
    switch (problem) {
    case FIN_QINIT_VORTEX: {
        if (nprm != 0 && nprm != 3) return set_err(FIN_ERR_ARG, "vortex: parameters are eps, xc, yc");
        const qinit::Vortex f{g, nprm ? prm[0] : 5.0, nprm ? prm[1] : 5.0, nprm ? prm[2] : 5.0};
        e = launch_sample(f, p.xlow, p.ylow, s->dx, s->dy, p.mx, p.my, q, s->plane, s->stream);
        break;
    }
    case FIN_QINIT_RIEMANN4: {
        if (nprm != 0 && nprm != 18) return set_err(FIN_ERR_ARG, "riemann4: parameters are xc, yc, 4 x (rho, u, v, p)");
        static const double def[18] = {0.8, 0.8, 1.5, 0.0, 0.0, 1.5, 0.5323, 1.206, 0.0, 0.3,
                                       0.138, 1.206, 1.206, 0.029, 0.5323, 0.0, 1.206, 0.3};
        const double* v = nprm ? prm : def;
        qinit::Riemann4 f;
        f.gamma = g; f.xc = v[0]; f.yc = v[1];
        for (int k = 0; k < 4; k++)
            for (int c = 0; c < 4; c++) f.s[k][c] = v[2 + 4 * k + c];
        e = launch_sample(f, p.xlow, p.ylow, s->dx, s->dy, p.mx, p.my, q, s->plane, s->stream);
        break;
    }
    case FIN_QINIT_SHOCK_ENTROPY:
        e = launch_sample(qinit::ShockEntropy{g}, p.xlow, p.ylow, s->dx, s->dy, p.mx, p.my, q, s->plane, s->stream);
        break;
    case FIN_QINIT_SHOCK_TUBE: {
        if (nprm != 1) return set_err(FIN_ERR_ARG, "shock tube: one parameter, OPT");
        e = launch_sample(qinit::ShockTube{g, int(prm[0])}, p.xlow, p.ylow, s->dx, s->dy, p.mx, p.my, q, s->plane,
                          s->stream);
        break;
    }
    case FIN_QINIT_VORTEX_EXACT2:
        e = launch_sample(qinit::VortexExact2{g}, p.xlow, p.ylow, s->dx, s->dy, p.mx, p.my, q, s->plane, s->stream);
        break;
    default:
        return set_err(FIN_ERR_ARG, "unknown initial-data problem");
    }
    if (e != cudaSuccess) return set_err(FIN_ERR_CUDA, std::string("k_sample: ") + cudaGetErrorString(e));
    s->launches++;
    s->t = t;
    s->ind_since = -1;
    CK(cudaMemsetAsync(s->slots + SLOT_STATUS, 0, sizeof(double), s->stream));
    int rc = compute_alpha(s, s->cur);
    if (rc) return rc;
    s->alpha_valid = true;
    return check_status(s);
}

int fin_get_state(fin_solver* s, double* q_host, double* t)
{
    if (!s || !q_host) return set_err(FIN_ERR_ARG, "null argument");
    int rc = ensure_aos(s);
    if (rc) return rc;
    const size_t n = s->aos_elems / MEQN;
    k_planes_to_aos<<<grid_blocks(n), 256, 0, s->stream>>>(s->q[s->cur], s->d_aos, s->p.mx, s->p.my, s->p.mbc,
                                                           s->plane, s->p.bc_xlow, s->p.bc_xhigh, s->p.bc_ylow,
                                                           s->p.bc_yhigh);
    s->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(q_host, s->d_aos, s->aos_elems * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (t) *t = s->t;
    return FIN_OK;
}

int fin_global_wave_spd(fin_solver* s, const double* q_host, double* alpha1, double* alpha2)
{
    if (!s || !q_host || !alpha1 || !alpha2) return set_err(FIN_ERR_ARG, "null argument");
    // use the next-state buffer as scratch so the solver's state is untouched
    const int buf = (s->cur + 3) % 4;
    int rc = upload(s, q_host, buf);
    if (rc) return rc;
    if ((rc = compute_alpha(s, buf))) return rc;
    double h[2];
    CK(cudaMemcpyAsync(h, alpha_slot(s, buf), sizeof(h), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    *alpha1 = h[0];
    *alpha2 = h[1];
    return check_status(s);
}

static int download_l_smax(fin_solver* s, int outb, double* L_host, double* smax_host);

int fin_construct_l(fin_solver* s, const double* q_host, double* L_host, double* smax_host)
{
    if (!s || !q_host || !L_host) return set_err(FIN_ERR_ARG, "null argument");
    const fin_params& p = s->p;
    const int buf = (s->cur + 3) % 4, outb = (s->cur + 2) % 4;
    int rc = upload(s, q_host, buf);
    if (rc) return rc;
    if (p.global_alpha && (rc = compute_alpha(s, buf))) return rc;
    if (smax_host) {
        if (!s->d_face_x) CK(cudaMalloc(&s->d_face_x, size_t(p.mx + 1) * p.my * sizeof(double)));
        if (!s->d_face_y) CK(cudaMalloc(&s->d_face_y, size_t(p.mx) * (p.my + 1) * sizeof(double)));
    }
    StageArgs a = base_args(s);
    a.qin = s->q[buf];
    a.A = nullptr; a.B = nullptr; a.qout = s->q[outb];
    a.a1 = 0.0; a.a2 = 0.0; a.bdt = 1.0;
    a.alpha_in = p.global_alpha ? alpha_slot(s, buf) : nullptr;
    a.face_alpha_x = smax_host ? s->d_face_x : nullptr;
    a.face_alpha_y = smax_host ? s->d_face_y : nullptr;
    if ((rc = launch_stage(s, a))) return rc;
    return download_l_smax(s, outb, L_host, smax_host);
}

// L (interior of the ghosted output, ghosts untouched: the reference leaves
// Lstar's ghost entries uninitialised) from q[outb], and smax max-accumulated
// from the per-face speeds, then the status word.
static int download_l_smax(fin_solver* s, int outb, double* L_host, double* smax_host)
{
    const fin_params& p = s->p;
    const size_t n = size_t(p.mx) * p.my;
    std::vector<double> hl(MEQN * n);
    for (int m = 0; m < MEQN; m++)
        CK(cudaMemcpyAsync(hl.data() + m * n, s->q[outb] + m * s->plane, n * sizeof(double), cudaMemcpyDeviceToHost,
                           s->stream));
    CK(cudaStreamSynchronize(s->stream));
    {
        const int sy = p.my + 2 * p.mbc;
        for (int i = 0; i < p.mx; i++)
            for (int j = 0; j < p.my; j++)
                for (int m = 0; m < MEQN; m++)
                    L_host[(size_t(i + p.mbc) * sy + (j + p.mbc)) * MEQN + m] = hl[m * n + size_t(i) * p.my + j];
    }
    if (smax_host) {
        std::vector<double> fx(size_t(p.mx + 1) * p.my), fy(size_t(p.mx) * (p.my + 1));
        CK(cudaMemcpyAsync(fx.data(), s->d_face_x, fx.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaMemcpyAsync(fy.data(), s->d_face_y, fy.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        // smax is dTensorBC3(mx+1, my+1, 2, mbc): max-accumulate (ConstructL.cpp:173,324)
        const int sy = p.my + 1 + 2 * p.mbc;
        auto at = [&](int i, int j, int m) -> double& {   // 1-based i, j, m
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
    CK(cudaStreamSynchronize(s->stream));
    return check_status(s);
}

int fin_set_indicator(fin_solver* s, const float* params, float z_threshold, int judge_every, double judge_tol)
{
    if (!s || !params) return set_err(FIN_ERR_ARG, "null argument");
    if (s->p.precision != FIN_PREC_HYBRID) return set_err(FIN_ERR_ARG, "the solver was not created in the hybrid form");
    if (!s->mlpP) CK(cudaMalloc(&s->mlpP, mlp::NPARAM * sizeof(float)));
    CK(cudaMemcpyAsync(s->mlpP, params, mlp::NPARAM * sizeof(float), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->zthr = z_threshold;
    // A face whose six stencil states are equal has all-zero features; when
    // the network's output for that row lies clearly below the threshold,
    // the indicator skips such faces (the same flags, less work).
    s->ind_skip_const = ind::zero_row_logit(params) < double(z_threshold) - 0.05;
    s->judge_every = judge_every;
    s->judge_tol = judge_tol;
    s->hyb_off = 0;
    s->ind_since = -1;
    if (s->ind_every < 1) s->ind_every = 1;
    return FIN_OK;
}

int fin_set_indicator_every(fin_solver* s, int every)
{
    if (!s) return set_err(FIN_ERR_ARG, "null argument");
    if (every < 1) return set_err(FIN_ERR_ARG, "the indicator period must be at least one step");
    s->ind_every = every;
    s->ind_since = -1;
    return FIN_OK;
}

int fin_hybrid_stats(fin_solver* s, long long* troubled_faces, long long* faces, long long* judges, long long* reverts)
{
    if (!s) return set_err(FIN_ERR_ARG, "null solver");
    if (s->ind_count) {
        unsigned long long c = 0;
        CK(cudaMemcpyAsync(&c, s->ind_count, sizeof(c), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        s->troubled_last = (long long)c;
    }
    if (troubled_faces) *troubled_faces = s->troubled_last;
    if (faces) *faces = s->faces;
    if (judges) *judges = s->judges;
    if (reverts) *reverts = s->reverts;
    return FIN_OK;
}

int fin_hybrid_flags(fin_solver* s, unsigned* words_host, size_t nwords)
{
    if (!s || !words_host) return set_err(FIN_ERR_ARG, "null argument");
    if (!s->flags) return set_err(FIN_ERR_ARG, "the solver holds no indicator flags");
    const size_t n = flag_words(s->p.mx, s->p.my);
    if (nwords < n) return set_err(FIN_ERR_SIZE, "flag buffer too small");
    CK(cudaMemcpyAsync(words_host, s->flags, n * sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return FIN_OK;
}

int fin_face_samples(fin_solver* s, long long offset, long long stride, long long max_n, float* X_host,
                     unsigned char* y_host, long long* n_out)
{
    if (!s || !X_host || !y_host || !n_out || stride < 1 || offset < 0) return set_err(FIN_ERR_ARG, "bad argument");
    const fin_params& p = s->p;
    const long long nf = (long long)(p.mx + 1) * p.my + (long long)p.mx * (p.my + 1);
    long long n = offset < nf ? (nf - offset + stride - 1) / stride : 0;
    if (n > max_n) n = max_n;
    *n_out = n;
    if (n == 0) return FIN_OK;
    int rc;
    if (p.global_alpha && !s->alpha_valid && (rc = compute_alpha(s, s->cur))) return rc;
    float* dX = nullptr;
    unsigned char* dy = nullptr;
    CK(cudaMallocAsync(&dX, size_t(n) * ind::NFEAT * sizeof(float), s->stream));
    CK(cudaMallocAsync(&dy, size_t(n), s->stream));
    k_face_samples<<<grid_blocks(size_t(n)), 256, 0, s->stream>>>(
        s->q[s->cur], s->plane, p.mx, p.my, p.bc_xlow, p.bc_xhigh, p.bc_ylow, p.bc_yhigh, p.gamma, p.epsilon,
        p.power_param, p.alpha_scaling, p.global_alpha ? alpha_slot(s, s->cur) : nullptr, offset, stride, n, dX, dy);
    s->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(X_host, dX, size_t(n) * ind::NFEAT * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(y_host, dy, size_t(n), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaFreeAsync(dX, s->stream));
    CK(cudaFreeAsync(dy, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return FIN_OK;
}

static int download_fg(fin_solver* s, double* F_host, double* G_host);

// ConstructIntegratedR, 1-state (lib/2d/ConstructIntegratedR.cpp:59-296).
int fin_construct_integrated_r(fin_solver* s, double dt, const double* q_host, double* F_host, double* G_host)
{
    if (!s || !q_host || !F_host || !G_host) return set_err(FIN_ERR_ARG, "null argument");
    if (!s->Fg) return set_err(FIN_ERR_ARG, "the solver was created for Runge-Kutta stepping (no F, G buffers)");
    const fin_params& p = s->p;
    const int buf = (s->cur + 3) % 4;
    int rc = upload(s, q_host, buf);
    if (rc) return rc;
    if ((rc = launch_intflux(s, p.time_order > 2 ? 1 : 0, s->q[buf], nullptr, dt, 0, 0, 0, 0))) return rc;
    return download_fg(s, F_host, G_host);
}

// s->Fg, s->Gg -> the interior and 3-cell ghost frame of ghosted host arrays.
static int download_fg(fin_solver* s, double* F_host, double* G_host)
{
    const fin_params& p = s->p;
    std::vector<double> hf(MEQN * s->gplane), hg(MEQN * s->gplane);
    CK(cudaMemcpyAsync(hf.data(), s->Fg, hf.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(hg.data(), s->Gg, hg.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const int sy = p.my + 2 * p.mbc;
    for (int i = -3; i < p.mx + 3; i++)
        for (int j = -3; j < p.my + 3; j++)
            for (int m = 0; m < MEQN; m++) {
                const size_t dst = (size_t(i + p.mbc) * sy + (j + p.mbc)) * MEQN + m;
                const size_t src = m * s->gplane + size_t(i + 3) * (p.my + 6) + (j + 3);
                F_host[dst] = hf[src];
                G_host[dst] = hg[src];
            }
    return FIN_OK;
}

// The 2-state and three-coefficient forms (ConstructIntegratedR.cpp:525-606,
// 608-700): q1 into the first scratch buffer, q2 into the second.
static int construct_integrated_r_two(fin_solver* s, int mode, double dt, double a1, double b1, double c1,
                                      const double* q1_host, double a2, double b2, double c2,
                                      const double* q2_host, double* F_host, double* G_host)
{
    if (!s || !q1_host || !q2_host || !F_host || !G_host) return set_err(FIN_ERR_ARG, "null argument");
    if (!s->Fg) return set_err(FIN_ERR_ARG, "the solver was created for Runge-Kutta stepping (no F, G buffers)");
    const int b1f = (s->cur + 3) % 4, b2f = (s->cur + 2) % 4;
    int rc = upload(s, q1_host, b1f);
    if (rc) return rc;
    if ((rc = upload(s, q2_host, b2f))) return rc;
    if ((rc = launch_intflux(s, mode, s->q[b1f], s->q[b2f], dt, a1, b1, a2, b2, c1, c2))) return rc;
    return download_fg(s, F_host, G_host);
}

int fin_construct_integrated_r2(fin_solver* s, double dt, double alpha1, double beta1, const double* q1_host,
                                double alpha2, double beta2, const double* q2_host, double* F_host, double* G_host)
{
    return construct_integrated_r_two(s, 2, dt, alpha1, beta1, 0.0, q1_host, alpha2, beta2, 0.0, q2_host, F_host,
                                      G_host);
}

int fin_construct_integrated_r3(fin_solver* s, double dt, double alpha1, double beta1, double charlie1,
                                const double* q1_host, double alpha2, double beta2, double charlie2,
                                const double* q2_host, double* F_host, double* G_host)
{
    return construct_integrated_r_two(s, 3, dt, alpha1, beta1, charlie1, q1_host, alpha2, beta2, charlie2, q2_host,
                                      F_host, G_host);
}

// ConstructLxWL (lib/2d/ConstructLxWL.cpp:30-414): the stage kernel in its
// F, G mode (the sampled time-integrated fluxes split in place of FluxFunc of
// q, ConstructLxWL.cpp:150-155) with no update (L alone), the per-face speeds
// for smax, and, when asked, the face fluxes Fhat / Ghat.
int fin_construct_lxwl(fin_solver* s, const double* q_host, const double* F_host, const double* G_host,
                       double* L_host, double* smax_host, double* Fhat_host, double* Ghat_host)
{
    if (!s || !q_host || !F_host || !G_host || !L_host) return set_err(FIN_ERR_ARG, "null argument");
    if (!s->Fg) return set_err(FIN_ERR_ARG, "the solver was created for Runge-Kutta stepping (no F, G buffers)");
    const fin_params& p = s->p;
    if (p.space_order != 5) return set_err(FIN_ERR_UNSUPPORTED, "ConstructLxWL is built for space_order 5");
    const int buf = (s->cur + 3) % 4, outb = (s->cur + 2) % 4;
    int rc = upload(s, q_host, buf);
    if (rc) return rc;
    if (p.global_alpha && (rc = compute_alpha(s, buf))) return rc;
    // F, G: ghosted host layout -> the (mx+6) x (my+6) frame planes
    {
        const int sy = p.my + 2 * p.mbc;
        std::vector<double> hf(MEQN * s->gplane, 0.0), hg(MEQN * s->gplane, 0.0);
        for (int i = -3; i < p.mx + 3; i++)
            for (int j = -3; j < p.my + 3; j++)
                for (int m = 0; m < MEQN; m++) {
                    const size_t src = (size_t(i + p.mbc) * sy + (j + p.mbc)) * MEQN + m;
                    const size_t dst = m * s->gplane + size_t(i + 3) * (p.my + 6) + (j + 3);
                    hf[dst] = F_host[src];
                    hg[dst] = G_host[src];
                }
        CK(cudaMemcpyAsync(s->Fg, hf.data(), hf.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
        CK(cudaMemcpyAsync(s->Gg, hg.data(), hg.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    }
    const size_t nx = size_t(p.mx + 1) * p.my, ny = size_t(p.mx) * (p.my + 1);
    if (smax_host) {
        if (!s->d_face_x) CK(cudaMalloc(&s->d_face_x, nx * sizeof(double)));
        if (!s->d_face_y) CK(cudaMalloc(&s->d_face_y, ny * sizeof(double)));
    }
    const bool fluxes = Fhat_host || Ghat_host;
    if (fluxes) {
        if (!s->mpp_fx) CK(cudaMalloc(&s->mpp_fx, MEQN * nx * sizeof(double)));
        if (!s->mpp_fy) CK(cudaMalloc(&s->mpp_fy, MEQN * ny * sizeof(double)));
    }
    StageArgs a = base_args(s);
    a.Fg = s->Fg; a.Gg = s->Gg; a.gplane = s->gplane;
    a.qin = s->q[buf];
    a.A = nullptr; a.B = nullptr; a.qout = s->q[outb];
    a.a1 = 0.0; a.a2 = 0.0; a.bdt = 1.0;
    a.alpha_in = p.global_alpha ? alpha_slot(s, buf) : nullptr;
    a.face_alpha_x = smax_host ? s->d_face_x : nullptr;
    a.face_alpha_y = smax_host ? s->d_face_y : nullptr;
    a.flux_x = fluxes ? s->mpp_fx : nullptr;
    a.flux_y = fluxes ? s->mpp_fy : nullptr;
    if ((rc = launch_stage(s, a))) return rc;
    if (fluxes) {
        std::vector<double> fx(MEQN * nx), fy(MEQN * ny);
        CK(cudaMemcpyAsync(fx.data(), s->mpp_fx, fx.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaMemcpyAsync(fy.data(), s->mpp_fy, fy.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        // Fhat: dTensorBC3(mx+1, my, meqn, mbc), Ghat: dTensorBC3(mx, my+1, meqn, mbc)
        // (ConstructLxWL.cpp:63-70); faces 1..mx+1 x 1..my and 1..mx x 1..my+1
        if (Fhat_host) {
            const int sy = p.my + 2 * p.mbc;
            for (int i = 0; i <= p.mx; i++)
                for (int j = 0; j < p.my; j++)
                    for (int m = 0; m < MEQN; m++)
                        Fhat_host[(size_t(i + p.mbc) * sy + (j + p.mbc)) * MEQN + m] =
                            fx[(size_t(m) * (p.mx + 1) + i) * p.my + j];
        }
        if (Ghat_host) {
            const int sy = p.my + 1 + 2 * p.mbc;
            for (int i = 0; i < p.mx; i++)
                for (int j = 0; j <= p.my; j++)
                    for (int m = 0; m < MEQN; m++)
                        Ghat_host[(size_t(i + p.mbc) * sy + (j + p.mbc)) * MEQN + m] =
                            fy[(size_t(m) * p.mx + i) * (p.my + 1) + j];
        }
    }
    return download_l_smax(s, outb, L_host, smax_host);
}

// UpdateSoln (lib/2d/UpdateSoln.cpp:14-38) on ghosted host arrays: every
// element, in the reference's order ((alpha1 q* + alpha2 q) + (beta dt) L),
// each product and sum rounded on its own.
int fin_update_soln(fin_solver* s, double alpha1, double alpha2, double beta, double dt, const double* qstar_host,
                    double t_star, const double* L_host, double* qnew_host, double* t_new)
{
    if (!s || !qstar_host || !L_host || !qnew_host || !t_new) return set_err(FIN_ERR_ARG, "null argument");
    const size_t n = s->aos_elems;
    if (!s->d_upd) CK(cudaMalloc(&s->d_upd, 4 * n * sizeof(double)));
    double* dqs = s->d_upd;
    double* dL = s->d_upd + n;
    double* dqn = s->d_upd + 2 * n;
    CK(cudaMemcpyAsync(dqs, qstar_host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(dL, L_host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(dqn, qnew_host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    k_update_soln<<<grid_blocks(n), 256, 0, s->stream>>>(dqs, dL, dqn, n, alpha1, alpha2, beta * dt);
    s->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(qnew_host, dqn, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    // UpdateSoln.cpp:27
    *t_new = alpha1 * t_star + alpha2 * *t_new + beta * dt;
    return FIN_OK;
}

// The fifth-order stepper's UpdateSoln (lib/2d/UpdateSoln.cpp:43-80) on
// ghosted host arrays; the reference leaves the times alone.
int fin_update_soln5(fin_solver* s, double g1, double g2, double g3, double delta, double beta, double dt,
                     const double* qold_host, const double* L_host, double* q1_host, double* q2_host)
{
    if (!s || !qold_host || !L_host || !q1_host || !q2_host) return set_err(FIN_ERR_ARG, "null argument");
    const size_t n = s->aos_elems;
    if (!s->d_upd) CK(cudaMalloc(&s->d_upd, 4 * n * sizeof(double)));
    double* dqo = s->d_upd;
    double* dL = s->d_upd + n;
    double* dq1 = s->d_upd + 2 * n;
    double* dq2 = s->d_upd + 3 * n;
    CK(cudaMemcpyAsync(dqo, qold_host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(dL, L_host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(dq1, q1_host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(dq2, q2_host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    k_update_soln5<<<grid_blocks(n), 256, 0, s->stream>>>(dqo, dL, dq1, dq2, n, g1, g2, g3, delta, beta * dt);
    s->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(q1_host, dq1, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(q2_host, dq2, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return FIN_OK;
}

// GetCFL (lib/2d/GetCFL.cpp:31-73) on a ghosted smax array: the maxima of
// smax(i,j,1) and smax(i,j,2) over i <= mx, j <= my on the device (NaN
// entries skipped: the reference's Max(a, b) = a > b ? a : b drops them),
// then max(dt S1/dx, dt S2/dy), which equals the reference's per-entry
// maximum because the rounded product and quotient are monotone in S.
int fin_get_cfl(fin_solver* s, double dt, double dtmax, const double* smax_host, double* cfl)
{
    if (!s || !smax_host || !cfl) return set_err(FIN_ERR_ARG, "null argument");
    if (dt > dtmax) return set_err(FIN_ERR_DT_BOUNDS, "dt is out of bounds");
    const fin_params& p = s->p;
    const size_t n = size_t(p.mx + 1 + 2 * p.mbc) * (p.my + 1 + 2 * p.mbc) * 2;
    int rc = ensure_aos(s);
    if (rc) return rc;
    if (n > s->aos_elems) return set_err(FIN_ERR_ARG, "smax larger than the staging buffer");
    CK(cudaMemcpyAsync(s->d_aos, smax_host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemsetAsync(s->slots + SLOT_SMAX_ALT, 0, 2 * sizeof(double), s->stream));
    const size_t cells = size_t(p.mx) * p.my;
    k_smax_max<<<grid_blocks(cells), 256, 0, s->stream>>>(s->d_aos, p.mx, p.my, p.mbc, s->slots + SLOT_SMAX_ALT);
    s->launches++;
    CK(cudaGetLastError());
    double h[2];
    CK(cudaMemcpyAsync(h, s->slots + SLOT_SMAX_ALT, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    double c = -100.0;
    c = Max(dt * h[0] / s->dx, c);
    c = Max(dt * h[1] / s->dy, c);
    *cfl = c;
    if (c > 1.0e8) return set_err(FIN_ERR_CFL_BOUNDS, "CFL number is out of bounds");
    return FIN_OK;
}

// GetCFL from the global wave speeds (lib/2d/GetCFL.cpp:76-101).
int fin_get_cfl_alpha(const fin_params* p, double dt, double dtmax, double alpha1, double alpha2, double* cfl)
{
    if (!p || !cfl) return set_err(FIN_ERR_ARG, "null argument");
    if (p->mx < 1 || p->my < 1 || !(p->xhigh > p->xlow) || !(p->yhigh > p->ylow))
        return set_err(FIN_ERR_ARG, "bad grid");
    if (dt > dtmax) return set_err(FIN_ERR_DT_BOUNDS, "dt is out of bounds");
    const double dx = (p->xhigh - p->xlow) / p->mx, dy = (p->yhigh - p->ylow) / p->my;
    double c = -100.0;
    c = Max(dt * alpha1 / dx, c);
    c = Max(dt * alpha2 / dy, c);
    *cfl = c;
    if (c > 1.0e8) return set_err(FIN_ERR_CFL_BOUNDS, "CFL number is out of bounds");
    return FIN_OK;
}

int fin_step_fixed(fin_solver* s, double dt, double* cfl_out)
{
    if (!s) return set_err(FIN_ERR_ARG, "null solver");
    int rc;
    if (!s->alpha_valid && (rc = compute_alpha(s, s->cur))) return rc;
    const int nxt = (s->cur + 3) % 4;
    CK(cudaEventRecord(s->ev0, s->stream));
    if ((rc = take_stages(s, dt, nxt))) return rc;
    CK(cudaEventRecord(s->ev1, s->stream));
    double cfl = 0.0;
    bool nonfinite = false;
    if ((rc = get_cfl(s, dt, 1e300, &cfl, &nonfinite))) return rc;
    if ((rc = collect_kernel_times(s))) return rc;
    settle_judge(s, nxt, dt, &cfl);
    if (nonfinite) return set_err(FIN_ERR_NONFINITE, "non-finite wave speed or state");
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    s->last_ms = ms;
    s->cur = nxt;
    if (s->ind_since >= 0) s->ind_since++;
    s->alpha_valid = true;
    s->t = s->t + dt;
    if (cfl_out) *cfl_out = cfl;
    return FIN_OK;
}

int fin_solve(fin_solver* s, double tend, double* dtv, int* nsteps_out)
{
    return fin_advance(s, tend, dtv, 0x7fffffff, nsteps_out);
}

// lib/2d/FinSolveRK.cpp:13-371, stopping early after max_steps accepted steps.
// Qnew's time after one RK step from t (UpdateSoln.cpp:27 applied per stage
// with SetRKinfo's coefficients, each product and sum rounded on its own;
// Qstar's time, *t_star, carries over between steps as in FinSolveRK).  The
// fifth-order method's ten-argument UpdateSoln leaves the times alone
// (UpdateSoln.cpp:44-80), so its Qnew keeps the step's start time.
static double rk_time(int order, double t, double dt, double* t_star)
{
    switch (order) {
    case 1:
        return 1.0 * t + 0.0 * t + 1.0 * dt;
    case 2:
        *t_star = 1.0 * t + 0.0 * *t_star + 1.0 * dt;
        return 0.5 * *t_star + 0.5 * t + 0.5 * dt;
    case 4: {
        double t1 = t, t2 = t;
        for (int s = 1; s <= 5; s++) t1 = 1.0 * t1 + 0.0 * t1 + (1.0 / 6.0) * dt;
        const double tmp = (t2 + 9.0 * t1) / 25.0;
        t2 = tmp;
        t1 = 15.0 * tmp - 5.0 * t1;
        for (int s = 6; s <= 9; s++) t1 = 1.0 * t1 + 0.0 * t1 + (1.0 / 6.0) * dt;
        return 1.0 * t2 + (3.0 / 5.0) * t1 + (1.0 / 10.0) * dt;
    }
    case 5:
        return t;
    default:
        *t_star = 1.0 * t + 0.0 * *t_star + 1.0 * dt;
        *t_star = 0.75 * t + 0.25 * *t_star + 0.25 * dt;
        return (2.0e0 / 3.0e0) * *t_star + (1.0e0 / 3.0e0) * t + (2.0e0 / 3.0e0) * dt;
    }
}

// Conservation totals of q[cur] (lib/2d/ConSoln.cpp:34-93, written by
// FinSolveRK.cpp:362 after every accepted step): computed and copied to
// pinned memory on the stream; the line goes to the file at the next
// synchronisation (flush_conservation), so no step waits for it.
static int queue_conservation(fin_solver* s)
{
    if (!s->cons_path) return FIN_OK;
    fin::io::launch_totals(s->stream, s->q[s->cur], MEQN, s->plane, size_t(s->p.mx) * s->p.my, s->dx * s->dy,
                           s->d_cons + MEQN, s->d_cons);
    s->launches += 2;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(s->h_cons, s->d_cons, MEQN * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    s->cons_pending = true;
    s->cons_t = s->t;
    return FIN_OK;
}

// After a synchronisation of the stream: the pending line, if any.
static int flush_conservation(fin_solver* s)
{
    if (!s->cons_pending) return FIN_OK;
    s->cons_pending = false;
    if (fin::io::append_conservation(*s->cons_path, s->cons_t, s->h_cons, MEQN))
        return set_err(FIN_ERR_ARG, "cannot write " + *s->cons_path);
    return FIN_OK;
}

int fin_advance(fin_solver* s, double tend, double* dtv, int max_steps, int* nsteps_out)
{
    if (!s || !dtv) return set_err(FIN_ERR_ARG, "null argument");
    const fin_params& p = s->p;
    const double CFL_max = p.max_cfl, CFL_target = p.desired_cfl;
    double t = s->t;
    double dt = dtv[1], cfl = 0.0;
    double t_star = s->t;   // Qstar.get_t()
    int n_step = 0, accepted = 0, rc = FIN_OK;
    if (!s->alpha_valid && (rc = compute_alpha(s, s->cur))) return rc;
    double ms_total = 0.0;
    CK(cudaEventRecord(s->ev0, s->stream));
    s->step_ms = 0.0;
    while (t < tend && accepted < max_steps) {
        int m_accept = 0;
        n_step = n_step + 1;
        if (n_step > p.nv) { rc = set_err(FIN_ERR_NSTEPS, "Exceeded allowed # of time steps"); break; }
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
            if ((rc = flush_conservation(s))) goto done;
            if ((rc = collect_kernel_times(s))) goto done;
            settle_judge(s, nxt, dt, &cfl);
            // Qnew's time after the step: RK3 keeps UpdateSoln.cpp:27's
            // bookkeeping over its stages; FinSolveMD.cpp:162 and
            // FinSolveLxW.cpp:175 set Qold.t + dt (= told + dt here).
            double t_new;
            if (p.time_stepping_method == FIN_TS_RK) t_new = rk_time(p.time_order, s->t, dt, &t_star);
            else t_new = s->t + dt;
            if (cfl > 0.0) dt = Min(dtv[2], dt * CFL_target / cfl);
            else dt = dtv[2];
            if (p.verbosity)
                printf("%s ... Step%5d   CFL =%6.3f   dt =%11.3e   t =%11.3e\n",
                       p.time_stepping_method == FIN_TS_RK ? "FinSolveRK2D"
                                                           : (p.time_stepping_method == FIN_TS_MD ? "FinSolveMD2D" : "FinSolveLxW2D"),
                       n_step, cfl, dt, t);
            if (cfl <= CFL_max && nonfinite) {
                rc = set_err(FIN_ERR_NONFINITE, "non-finite wave speed or state in an accepted step");
                goto done;
            }
            if (cfl <= CFL_max) {
                m_accept = 1;
                s->cur = nxt;          // accept: q^{n+1} becomes q^n (alpha slot travels with it)
                if (s->ind_since >= 0) s->ind_since++;
                s->t = t_new;
            } else {
                t = told;              // reject: q^n was never overwritten
                s->t = t_old_q;
                if (p.verbosity) printf("FinSolveRK2D rejecting step...CFL number too large\n");
            }
        }
        accepted++;
        if ((rc = queue_conservation(s))) goto done;   // ConSoln(Qnew), FinSolveRK.cpp:362
    }
    dtv[1] = dt;
done:
    {
        cudaError_t e1 = cudaEventRecord(s->ev1, s->stream);
        if (e1 == cudaSuccess) e1 = cudaEventSynchronize(s->ev1);
        float ms = 0.f;
        if (e1 == cudaSuccess) e1 = cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        if (e1 == cudaSuccess) ms_total = ms;
        if (e1 == cudaSuccess) {
            const int rf = flush_conservation(s);
            if (!rc) rc = rf;
        }
    }
    s->last_ms = ms_total;
    if (nsteps_out) *nsteps_out = accepted;
    return rc;
}

int fin_fma_peak(int fp64, double* tflops)
{
    if (!tflops) return set_err(FIN_ERR_ARG, "null argument");
    int dev = 0, nsm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    void* out = nullptr;
    CK(cudaMalloc(&out, 64));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const int threads = 256, blocks = nsm * 8, iters = 1 << 14;
    double best = 0.0;
    for (int rep = 0; rep < 4; rep++) {
        CK(cudaEventRecord(e0, 0));
        if (fp64) k_fma_peak<double><<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
        else k_fma_peak<float><<<blocks, threads>>>((float*)out, iters, 0.999999f, 1e-7f);
        CK(cudaEventRecord(e1, 0));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        const double flops = 2.0 * 8.0 * double(iters) * threads * blocks;
        if (rep > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *tflops = best;
    return FIN_OK;
}

int fin_set_kernel_timing(fin_solver* s, int on)
{
    if (!s) return set_err(FIN_ERR_ARG, "null solver");
    s->time_kernels = on != 0;
    s->kernel_ms = 0.0;
    s->kernel_launches = 0;
    s->ind_ms = 0.0;
    s->ind_launches = 0;
    s->ind_timed = false;
    return FIN_OK;
}

int fin_indicator_time(fin_solver* s, double* ms, long long* launches)
{
    if (!s || !ms || !launches) return set_err(FIN_ERR_ARG, "null argument");
    *ms = s->ind_ms;
    *launches = s->ind_launches;
    return FIN_OK;
}

int fin_kernel_time(fin_solver* s, double* ms, long long* launches)
{
    if (!s || !ms || !launches) return set_err(FIN_ERR_ARG, "null argument");
    *ms = s->kernel_ms;
    *launches = s->kernel_launches;
    return FIN_OK;
}

int fin_conservation_totals(fin_solver* s, double* totals)
{
    if (!s || !totals) return set_err(FIN_ERR_ARG, "null argument");
    // Host-side compensated sum over a device->host copy of the planes.
    const size_t n = size_t(s->p.mx) * s->p.my;
    std::vector<double> h(n);
    for (int m = 0; m < MEQN; m++) {
        CK(cudaMemcpyAsync(h.data(), s->q[s->cur] + m * s->plane, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        double sum = 0.0, comp = 0.0;
        for (size_t k = 0; k < n; k++) {
            const double y = s->dx * s->dy * h[k] - comp;
            const double tt = sum + y;
            comp = (tt - sum) - y;
            sum = tt;
        }
        totals[m] = sum;
    }
    return FIN_OK;
}

int fin_set_conservation_file(fin_solver* s, const char* outdir)
{
    if (!s) return set_err(FIN_ERR_ARG, "null solver");
    if (s->cons_pending) {
        CK(cudaStreamSynchronize(s->stream));
        int rc = flush_conservation(s);
        if (rc) return rc;
    }
    delete s->cons_path;
    s->cons_path = nullptr;
    if (!outdir) return FIN_OK;
    struct stat st;
    if (stat(outdir, &st) != 0 || !S_ISDIR(st.st_mode)) return set_err(FIN_ERR_ARG, std::string("no directory ") + outdir);
    if (!s->d_cons) CK(cudaMalloc(&s->d_cons, (MEQN + 2 * MEQN * fin::io::NCHUNK) * sizeof(double)));
    if (!s->h_cons) CK(cudaMallocHost(&s->h_cons, MEQN * sizeof(double)));
    s->cons_path = new std::string(std::string(outdir) + "/conservation.dat");
    return FIN_OK;
}

int fin_write_conservation(fin_solver* s)
{
    if (!s) return set_err(FIN_ERR_ARG, "null solver");
    if (!s->cons_path) return set_err(FIN_ERR_ARG, "no conservation file set (fin_set_conservation_file)");
    int rc = queue_conservation(s);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->stream));
    return flush_conservation(s);
}

int fin_output_frame(fin_solver* s, int nframe, const char* outdir)
{
    if (!s || !outdir || nframe < 0) return set_err(FIN_ERR_ARG, "bad argument");
    if (!s->writer) s->writer = new fin::io::FrameWriter();
    char name[32];
    std::snprintf(name, sizeof(name), "/q%04d.dat", nframe);
    const std::string qpath = std::string(outdir) + name;
    std::snprintf(name, sizeof(name), "/a%04d.dat", nframe);
    const std::string apath = std::string(outdir) + name;
    // the Euler path holds no aux planes (its AuxFunc sets none,
    // apps/2d/euler/lib/AuxFunc.cpp:10-13): maux planes of zeros
    const int rc = s->writer->start(s->stream, s->q[s->cur], MEQN, nullptr, s->p.maux, s->plane, s->p.mx, s->p.my,
                                    s->t, qpath, apath);
    if (rc) return set_err(rc, s->writer->err());
    s->launches++;
    return FIN_OK;
}

int fin_output_wait(fin_solver* s)
{
    if (!s) return set_err(FIN_ERR_ARG, "null solver");
    if (!s->writer) return FIN_OK;
    const int rc = s->writer->wait();
    if (rc) return set_err(rc, s->writer->err());
    return FIN_OK;
}

int fin_read_frame(fin_solver* s, const char* path)
{
    if (!s || !path) return set_err(FIN_ERR_ARG, "null argument");
    if (s->writer) {   // a frame still being written may be the one read
        const int rw = s->writer->wait();
        if (rw) return set_err(rw, s->writer->err());
    }
    const size_t n = size_t(s->p.mx) * s->p.my * MEQN;
    double* stage = nullptr;
    CK(cudaMalloc(&stage, n * sizeof(double)));
    double t = 0.0;
    std::string msg;
    const int rc = fin::io::read_frame(path, s->stream, s->q[s->cur], MEQN, s->plane, s->p.mx, s->p.my, stage, &t, &msg);
    cudaFree(stage);
    if (rc) return set_err(rc, msg);
    s->launches++;
    s->t = t;
    s->ind_since = -1;
    CK(cudaMemsetAsync(s->slots + SLOT_STATUS, 0, sizeof(double), s->stream));
    int r2 = compute_alpha(s, s->cur);
    if (r2) return r2;
    s->alpha_valid = true;
    return check_status(s);
}

int fin_write_qhelp(const fin_params* p, const char* outdir)
{
    if (!p || !outdir) return set_err(FIN_ERR_ARG, "null argument");
    const std::string path = std::string(outdir) + "/qhelp.dat";
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return set_err(FIN_ERR_ARG, "cannot open " + path);
    // lib/2d/WriteQhelp.cpp:33-42, field by field
    std::fprintf(f, "%16d   : ndims   \n", 2);
    std::fprintf(f, "%16d   : meqn    \n", p->meqn);
    std::fprintf(f, "%16d   : maux    \n", p->maux);
    std::fprintf(f, "%16d   : nout    \n", p->nout);
    std::fprintf(f, "%16d   : mx      \n", p->mx);
    std::fprintf(f, "%16d   : my      \n", p->my);
    std::fprintf(f, "%16.8e : xlow    \n", p->xlow);
    std::fprintf(f, "%16.8e : xhigh   \n", p->xhigh);
    std::fprintf(f, "%16.8e : ylow    \n", p->ylow);
    std::fprintf(f, "%16.8e : yhigh   \n", p->yhigh);
    return std::fclose(f) == 0 ? FIN_OK : set_err(FIN_ERR_ARG, "write failed: " + path);
}

int fin_last_kernel_ms(fin_solver* s, double* ms)
{
    if (!s || !ms) return set_err(FIN_ERR_ARG, "null argument");
    *ms = s->last_ms;
    return FIN_OK;
}

int fin_launch_count(fin_solver* s, long long* launches)
{
    if (!s || !launches) return set_err(FIN_ERR_ARG, "null argument");
    *launches = s->launches;
    return FIN_OK;
}

int fin_device_layout(fin_solver* s, size_t* plane_stride, size_t* row_stride)
{
    if (!s) return set_err(FIN_ERR_ARG, "null solver");
    if (plane_stride) *plane_stride = s->plane;
    if (row_stride) *row_stride = size_t(s->p.my);
    return FIN_OK;
}

int fin_state_device_ptr(fin_solver* s, double** q_dev)
{
    if (!s || !q_dev) return set_err(FIN_ERR_ARG, "null argument");
    *q_dev = s->q[s->cur];
    return FIN_OK;
}

}  // extern "C"
