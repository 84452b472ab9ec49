// Batched solver: many independent 2D Euler problems of uneven grid sizes
// advanced together to a common end time, each with its own adaptive dt.
//
// Per problem the arithmetic is the single-problem solver's (the same stage
// kernel body, stage_tile, and FinSolveRK's time-step control of
// lib/2d/FinSolveRK.cpp:77-364), so every problem's result agrees with a
// separate fin_solve of it to rounding (the compiler may fuse a multiply-add
// differently in the two kernels).  What changes is the schedule:
//   * the step's control runs on the device, one thread per problem
//     (k_batch_prep: the attempt's dt, buffers and stage arguments;
//     k_batch_ctl: GetCFL, accept / reject, the next dt, done);
//   * each stage is ONE persistent launch over the tiles of all active
//     problems: CTAs take tiles from a work queue (an atomic counter), map a
//     tile to its problem by binary search in the tiles' prefix sums and run
//     the stage on it;
//   * a step (prep, three stages, control) is captured once in a CUDA graph
//     and replayed; the host reads one counter of active problems every few
//     replays;
//   * the tile shape is picked by timing each built shape on the batch itself
//     (the autotuner) before the first step.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>
#include "finess_b200.h"
#include "fin_stage.cuh"

using namespace fin;

namespace {

thread_local std::string g_berr;
int berr(int code, const std::string& m)
{
    g_berr = m;
    return code;
}
#define BCK(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return berr(FIN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Per-problem state on the device: geometry, buffers and FinSolveRK's host
// variables.
struct BProb {
    int mx, my, nv, pad;
    size_t plane;
    double dx, dy, rdx, rdy;
    double* q[4];
    int bc[4];
    double t_loop;     // FinSolveRK's t
    double t_state;    // Qnew.get_t()
    double told;       // start of the current attempt
    double dt;         // the attempt's dt, then the next dt
    double tend, max_dt, cfl_target, cfl_max;
    int cur, nxt, q1, q2;
    int active, fresh, n_step, accepted;
    int err;           // FIN_* code of a failed problem (0: none)
    unsigned int status;
    double smax[2];
    double alpha[4][2];
};

// ---- device control ------------------------------------------------------
// The attempt of every active problem: FinSolveRK.cpp:77-100 (step count,
// clip of dt to tend) and the stage arguments of SetRKinfo.cpp:50-64.
__global__ void k_batch_prep(BProb* pr, int n, StageArgs* args, const StageArgs tmpl, int global_alpha)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    BProb& b = pr[p];
    if (!b.active) return;
    if (b.fresh) {
        b.n_step++;
        if (b.n_step > b.nv) {
            b.err = FIN_ERR_NSTEPS;
            b.active = 0;
            return;
        }
        b.fresh = 0;
    }
    b.told = b.t_loop;
    if (b.told + b.dt > b.tend) b.dt = b.tend - b.told;
    b.nxt = (b.cur + 3) % 4;
    int reg[2] = {0, 0}, k = 0;
    for (int q = 0; q < 4 && k < 2; q++)
        if (q != b.cur && q != b.nxt) reg[k++] = q;
    b.q1 = reg[0];
    b.q2 = reg[1];
    b.smax[0] = b.smax[1] = 0.0;
    b.status = 0;
    b.alpha[b.q1][0] = b.alpha[b.q1][1] = 0.0;
    b.alpha[b.q2][0] = b.alpha[b.q2][1] = 0.0;
    b.alpha[b.nxt][0] = b.alpha[b.nxt][1] = 0.0;
    const double dt = b.dt;
    for (int s = 0; s < 3; s++) {
        StageArgs a = tmpl;
        a.mx = b.mx;
        a.my = b.my;
        a.plane = b.plane;
        a.rdx = b.rdx;
        a.rdy = b.rdy;
        a.bc[0] = b.bc[0]; a.bc[1] = b.bc[1]; a.bc[2] = b.bc[2]; a.bc[3] = b.bc[3];
        a.status = &b.status;
        a.smax_out = b.smax;
        const int in = s == 0 ? b.cur : (s == 1 ? b.q1 : b.q2);
        const int out = s == 0 ? b.q1 : (s == 1 ? b.q2 : b.nxt);
        a.qin = b.q[in];
        a.qout = b.q[out];
        if (s == 0) { a.A = b.q[b.cur]; a.B = nullptr; a.a1 = 1.0; a.a2 = 0.0; a.bdt = 1.0 * dt; }
        if (s == 1) { a.A = b.q[b.cur]; a.B = b.q[b.q1]; a.a1 = 0.75; a.a2 = 0.25; a.bdt = 0.25 * dt; }
        if (s == 2) {
            a.A = b.q[b.q2]; a.B = b.q[b.cur]; a.a1 = 2.0e0 / 3.0e0; a.a2 = 1.0e0 / 3.0e0;
            a.bdt = (2.0e0 / 3.0e0) * dt;
        }
        a.alpha_in = global_alpha ? b.alpha[in] : nullptr;
        a.alpha_out = b.alpha[out];
        args[size_t(s) * n + p] = a;
    }
}

// GetCFL (lib/2d/GetCFL.cpp:31-73) and FinSolveRK.cpp:300-357 per problem:
// CFL from the step's face-speed maxima, Qnew's time, the next dt, accept or
// reject; counts the problems still active.
__global__ void k_batch_ctl(BProb* pr, int n, int* nactive)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    BProb& b = pr[p];
    if (!b.active) return;
    const double dt = b.dt;
    if (dt > b.max_dt) {
        b.err = FIN_ERR_DT_BOUNDS;
        b.active = 0;
        return;
    }
    double c = -100.0;
    c = Max(__ddiv_rn(__dmul_rn(dt, b.smax[0]), b.dx), c);
    c = Max(__ddiv_rn(__dmul_rn(dt, b.smax[1]), b.dy), c);
    if (c > 1.0e8) {
        b.err = FIN_ERR_CFL_BOUNDS;
        b.active = 0;
        return;
    }
    const bool nonfinite = (b.status & 1u) != 0;
    // Qnew's time after the three stages (UpdateSoln.cpp:27 per stage), each
    // product and sum rounded on its own as on the host
    double t_star = __dadd_rn(__dadd_rn(__dmul_rn(1.0, b.told), 0.0), __dmul_rn(1.0, dt));
    t_star = __dadd_rn(__dadd_rn(__dmul_rn(0.75, b.told), __dmul_rn(0.25, t_star)), __dmul_rn(0.25, dt));
    const double t_new = __dadd_rn(__dadd_rn(__dmul_rn(2.0e0 / 3.0e0, t_star), __dmul_rn(1.0e0 / 3.0e0, b.told)),
                                   __dmul_rn(2.0e0 / 3.0e0, dt));
    b.dt = c > 0.0 ? Min(b.max_dt, __ddiv_rn(__dmul_rn(dt, b.cfl_target), c)) : b.max_dt;
    if (c <= b.cfl_max) {
        if (nonfinite) {
            b.err = FIN_ERR_NONFINITE;
            b.active = 0;
            return;
        }
        b.cur = b.nxt;
        b.t_state = t_new;
        b.t_loop = __dadd_rn(b.told, dt);
        b.accepted++;
        b.fresh = 1;
    } else {
        b.t_loop = b.told;   // reject: q^n was never overwritten
    }
    if (!(b.t_loop < b.tend)) b.active = 0;
    if (b.active) atomicAdd(nactive, 1);
}

// The work queue of a step: the active problems (act[0 .. na-1]) and the
// prefix sums of their tile counts (tile0[0 .. na], tile0[na] = total), for
// the tile shape TI x TJ.  One CTA of 1024 threads, chunks of 1024 problems.
__global__ void __launch_bounds__(1024) k_batch_queue(const BProb* pr, int n, int TI, int TJ, int* act,
                                                      long long* tile0, int* nact_out)
{
    __shared__ long long sc[1024];
    __shared__ int si[1024];
    __shared__ long long base_t;
    __shared__ int base_i;
    const int tid = threadIdx.x;
    if (tid == 0) { base_t = 0; base_i = 0; }
    __syncthreads();
    for (int c0 = 0; c0 < n; c0 += 1024) {
        const int p = c0 + tid;
        const bool on = p < n && pr[p].active;
        const long long nt = on ? (long long)((pr[p].mx + TI - 1) / TI) * ((pr[p].my + TJ - 1) / TJ) : 0;
        sc[tid] = nt;
        si[tid] = on ? 1 : 0;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {   // inclusive scans (Hillis-Steele)
            const long long vt = tid >= o ? sc[tid - o] : 0;
            const int vi = tid >= o ? si[tid - o] : 0;
            __syncthreads();
            sc[tid] += vt;
            si[tid] += vi;
            __syncthreads();
        }
        if (on) {
            const int k = base_i + si[tid] - 1;
            act[k] = p;
            tile0[k] = base_t + sc[tid] - nt;
        }
        __syncthreads();
        if (tid == 0) {
            base_t += sc[1023];
            base_i += si[1023];
        }
        __syncthreads();
    }
    if (tid == 0) {
        tile0[base_i] = base_t;
        *nact_out = base_i;
    }
}

// One stage over every active problem: persistent CTAs take tiles from the
// work queue and find the tile's problem by binary search in the prefix sums.
template <class R, int VER, bool P2, class Cfg>
__global__ void __launch_bounds__(Cfg::NT, MinBlocks<R>::value)
k_stage_batch(const BProb* pr, const int* act, const long long* tile0, const int* nact, const StageArgs* args,
              unsigned long long* queue)
{
    __shared__ long long s_tile;
    const int na = *nact;
    const long long total = tile0[na];
    for (;;) {
        __syncthreads();   // the previous tile's shared memory is free
        if (threadIdx.x == 0) s_tile = (long long)atomicAdd(queue, 1ull);
        __syncthreads();
        const long long t = s_tile;
        if (t >= total) return;
        int lo = 0, hi = na - 1;   // the entry whose tiles contain t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tile0[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const int p = act[lo];
        const int lt = int(t - tile0[lo]), tj = (pr[p].my + Cfg::TJ - 1) / Cfg::TJ;
        stage_tile<R, VER, P2, Cfg>(args[p], (lt / tj) * Cfg::TI, (lt % tj) * Cfg::TJ);
    }
}

// Tile shapes the autotuner chooses from.
using BatchCfgA = TileCfg<15, 16, 256>;
using BatchCfgB = TileCfg<7, 32, 256>;
constexpr int NCFG = 2;

}  // namespace

struct fin_batch {
    int n;
    fin_params tmpl_p;          // shared parameters (from problem 0)
    std::vector<fin_params> p;
    std::vector<BProb> hb;      // host mirror
    BProb* db;
    StageArgs* dargs;
    int* dact;                  // active problems of the step
    long long* dtile0;          // prefix sums of their tiles
    int* dnact;                 // their count
    unsigned long long* dqueue; // three work-queue counters
    int* dactive;
    double* d_aos;              // staging for host-layout copies (largest problem)
    size_t aos_max;
    cudaStream_t stream;
    cudaEvent_t ev0, ev1;
    cudaGraphExec_t graph;
    int cfg;                    // chosen tile shape (-1: not yet tuned)
    double tune_ms[NCFG];
    double last_ms;
    long long replays;
};

namespace {

StageArgs template_args(const fin_params& p)
{
    StageArgs a;
    memset(&a, 0, sizeof(a));
    a.gamma = p.gamma;
    a.eps = p.epsilon;
    a.pw = p.power_param;
    a.alpha_scaling = p.alpha_scaling;
    a.gamma_f = float(p.gamma);
    a.eps_f = float(p.epsilon);
    a.pw_f = float(p.power_param);
    a.alpha_scaling_f = float(p.alpha_scaling);
    return a;
}

template <class Cfg, class R, int VER, bool P2>
int launch_batch_kernel(fin_batch* b, int cfgi, int stage)
{
    auto kern = k_stage_batch<R, VER, P2, Cfg>;
    const size_t smem = Cfg::template smem_bytes<R>();
    static int grid = 0;   // per instantiation: resident CTAs on the device
    if (!grid) {
        BCK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        int per_sm = 0, dev = 0, nsm = 0;
        BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Cfg::NT, smem));
        BCK(cudaGetDevice(&dev));
        BCK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        grid = std::max(1, per_sm) * nsm;
    }
    kern<<<grid, Cfg::NT, smem, b->stream>>>(b->db, b->dact, b->dtile0, b->dnact, b->dargs + size_t(stage) * b->n,
                                             b->dqueue + stage);
    BCK(cudaGetLastError());
    return FIN_OK;
}

template <class Cfg>
int launch_batch_stage(fin_batch* b, int cfgi, int stage)
{
    const bool f32 = b->tmpl_p.precision == FIN_PREC_FP32;
    const bool p2 = b->tmpl_p.power_param == 2.0;
    switch (b->tmpl_p.weno_version) {
    case FIN_WENO_JS:
        if (f32) return p2 ? launch_batch_kernel<Cfg, float, FIN_WENO_JS, true>(b, cfgi, stage)
                           : launch_batch_kernel<Cfg, float, FIN_WENO_JS, false>(b, cfgi, stage);
        return p2 ? launch_batch_kernel<Cfg, double, FIN_WENO_JS, true>(b, cfgi, stage)
                  : launch_batch_kernel<Cfg, double, FIN_WENO_JS, false>(b, cfgi, stage);
    case FIN_WENO_Z:
        if (f32) return p2 ? launch_batch_kernel<Cfg, float, FIN_WENO_Z, true>(b, cfgi, stage)
                           : launch_batch_kernel<Cfg, float, FIN_WENO_Z, false>(b, cfgi, stage);
        return p2 ? launch_batch_kernel<Cfg, double, FIN_WENO_Z, true>(b, cfgi, stage)
                  : launch_batch_kernel<Cfg, double, FIN_WENO_Z, false>(b, cfgi, stage);
    default:
        return f32 ? launch_batch_kernel<Cfg, float, FIN_WENO_FD, true>(b, cfgi, stage)
                   : launch_batch_kernel<Cfg, double, FIN_WENO_FD, true>(b, cfgi, stage);
    }
}

int launch_queue(fin_batch* b, int cfgi)
{
    const int TI = cfgi == 0 ? BatchCfgA::TI : BatchCfgB::TI, TJ = cfgi == 0 ? BatchCfgA::TJ : BatchCfgB::TJ;
    k_batch_queue<<<1, 1024, 0, b->stream>>>(b->db, b->n, TI, TJ, b->dact, b->dtile0, b->dnact);
    BCK(cudaGetLastError());
    return FIN_OK;
}

int launch_stage_cfg(fin_batch* b, int cfgi, int stage)
{
    return cfgi == 0 ? launch_batch_stage<BatchCfgA>(b, 0, stage) : launch_batch_stage<BatchCfgB>(b, 1, stage);
}

// One step of every active problem: prep, three stages, control.
int enqueue_step(fin_batch* b)
{
    const int nb = (b->n + 127) / 128;
    k_batch_prep<<<nb, 128, 0, b->stream>>>(b->db, b->n, b->dargs, template_args(b->tmpl_p), b->tmpl_p.global_alpha);
    BCK(cudaGetLastError());
    int rq = launch_queue(b, b->cfg);
    if (rq) return rq;
    BCK(cudaMemsetAsync(b->dqueue, 0, 3 * sizeof(unsigned long long), b->stream));
    for (int s = 0; s < 3; s++) {
        const int rc = launch_stage_cfg(b, b->cfg, s);
        if (rc) return rc;
    }
    BCK(cudaMemsetAsync(b->dactive, 0, sizeof(int), b->stream));
    k_batch_ctl<<<nb, 128, 0, b->stream>>>(b->db, b->n, b->dactive);
    BCK(cudaGetLastError());
    return FIN_OK;
}

// The autotuner: each tile shape times stage 1 of the current attempt (which
// writes only the first stage register), best of three; the control state is
// restored afterwards.
int autotune(fin_batch* b)
{
    std::vector<BProb> save(b->n);
    BCK(cudaMemcpyAsync(save.data(), b->db, b->n * sizeof(BProb), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    const int nb = (b->n + 127) / 128;
    k_batch_prep<<<nb, 128, 0, b->stream>>>(b->db, b->n, b->dargs, template_args(b->tmpl_p), b->tmpl_p.global_alpha);
    BCK(cudaGetLastError());
    for (int c = 0; c < NCFG; c++) {
        double best = 1e30;
        const int rq = launch_queue(b, c);
        if (rq) return rq;
        for (int rep = 0; rep < 3; rep++) {
            BCK(cudaMemsetAsync(b->dqueue, 0, sizeof(unsigned long long), b->stream));
            BCK(cudaEventRecord(b->ev0, b->stream));
            const int rc = launch_stage_cfg(b, c, 0);
            if (rc) return rc;
            BCK(cudaEventRecord(b->ev1, b->stream));
            BCK(cudaEventSynchronize(b->ev1));
            float ms = 0.f;
            BCK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
            best = std::min(best, double(ms));
        }
        b->tune_ms[c] = best;
    }
    b->cfg = b->tune_ms[1] < b->tune_ms[0] ? 1 : 0;
    BCK(cudaMemcpyAsync(b->db, save.data(), b->n * sizeof(BProb), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    return FIN_OK;
}

int build_graph(fin_batch* b)
{
    if (b->graph) return FIN_OK;
    cudaGraph_t g;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_step(b);
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return berr(FIN_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    const cudaError_t e2 = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) return berr(FIN_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2));
    return FIN_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* fin_batch_last_error(void) { return g_berr.c_str(); }

int fin_batch_create(const fin_params* params, int nprob, fin_batch** out)
{
    if (!params || !out || nprob < 1) return berr(FIN_ERR_ARG, "null argument or empty batch");
    *out = nullptr;
    const fin_params& p0 = params[0];
    for (int k = 0; k < nprob; k++) {
        const fin_params& p = params[k];
        if (p.physics != FIN_PHYS_EULER || p.meqn != 5) return berr(FIN_ERR_UNSUPPORTED, "only 2D Euler (meqn 5)");
        if (p.time_stepping_method != FIN_TS_RK || p.time_order != 3)
            return berr(FIN_ERR_UNSUPPORTED, "the batch runs SSP-RK3");
        if (p.precision != FIN_PREC_FP64 && p.precision != FIN_PREC_FP32)
            return berr(FIN_ERR_UNSUPPORTED, "the batch runs the FP64 or FP32 form");
        if (p.space_order != 5 || p.mbc < 3 || p.mx < 1 || p.my < 1) return berr(FIN_ERR_ARG, "grid or order");
        if (p.weno_version != FIN_WENO_FD && p.weno_version != FIN_WENO_JS && p.weno_version != FIN_WENO_Z)
            return berr(FIN_ERR_ARG, "Requested WENO Reconstruction not implemented.");
        if (p.precision != p0.precision || p.weno_version != p0.weno_version || p.power_param != p0.power_param ||
            p.epsilon != p0.epsilon || p.gamma != p0.gamma || p.alpha_scaling != p0.alpha_scaling ||
            p.global_alpha != p0.global_alpha)
            return berr(FIN_ERR_ARG, "problems of a batch share precision, WENO and physics parameters");
        const int bcs[4] = {p.bc_xlow, p.bc_xhigh, p.bc_ylow, p.bc_yhigh};
        for (int bc : bcs)
            if (bc != FIN_BC_PERIODIC && bc != FIN_BC_TRANSMISSIVE) return berr(FIN_ERR_ARG, "bad boundary condition");
        if ((p.bc_xlow == FIN_BC_PERIODIC) != (p.bc_xhigh == FIN_BC_PERIODIC) ||
            (p.bc_ylow == FIN_BC_PERIODIC) != (p.bc_yhigh == FIN_BC_PERIODIC))
            return berr(FIN_ERR_ARG, "periodic boundaries come in pairs");
        if ((p.bc_xlow == FIN_BC_PERIODIC && p.mx < 3) || (p.bc_ylow == FIN_BC_PERIODIC && p.my < 3))
            return berr(FIN_ERR_ARG, "periodic direction shorter than the stencil halo");
        if (!(p.xhigh > p.xlow) || !(p.yhigh > p.ylow)) return berr(FIN_ERR_ARG, "empty domain");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return berr(FIN_ERR_NO_DEVICE, "no CUDA device");
    fin_batch* b = new fin_batch();
    b->n = nprob;
    b->tmpl_p = p0;
    b->p.assign(params, params + nprob);
    b->hb.assign(nprob, BProb());
    b->cfg = -1;
    auto fail = [&](cudaError_t e, const char* what) {
        fin_batch_destroy(b);
        return berr(FIN_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaEventCreate(&b->ev0)) != cudaSuccess) return fail(e, "event");
    if ((e = cudaEventCreate(&b->ev1)) != cudaSuccess) return fail(e, "event");
    for (int k = 0; k < nprob; k++) {
        const fin_params& p = params[k];
        BProb& h = b->hb[k];
        memset(&h, 0, sizeof(h));
        h.mx = p.mx;
        h.my = p.my;
        h.nv = p.nv;
        h.plane = (size_t(p.mx) * p.my + 31) / 32 * 32;
        h.dx = (p.xhigh - p.xlow) / p.mx;
        h.dy = (p.yhigh - p.ylow) / p.my;
        h.rdx = 1.0 / h.dx;
        h.rdy = 1.0 / h.dy;
        h.bc[0] = p.bc_xlow; h.bc[1] = p.bc_xhigh; h.bc[2] = p.bc_ylow; h.bc[3] = p.bc_yhigh;
        h.max_dt = p.max_dt;
        h.cfl_target = p.desired_cfl;
        h.cfl_max = p.max_cfl;
        for (int q = 0; q < 4; q++)
            if ((e = cudaMalloc(&h.q[q], MEQN * h.plane * sizeof(double))) != cudaSuccess) return fail(e, "cudaMalloc state");
        b->aos_max = std::max(b->aos_max, size_t(p.mx + 2 * p.mbc) * (p.my + 2 * p.mbc) * MEQN);
    }
    if ((e = cudaMalloc(&b->dact, nprob * sizeof(int))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->dtile0, (nprob + 1) * sizeof(long long))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->dnact, sizeof(int))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->db, nprob * sizeof(BProb))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->dargs, 3 * size_t(nprob) * sizeof(StageArgs))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->dqueue, 3 * sizeof(unsigned long long))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->dactive, sizeof(int))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->d_aos, b->aos_max * sizeof(double))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMemcpy(b->db, b->hb.data(), nprob * sizeof(BProb), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "cudaMemcpy");
    *out = b;
    return FIN_OK;
}

int fin_batch_destroy(fin_batch* b)
{
    if (!b) return FIN_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (BProb& h : b->hb)
        for (int q = 0; q < 4; q++) cudaFree(h.q[q]);
    cudaFree(b->dact);
    cudaFree(b->dtile0);
    cudaFree(b->dnact);
    cudaFree(b->db);
    cudaFree(b->dargs);
    cudaFree(b->dqueue);
    cudaFree(b->dactive);
    cudaFree(b->d_aos);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return FIN_OK;
}

// Problem k's state from the reference's ghosted layout (as fin_set_state):
// q^n in buffer 0 and its global wave speeds.
int fin_batch_set_state(fin_batch* b, int k, const double* q_host, double t)
{
    if (!b || !q_host || k < 0 || k >= b->n) return berr(FIN_ERR_ARG, "bad argument");
    const fin_params& p = b->p[k];
    BProb& h = b->hb[k];
    BCK(cudaMemcpyAsync(&h, b->db + k, sizeof(BProb), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    const size_t ne = size_t(p.mx + 2 * p.mbc) * (p.my + 2 * p.mbc) * MEQN;
    BCK(cudaMemcpyAsync(b->d_aos, q_host, ne * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    const size_t n = size_t(p.mx) * p.my;
    const int g = int(std::min<size_t>((n + 255) / 256, 148 * 16));
    k_aos_to_planes<<<g, 256, 0, b->stream>>>(b->d_aos, h.q[0], p.mx, p.my, p.mbc, h.plane);
    BCK(cudaGetLastError());
    h.cur = 0;
    h.t_loop = h.t_state = t;
    h.err = 0;
    h.active = 0;
    for (int q = 0; q < 4; q++) h.alpha[q][0] = h.alpha[q][1] = 0.0;
    h.status = 0;
    BCK(cudaMemcpyAsync(b->db + k, &h, sizeof(BProb), cudaMemcpyHostToDevice, b->stream));
    char* dk = reinterpret_cast<char*>(b->db + k);
    k_wave_spd_max<<<g, 256, 0, b->stream>>>(h.q[0], p.mx, p.my, h.plane, p.gamma,
                                              reinterpret_cast<double*>(dk + offsetof(BProb, alpha)),
                                              reinterpret_cast<unsigned int*>(dk + offsetof(BProb, status)));
    BCK(cudaGetLastError());
    BCK(cudaStreamSynchronize(b->stream));
    return FIN_OK;
}

int fin_batch_get_state(fin_batch* b, int k, double* q_host, double* t)
{
    if (!b || !q_host || k < 0 || k >= b->n) return berr(FIN_ERR_ARG, "bad argument");
    const fin_params& p = b->p[k];
    BProb& h = b->hb[k];
    BCK(cudaMemcpyAsync(&h, b->db + k, sizeof(BProb), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    const size_t n = size_t(p.mx) * p.my;
    const int g = int(std::min<size_t>((n + 255) / 256, 148 * 16));
    k_planes_to_aos<<<g, 256, 0, b->stream>>>(h.q[h.cur], b->d_aos, p.mx, p.my, p.mbc, h.plane, p.bc_xlow,
                                              p.bc_xhigh, p.bc_ylow, p.bc_yhigh);
    BCK(cudaGetLastError());
    const size_t ne = size_t(p.mx + 2 * p.mbc) * (p.my + 2 * p.mbc) * MEQN;
    BCK(cudaMemcpyAsync(q_host, b->d_aos, ne * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    if (t) *t = h.t_state;
    return FIN_OK;
}

int fin_batch_solve(fin_batch* b, double tend, double* dtv1, int* steps)
{
    if (!b || !dtv1) return berr(FIN_ERR_ARG, "null argument");
    BCK(cudaMemcpyAsync(b->hb.data(), b->db, b->n * sizeof(BProb), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    int nact = 0;
    for (int k = 0; k < b->n; k++) {
        BProb& h = b->hb[k];
        h.tend = tend;
        h.dt = dtv1[k];
        h.t_loop = h.t_state;
        h.active = h.t_loop < tend ? 1 : 0;
        h.fresh = 1;
        h.n_step = 0;
        h.accepted = 0;
        h.err = 0;
        nact += h.active;
    }
    BCK(cudaMemcpyAsync(b->db, b->hb.data(), b->n * sizeof(BProb), cudaMemcpyHostToDevice, b->stream));
    int rc;
    long long reps = 0;
    BCK(cudaEventRecord(b->ev0, b->stream));
    if (nact > 0) {
        if (b->cfg < 0 && (rc = autotune(b))) return rc;
        if ((rc = build_graph(b))) return rc;
        BCK(cudaEventRecord(b->ev0, b->stream));
        const int chunk = 8;   // replays between the host's looks at the active count
        while (nact > 0) {
            for (int r = 0; r < chunk; r++) BCK(cudaGraphLaunch(b->graph, b->stream));
            reps += chunk;
            BCK(cudaMemcpyAsync(&nact, b->dactive, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
            BCK(cudaStreamSynchronize(b->stream));
        }
    }
    BCK(cudaEventRecord(b->ev1, b->stream));
    BCK(cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    BCK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->last_ms = ms;
    b->replays = reps;
    BCK(cudaMemcpyAsync(b->hb.data(), b->db, b->n * sizeof(BProb), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    int first = -1;
    for (int k = 0; k < b->n; k++) {
        dtv1[k] = b->hb[k].dt;
        if (steps) steps[k] = b->hb[k].accepted;
        if (b->hb[k].err && first < 0) first = k;
    }
    if (first >= 0)
        return berr(b->hb[first].err, "problem " + std::to_string(first) + " failed (code " +
                                          std::to_string(b->hb[first].err) + ")");
    return FIN_OK;
}

int fin_batch_stats(fin_batch* b, double* device_ms, long long* replays, int* tile_cfg, double* tune_ms)
{
    if (!b) return berr(FIN_ERR_ARG, "null batch");
    if (device_ms) *device_ms = b->last_ms;
    if (replays) *replays = b->replays;
    if (tile_cfg) *tile_cfg = b->cfg;
    if (tune_ms)
        for (int c = 0; c < NCFG; c++) tune_ms[c] = b->tune_ms[c];
    return FIN_OK;
}

}  // extern "C"
