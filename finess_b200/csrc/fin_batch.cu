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
// The hybrid form (FP32 bulk, troubled-face network, judge step) keeps the
// single-problem schedule per problem (the indicator on q^n every ind_every
// accepted steps, every judge_every-th hybrid step judged against a
// full-WENO step from the same state, judge_every plain steps after a
// revert), decided by k_batch_prep and k_batch_ctl per problem.  A step
// then runs, each over a work queue of its own problems:
//   indicator (problems due for it) -> three hybrid stages (problems in the
//   hybrid form this attempt) -> three plain FP32 stages (problems in the
//   plain form, and the judge steps into a fifth buffer) -> the judge's
//   state difference -> control.
// Its tiles are the hybrid kernels' 15 x 16 (the flag masks' layout).
#include <cuda_runtime.h>
#include <algorithm>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>
#include "finess_b200.h"
#include "fin_stage.cuh"
#include "fin_stage_hyb.cuh"
#include "fin_hybrid.cuh"
#include "fin_mlp.cuh"
#include "fin_tmap.h"

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
    double* q[5];      // q[4]: the judge step's result (hybrid form only)
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
    // hybrid form
    unsigned* flags;        // troubled-face masks of q[cur] (flag_wx / flag_wy layout)
    int use_hyb;            // this attempt runs the hybrid stages
    int run_ind;            // ... after the indicator on q[cur]
    int judge;              // ... and is judged (full-WENO stages into q[4])
    int hyb_off;            // attempts left in the plain form after a revert
    int ind_since;          // accepted steps since the indicator's last run; -1: flags not valid for q[cur]
    unsigned int status_full;
    long long hstep, judges, reverts;
    double smax_full[2];    // the judge stages' face-speed maxima
    double aj[3][2];        // the judge stages' global alphas
    double diff[2];         // max |q_hybrid - q_full|, max |q_full|
    int tslot[5];           // tensor maps of q[k]: entries 2 tslot[k] (tile + halo box), +1 (interior box)
    int tmok;               // the maps exist (even my): the hybrid stages stage tiles by TMA
};

// Hybrid-form schedule shared by the problems of a batch (on = 0: no
// indicator, every attempt in the plain form).
struct BHyb {
    int on, ind_every, judge_every;
    double judge_tol;
};

// ---- device control ------------------------------------------------------
// The attempt of every active problem: FinSolveRK.cpp:77-100 (step count,
// clip of dt to tend) and the stage arguments of SetRKinfo.cpp:50-64.  In
// the hybrid form also the attempt's form (fin_solve's take_stages: the
// indicator when its flags are stale, the judge every judge_every-th hybrid
// attempt, the plain form while hyb_off counts down); args then holds the
// hybrid stages and args_p the plain ones (the whole step of a problem in
// the plain form, or the judge's stages from q^n through the same two stage
// registers into q[4], with their own maxima, alphas and status).
__global__ void k_batch_prep(BProb* pr, int n, StageArgs* args, StageArgs* args_p, const StageArgs tmpl,
                             int global_alpha, const BHyb h, unsigned long long* cnt, const CUtensorMap* tm)
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
    b.use_hyb = b.run_ind = b.judge = 0;
    if (h.on) {
        if (b.hyb_off == 0) {
            b.use_hyb = 1;
            if (b.ind_since < 0 || b.ind_since >= h.ind_every) {
                b.run_ind = 1;
                b.ind_since = 0;
                atomicAdd(cnt + 1, (unsigned long long)(b.mx + 1) * b.my + (unsigned long long)b.mx * (b.my + 1));
            }
            b.hstep++;
            b.judge = h.judge_every > 0 && b.hstep % h.judge_every == 0;
        } else {
            b.hyb_off--;
        }
        b.smax_full[0] = b.smax_full[1] = 0.0;
        b.status_full = 0;
        b.diff[0] = b.diff[1] = 0.0;
        for (int s = 0; s < 3; s++) b.aj[s][0] = b.aj[s][1] = 0.0;
    }
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
        if (!h.on) {
            args[size_t(s) * n + p] = a;
            continue;
        }
        StageArgs ah = a;
        ah.flags = b.flags;
        if (b.tmok) {   // q_in's tile + halo and the other operand (always q^n) by TMA
            const CUtensorMap* tp = tm + size_t(p) * 10;
            ah.tma = 1;
            ah.gtm_in = tp + 2 * b.tslot[in];
            ah.gtm_A = tp + 2 * b.tslot[b.cur] + 1;
        }
        args[size_t(s) * n + p] = ah;
        if (b.use_hyb && b.judge) {
            a.status = &b.status_full;
            a.smax_out = b.smax_full;
            if (s == 2) a.qout = b.q[4];
            a.alpha_in = global_alpha ? (s == 0 ? b.alpha[b.cur] : b.aj[s - 1]) : nullptr;
            a.alpha_out = b.aj[s];
        }
        args_p[size_t(s) * n + p] = a;
    }
}

// GetCFL (lib/2d/GetCFL.cpp:31-73) and FinSolveRK.cpp:300-357 per problem:
// CFL from the step's face-speed maxima, Qnew's time, the next dt, accept or
// reject; counts the problems still active.  A judged hybrid attempt is
// settled first (fin_solve's settle_judge): the hybrid result stays unless
// it differs from the full-WENO one by more than judge_tol (relative
// L-infinity); then the full result takes its place (a pointer swap), its
// maxima give the CFL, and the problem runs judge_every attempts in the
// plain form.
__global__ void k_batch_ctl(BProb* pr, int n, int* nactive, const BHyb h)
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
    double sx = b.smax[0], sy = b.smax[1];
    unsigned int st = b.status;
    if (b.use_hyb && b.judge) {
        b.judges++;
        const double d = b.diff[0], m = b.diff[1];
        if (!(d <= h.judge_tol * (m > 0 ? m : 1.0))) {
            b.reverts++;
            b.hyb_off = h.judge_every;
            b.ind_since = -1;
            double* t = b.q[4];
            b.q[4] = b.q[b.nxt];
            b.q[b.nxt] = t;
            const int ts = b.tslot[4];
            b.tslot[4] = b.tslot[b.nxt];
            b.tslot[b.nxt] = ts;
            b.alpha[b.nxt][0] = b.aj[2][0];
            b.alpha[b.nxt][1] = b.aj[2][1];
            sx = b.smax_full[0];
            sy = b.smax_full[1];
            st = b.status_full | (st & ~3u);   // the indicator's wait bits stay
        }
    }
    if (st & 28u) {   // a bounded device wait ran out, or a misaligned TMA destination
        b.err = FIN_ERR_CUDA;
        b.active = 0;
        return;
    }
    double c = -100.0;
    c = Max(__ddiv_rn(__dmul_rn(dt, sx), b.dx), c);
    c = Max(__ddiv_rn(__dmul_rn(dt, sy), b.dy), c);
    if (c > 1.0e8) {
        b.err = FIN_ERR_CFL_BOUNDS;
        b.active = 0;
        return;
    }
    const bool nonfinite = (st & 1u) != 0;
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
        if (b.ind_since >= 0) b.ind_since++;
    } else {
        b.t_loop = b.told;   // reject: q^n was never overwritten
    }
    if (!(b.t_loop < b.tend)) b.active = 0;
    if (b.active) atomicAdd(nactive, 1);
}

// Work queues of a step, one per selector: the problems it selects
// (act[0 .. na-1]) and the prefix sums of their tile counts (tile0[0 .. na],
// tile0[na] = total) for the tile shape TI x TJ.  Selectors: 0 every active
// problem (the plain forms); hybrid form: 1 the indicator's problems, 2 the
// hybrid stages', 3 the plain stages' (plain-form attempts and judges).
enum { QSEL_ALL = 0, QSEL_IND = 1, QSEL_HYB = 2, QSEL_PLAIN = 3, NQSEL = 4 };

__device__ __forceinline__ bool queue_selects(const BProb& b, int sel)
{
    if (!b.active) return false;
    switch (sel) {
    case QSEL_IND: return b.run_ind != 0;
    case QSEL_HYB: return b.use_hyb != 0;
    case QSEL_PLAIN: return !b.use_hyb || b.judge;
    default: return true;
    }
}

// One CTA of 1024 threads, chunks of 1024 problems; selector k's queue goes
// to act + k n, tile0 + k (n + 1), nact_out[k], for each k in selmask.
__global__ void __launch_bounds__(1024) k_batch_queue(const BProb* pr, int n, int TI, int TJ, unsigned selmask,
                                                      int* act, long long* tile0, int* nact_out)
{
    __shared__ long long sc[1024];
    __shared__ int si[1024];
    __shared__ long long base_t;
    __shared__ int base_i;
    const int tid = threadIdx.x;
    for (int sel = 0; sel < NQSEL; sel++) {
        if (!((selmask >> sel) & 1u)) continue;
        int* act_s = act + size_t(sel) * n;
        long long* tile0_s = tile0 + size_t(sel) * (n + 1);
        if (tid == 0) { base_t = 0; base_i = 0; }
        __syncthreads();
        for (int c0 = 0; c0 < n; c0 += 1024) {
            const int p = c0 + tid;
            const bool on = p < n && queue_selects(pr[p], sel);
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
                act_s[k] = p;
                tile0_s[k] = base_t + sc[tid] - nt;
            }
            __syncthreads();
            if (tid == 0) {
                base_t += sc[1023];
                base_i += si[1023];
            }
            __syncthreads();
        }
        if (tid == 0) {
            tile0_s[base_i] = base_t;
            nact_out[sel] = base_i;
        }
        __syncthreads();
    }
}

// The walk of a work queue shared by the batch kernels: persistent CTAs take
// tiles from an atomic counter, find the tile's problem by binary search in
// the prefix sums and run body(p, i0, j0) on it, until the queue is empty or
// body returns false (uniformly across the CTA).  The counter is bumped for
// the next tile when a tile starts, so the atomic's round trip overlaps the
// tile's work (the result is first needed after body).
template <int TI, int TJ, class F>
__device__ __forceinline__ void walk_queue(const BProb* pr, const int* act, const long long* tile0, const int* nact,
                                           unsigned long long* queue, F&& body)
{
    __shared__ long long s_tile;
    const int na = *nact;
    const long long total = tile0[na];
    if (threadIdx.x == 0) s_tile = (long long)atomicAdd(queue, 1ull);
    __syncthreads();
    long long t = s_tile;
    while (t < total) {
        unsigned long long nx = 0;
        if (threadIdx.x == 0) nx = atomicAdd(queue, 1ull);
        int lo = 0, hi = na - 1;   // the entry whose tiles contain t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tile0[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const int p = act[lo];
        const int lt = int(t - tile0[lo]), tj = (pr[p].my + TJ - 1) / TJ;
        if (!body(p, (lt / tj) * TI, (lt % tj) * TJ)) return;
        __syncthreads();   // the tile's shared memory and s_tile are free
        if (threadIdx.x == 0) s_tile = (long long)nx;
        __syncthreads();
        t = s_tile;
    }
}

// One stage over the problems of a queue (stage_tile, the body of k_stage).
template <class R, int VER, bool P2, class Cfg>
__global__ void __launch_bounds__(Cfg::NT, MinBlocks<R>::value)
k_stage_batch(const BProb* pr, const int* act, const long long* tile0, const int* nact, const StageArgs* args,
              unsigned long long* queue)
{
    walk_queue<Cfg::TI, Cfg::TJ>(pr, act, tile0, nact, queue, [&](int p, int i0, int j0) {
        stage_tile<R, VER, P2, Cfg>(args[p], i0, j0);
        return true;
    });
}

// One hybrid stage over the problems of a queue (stage_hyb_tile, the body of
// k_stage_hyb, with the tile staged by loads: args have tma = 0).
template <int VER, bool P2, class Cfg>
__global__ void __launch_bounds__(Cfg::NT, FIN_HYB_CTAS)
k_stage_hyb_batch(const BProb* pr, const int* act, const long long* tile0, const int* nact, const StageArgs* args,
                  unsigned long long* queue)
{
    walk_queue<Cfg::TI, Cfg::TJ>(pr, act, tile0, nact, queue, [&](int p, int i0, int j0) {
        stage_hyb_tile<VER, P2, Cfg>(args[p], i0, j0);
        return true;
    });
}

// Clears, per tile of the indicator's queue, the flag words that hold the
// tile's faces: the x faces of rows i0 .. i0+TI-1 (and row mx for the last
// tile row), the y faces of rows i0 .. i0+TI-1 at columns j0 .. j0+TJ.  A
// word shared with a neighbouring tile is cleared by both, all before the
// indicator sets any bit (a launch of its own); bits that no face owns are
// zero from the allocation.
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) k_batch_clear_flags(BProb* pr, const int* act, const long long* tile0,
                                                               const int* nact, unsigned long long* queue)
{
    static_assert(Cfg::TJ == 16 && Cfg::TI < 32, "one word per x-face row, two per y-face row");
    walk_queue<Cfg::TI, Cfg::TJ>(pr, act, tile0, nact, queue, [&](int p, int i0, int j0) {
        const BProb& b = pr[p];
        const int mx = b.mx, my = b.my, wx = flag_wx(my), wy = flag_wy(my), t = threadIdx.x, k = j0 >> 5;
        if (t <= Cfg::TI) {
            const int gi = i0 + t;
            if (t < Cfg::TI ? gi <= mx : gi == mx) b.flags[size_t(gi) * wx + k] = 0u;
        } else if (t >= 32 && t < 32 + Cfg::TI) {
            const int gi = i0 + t - 32;
            if (gi < mx) {
                unsigned* row = b.flags + size_t(mx + 1) * wx + size_t(gi) * wy;
                row[k] = 0u;
                if (((j0 + Cfg::TJ) >> 5) != k && ((j0 + Cfg::TJ) >> 5) < wy) row[(j0 + Cfg::TJ) >> 5] = 0u;
            }
        }
        return true;
    });
}

// stage_remap with asynchronous copies (cp.async, 8 bytes each): the loads
// land in stg while the CTA works on the previous tile; cp.async.wait_all and
// a barrier before stg is read.
template <class Cfg>
__device__ __forceinline__ void stage_remap_async(double* stg, const double* q, size_t plane, int i0, int j0, int mx,
                                                  int my, const int* bc, int tid)
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
        for (int m = 0; m < MEQN; m++) {
            const uint32_t dst = tc::smem_addr(stg + (m * RI + ii) * Cfg::SJ + jj + 1);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(q + m * plane + g) : "memory");
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The indicator over the problems of a queue: per tile q[cur]'s tile + halo
// (asynchronous copies issued while the previous tile's network runs),
// then indicator_tile (the body of k_indicator) into the problem's flags;
// troubled faces counted into *count.
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT, 3)
k_indicator_batch(BProb* pr, const int* act, const long long* tile0, const int* nact, const float* P, float gamma,
                  float zthr, unsigned long long* count, unsigned long long* queue, int skip_const)
{
    const int na = *nact;
    const long long total = tile0[na];
    if ((long long)blockIdx.x >= total) return;   // no tile for this CTA: skip the set-up
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ long long s_next;
    IndTile<Cfg>& S = *reinterpret_cast<IndTile<Cfg>*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    ind::load_ind_weights(S.w, P, tid, Cfg::NT);
    if (warp == 0) tc::tmem_alloc(&S.tmem, 128);
    if (tid == 0) {
        tc::mbar_init(&S.mbar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        S.abort = 0;
        S.cnt = 0;
        s_next = (long long)atomicAdd(queue, 1ull);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem;
    uint32_t mma_phase = 0;
    // tile t -> problem and tile origin (binary search in the prefix sums)
    auto locate = [&](long long t, int& p, int& i0, int& j0) {
        int lo = 0, hi = na - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tile0[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        p = act[lo];
        const int lt = int(t - tile0[lo]), tj = (pr[p].my + Cfg::TJ - 1) / Cfg::TJ;
        i0 = (lt / tj) * Cfg::TI;
        j0 = (lt % tj) * Cfg::TJ;
    };
    auto prefetch = [&](int p, int i0, int j0) {
        const BProb& b = pr[p];
        stage_remap_async<Cfg>(S.stg, b.q[b.cur], b.plane, i0, j0, b.mx, b.my, b.bc, tid);
    };
    long long t = s_next;
    int p = 0, i0 = 0, j0 = 0;
    if (t < total) {
        locate(t, p, i0, j0);
        prefetch(p, i0, j0);
    }
    while (t < total) {
        cp_async_wait_all();
        __syncthreads();
        stage_convert<Cfg, float>(S.stg, S.qs, tid);
        if (tid == 0) s_next = (long long)atomicAdd(queue, 1ull);
        __syncthreads();   // qs complete, stg free, the next tile published
        const long long tn = s_next;
        int pn = 0, in0 = 0, jn0 = 0;
        if (tn < total) {
            locate(tn, pn, in0, jn0);
            prefetch(pn, in0, jn0);
        }
        BProb& b = pr[p];
        indicator_tile<Cfg>(S, b.mx, b.my, gamma, zthr, b.flags, i0, j0, tmem, mma_phase, skip_const != 0);
        if (S.abort) {
            if (tid == 0) atomicOr(&b.status, 4u);
            break;
        }
        t = tn;
        p = pn;
        i0 = in0;
        j0 = jn0;
    }
    cp_async_wait_all();   // no copy stays in flight into released shared memory
    __syncthreads();
    if (tid == 0 && S.cnt) atomicAdd(count, (unsigned long long)S.cnt);
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tmem, 128);
}

// The judge's comparison over the plain queue's tiles of the judged
// problems: max |q[nxt] - q[4]| (NaN wins) and max |q[4]| over all planes,
// as fin_solve's k_max_diff, into the problem's diff.
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) k_batch_diff(BProb* pr, const int* act, const long long* tile0,
                                                        const int* nact, unsigned long long* queue)
{
    __shared__ double red[2][Cfg::NT / 32];
    walk_queue<Cfg::TI, Cfg::TJ>(pr, act, tile0, nact, queue, [&](int p, int i0, int j0) {
        BProb& b = pr[p];
        if (!b.judge) return true;
        const double* qa = b.q[b.nxt];
        const double* qb = b.q[4];
        double d = 0.0, m = 0.0;
        for (int c = threadIdx.x; c < Cfg::TI * Cfg::TJ; c += Cfg::NT) {
            const int gi = i0 + c / Cfg::TJ, gj = j0 + c % Cfg::TJ;
            if (gi >= b.mx || gj >= b.my) continue;
            const size_t g = size_t(gi) * b.my + gj;
#pragma unroll
            for (int k = 0; k < MEQN; k++) {
                const double va = qa[k * b.plane + g], vb = qb[k * b.plane + g];
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
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) { red[0][w] = d; red[1][w] = m; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 0; k < Cfg::NT / 32; k++) {
                d = red[0][k] > d || red[0][k] != red[0][k] ? red[0][k] : d;
                m = Max(m, red[1][k]);
            }
            atomic_max_nonneg(b.diff, d != d ? __longlong_as_double(0x7ff0000000000000ll) : d);
            atomic_max_nonneg(b.diff + 1, m);
        }
        return true;
    });
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
    StageArgs* dargs;           // stage arguments (3 x n); hybrid form: the hybrid stages
    StageArgs* dargs_p;         // hybrid form: the plain stages (3 x n)
    int* dact;                  // the queues' problems (NQSEL x n)
    long long* dtile0;          // prefix sums of their tiles (NQSEL x (n + 1))
    int* dnact;                 // their counts (NQSEL)
    unsigned long long* dqueue; // work-queue counters (NCOUNTER)
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
    // hybrid form
    bool hyb;                   // created in the hybrid form with WENO-JS or WENO-Z
    float* mlpP;                // network parameters (null: none given yet, the plain FP32 form runs)
    float zthr;
    bool ind_skip_const;
    BHyb hs;
    unsigned* dflags;           // every problem's flag masks
    unsigned long long* dcount; // troubled faces and faces the indicator ran on
    CUtensorMap* dtm;           // per problem and buffer slot: tile + halo box, interior box
    // kernel timing (steps launched one by one with events between the
    // launch groups instead of graph replays)
    bool timing;
    std::vector<cudaEvent_t> tev;
    double tms[5];              // control, indicator, hybrid stages, plain stages, judge difference
};

namespace {

// Work-queue counters of a step: the stages of the plain forms use 0-2; the
// hybrid form the indicator 0, hybrid stages 1-3, plain stages 4-6, judge 7,
// the flag clearing 8.
constexpr int NCOUNTER = 9;
// Steps between the host's looks at the active count, and the events a
// timed step records.
constexpr int CHUNK = 8, NSTEPEV = 7;

bool hybrid_on(const fin_batch* b) { return b->hyb && b->mlpP != nullptr; }

BHyb schedule(const fin_batch* b)
{
    BHyb h = b->hs;
    h.on = hybrid_on(b) ? 1 : 0;
    return h;
}

struct QueueRef {
    const int* act;
    const long long* tile0;
    const int* nact;
};

QueueRef queue_ref(const fin_batch* b, int sel)
{
    return {b->dact + size_t(sel) * b->n, b->dtile0 + size_t(sel) * (b->n + 1), b->dnact + sel};
}

// Resident CTAs of a kernel on the device (persistent grid).
template <class K>
int resident_grid(K kern, int nt, size_t smem, int* grid)
{
    if (*grid) return FIN_OK;
    BCK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int per_sm = 0, dev = 0, nsm = 0;
    BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, smem));
    BCK(cudaGetDevice(&dev));
    BCK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    *grid = std::max(1, per_sm) * nsm;
    return FIN_OK;
}

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
int launch_batch_kernel(fin_batch* b, QueueRef q, const StageArgs* args, unsigned long long* counter)
{
    auto kern = k_stage_batch<R, VER, P2, Cfg>;
    const size_t smem = Cfg::template smem_bytes<R>();
    static int grid = 0;   // per instantiation: resident CTAs on the device
    const int rg = resident_grid(kern, Cfg::NT, smem, &grid);
    if (rg) return rg;
    kern<<<grid, Cfg::NT, smem, b->stream>>>(b->db, q.act, q.tile0, q.nact, args, counter);
    BCK(cudaGetLastError());
    return FIN_OK;
}

// A plain stage (FP64, or FP32 for the FP32 and hybrid forms).
template <class Cfg>
int launch_batch_stage(fin_batch* b, QueueRef q, const StageArgs* args, unsigned long long* counter)
{
    const bool f32 = b->tmpl_p.precision != FIN_PREC_FP64;
    const bool p2 = b->tmpl_p.power_param == 2.0;
    switch (b->tmpl_p.weno_version) {
    case FIN_WENO_JS:
        if (f32) return p2 ? launch_batch_kernel<Cfg, float, FIN_WENO_JS, true>(b, q, args, counter)
                           : launch_batch_kernel<Cfg, float, FIN_WENO_JS, false>(b, q, args, counter);
        return p2 ? launch_batch_kernel<Cfg, double, FIN_WENO_JS, true>(b, q, args, counter)
                  : launch_batch_kernel<Cfg, double, FIN_WENO_JS, false>(b, q, args, counter);
    case FIN_WENO_Z:
        if (f32) return p2 ? launch_batch_kernel<Cfg, float, FIN_WENO_Z, true>(b, q, args, counter)
                           : launch_batch_kernel<Cfg, float, FIN_WENO_Z, false>(b, q, args, counter);
        return p2 ? launch_batch_kernel<Cfg, double, FIN_WENO_Z, true>(b, q, args, counter)
                  : launch_batch_kernel<Cfg, double, FIN_WENO_Z, false>(b, q, args, counter);
    default:
        return f32 ? launch_batch_kernel<Cfg, float, FIN_WENO_FD, true>(b, q, args, counter)
                   : launch_batch_kernel<Cfg, double, FIN_WENO_FD, true>(b, q, args, counter);
    }
}

template <int VER, bool P2>
int launch_hyb_kernel(fin_batch* b, QueueRef q, const StageArgs* args, unsigned long long* counter)
{
    auto kern = k_stage_hyb_batch<VER, P2, HybCfg>;
    const size_t smem = HybSmem<HybCfg>::BYTES;
    static int grid = 0;
    const int rg = resident_grid(kern, HybCfg::NT, smem, &grid);
    if (rg) return rg;
    kern<<<grid, HybCfg::NT, smem, b->stream>>>(b->db, q.act, q.tile0, q.nact, args, counter);
    BCK(cudaGetLastError());
    return FIN_OK;
}

// A hybrid stage (the form is built for WENO-JS and WENO-Z).
int launch_hyb_stage(fin_batch* b, QueueRef q, const StageArgs* args, unsigned long long* counter)
{
    const bool p2 = b->tmpl_p.power_param == 2.0;
    if (b->tmpl_p.weno_version == FIN_WENO_JS)
        return p2 ? launch_hyb_kernel<FIN_WENO_JS, true>(b, q, args, counter)
                  : launch_hyb_kernel<FIN_WENO_JS, false>(b, q, args, counter);
    return p2 ? launch_hyb_kernel<FIN_WENO_Z, true>(b, q, args, counter)
              : launch_hyb_kernel<FIN_WENO_Z, false>(b, q, args, counter);
}

int launch_indicator(fin_batch* b, QueueRef q, unsigned long long* counter)
{
    auto kern = k_indicator_batch<HybCfg>;
    const size_t smem = sizeof(IndTile<HybCfg>);
    static int grid = 0;
    if (!grid) {
        // three CTAs per SM, as the kernel is laid out for (registers and
        // shared memory; 3 x 128 of the SM's 512 TMEM columns).  The
        // occupancy calculator reported one CTA per SM for this kernel, so
        // the grid is set from the layout.
        BCK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        int nsm = 0, dev = 0;
        BCK(cudaGetDevice(&dev));
        BCK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        grid = 3 * nsm;
    }
    kern<<<grid, HybCfg::NT, smem, b->stream>>>(b->db, q.act, q.tile0, q.nact, b->mlpP, float(b->tmpl_p.gamma),
                                                b->zthr, b->dcount, counter, b->ind_skip_const ? 1 : 0);
    BCK(cudaGetLastError());
    return FIN_OK;
}

int launch_clear_flags(fin_batch* b, QueueRef q, unsigned long long* counter)
{
    k_batch_clear_flags<HybCfg><<<148 * 4, HybCfg::NT, 0, b->stream>>>(b->db, q.act, q.tile0, q.nact, counter);
    BCK(cudaGetLastError());
    return FIN_OK;
}

int launch_diff(fin_batch* b, QueueRef q, unsigned long long* counter)
{
    k_batch_diff<HybCfg><<<148 * 4, HybCfg::NT, 0, b->stream>>>(b->db, q.act, q.tile0, q.nact, counter);
    BCK(cudaGetLastError());
    return FIN_OK;
}

int launch_queue(fin_batch* b, int TI, int TJ, unsigned selmask)
{
    k_batch_queue<<<1, 1024, 0, b->stream>>>(b->db, b->n, TI, TJ, selmask, b->dact, b->dtile0, b->dnact);
    BCK(cudaGetLastError());
    return FIN_OK;
}

int launch_queue_cfg(fin_batch* b, int cfgi)
{
    return cfgi == 0 ? launch_queue(b, BatchCfgA::TI, BatchCfgA::TJ, 1u << QSEL_ALL)
                     : launch_queue(b, BatchCfgB::TI, BatchCfgB::TJ, 1u << QSEL_ALL);
}

int launch_stage_cfg(fin_batch* b, int cfgi, QueueRef q, const StageArgs* args, unsigned long long* counter)
{
    return cfgi == 0 ? launch_batch_stage<BatchCfgA>(b, q, args, counter)
                     : launch_batch_stage<BatchCfgB>(b, q, args, counter);
}

int launch_prep(fin_batch* b, const BHyb& h)
{
    const int nb = (b->n + 127) / 128;
    k_batch_prep<<<nb, 128, 0, b->stream>>>(b->db, b->n, b->dargs, b->dargs_p, template_args(b->tmpl_p),
                                            b->tmpl_p.global_alpha, h, b->dcount, b->dtm);
    BCK(cudaGetLastError());
    return FIN_OK;
}

// One step of every active problem: prep, three stages, control; in the
// hybrid form prep, the indicator, three hybrid and three plain stages, the
// judge's difference, control.  ev (kernel timing, else null): NSTEPEV
// events recorded between the launch groups (see fin_batch_kernel_times).
int enqueue_step(fin_batch* b, cudaEvent_t* ev = nullptr)
{
    const int nb = (b->n + 127) / 128;
    const BHyb h = schedule(b);
    auto mark = [&](int k) -> cudaError_t { return ev ? cudaEventRecord(ev[k], b->stream) : cudaSuccess; };
    int rc;
    BCK(mark(0));
    if ((rc = launch_prep(b, h))) return rc;
    if (!h.on) {
        if ((rc = launch_queue_cfg(b, b->cfg))) return rc;
        BCK(cudaMemsetAsync(b->dqueue, 0, 3 * sizeof(unsigned long long), b->stream));
        BCK(mark(1));
        BCK(mark(2));
        BCK(mark(3));
        for (int s = 0; s < 3; s++)
            if ((rc = launch_stage_cfg(b, b->cfg, queue_ref(b, QSEL_ALL), b->dargs + size_t(s) * b->n, b->dqueue + s)))
                return rc;
        BCK(mark(4));
    } else {
        static_assert(HybCfg::TI == BatchCfgA::TI && HybCfg::TJ == BatchCfgA::TJ, "one tile shape for all queues");
        if ((rc = launch_queue(b, HybCfg::TI, HybCfg::TJ, (1u << QSEL_IND) | (1u << QSEL_HYB) | (1u << QSEL_PLAIN))))
            return rc;
        BCK(cudaMemsetAsync(b->dqueue, 0, NCOUNTER * sizeof(unsigned long long), b->stream));
        BCK(mark(1));
        if ((rc = launch_clear_flags(b, queue_ref(b, QSEL_IND), b->dqueue + 8))) return rc;
        if ((rc = launch_indicator(b, queue_ref(b, QSEL_IND), b->dqueue))) return rc;
        BCK(mark(2));
        for (int s = 0; s < 3; s++)
            if ((rc = launch_hyb_stage(b, queue_ref(b, QSEL_HYB), b->dargs + size_t(s) * b->n, b->dqueue + 1 + s)))
                return rc;
        BCK(mark(3));
        for (int s = 0; s < 3; s++)
            if ((rc = launch_batch_stage<BatchCfgA>(b, queue_ref(b, QSEL_PLAIN), b->dargs_p + size_t(s) * b->n,
                                                    b->dqueue + 4 + s)))
                return rc;
        BCK(mark(4));
        if ((rc = launch_diff(b, queue_ref(b, QSEL_PLAIN), b->dqueue + 7))) return rc;
    }
    BCK(mark(5));
    BCK(cudaMemsetAsync(b->dactive, 0, sizeof(int), b->stream));
    k_batch_ctl<<<nb, 128, 0, b->stream>>>(b->db, b->n, b->dactive, h);
    BCK(cudaGetLastError());
    BCK(mark(6));
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
    BHyb off = b->hs;
    off.on = 0;
    int rc;
    if ((rc = launch_prep(b, off))) return rc;
    for (int c = 0; c < NCFG; c++) {
        double best = 1e30;
        if ((rc = launch_queue_cfg(b, c))) return rc;
        for (int rep = 0; rep < 3; rep++) {
            BCK(cudaMemsetAsync(b->dqueue, 0, sizeof(unsigned long long), b->stream));
            BCK(cudaEventRecord(b->ev0, b->stream));
            if ((rc = launch_stage_cfg(b, c, queue_ref(b, QSEL_ALL), b->dargs, b->dqueue))) return rc;
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
        if (p.precision != FIN_PREC_FP64 && p.precision != FIN_PREC_FP32 && p.precision != FIN_PREC_HYBRID)
            return berr(FIN_ERR_UNSUPPORTED, "the batch runs the FP64, FP32 or hybrid form");
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
    b->hyb = p0.precision == FIN_PREC_HYBRID && p0.weno_version != FIN_WENO_FD;
    b->hs.on = 0;
    b->hs.ind_every = 1;
    b->hs.judge_every = 20;
    b->hs.judge_tol = 1e-3;
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
        for (int q = 0; q < (b->hyb ? 5 : 4); q++)
            if ((e = cudaMalloc(&h.q[q], MEQN * h.plane * sizeof(double))) != cudaSuccess) return fail(e, "cudaMalloc state");
        h.ind_since = -1;
        for (int q = 0; q < 5; q++) h.tslot[q] = q;
        b->aos_max = std::max(b->aos_max, size_t(p.mx + 2 * p.mbc) * (p.my + 2 * p.mbc) * MEQN);
    }
    if (b->hyb) {
        // one allocation for every problem's flag masks (cleared per run by
        // k_batch_clear_flags; bits that no face owns stay zero from here)
        size_t words = 0;
        for (const fin_params& p : b->p) words += flag_words(p.mx, p.my);
        if ((e = cudaMalloc(&b->dflags, words * sizeof(unsigned))) != cudaSuccess) return fail(e, "cudaMalloc flags");
        if ((e = cudaMemset(b->dflags, 0, words * sizeof(unsigned))) != cudaSuccess) return fail(e, "memset flags");
        size_t off = 0;
        for (int k = 0; k < nprob; k++) {
            b->hb[k].flags = b->dflags + off;
            off += flag_words(b->p[k].mx, b->p[k].my);
        }
        if ((e = cudaMalloc(&b->dargs_p, 3 * size_t(nprob) * sizeof(StageArgs))) != cudaSuccess)
            return fail(e, "cudaMalloc");
        // tensor maps of every state buffer (grids with even my), written
        // once: the judge's buffer swaps permute the slots, not the maps
        std::vector<CUtensorMap> tms(size_t(nprob) * 10);
        memset(tms.data(), 0, tms.size() * sizeof(CUtensorMap));
        for (int k = 0; k < nprob; k++) {
            BProb& h = b->hb[k];
            bool ok = true;
            for (int q = 0; q < 5 && ok; q++)
                ok = make_state_map(&tms[size_t(k) * 10 + 2 * q], h.q[q], h.mx, h.my, h.plane, HybCfg::SJ, HybCfg::RI) &&
                     make_state_map(&tms[size_t(k) * 10 + 2 * q + 1], h.q[q], h.mx, h.my, h.plane, HybCfg::TJ,
                                    HybCfg::TI);
            h.tmok = ok ? 1 : 0;
        }
        if ((e = cudaMalloc(&b->dtm, tms.size() * sizeof(CUtensorMap))) != cudaSuccess) return fail(e, "cudaMalloc");
        if ((e = cudaMemcpy(b->dtm, tms.data(), tms.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return fail(e, "cudaMemcpy");
    }
    if ((e = cudaMalloc(&b->dcount, 2 * sizeof(unsigned long long))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMemset(b->dcount, 0, 2 * sizeof(unsigned long long))) != cudaSuccess) return fail(e, "memset");
    if ((e = cudaMalloc(&b->dact, NQSEL * size_t(nprob) * sizeof(int))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->dtile0, NQSEL * size_t(nprob + 1) * sizeof(long long))) != cudaSuccess)
        return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->dnact, NQSEL * sizeof(int))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->db, nprob * sizeof(BProb))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->dargs, 3 * size_t(nprob) * sizeof(StageArgs))) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->dqueue, NCOUNTER * sizeof(unsigned long long))) != cudaSuccess) return fail(e, "cudaMalloc");
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
    // the judge's pointer swaps only permute a problem's five buffers
    for (BProb& h : b->hb)
        for (int q = 0; q < 5; q++) cudaFree(h.q[q]);
    cudaFree(b->dflags);
    cudaFree(b->dcount);
    cudaFree(b->dtm);
    cudaFree(b->mlpP);
    cudaFree(b->dargs_p);
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
    for (cudaEvent_t e : b->tev)
        if (e) cudaEventDestroy(e);
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
    h.ind_since = -1;   // the flags no longer describe q[cur]
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
        // the hybrid form's kernels are built for one tile shape (15 x 16)
        if (b->cfg < 0 && hybrid_on(b)) b->cfg = 0;
        if (b->cfg < 0 && (rc = autotune(b))) return rc;
        if (!b->timing && (rc = build_graph(b))) return rc;
        BCK(cudaEventRecord(b->ev0, b->stream));
        while (nact > 0) {
            for (int r = 0; r < CHUNK; r++) {
                if (!b->timing) BCK(cudaGraphLaunch(b->graph, b->stream));
                else if ((rc = enqueue_step(b, b->tev.data() + r * NSTEPEV))) return rc;
            }
            reps += CHUNK;
            BCK(cudaMemcpyAsync(&nact, b->dactive, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
            BCK(cudaStreamSynchronize(b->stream));
            for (int r = 0; b->timing && r < CHUNK; r++) {
                const cudaEvent_t* e = b->tev.data() + r * NSTEPEV;
                float m[6];
                for (int k = 0; k < 6; k++) BCK(cudaEventElapsedTime(&m[k], e[k], e[k + 1]));
                b->tms[0] += m[0] + m[5];
                for (int k = 1; k < 5; k++) b->tms[k] += m[k];
            }
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

int fin_batch_set_indicator(fin_batch* b, const float* params, float z_threshold, int judge_every, double judge_tol)
{
    if (!b || !params) return berr(FIN_ERR_ARG, "null argument");
    if (b->tmpl_p.precision != FIN_PREC_HYBRID) return berr(FIN_ERR_ARG, "the batch was not created in the hybrid form");
    if (!b->hyb) return FIN_OK;   // WENO FD: every face takes the linear flux already
    if (!b->mlpP) BCK(cudaMalloc(&b->mlpP, mlp::NPARAM * sizeof(float)));
    BCK(cudaMemcpyAsync(b->mlpP, params, mlp::NPARAM * sizeof(float), cudaMemcpyHostToDevice, b->stream));
    b->zthr = z_threshold;
    b->ind_skip_const = ind::zero_row_logit(params) < double(z_threshold) - 0.05;   // as fin_set_indicator
    b->hs.judge_every = judge_every;
    b->hs.judge_tol = judge_tol;
    BCK(cudaMemcpyAsync(b->hb.data(), b->db, b->n * sizeof(BProb), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    for (BProb& h : b->hb) {
        h.hyb_off = 0;
        h.ind_since = -1;
    }
    BCK(cudaMemcpyAsync(b->db, b->hb.data(), b->n * sizeof(BProb), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    if (b->graph) {   // the step's schedule is captured in the graph
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return FIN_OK;
}

int fin_batch_set_indicator_every(fin_batch* b, int every)
{
    if (!b) return berr(FIN_ERR_ARG, "null argument");
    if (every < 1) return berr(FIN_ERR_ARG, "the indicator period must be at least one step");
    b->hs.ind_every = every;
    BCK(cudaMemcpyAsync(b->hb.data(), b->db, b->n * sizeof(BProb), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    for (BProb& h : b->hb) h.ind_since = -1;
    BCK(cudaMemcpyAsync(b->db, b->hb.data(), b->n * sizeof(BProb), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return FIN_OK;
}

int fin_batch_set_kernel_timing(fin_batch* b, int on)
{
    if (!b) return berr(FIN_ERR_ARG, "null batch");
    if (on && b->tev.empty()) {
        b->tev.assign(CHUNK * NSTEPEV, nullptr);
        for (cudaEvent_t& e : b->tev) BCK(cudaEventCreate(&e));
    }
    b->timing = on != 0;
    for (double& t : b->tms) t = 0.0;
    return FIN_OK;
}

int fin_batch_kernel_times(fin_batch* b, double* ms)
{
    if (!b || !ms) return berr(FIN_ERR_ARG, "null argument");
    for (int k = 0; k < 5; k++) ms[k] = b->tms[k];
    return FIN_OK;
}

int fin_batch_hybrid_stats(fin_batch* b, long long* troubled_faces, long long* faces, long long* judges,
                           long long* reverts)
{
    if (!b) return berr(FIN_ERR_ARG, "null batch");
    unsigned long long c[2] = {0, 0};
    BCK(cudaMemcpyAsync(c, b->dcount, sizeof(c), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaMemcpyAsync(b->hb.data(), b->db, b->n * sizeof(BProb), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    long long j = 0, r = 0;
    for (const BProb& h : b->hb) {
        j += h.judges;
        r += h.reverts;
    }
    if (troubled_faces) *troubled_faces = (long long)c[0];
    if (faces) *faces = (long long)c[1];
    if (judges) *judges = j;
    if (reverts) *reverts = r;
    return FIN_OK;
}

}  // extern "C"
