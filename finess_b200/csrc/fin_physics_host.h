// Host driver of the application callback surface (fin_physics.cuh): what
// lib/2d's ConstructL, GlobalWaveSpd, UpdateSoln, GetCFL and FinSolveRK do
// for an application, with the application's physics policy on the device.
// Header-only: an application includes it in its own .cu file and
// instantiates fin::phys::Driver<ItsPhysics, ItsHooks>.
//
// Hooks (lib/2d/hooks.h:6-10): the Hooks type's member functions are called
// where FinSolveRK.cpp:112-211 calls BeforeFullTimeStep, BeforeStep,
// AfterStep and AfterFullTimeStep, with the device state planes (plane m of
// a state at q + m * grid.plane, cell (i, j) at i * grid.my + j) and the
// driver's stream, on which they enqueue their own device work.  Because a
// hook may change the state, each stage's global alpha is computed from its
// input after the hooks (one extra pass of k_phys_wave_spd per stage).
//
// Arrays at the boundary are the reference's ghosted layout (q(i, j, m), m
// fastest, i slowest, mbc ghost cells), as the library's C ABI takes them.
#pragma once
#include <cuda_runtime.h>
#include <cstring>
#include <utility>
#include <vector>
#include "finess_b200.h"
#include "fin_physics.cuh"

namespace fin {
namespace phys {

struct Grid {
    int mx, my;
    size_t plane;
    double xlow, ylow, dx, dy;
};

// No hooks: the reference's lib/2d/blanks versions do nothing either.
struct NoHooks {
    void before_full_time_step(double, const double*, double*, const Grid&, cudaStream_t) const {}
    void before_step(double, double*, const Grid&, cudaStream_t) const {}
    void after_step(double, double*, const Grid&, cudaStream_t) const {}
    void after_full_time_step(double, const double*, double*, const Grid&, cudaStream_t) const {}
};

template <int M>
__global__ void k_ghosted_to_planes(const double* aos, double* planes, int mx, int my, int mbc, size_t plane)
{
    const size_t n = size_t(mx) * my;
    const int sy = my + 2 * mbc;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        const int i = int(g / my), j = int(g - size_t(i) * my);
        const size_t src = (size_t(i + mbc) * sy + (j + mbc)) * M;
        for (int m = 0; m < M; m++) planes[m * plane + g] = aos[src + m];
    }
}

// planes -> the whole ghosted array, ghosts by the boundary remap (what
// SetBndValues leaves there)
template <int M>
__global__ void k_planes_to_ghosted(const double* planes, double* aos, int mx, int my, int mbc, size_t plane, int b0,
                                    int b1, int b2, int b3)
{
    const int sx = mx + 2 * mbc, sy = my + 2 * mbc;
    const size_t n = size_t(sx) * sy;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
        const int ii = int(e / sy), jj = int(e - size_t(ii) * sy);
        const size_t g = size_t(bc_remap(ii - mbc, mx, b0, b1)) * my + bc_remap(jj - mbc, my, b2, b3);
        for (int m = 0; m < M; m++) aos[e * M + m] = planes[m * plane + g];
    }
}

template <class Phys, class Hooks = NoHooks>
class Driver {
public:
    static constexpr int M = Phys::MEQN;

    Driver(const fin_params& p, const Phys& phys, const Hooks& hooks = Hooks()) : p_(p), phys_(phys), hooks_(hooks) {}
    ~Driver()
    {
        if (stream_) cudaStreamSynchronize(stream_);
        for (double* b : q_) cudaFree(b);
        cudaFree(aos_);
        cudaFree(slots_);
        cudaFree(face_x_);
        cudaFree(face_y_);
        if (stream_) cudaStreamDestroy(stream_);
    }

    // Validates the parameters and allocates the device buffers.
    int init()
    {
        if (p_.meqn != M || p_.mx < 1 || p_.my < 1 || p_.mbc < 3 || p_.space_order != 5) return FIN_ERR_ARG;
        if (p_.weno_version != FIN_WENO_JS && p_.weno_version != FIN_WENO_Z && p_.weno_version != FIN_WENO_FD)
            return FIN_ERR_ARG;
        for (int b : {p_.bc_xlow, p_.bc_xhigh, p_.bc_ylow, p_.bc_yhigh})
            if (b != FIN_BC_PERIODIC && b != FIN_BC_TRANSMISSIVE) return FIN_ERR_ARG;
        g_.mx = p_.mx;
        g_.my = p_.my;
        g_.plane = (size_t(p_.mx) * p_.my + 31) / 32 * 32;
        g_.xlow = p_.xlow;
        g_.ylow = p_.ylow;
        g_.dx = (p_.xhigh - p_.xlow) / p_.mx;
        g_.dy = (p_.yhigh - p_.ylow) / p_.my;
        aos_n_ = size_t(p_.mx + 2 * p_.mbc) * (p_.my + 2 * p_.mbc) * M;
        if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess) return FIN_ERR_CUDA;
        for (double*& b : q_)
            if (cudaMalloc(&b, M * g_.plane * sizeof(double)) != cudaSuccess) return FIN_ERR_CUDA;
        if (cudaMalloc(&aos_, aos_n_ * sizeof(double)) != cudaSuccess) return FIN_ERR_CUDA;
        if (cudaMalloc(&slots_, 8 * sizeof(double)) != cudaSuccess) return FIN_ERR_CUDA;
        if (cudaFuncSetAttribute(k_phys_stage<Phys, FIN_WENO_JS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(Tile<M>::BYTES)) != cudaSuccess ||
            cudaFuncSetAttribute(k_phys_stage<Phys, FIN_WENO_JS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(Tile<M>::BYTES)) != cudaSuccess ||
            cudaFuncSetAttribute(k_phys_stage<Phys, FIN_WENO_Z, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(Tile<M>::BYTES)) != cudaSuccess ||
            cudaFuncSetAttribute(k_phys_stage<Phys, FIN_WENO_Z, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(Tile<M>::BYTES)) != cudaSuccess ||
            cudaFuncSetAttribute(k_phys_stage<Phys, FIN_WENO_FD, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(Tile<M>::BYTES)) != cudaSuccess)
            return FIN_ERR_CUDA;
        return FIN_OK;
    }

    const Grid& grid() const { return g_; }
    cudaStream_t stream() const { return stream_; }
    double time() const { return t_; }

    // StateVars construction: the interior of a ghosted host array.
    int set_state(const double* q_host, double t)
    {
        int rc = upload(q_host, 0);
        if (rc) return rc;
        cur_ = 0;
        t_ = t;
        return sync();
    }

    // The state back, ghosts filled as SetBndValues would.
    int get_state(double* q_host, double* t)
    {
        k_planes_to_ghosted<M><<<blocks(aos_n_ / M), 256, 0, stream_>>>(q_[cur_], aos_, p_.mx, p_.my, p_.mbc, g_.plane,
                                                                       p_.bc_xlow, p_.bc_xhigh, p_.bc_ylow,
                                                                       p_.bc_yhigh);
        if (cudaGetLastError() != cudaSuccess) return FIN_ERR_CUDA;
        if (cudaMemcpyAsync(q_host, aos_, aos_n_ * sizeof(double), cudaMemcpyDeviceToHost, stream_) != cudaSuccess)
            return FIN_ERR_CUDA;
        if (t) *t = t_;
        return sync();
    }

    // GlobalWaveSpd (lib/2d/GlobalWaveSpd.cpp:20-80) of a host state.
    int global_wave_spd(const double* q_host, double* a1, double* a2)
    {
        int rc = upload(q_host, 3);
        if (rc) return rc;
        if ((rc = wave_spd(3, slots_))) return rc;
        double h[2];
        if (cudaMemcpyAsync(h, slots_, sizeof(h), cudaMemcpyDeviceToHost, stream_) != cudaSuccess) return FIN_ERR_CUDA;
        if ((rc = sync())) return rc;
        *a1 = h[0];
        *a2 = h[1];
        return status();
    }

    // ConstructL (lib/2d/ConstructL.cpp:13-408) of a host state: L's interior
    // into the ghosted L_host (ghosts untouched); smax_host (may be NULL) the
    // ghosted (mx+1, my+1, 2) array, max-accumulated as ConstructL.cpp:173,324.
    int construct_l(const double* q_host, double* L_host, double* smax_host)
    {
        int rc = upload(q_host, 3);
        if (rc) return rc;
        if (p_.global_alpha && (rc = wave_spd(3, slots_))) return rc;
        const size_t nx = size_t(p_.mx + 1) * p_.my, ny = size_t(p_.mx) * (p_.my + 1);
        if (smax_host && !face_x_) {
            if (cudaMalloc(&face_x_, nx * sizeof(double)) != cudaSuccess) return FIN_ERR_CUDA;
            if (cudaMalloc(&face_y_, ny * sizeof(double)) != cudaSuccess) return FIN_ERR_CUDA;
        }
        StageArgs a = args();
        a.qin = q_[3];
        a.qout = q_[2];
        a.bdt = 1.0;
        a.alpha_in = p_.global_alpha ? slots_ : nullptr;
        a.face_alpha_x = smax_host ? face_x_ : nullptr;
        a.face_alpha_y = smax_host ? face_y_ : nullptr;
        if ((rc = launch(a))) return rc;
        const size_t n = size_t(p_.mx) * p_.my;
        std::vector<double> hl(M * g_.plane);
        if (cudaMemcpyAsync(hl.data(), q_[2], hl.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_) != cudaSuccess)
            return FIN_ERR_CUDA;
        std::vector<double> fx(smax_host ? nx : 0), fy(smax_host ? ny : 0);
        if (smax_host) {
            if (cudaMemcpyAsync(fx.data(), face_x_, nx * sizeof(double), cudaMemcpyDeviceToHost, stream_) != cudaSuccess ||
                cudaMemcpyAsync(fy.data(), face_y_, ny * sizeof(double), cudaMemcpyDeviceToHost, stream_) != cudaSuccess)
                return FIN_ERR_CUDA;
        }
        if ((rc = sync())) return rc;
        const int sy = p_.my + 2 * p_.mbc;
        for (int i = 0; i < p_.mx; i++)
            for (int j = 0; j < p_.my; j++)
                for (int m = 0; m < M; m++)
                    L_host[(size_t(i + p_.mbc) * sy + (j + p_.mbc)) * M + m] = hl[m * g_.plane + size_t(i) * p_.my + j];
        (void)n;
        if (smax_host) {
            const int ss = p_.my + 1 + 2 * p_.mbc;
            for (int i = 0; i <= p_.mx; i++)
                for (int j = 0; j < p_.my; j++) {
                    double& d = smax_host[(size_t(i + p_.mbc) * ss + (j + p_.mbc)) * 2 + 0];
                    d = Max(d, fx[size_t(i) * p_.my + j]);
                }
            for (int i = 0; i < p_.mx; i++)
                for (int j = 0; j <= p_.my; j++) {
                    double& d = smax_host[(size_t(i + p_.mbc) * ss + (j + p_.mbc)) * 2 + 1];
                    d = Max(d, fy[size_t(i) * (p_.my + 1) + j]);
                }
        }
        return status();
    }

    // One SSP-RK3 step of exactly dt (FinSolveRK.cpp:112-211 with the hooks,
    // SetRKinfo.cpp:50-64's coefficients) from the state into itself;
    // *cfl receives GetCFL's value (GetCFL.cpp:31-73).
    int step_fixed(double dt, double* cfl)
    {
        const int qn = cur_, q1 = (cur_ + 1) % 3, nx = (cur_ + 2) % 3;
        int rc;
        if (cudaMemsetAsync(slots_ + 2, 0, 2 * sizeof(double), stream_) != cudaSuccess) return FIN_ERR_CUDA;
        hooks_.before_full_time_step(dt, q_[qn], q_[qn], g_, stream_);
        // stage 1: Qstar = 1 Qnew + 0 Qstar + (1 dt) L(Qnew)
        if ((rc = stage(dt, qn, qn, 1.0, -1, 0.0, 1.0 * dt, q1))) return rc;
        // stage 2: Qstar = 0.75 Qnew + 0.25 Qstar + (0.25 dt) L(Qstar)
        if ((rc = stage(dt, q1, qn, 0.75, q1, 0.25, 0.25 * dt, q1, true))) return rc;
        // stage 3: Qnew = (2/3) Qstar + (1/3) Qnew + ((2/3) dt) L(Qstar)
        if ((rc = stage(dt, q1, q1, 2.0e0 / 3.0e0, qn, 1.0e0 / 3.0e0, (2.0e0 / 3.0e0) * dt, nx))) return rc;
        hooks_.after_full_time_step(dt, q_[qn], q_[nx], g_, stream_);
        double h[2];
        if (cudaMemcpyAsync(h, slots_ + 2, sizeof(h), cudaMemcpyDeviceToHost, stream_) != cudaSuccess)
            return FIN_ERR_CUDA;
        if ((rc = sync())) return rc;
        double c = -100.0;
        c = Max(dt * h[0] / g_.dx, c);
        c = Max(dt * h[1] / g_.dy, c);
        if (cfl) *cfl = c;
        cur_ = nx;
        t_ = t_ + dt;
        return status();
    }

private:
    fin_params p_;
    Phys phys_;
    Hooks hooks_;
    Grid g_{};
    size_t aos_n_ = 0;
    cudaStream_t stream_ = nullptr;
    double* q_[4] = {nullptr, nullptr, nullptr, nullptr};   // three state registers + a scratch buffer
    double* aos_ = nullptr;
    double* slots_ = nullptr;   // [0..1] alpha of a stage input, [2..3] face-speed maxima, [4] status
    double* face_x_ = nullptr;
    double* face_y_ = nullptr;
    int cur_ = 0;
    double t_ = 0.0;

    static unsigned blocks(size_t n)
    {
        size_t b = (n + 255) / 256;
        return unsigned(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
    }
    int sync() { return cudaStreamSynchronize(stream_) == cudaSuccess ? FIN_OK : FIN_ERR_CUDA; }
    int status()
    {
        unsigned st = 0;
        if (cudaMemcpy(&st, slots_ + 4, sizeof(st), cudaMemcpyDeviceToHost) != cudaSuccess) return FIN_ERR_CUDA;
        if (st & 1u) {
            cudaMemset(slots_ + 4, 0, sizeof(double));
            return FIN_ERR_NONFINITE;
        }
        return FIN_OK;
    }
    int upload(const double* q_host, int buf)
    {
        if (cudaMemcpyAsync(aos_, q_host, aos_n_ * sizeof(double), cudaMemcpyHostToDevice, stream_) != cudaSuccess)
            return FIN_ERR_CUDA;
        k_ghosted_to_planes<M><<<blocks(size_t(p_.mx) * p_.my), 256, 0, stream_>>>(aos_, q_[buf], p_.mx, p_.my,
                                                                                 p_.mbc, g_.plane);
        return cudaGetLastError() == cudaSuccess ? FIN_OK : FIN_ERR_CUDA;
    }
    int wave_spd(int buf, double* out)
    {
        if (cudaMemsetAsync(out, 0, 2 * sizeof(double), stream_) != cudaSuccess) return FIN_ERR_CUDA;
        k_phys_wave_spd<Phys><<<blocks(size_t(p_.mx) * p_.my), 256, 0, stream_>>>(
            phys_, q_[buf], p_.mx, p_.my, g_.plane, g_.xlow, g_.ylow, g_.dx, g_.dy, out,
            reinterpret_cast<unsigned*>(slots_ + 4));
        return cudaGetLastError() == cudaSuccess ? FIN_OK : FIN_ERR_CUDA;
    }
    StageArgs args() const
    {
        StageArgs a;
        memset(&a, 0, sizeof(a));
        a.mx = p_.mx;
        a.my = p_.my;
        a.plane = g_.plane;
        a.xlow = g_.xlow;
        a.ylow = g_.ylow;
        a.dx = g_.dx;
        a.dy = g_.dy;
        a.eps = p_.epsilon;
        a.pw = p_.power_param;
        a.alpha_scaling = p_.alpha_scaling;
        a.status = reinterpret_cast<unsigned*>(slots_ + 4);
        a.bc[0] = p_.bc_xlow; a.bc[1] = p_.bc_xhigh; a.bc[2] = p_.bc_ylow; a.bc[3] = p_.bc_yhigh;
        return a;
    }
    int launch(const StageArgs& a)
    {
        dim3 grid((p_.my + Tile<M>::TJ - 1) / Tile<M>::TJ, (p_.mx + Tile<M>::TI - 1) / Tile<M>::TI);
        const size_t sm = Tile<M>::BYTES;
        const bool p2 = p_.power_param == 2.0;
        if (p_.weno_version == FIN_WENO_JS) {
            if (p2) k_phys_stage<Phys, FIN_WENO_JS, true><<<grid, 256, sm, stream_>>>(a, phys_);
            else k_phys_stage<Phys, FIN_WENO_JS, false><<<grid, 256, sm, stream_>>>(a, phys_);
        } else if (p_.weno_version == FIN_WENO_Z) {
            if (p2) k_phys_stage<Phys, FIN_WENO_Z, true><<<grid, 256, sm, stream_>>>(a, phys_);
            else k_phys_stage<Phys, FIN_WENO_Z, false><<<grid, 256, sm, stream_>>>(a, phys_);
        } else {
            k_phys_stage<Phys, FIN_WENO_FD, true><<<grid, 256, sm, stream_>>>(a, phys_);
        }
        return cudaGetLastError() == cudaSuccess ? FIN_OK : FIN_ERR_CUDA;
    }
    // One stage: BeforeStep(in), alpha of in, then out = a1 A + a2 B + bdt L(in)
    // (A, B < 0: term absent), then AfterStep(out).  With in_place the stage
    // writes over its input register (Qstar of stage 2): the output goes to
    // the scratch buffer and is swapped in.
    int stage(double dt, int in, int A, double a1, int B, double a2, double bdt, int out, bool in_place = false)
    {
        hooks_.before_step(dt, q_[in], g_, stream_);
        int rc;
        if (p_.global_alpha && (rc = wave_spd(in, slots_))) return rc;
        StageArgs a = args();
        a.qin = q_[in];
        a.A = A >= 0 ? q_[A] : nullptr;
        a.a1 = a1;
        a.B = B >= 0 ? q_[B] : nullptr;
        a.a2 = a2;
        a.bdt = bdt;
        a.qout = in_place ? q_[3] : q_[out];
        a.alpha_in = p_.global_alpha ? slots_ : nullptr;
        a.smax_out = slots_ + 2;
        if ((rc = launch(a))) return rc;
        if (in_place) std::swap(q_[3], q_[out]);
        hooks_.after_step(dt, q_[out], g_, stream_);
        return FIN_OK;
    }
};

}  // namespace phys
}  // namespace fin
