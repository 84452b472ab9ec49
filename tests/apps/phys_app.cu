// A FINESS-style application written against the device callback surface
// (fin_physics.cuh, fin_physics_host.h), built into its own library the way
// an application links its callbacks: test infrastructure for
// tests/test_gpu_physics.py.
//
// Physics 1, linear advection-acoustics (meqn 3, q = (p, u, v)):
//   q_t + f(q)_x + g(q)_y = 0,  f = (ax p + K u, ax u + p/rho0, ax v),
//                               g = (ay p + K v, ay u, ay v + p/rho0),
// speeds a_n - c, a_n, a_n + c with c = sqrt(K/rho0), impedance Z = rho0 c;
// in x the right eigenvectors are (-Z, 1, 0), (0, 0, 1), (Z, 1, 0) and the
// left ones (-1/(2Z), 1/2, 0), (0, 0, 1), (1/(2Z), 1/2, 0); in y u and v trade
// places.  Optional hooks (lib/2d/hooks.h): BeforeStep adds h0 to p, AfterStep
// scales u by h1.
// Physics 2, the library's Euler callbacks as a policy (fin::phys::EulerPhys).
#include <cmath>
#include "fin_physics_host.h"

namespace {

struct AdvAcoustics {
    static constexpr int MEQN = 3;
    double K, rho0, ax, ay;
    struct Face { int ixy; double Z; };
    __device__ double c() const { return sqrt(K / rho0); }
    __device__ void flux(double, double, const double* q, double* f, double* g) const
    {
        f[0] = ax * q[0] + K * q[1];
        f[1] = ax * q[1] + q[0] / rho0;
        f[2] = ax * q[2];
        g[0] = ay * q[0] + K * q[2];
        g[1] = ay * q[1];
        g[2] = ay * q[2] + q[0] / rho0;
    }
    __device__ void wave_speed(double nx, double ny, double, double, const double*, const double*, double& s1,
                               double& s2) const
    {
        const double an = ax * nx + ay * ny;
        s1 = an - c();
        s2 = an + c();
    }
    __device__ Face face(int ixy, const double*) const { return Face{ixy, rho0 * c()}; }
    __device__ void left(const Face& f, const double* v, double* w) const
    {
        const int n = f.ixy == 1 ? 1 : 2, t = f.ixy == 1 ? 2 : 1;   // normal, tangential velocity
        w[0] = -v[0] / (2.0 * f.Z) + 0.5 * v[n];
        w[1] = v[t];
        w[2] = v[0] / (2.0 * f.Z) + 0.5 * v[n];
    }
    __device__ void right(const Face& f, const double* w, double* v) const
    {
        const int n = f.ixy == 1 ? 1 : 2, t = f.ixy == 1 ? 2 : 1;
        v[0] = -f.Z * w[0] + f.Z * w[2];
        v[n] = w[0] + w[2];
        v[t] = w[1];
    }
};

__global__ void k_add(double* q, size_t n, double h)
{
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
        q[k] = q[k] + h;
}
__global__ void k_scale(double* q, size_t n, double h)
{
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
        q[k] = q[k] * h;
}

struct AcousticHooks : fin::phys::NoHooks {
    double h0 = 0.0, h1 = 1.0;
    void before_step(double, double* q, const fin::phys::Grid& g, cudaStream_t s) const
    {
        k_add<<<64, 256, 0, s>>>(q, size_t(g.mx) * g.my, h0);   // plane 0: p
    }
    void after_step(double, double* q, const fin::phys::Grid& g, cudaStream_t s) const
    {
        k_scale<<<64, 256, 0, s>>>(q + g.plane, size_t(g.mx) * g.my, h1);   // plane 1: u
    }
};

struct AppBase {
    virtual ~AppBase() {}
    virtual int set_state(const double* q, double t) = 0;
    virtual int get_state(double* q, double* t) = 0;
    virtual int construct_l(const double* q, double* L, double* smax) = 0;
    virtual int global_wave_spd(const double* q, double* a1, double* a2) = 0;
    virtual int step_fixed(double dt, double* cfl) = 0;
};

template <class Phys, class Hooks>
struct App : AppBase {
    fin::phys::Driver<Phys, Hooks> d;
    App(const fin_params& p, const Phys& ph, const Hooks& h) : d(p, ph, h) {}
    int set_state(const double* q, double t) override { return d.set_state(q, t); }
    int get_state(double* q, double* t) override { return d.get_state(q, t); }
    int construct_l(const double* q, double* L, double* smax) override { return d.construct_l(q, L, smax); }
    int global_wave_spd(const double* q, double* a1, double* a2) override { return d.global_wave_spd(q, a1, a2); }
    int step_fixed(double dt, double* cfl) override { return d.step_fixed(dt, cfl); }
};

// The library's reciprocal (fin_device.cuh: Newton-Raphson refinement of
// rcp.approx) beside CUDA's correctly rounded division, for a sweep of
// arguments.
__global__ void k_rcp_probe(const double* x, double* r64, double* div64, float* r32, int n)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        r64[k] = fin::rcp(x[k]);
        div64[k] = __ddiv_rn(1.0, x[k]);
        r32[k] = fin::rcp(float(x[k]));
    }
}

}  // namespace

extern "C" {

// rcp(x) (FP64 and FP32) and 1/x of n host values through the device.
int app_rcp_probe(const double* x, double* r64, double* div64, float* r32, int n)
{
    double *dx = nullptr, *d64 = nullptr, *dd = nullptr;
    float* d32 = nullptr;
    if (cudaMalloc(&dx, n * sizeof(double)) != cudaSuccess || cudaMalloc(&d64, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dd, n * sizeof(double)) != cudaSuccess || cudaMalloc(&d32, n * sizeof(float)) != cudaSuccess)
        return FIN_ERR_CUDA;
    cudaMemcpy(dx, x, n * sizeof(double), cudaMemcpyHostToDevice);
    k_rcp_probe<<<(n + 255) / 256, 256>>>(dx, d64, dd, d32, n);
    int rc = cudaGetLastError() == cudaSuccess ? FIN_OK : FIN_ERR_CUDA;
    cudaMemcpy(r64, d64, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(div64, dd, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(r32, d32, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = FIN_ERR_CUDA;
    cudaFree(dx);
    cudaFree(d64);
    cudaFree(dd);
    cudaFree(d32);
    return rc;
}

// kind 0: advection-acoustics, prm = (K, rho0, ax, ay); kind 1: the same with
// the hooks, prm = (K, rho0, ax, ay, h0, h1); kind 2: EulerPhys (gamma of p).
int app_create(int kind, const fin_params* p, const double* prm, void** out)
{
    if (!p || !out) return FIN_ERR_ARG;
    AppBase* a = nullptr;
    if (kind == 0 || kind == 1) {
        const AdvAcoustics ph{prm[0], prm[1], prm[2], prm[3]};
        AcousticHooks h;
        if (kind == 1) { h.h0 = prm[4]; h.h1 = prm[5]; }
        auto* x = new App<AdvAcoustics, AcousticHooks>(*p, ph, h);
        int rc = x->d.init();
        if (rc) { delete x; return rc; }
        a = x;
    } else if (kind == 2) {
        auto* x = new App<fin::phys::EulerPhys, fin::phys::NoHooks>(*p, fin::phys::EulerPhys{p->gamma}, {});
        int rc = x->d.init();
        if (rc) { delete x; return rc; }
        a = x;
    } else {
        return FIN_ERR_ARG;
    }
    *out = a;
    return FIN_OK;
}
int app_destroy(void* h) { delete static_cast<AppBase*>(h); return FIN_OK; }
int app_set_state(void* h, const double* q, double t) { return static_cast<AppBase*>(h)->set_state(q, t); }
int app_get_state(void* h, double* q, double* t) { return static_cast<AppBase*>(h)->get_state(q, t); }
int app_construct_l(void* h, const double* q, double* L, double* smax)
{
    return static_cast<AppBase*>(h)->construct_l(q, L, smax);
}
int app_global_wave_spd(void* h, const double* q, double* a1, double* a2)
{
    return static_cast<AppBase*>(h)->global_wave_spd(q, a1, a2);
}
int app_step_fixed(void* h, double dt, double* cfl) { return static_cast<AppBase*>(h)->step_fixed(dt, cfl); }

}  // extern "C"
