// Element-wise kernels of the higher-order Runge-Kutta steps of FinSolveRK
// (lib/2d/FinSolveRK.cpp:213-305) that are not a stage of the form
// q_out = a1 A + a2 B + beta dt L (those run through the stage kernel):
//   * the register swap between stages 5 and 6 of the ten-stage fourth-order
//     method (:239-247);
//   * the update of the eight-stage fifth-order method (the ten-argument
//     UpdateSoln, lib/2d/UpdateSoln.cpp:44-80), whose L comes from the stage
//     kernel with a1 = a2 = 0 and beta dt = 1.
// Each writes its new state and that state's global wave speeds
// (GlobalWaveSpd.cpp:71-76), which the next stage takes as its alpha.  All
// arithmetic is correctly rounded FP64 in the reference's order.
#pragma once
#include "fin_stage.cuh"

namespace fin {
namespace rk {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// GlobalWaveSpd.cpp:71-76 of one cell: |u1| + c and |u2| + c (SetWaveSpd.cpp
// with Ql = Qr), with c = sqrt(|gamma p / rho|).
__device__ __forceinline__ void cell_speeds(const double* Q, double gamma, double& sx, double& sy)
{
    const double rho = Q[0];
    const double u1 = dvd(Q[1], rho), u2 = dvd(Q[2], rho), u3 = dvd(Q[3], rho);
    const double ke = add(add(mul(u1, u1), mul(u2, u2)), mul(u3, u3));
    const double press = mul(sub(gamma, 1.0e0), sub(Q[4], mul(mul(0.5e0, rho), ke)));
    const double c = sqrt(fabs(dvd(mul(gamma, press), rho)));
    sx = add(fabs(u1), c);
    sy = add(fabs(u2), c);
}

// Block maximum of the two speeds into alpha_out (finite values only; a
// non-finite one sets status bit 0).
__device__ __forceinline__ void reduce_speeds(double sx, double sy, bool nonfinite, double* alpha_out,
                                              unsigned int* status)
{
    __shared__ double red[2][8];
    for (int o = 16; o > 0; o >>= 1) {
        sx = Max(sx, __shfl_xor_sync(0xffffffffu, sx, o));
        sy = Max(sy, __shfl_xor_sync(0xffffffffu, sy, o));
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = sx;
        red[1][threadIdx.x >> 5] = sy;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < int(blockDim.x >> 5); w++) {
            sx = Max(sx, red[0][w]);
            sy = Max(sy, red[1][w]);
        }
        if (alpha_out) {
            atomic_max_nonneg(alpha_out, sx);
            atomic_max_nonneg(alpha_out + 1, sy);
        }
    }
    if (nonfinite) atomicOr(status, 1u);
}

// Fourth order, between stages 5 and 6 (FinSolveRK.cpp:239-247):
//   q2 <- (q2 + 9 q1) / 25;  q1 <- 15 q2 - 5 q1   (q1 in place)
__global__ void __launch_bounds__(256) k_rk4_swap(const double* __restrict__ q2_in, double* __restrict__ q2_out,
                                                  double* __restrict__ q1, size_t plane, size_t n, double gamma,
                                                  double* alpha_out, unsigned int* status)
{
    double sx = 0.0, sy = 0.0;
    bool nonfinite = false;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        double Q[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            const double a = q1[m * plane + g];
            const double tmp = dvd(add(q2_in[m * plane + g], mul(9.0, a)), 25.0);
            q2_out[m * plane + g] = tmp;
            Q[m] = sub(mul(15.0, tmp), mul(5.0, a));
            q1[m * plane + g] = Q[m];
        }
        double a, b;
        cell_speeds(Q, gamma, a, b);
        if (!(a <= 1e300) || !(b <= 1e300)) nonfinite = true;
        else {
            sx = Max(sx, a);
            sy = Max(sy, b);
        }
    }
    reduce_speeds(sx, sy, nonfinite, alpha_out, status);
}

// Fifth order, one stage's update (UpdateSoln.cpp:66-78):
//   s1 = q1;  s2 = q2 + delta s1;  q2 <- s2;
//   q1 <- g1 s1 + g2 s2 + g3 qold + (beta dt) L
// q2_in null: q2 = 0 (FinSolveRK.cpp:280 clears it at each step).
__global__ void __launch_bounds__(256) k_rk5_update(const double* __restrict__ q1_in, double* __restrict__ q1_out,
                                                    const double* __restrict__ q2_in, double* __restrict__ q2_out,
                                                    const double* __restrict__ qold, const double* __restrict__ L,
                                                    size_t plane, size_t n, double g1, double g2, double g3,
                                                    double delta, double bdt, double gamma, double* alpha_out,
                                                    unsigned int* status)
{
    double sx = 0.0, sy = 0.0;
    bool nonfinite = false;
    for (size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < n; g += size_t(gridDim.x) * blockDim.x) {
        double Q[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            const size_t k = m * plane + g;
            const double s1 = q1_in[k];
            const double s2 = add(q2_in ? q2_in[k] : 0.0, mul(delta, s1));
            q2_out[k] = s2;
            const double s3 = qold[k];
            Q[m] = add(add(add(mul(g1, s1), mul(g2, s2)), mul(g3, s3)), mul(bdt, L[k]));
            q1_out[k] = Q[m];
        }
        double a, b;
        cell_speeds(Q, gamma, a, b);
        if (!(a <= 1e300) || !(b <= 1e300)) nonfinite = true;
        else {
            sx = Max(sx, a);
            sy = Max(sy, b);
        }
    }
    reduce_speeds(sx, sy, nonfinite, alpha_out, status);
}

// SetRKinfo.cpp:86-126, the fifth-order method's coefficients (delta,
// gamma rows 1-3, beta for stages 1-8).
struct Rk5Coef {
    double delta[8], g1[8], g2[8], g3[8], beta[8];
};
inline Rk5Coef rk5_coefficients()
{
    Rk5Coef c = {
        {1.0e0, 1.528486658778845e00, 4.720094096662784e-02, 8.801244253465348e-01, 1.019066090228480e+00,
         1.049772291176110e+01, -4.254616508506826e+00, 0.0},
        {0.0, -1.552288007713033e+01, 4.127286635722417e-01, -1.011819196331377e+00, -2.765748383780848e-01,
         5.075770311217778e-02, 6.999810478513669e+00, -1.114908881433104e+01},
        {1.0, 6.534691420958578e+00, 2.280056542904473e-01, 1.308684311397668e+00, 4.769419552531064e-01,
         -6.368809762042849e-03, 9.339446057238532e-02, 9.556626047962331e-01},
        {0.0, 0.0, 0.0, -2.510747784045939e+00, -8.576822794622042e-01, 1.044599944472272e+00,
         -7.000810861049136e+00, 1.906311811144179e+00},
        {8.653258038183180e-02, 9.544677980851571e-01, 2.651941386774408e-01, 2.736914413910379e-01,
         5.999778649323600e-01, 4.433177471748104e-03, 5.309971130968292e-03, 5.830861806762871e-01}};
    return c;
}

}  // namespace rk
}  // namespace fin
