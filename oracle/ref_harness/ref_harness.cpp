// Harness that links the reference's own, unmodified hot-path sources
// (lib/2d/ConstructL.cpp, lib/WenoReconstruct.cpp, lib/2d/FinSolveRK.cpp, ...
// and apps/2d/euler/lib/*.cpp) into oracle/_ref/libfinref.so and drives them
// through a small extern "C" API.  TEST INFRASTRUCTURE ONLY: it is the
// checker for the CUDA path and the CPU baseline of bench.py, never part of
// the product.
//
// What the harness supplies itself (the parts an application supplies in
// the reference):
//  * global_ini_params (IniParams.h beside this file);
//  * SetBndValues as an index remap per side, periodic or transmissive,
//    corners included (apps/2d/euler/test_exact2/SetBndValues.cpp:8-199 and
//    apps/2d/euler/riemann_test/SetBndValues.cpp:9-115 are the patterns);
//  * empty hooks (lib/2d/hooks.h:6-10), an empty SourceTermFunc, and a
//    ConSoln that writes no file (lib/2d/ConSoln.cpp writes conservation.dat).
#include <cstdio>
#include <cstring>
#include <cmath>
#include <stdexcept>
#include "IniParams.h"
#include "tensors.h"
#include "StateVars.h"
#include "finess_b200.h"

IniParams global_ini_params;

// ---- declarations of reference library functions driven from here -------
void ConstructL(StateVars& Q, dTensorBC3& Lstar, dTensorBC3& smax);
void GlobalWaveSpd(const StateVars& Q, double& alpha1, double& alpha2);
void FinSolveRK(StateVars& Qnew, double tend, double dtv[]);
void FinSolveMD(StateVars& Qnew, double tend, double dtv[]);
void FinSolveLxW(StateVars& Qnew, double tend, double dtv[]);
void ConstructIntegratedR(double dt, const StateVars& Q,
    dTensorBC3& smax, dTensorBC3& F, dTensorBC3& G);
void ConstructIntegratedR(double dt, double alpha1, double beta1, const StateVars& Q1,
    double alpha2, double beta2, const StateVars& Q2,
    dTensorBC3& smax, dTensorBC3& F, dTensorBC3& G);
void ConstructLxWL(const StateVars& Q, const dTensorBC3& F, const dTensorBC3& G,
    dTensorBC3& Lstar, dTensorBC3& smax);

void DFluxFunc(const dTensor2&, const dTensor2&, const dTensor2&, dTensor4&);
void D2FluxFunc(const dTensor2&, const dTensor2&, const dTensor2&, dTensor5&);

static int g_bc[4] = {FIN_BC_PERIODIC, FIN_BC_PERIODIC, FIN_BC_PERIODIC, FIN_BC_PERIODIC};

static int remap(int k, int n, int bc_lo, int bc_hi)
{
    if (k < 1) return bc_lo == FIN_BC_PERIODIC ? k + n : 1;
    if (k > n) return bc_hi == FIN_BC_PERIODIC ? k - n : n;
    return k;
}

// ---- application-supplied callbacks --------------------------------------
void SetBndValues(StateVars& Q)
{
    dTensorBC3& q = Q.ref_q();
    dTensorBC3& aux = Q.ref_aux();
    const int mx = global_ini_params.get_mx(), my = global_ini_params.get_my();
    const int mbc = global_ini_params.get_mbc(), meqn = global_ini_params.get_meqn();
    const int maux = global_ini_params.get_maux();
    for (int i = 1 - mbc; i <= mx + mbc; i++)
        for (int j = 1 - mbc; j <= my + mbc; j++) {
            if (i >= 1 && i <= mx && j >= 1 && j <= my) continue;
            const int si = remap(i, mx, g_bc[0], g_bc[1]);
            const int sj = remap(j, my, g_bc[2], g_bc[3]);
            for (int m = 1; m <= meqn; m++) q.set(i, j, m, q.get(si, sj, m));
            for (int m = 1; m <= maux; m++) aux.set(i, j, m, aux.get(si, sj, m));
        }
}
// The MPP limiter branch of FinSolveLxW (off in every configuration here)
// links ConstructLFL.cpp, which calls these one-direction BC variants.
void SetBndValuesX(StateVars& Q) { SetBndValues(Q); }
void SetBndValuesY(StateVars& Q) { SetBndValues(Q); }
void SourceTermFunc(const dTensor2&, const dTensor2&, const dTensor2&, dTensor2& source)
{
    source.setall(0.);
}
void AfterQinit(StateVars&) {}
void BeforeFullTimeStep(double, StateVars&, StateVars&) {}
void AfterFullTimeStep(double, StateVars&, StateVars&) {}
void BeforeStep(double, StateVars&) {}
void AfterStep(double, StateVars&) {}
// FinSolveRK / FinSolveMD / FinSolveLxW call ConSoln once per accepted step
// (FinSolveRK.cpp:362): the harness counts the calls instead of writing
// conservation.dat, which gives the number of accepted steps of a run.
static long long g_accepted_steps = 0;
void ConSoln(const StateVars&) { ++g_accepted_steps; }

// ---- helpers -------------------------------------------------------------
static void load(dTensorBC3& t, const double* src)
{
    const int n = t.numel();
    for (int k = 0; k < n; k++) t.vset(k, src[k]);
}
static void store(const dTensorBC3& t, double* dst)
{
    const int n = t.numel();
    for (int k = 0; k < n; k++) dst[k] = t.vget(k);
}

extern "C" {

int ref_setup(const fin_params* p)
{
    IniParams& g = global_ini_params;
    g.meqn = p->meqn; g.maux = p->maux;
    g.space_order = p->space_order; g.time_order = p->time_order;
    g.global_alpha = p->global_alpha != 0; g.source_term = p->source_term != 0;
    g.nv = p->nv; g.verbosity = p->verbosity;
    g.initial_dt = p->initial_dt; g.max_dt = p->max_dt;
    g.max_cfl = p->max_cfl; g.desired_cfl = p->desired_cfl;
    g.mx = p->mx; g.my = p->my; g.mbc = p->mbc;
    g.xlow = p->xlow; g.xhigh = p->xhigh; g.ylow = p->ylow; g.yhigh = p->yhigh;
    g.weno_version = (IniParams::WenoVersion::enum_type)p->weno_version;
    g.epsilon = p->epsilon; g.power_param = p->power_param; g.alpha_scaling = p->alpha_scaling;
    g.gamma = p->gamma;
    g.mpp_limiter = p->mpp_limiter != 0;
    g.time_stepping_method = p->time_stepping_method == FIN_TS_MD    ? IniParams::TimeSteppingMethod::MD
                             : p->time_stepping_method == FIN_TS_LXW ? IniParams::TimeSteppingMethod::LxW
                                                                     : IniParams::TimeSteppingMethod::RK;
    g_bc[0] = p->bc_xlow; g_bc[1] = p->bc_xhigh; g_bc[2] = p->bc_ylow; g_bc[3] = p->bc_yhigh;
    return 0;
}

static StateVars* make_state(const double* q, double t)
{
    const IniParams& g = global_ini_params;
    StateVars* Q = new StateVars(t, g.mx, g.my, g.meqn, g.maux, g.mbc);
    load(Q->ref_q(), q);
    Q->ref_aux().setall(0.);
    return Q;
}

// Apply the harness SetBndValues in place on a ghosted host array.
int ref_set_bnd(double* q)
{
    StateVars* Q = make_state(q, 0.0);
    SetBndValues(*Q);
    store(Q->ref_q(), q);
    delete Q;
    return 0;
}

// ConstructL on q as given (ghosts included, no BC applied here).
// L: ghosted (mx,my,meqn); smax: ghosted (mx+1,my+1,2), max-accumulated.
int ref_construct_l(const double* q, double* L, double* smax)
{
    const IniParams& g = global_ini_params;
    StateVars* Q = make_state(q, 0.0);
    dTensorBC3 Lstar(g.mx, g.my, g.meqn, g.mbc);
    dTensorBC3 sm(g.mx + 1, g.my + 1, 2, g.mbc);
    Lstar.setall(0.);
    load(sm, smax);
    int rc = 0;
    try { ConstructL(*Q, Lstar, sm); } catch (std::exception&) { rc = FIN_ERR_ARG; }
    store(Lstar, L);
    store(sm, smax);
    delete Q;
    return rc;
}

int ref_global_wave_spd(const double* q, double* alpha12)
{
    StateVars* Q = make_state(q, 0.0);
    GlobalWaveSpd(*Q, alpha12[0], alpha12[1]);
    delete Q;
    return 0;
}

// Time-integrated fluxes F, G of ConstructIntegratedR (1-state form).
int ref_construct_integrated_r(double dt, const double* q, double* F, double* G)
{
    const IniParams& g = global_ini_params;
    StateVars* Q = make_state(q, 0.0);
    dTensorBC3 sm(g.mx + 1, g.my + 1, 2, g.mbc);
    dTensorBC3 Ft(g.mx, g.my, g.meqn, g.mbc), Gt(g.mx, g.my, g.meqn, g.mbc);
    Ft.setall(0.); Gt.setall(0.); sm.setall(0.);
    ConstructIntegratedR(dt, *Q, sm, Ft, Gt);
    store(Ft, F); store(Gt, G);
    delete Q;
    return 0;
}

// FinSolveRK (method 0), FinSolveLxW (2) or FinSolveMD (3) from t to tend.
// q is in/out (ghosted), dtv[0..2] as RunFinpack.cpp:62-63 (dtv[1], dtv[2]).
int ref_finsolve(int method, double* q, double* t, double tend, double* dtv)
{
    StateVars* Q = make_state(q, *t);
    int rc = 0;
    g_accepted_steps = 0;
    try {
        if (method == FIN_TS_RK) FinSolveRK(*Q, tend, dtv);
        else if (method == FIN_TS_MD) FinSolveMD(*Q, tend, dtv);
        else if (method == FIN_TS_LXW) FinSolveLxW(*Q, tend, dtv);
        else rc = FIN_ERR_ARG;
    } catch (std::exception&) { rc = FIN_ERR_ARG; }
    store(Q->ref_q(), q);
    *t = Q->get_t();
    delete Q;
    return rc;
}

// Accepted steps of the last ref_finsolve call.
long long ref_last_steps(void) { return g_accepted_steps; }

// Jacobian and Hessian of the application's flux at one state (DFluxFunc,
// D2FluxFunc): A[(d*5+m)*5+k], H[((d*5+m)*5+k1)*5+k2], d = 0 (f) or 1 (g).
int ref_flux_derivs(const double* Q, double* A, double* H)
{
    dTensor2 xp(1, 2), q(1, 5), aux(1, 1);
    xp.setall(0.); aux.setall(0.);
    for (int m = 1; m <= 5; m++) q.set(1, m, Q[m - 1]);
    dTensor4 D(1, 5, 5, 2);
    dTensor5 D2(1, 5, 5, 5, 2);
    DFluxFunc(xp, q, aux, D);
    D2FluxFunc(xp, q, aux, D2);
    for (int d = 0; d < 2; d++)
        for (int m = 0; m < 5; m++)
            for (int k = 0; k < 5; k++) {
                A[(d * 5 + m) * 5 + k] = D.get(1, m + 1, k + 1, d + 1);
                for (int k2 = 0; k2 < 5; k2++)
                    H[((d * 5 + m) * 5 + k) * 5 + k2] = D2.get(1, m + 1, k + 1, k2 + 1, d + 1);
            }
    return 0;
}

}  // extern "C"
