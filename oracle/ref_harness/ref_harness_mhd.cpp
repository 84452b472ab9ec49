// Harness that links the reference's own, unmodified ideal-MHD sources
// (lib/2d/ConstructL.cpp with apps/2d/mhd/lib/*.cpp: the MHD callbacks,
// FinSolveRK, UpdateSoln, ConstructHJ_L, AfterStep and GetCFL, and the
// Orszag-Tang case's QinitFunc, AfterQinit and SetBndValues) into
// oracle/_ref/libfinref_mhd.so and drives them through a small extern "C"
// API.  TEST INFRASTRUCTURE ONLY: it is the checker for the CUDA path and
// the CPU baseline of bench.py, never part of the product.
//
// What the harness supplies itself (the parts an application supplies in
// the reference): global_ini_params (IniParams.h beside this file), empty
// hooks (lib/2d/hooks.h:6-10), a ConSoln that writes no file, and the
// four-argument QinitFunc adapter of lib/2d/RunFinpack.cpp:143-149.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <stdexcept>
#include "IniParams.h"
#include "tensors.h"
#include "StateVars.h"
#include "finess_b200.h"

IniParams global_ini_params;

void ConstructL(StateVars& Q, dTensorBC3& Lstar, dTensorBC3& smax);
void GlobalWaveSpd(const StateVars& Q, double& alpha1, double& alpha2);
void FinSolveRK(StateVars& Qnew, double tend, double dtv[]);
void ConstructHJ_L_Order1(const StateVars& Q, dTensorBC3& Lauxstar);
void AfterStep(double dt, StateVars& Q);
void SetBndValues(StateVars& Q);
void AfterQinit(StateVars& Qnew);
void QinitFunc(const dTensor2& xpts, dTensor2& qvals);
void SampleFunction(int istart, int iend, int jstart, int jend, const dTensorBC3& qin, const dTensorBC3& auxin,
                    dTensorBC3& Fout, void (*Func)(const dTensor2&, const dTensor2&, const dTensor2&, dTensor2&));

// ---- application-supplied hooks ------------------------------------------
void BeforeFullTimeStep(double, StateVars&, StateVars&) {}
void AfterFullTimeStep(double, StateVars&, StateVars&) {}
void BeforeStep(double, StateVars&) {}
void ConSoln(const StateVars&) {}

static void QinitFunc4(const dTensor2& xpts, const dTensor2&, const dTensor2&, dTensor2& qvals)
{
    QinitFunc(xpts, qvals);
}

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

static StateVars* make_state(const double* q, const double* aux, double t)
{
    const IniParams& g = global_ini_params;
    StateVars* Q = new StateVars(t, g.mx, g.my, g.meqn, g.maux, g.mbc);
    load(Q->ref_q(), q);
    load(Q->ref_aux(), aux);
    return Q;
}

extern "C" {

int ref_mhd_setup(const fin_params* p)
{
    IniParams& g = global_ini_params;
    g.meqn = p->meqn; g.maux = p->maux;
    g.space_order = p->space_order; g.time_order = p->time_order;
    g.global_alpha = p->global_alpha != 0; g.source_term = p->source_term != 0;
    g.mpp_limiter = false;
    g.nv = p->nv; g.verbosity = p->verbosity;
    g.initial_dt = p->initial_dt; g.max_dt = p->max_dt;
    g.max_cfl = p->max_cfl; g.desired_cfl = p->desired_cfl;
    g.mx = p->mx; g.my = p->my; g.mbc = p->mbc;
    g.xlow = p->xlow; g.xhigh = p->xhigh; g.ylow = p->ylow; g.yhigh = p->yhigh;
    g.weno_version = (IniParams::WenoVersion::enum_type)p->weno_version;
    g.epsilon = p->epsilon; g.power_param = p->power_param; g.alpha_scaling = p->alpha_scaling;
    g.gamma = p->gamma;
    g.constrained_transport = p->constrained_transport != 0;
    return 0;
}

// RunFinpack.cpp:77-83: QinitFunc sampled on every ghosted cell, then AfterQinit.
int ref_mhd_qinit(double* q, double* aux)
{
    const IniParams& g = global_ini_params;
    StateVars Q(0.0, g.mx, g.my, g.meqn, g.maux, g.mbc);
    Q.ref_q().setall(0.);
    Q.ref_aux().setall(0.);
    SampleFunction(1 - g.mbc, g.mx + g.mbc, 1 - g.mbc, g.my + g.mbc, Q.ref_q(), Q.ref_aux(), Q.ref_q(), &QinitFunc4);
    AfterQinit(Q);
    store(Q.ref_q(), q);
    store(Q.ref_aux(), aux);
    return 0;
}

int ref_mhd_set_bnd(double* q, double* aux)
{
    StateVars* Q = make_state(q, aux, 0.0);
    SetBndValues(*Q);
    store(Q->ref_q(), q);
    store(Q->ref_aux(), aux);
    delete Q;
    return 0;
}

// ConstructL on (q, aux) as given (no BC applied here).
int ref_mhd_construct_l(const double* q, const double* aux, double* L, double* smax)
{
    const IniParams& g = global_ini_params;
    StateVars* Q = make_state(q, aux, 0.0);
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

int ref_mhd_global_wave_spd(const double* q, const double* aux, double* alpha12)
{
    StateVars* Q = make_state(q, aux, 0.0);
    GlobalWaveSpd(*Q, alpha12[0], alpha12[1]);
    delete Q;
    return 0;
}

int ref_mhd_construct_hj_l(const double* q, const double* aux, double* Laux)
{
    const IniParams& g = global_ini_params;
    StateVars* Q = make_state(q, aux, 0.0);
    dTensorBC3 La(g.mx, g.my, g.maux, g.mbc);
    ConstructHJ_L_Order1(*Q, La);
    store(La, Laux);
    delete Q;
    return 0;
}

int ref_mhd_after_step(double* q, const double* aux)
{
    StateVars* Q = make_state(q, aux, 0.0);
    AfterStep(0.0, *Q);
    store(Q->ref_q(), q);
    delete Q;
    return 0;
}

// FinSolveRK (apps/2d/mhd/lib/FinSolveRK.cpp) from t to tend; q, aux in/out.
int ref_mhd_finsolve(double* q, double* aux, double* t, double tend, double* dtv)
{
    StateVars* Q = make_state(q, aux, *t);
    int rc = 0;
    try { FinSolveRK(*Q, tend, dtv); } catch (std::exception&) { rc = FIN_ERR_ARG; }
    store(Q->ref_q(), q);
    store(Q->ref_aux(), aux);
    *t = Q->get_t();
    delete Q;
    return rc;
}

}  // extern "C"
