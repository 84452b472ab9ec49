/*
 * finess_oracle.h -- CPU restatement (plain C, FP64) of the reference's 2D
 * WENO right-hand side and time steppers.  TEST INFRASTRUCTURE ONLY: it is
 * the checker for the CUDA path (tests, smoke(), bench.py's CPU baseline)
 * and never part of the product.
 *
 * Arrays use the reference's ghosted dTensorBC3 layout (lib/tensors.h:267-273):
 *   idx(i,j,m) = ((i+mbc-1)*(my+2*mbc) + (j+mbc-1))*meqn + (m-1).
 */
#ifndef FINESS_ORACLE_H
#define FINESS_ORACLE_H

#include "finess_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* SetBndValues as a per-side index remap, corners included. */
void oracle_set_bnd(const fin_params* p, double* q);

/* GlobalWaveSpd (lib/2d/GlobalWaveSpd.cpp:20-80). */
void oracle_global_wave_spd(const fin_params* p, const double* q, double* alpha1, double* alpha2);

/* ConstructL (lib/2d/ConstructL.cpp:13-408) on q as given (ghosts used as
 * they are).  L ghosted (mx,my,meqn), interior written; smax ghosted
 * (mx+1,my+1,2), max-accumulated.  Returns 0, or FIN_ERR_ARG for an
 * unsupported (weno_version, space_order). */
int oracle_construct_l(const fin_params* p, const double* q, double* L, double* smax);

/* Point-value WENO reconstructions of one 5-point stencil
 * (lib/WenoReconstruct.cpp:90-141, 385-438, 580-616). */
double oracle_weno5(int weno_version, double eps, double power_param, const double u[5]);

/* Nonlinear JS5 weights omega_k = omt_k/omts for one stencil
 * (lib/WenoReconstruct.cpp:121-134); used to label troubled stencils. */
void oracle_weno_js5_weights(double eps, double power_param, const double u[5], double w[3]);

/* FinSolveRK / FinSolveMD / FinSolveLxW from *t to tend (q in/out, ghosted).
 * dtv[1], dtv[2] as in lib/2d/RunFinpack.cpp:62-63.  nsteps may be NULL. */
int oracle_finsolve(const fin_params* p, double* q, double* t, double tend, double* dtv, int* nsteps);

/* One step of exactly dt with no CFL control; *cfl receives GetCFL's value. */
int oracle_step_fixed(const fin_params* p, double* q, double dt, double* cfl);

/* ConstructIntegratedR, 1-state form (lib/2d/ConstructIntegratedR.cpp:59-296):
 * time-integrated fluxes F, G (ghosted (mx,my,meqn)) from q with BCs applied. */
int oracle_construct_integrated_r(const fin_params* p, double dt, const double* q, double* F, double* G);

/* ConstructLxWL (lib/2d/ConstructLxWL.cpp:30-414): ConstructL's splitting
 * applied to the sampled F, G. */
int oracle_construct_lxwl(const fin_params* p, const double* q, const double* F, const double* G,
                          double* L, double* smax);

/* ConSoln totals (lib/2d/ConSoln.cpp:52-64): naive serial sum of dx*dy*q. */
void oracle_conservation_totals(const fin_params* p, const double* q, double* totals);

/* Troubled-cell indicator features (20 per face) and labels of every face,
 * x faces then y faces (the device kernel's enumeration). */
void oracle_face_samples(const fin_params* p, const double* q, double* X, unsigned char* y);

/* ---- ideal MHD (mhd_oracle.c): q ghosted (mx,my,8), aux ghosted (mx,my,1) ---- */
/* Doubly periodic SetBndValues of apps/2d/mhd/orszag_tang (aux may be NULL). */
void oracle_mhd_set_bnd(const fin_params* p, double* q, double* aux);
void oracle_mhd_global_wave_spd(const fin_params* p, const double* q, double* alpha1, double* alpha2);
/* ConstructL with the MHD callbacks; L interior written, smax max-accumulated. */
int oracle_mhd_construct_l(const fin_params* p, const double* q, double* L, double* smax);
/* ConstructHJ_L_Order1 (apps/2d/mhd/lib/ConstructHJ_L.cpp:29-113); needs mbc >= 5. */
int oracle_mhd_construct_hj_l(const fin_params* p, const double* q, const double* aux, double* Laux);
/* AfterStep (apps/2d/mhd/lib/AfterStep.cpp:13-60): B1, B2 from aux when
 * p->constrained_transport is set. */
void oracle_mhd_after_step(const fin_params* p, double* q, const double* aux);
/* One SSP-RK3 step of exactly dt (no CFL control); *cfl: the MHD GetCFL. */
int oracle_mhd_step_fixed(const fin_params* p, double* q, double* aux, double dt, double* cfl);
/* apps/2d/mhd/lib/FinSolveRK.cpp:17-395 (time_order 3) from *t to tend. */
int oracle_mhd_finsolve(const fin_params* p, double* q, double* aux, double* t, double tend, double* dtv,
                        int* nsteps);
/* Features (20 per face) and labels of the MHD troubled-face indicator,
 * x faces then y faces (the device kernel's enumeration). */
void oracle_mhd_face_samples(const fin_params* p, const double* q, double* X, unsigned char* y);
/* Orszag-Tang initial state (QinitFunc + AfterQinit), ghosts filled. */
void oracle_orszag_tang(const fin_params* p, double* q, double* aux);

#ifdef __cplusplus
}
#endif
#endif
