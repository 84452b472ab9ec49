/*
 * finess_b200.h -- C ABI of the B200 (sm_100a) implementation of FINESS's
 * 2D finite-difference WENO right-hand side and time steppers.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an
 * int status (FIN_OK == 0) and never exits the process.  The C++ relink shims
 * (finess_b200/csrc/shim/*.cpp, one file per reference symbol) map these
 * statuses back onto the reference's own conventions (printf + exit(1),
 * std::logic_error).
 *
 * Array layout at this boundary is the reference's own dTensorBC3 layout
 * (lib/tensors.h:267-273, lib/tensors.cpp:650-667): a ghosted array
 *   q(i, j, m),  i = 1-mbc .. mx+mbc,  j = 1-mbc .. my+mbc,  m = 1 .. meqn,
 * stored with m fastest and i slowest:
 *   idx = ((i+mbc-1)*(my+2*mbc) + (j+mbc-1))*meqn + (m-1).
 * "host" entry points take host pointers (pageable or pinned) in that layout;
 * "_dev" entry points take device pointers in the device layout described
 * with fin_device_layout().
 */
#ifndef FINESS_B200_H
#define FINESS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FIN_ABI_VERSION 2

/* ---- status codes ---------------------------------------------------- */
enum {
    FIN_OK = 0,
    FIN_ERR_ARG = 1,          /* bad argument / unsupported parameter combination */
    FIN_ERR_CUDA = 2,         /* a CUDA runtime call failed (see fin_last_error) */
    FIN_ERR_NO_DEVICE = 3,    /* no sm_100 device visible */
    FIN_ERR_NSTEPS = 4,       /* more than nv steps in one frame (FinSolveRK.cpp:84-92) */
    FIN_ERR_DT_BOUNDS = 5,    /* dt > max_dt (GetCFL.cpp:43-48) */
    FIN_ERR_CFL_BOUNDS = 6,   /* cfl > 1e8 (GetCFL.cpp:61-66) */
    FIN_ERR_NONFINITE = 7,    /* NaN/Inf met in a wave speed or the state */
    FIN_ERR_UNSUPPORTED = 8,  /* valid in the reference, not built here */
    FIN_ERR_SIZE = 9          /* a size beyond a documented maximum */
};

/* ---- enumerations (numeric values follow the reference's enum order) -- */
enum fin_weno_version { FIN_WENO_FD = 0, FIN_WENO_JS = 1, FIN_WENO_Z = 2 };
enum fin_time_stepping { FIN_TS_RK = 0, FIN_TS_LXW = 2, FIN_TS_MD = 3 };
enum fin_bc { FIN_BC_PERIODIC = 0, FIN_BC_TRANSMISSIVE = 1 };
enum fin_physics { FIN_PHYS_EULER = 0, FIN_PHYS_MHD = 1 };
enum fin_precision {
    FIN_PREC_FP64 = 0,     /* plain method, FP64 everywhere (the parity form) */
    FIN_PREC_FP32 = 1,     /* FP32 reconstruction/splitting/projection, FP64 state */
    FIN_PREC_HYBRID = 2    /* FP32 bulk + troubled-cell indicator: linear FD5 on smooth cells */
};

/* Parameters of one problem: the fields of parameters.ini that the
 * reference's hot path reads (python/finess/params/{finess,dim2,weno,euler}.py). */
typedef struct fin_params {
    /* [finess] */
    int meqn, maux;
    int space_order, time_order;
    int time_stepping_method;      /* enum fin_time_stepping */
    int global_alpha, source_term;
    int nv, verbosity;
    double initial_dt, max_dt, max_cfl, desired_cfl;
    /* [grid] */
    int mx, my, mbc;
    double xlow, xhigh, ylow, yhigh;
    /* [weno] */
    int weno_version;              /* enum fin_weno_version */
    double epsilon, power_param, alpha_scaling;
    /* [euler] */
    double gamma;
    /* boundary conditions applied as an index remap (the apps' SetBndValues) */
    int bc_xlow, bc_xhigh, bc_ylow, bc_yhigh;  /* enum fin_bc */
    /* this library */
    int physics;                   /* enum fin_physics */
    int precision;                 /* enum fin_precision */
    /* frame loop of RunFinpack (lib/2d/RunFinpack.cpp:95-130) */
    double tfinal;
    int nout;
    /* [mhd] (python/finess/params/mhd.py:20-26): rebuild B1, B2 from the
     * potential A3 after every stage (apps/2d/mhd/lib/AfterStep.cpp:31-56) */
    int constrained_transport;
    /* [finess] mpp_limiter (python/finess/params/finess.py:21-26): the
     * Lax-Wendroff step limits its fluxes toward Lax-Friedrichs ones to keep
     * density and pressure positive (FinSolveLxW.cpp:126-151); the
     * reference reads it only in FinSolveLxW */
    int mpp_limiter;
} fin_params;

/* Defaults of python/finess/params/finess.py, weno.py, euler.py and mhd.py. */
void fin_params_default(fin_params* p);

/* Reads an application's parameters.ini (sections [finess], [grid], [weno],
 * [euler] with the keys, defaults and checks of the reference's parameter
 * specs, python/finess/params/{finess,dim2,weno,euler}.py, which its build
 * compiles into IniParams, python/finess/params/params.py:358-497), plus an
 * optional [finess_b200] section: bc_xlow/bc_xhigh/bc_ylow/bc_yhigh =
 * periodic|transmissive and precision = fp64|fp32|hybrid.  Returns
 * FIN_ERR_ARG with fin_ini_last_error() set when a check fails, where the
 * reference's terminate() would throw (lib/sys/util.h:38-43). */
int fin_params_from_ini(const char* path, fin_params* p);
const char* fin_ini_last_error(void);

/* Last error message of the calling thread (never NULL). */
const char* fin_last_error(void);

/* ABI version of the loaded library (FIN_ABI_VERSION it was built with). */
int fin_abi_version(void);

/* ---- solver handle ---------------------------------------------------- */
typedef struct fin_solver fin_solver;

/* Allocates the device state for one problem on the current CUDA device.
 * Replaces the StateVars/dTensorBC3 allocations of FinSolveRK.cpp:44-70. */
int fin_create(const fin_params* p, fin_solver** out);
int fin_destroy(fin_solver* s);

/* Copies a host state (reference ghosted layout, interior used) to the device
 * and sets t.  Replaces StateVars construction + QinitFunc sampling. */
int fin_set_state(fin_solver* s, const double* q_host, double t);
/* Initial data sampled on the device into the state and t set: SampleFunction
 * (lib/2d/SampleFunction.cpp:62-125) with a QinitFunc (lib/2d/app_defined.h:7)
 * evaluated at the interior cell centres xlow + (i - 1/2) dx,
 * ylow + (j - 1/2) dy, as RunFinpack.cpp:80 does before the first frame.
 * Replaces StateVars construction + host sampling + fin_set_state.
 * problem / prm (nprm values; 0 = the defaults in brackets):
 *   FIN_QINIT_VORTEX         isentropic vortex on the background (1, 1, 1, 1):
 *                            eps, xc, yc [5, 5, 5]
 *   FIN_QINIT_RIEMANN4       four-quadrant Riemann problem: xc, yc, then
 *                            (rho, u, v, p) of the upper-right, upper-left,
 *                            lower-left, lower-right quadrants [interface
 *                            (0.8, 0.8), the benchmark's states]
 *   FIN_QINIT_SHOCK_ENTROPY  shock / entropy-wave interaction on [-5,5]x[0,1]
 *   FIN_QINIT_SHOCK_TUBE     apps/2d/euler/riemann_test/QinitFunc.cpp: OPT
 *   FIN_QINIT_VORTEX_EXACT2  apps/2d/euler/test_exact2/QinitFunc.cpp
 * Applications with their own initial data instantiate the device template
 * fin::launch_sample<Functor> of finess_b200/csrc/fin_sample.cuh. */
#define FIN_QINIT_VORTEX 1
#define FIN_QINIT_RIEMANN4 2
#define FIN_QINIT_SHOCK_ENTROPY 3
#define FIN_QINIT_SHOCK_TUBE 4
#define FIN_QINIT_VORTEX_EXACT2 5
int fin_set_state_qinit(fin_solver* s, int problem, const double* prm, int nprm, double t);

/* Copies the device state back (interior written; ghosts filled by the BC
 * remap, as SetBndValues would). */
int fin_get_state(fin_solver* s, double* q_host, double* t);

/* ConstructL (lib/2d/ConstructL.cpp:13-408) on a host state.
 *   q_host:  ghosted input state (only interior cells read; ghosts come
 *            from the BC remap, i.e. SetBndValues is applied first);
 *   L_host:  ghosted output, interior written, ghosts untouched
 *            (the reference leaves them uninitialised);
 *   smax_host: optional (may be NULL), ghosted (mx+1, my+1, 2) array that
 *            is max-accumulated exactly as ConstructL.cpp:173,324 do.
 * GlobalWaveSpd (lib/2d/GlobalWaveSpd.cpp:20-80) runs first when
 * global_alpha is set. */
int fin_construct_l(fin_solver* s, const double* q_host, double* L_host, double* smax_host);

/* GlobalWaveSpd (lib/2d/GlobalWaveSpd.cpp:20-80) on a host state. */
int fin_global_wave_spd(fin_solver* s, const double* q_host, double* alpha1, double* alpha2);

/* FinSolveRK / FinSolveMD / FinSolveLxW on the device state, advancing it
 * from its t to tend (lib/2d/FinSolveRK.cpp:13-371, FinSolveMD.cpp:21-291,
 * FinSolveLxW.cpp:16-245).  dtv[1] is the starting dt and receives the next
 * dt; dtv[2] is max_dt (lib/2d/RunFinpack.cpp:62-63).  dtv has >= 3 entries.
 * nsteps_out (may be NULL) receives the number of accepted steps. */
int fin_solve(fin_solver* s, double tend, double* dtv, int* nsteps_out);

/* fin_solve that stops after max_steps accepted steps (or at tend).  The
 * device time of the whole call, host waits included, is then available
 * from fin_last_kernel_ms. */
int fin_advance(fin_solver* s, double tend, double* dtv, int max_steps, int* nsteps_out);

/* ConstructIntegratedR, 1-state form (lib/2d/ConstructIntegratedR.cpp:59-296):
 * the time-integrated fluxes F = f + dt/2 (f_t + dt/3 f_tt) (f_tt when
 * time_order > 2) on the interior and the 3-cell ghost frame, written into
 * ghosted host arrays F_host, G_host (other ghost entries untouched).  Needs a
 * solver created with Lax-Wendroff or multiderivative stepping (mbc >= 5). */
int fin_construct_integrated_r(fin_solver* s, double dt, const double* q_host, double* F_host, double* G_host);

/* ConstructIntegratedR, 2-state form (lib/2d/ConstructIntegratedR.cpp:
 * 525-606, declared lib/2d/constructs.h:19-24): F = alpha1 R(q1) + dt beta1
 * f_t(q1) + alpha2 R(q2) + dt beta2 f_t(q2), and G alike; arrays as the
 * 1-state form. */
int fin_construct_integrated_r2(fin_solver* s, double dt, double alpha1, double beta1, const double* q1_host,
                                double alpha2, double beta2, const double* q2_host, double* F_host, double* G_host);

/* ConstructIntegratedR, three-coefficient form (lib/2d/ConstructIntegratedR.
 * cpp:608-700, declared lib/2d/constructs.h:26-31), used by the fifth-order
 * multiderivative stepper: adds charlie1 dt^2 f_tt(q1) + charlie2 dt^2
 * f_tt(q2) to the 2-state sum. */
int fin_construct_integrated_r3(fin_solver* s, double dt, double alpha1, double beta1, double charlie1,
                                const double* q1_host, double alpha2, double beta2, double charlie2,
                                const double* q2_host, double* F_host, double* G_host);

/* ConstructLxWL (lib/2d/ConstructLxWL.cpp:30-414, declared lib/2d/
 * constructs.h:44-51): ConstructL's split, reconstruction and projection
 * applied to the sampled time-integrated fluxes F, G (ghosted host arrays
 * whose interior and 3-cell ghost frame are read) instead of FluxFunc of q.
 * L_host and smax_host as fin_construct_l.  Fhat_host, Ghat_host (may be
 * NULL: the overload without them) receive the face fluxes in the ghosted
 * (mx+1, my, meqn) and (mx, my+1, meqn) layouts, faces 1..mx+1 / 1..my+1
 * written.  Needs a solver created with Lax-Wendroff or multiderivative
 * stepping. */
int fin_construct_lxwl(fin_solver* s, const double* q_host, const double* F_host, const double* G_host,
                       double* L_host, double* smax_host, double* Fhat_host, double* Ghat_host);

/* UpdateSoln, orders 1-4 (lib/2d/UpdateSoln.cpp:14-38, declared lib/2d/
 * FinSolveRK.h:21-22): qnew = alpha1 qstar + alpha2 qnew + (beta dt) L over
 * every element of the ghosted arrays (ghosts included, in the reference's
 * operation order, correctly rounded), and *t_new = alpha1 t_star + alpha2
 * *t_new + beta dt. */
int fin_update_soln(fin_solver* s, double alpha1, double alpha2, double beta, double dt, const double* qstar_host,
                    double t_star, const double* L_host, double* qnew_host, double* t_new);

/* UpdateSoln, the fifth-order stepper's form (lib/2d/UpdateSoln.cpp:43-80,
 * declared lib/2d/FinSolveRK.h:25-29): over every element, q2 = q2 + delta
 * q1, then q1 = g1 q1 + g2 q2 + g3 qold + (beta dt) L; times untouched. */
int fin_update_soln5(fin_solver* s, double g1, double g2, double g3, double delta, double beta, double dt,
                     const double* qold_host, const double* L_host, double* q1_host, double* q2_host);

/* GetCFL (lib/2d/GetCFL.cpp:31-73, declared lib/2d/misc2d.h:7): the maximum
 * of dt smax(i,j,1)/dx and dt smax(i,j,2)/dy over i <= mx, j <= my of the
 * ghosted (mx+1, my+1, 2) host array smax_host (NaN entries skipped, as the
 * reference's Max does).  Returns FIN_ERR_DT_BOUNDS when dt > dtmax and
 * FIN_ERR_CFL_BOUNDS when the CFL number exceeds 1e8 (*cfl is set then too);
 * the relink shim turns these into the reference's message and exit(1). */
int fin_get_cfl(fin_solver* s, double dt, double dtmax, const double* smax_host, double* cfl);

/* GetCFL from the global wave speeds (lib/2d/GetCFL.cpp:76-101, declared
 * lib/2d/misc2d.h:8): max(dt alpha1/dx, dt alpha2/dy), same errors. */
int fin_get_cfl_alpha(const fin_params* p, double dt, double dtmax, double alpha1, double alpha2, double* cfl);

/* One time step of exactly dt with no CFL control (benchmarking and
 * per-step parity); cfl_out (may be NULL) receives GetCFL's value for it. */
int fin_step_fixed(fin_solver* s, double dt, double* cfl_out);

/* Per-component totals sum(dx*dy*q) over interior cells, accumulated in FP64
 * with compensated summation (lib/2d/ConSoln.cpp:52-64). totals[meqn]. */
int fin_conservation_totals(fin_solver* s, double* totals);

/* ---- output files ----------------------------------------------------- */
/* The reference's frame files from the device state, in its formats:
 * q%04d.dat and a%04d.dat (void Output(const StateVars&, int nframe),
 * lib/2d/Output.cpp:12-62: a header line with t, then every value of
 * component m = 1..meqn (maux for the aux file), j = 1..my, i = 1..mx (i
 * fastest) as "%24.16e\n", i.e. setprecision(16), setw(24), scientific),
 * written under outdir.  Asynchronous: the state is reordered on the device
 * and copied to pinned host memory on a side stream, then host threads
 * format and write the files while the solver goes on; fin_output_wait
 * returns when they are on disk (the next fin_output_frame, fin_read_frame
 * and fin_destroy wait too).  The Euler path holds no aux planes (its
 * AuxFunc sets none, apps/2d/euler/lib/AuxFunc.cpp:10-13): a%04d.dat gets
 * maux planes of zeros. */
int fin_output_frame(fin_solver* s, int nframe, const char* outdir);
int fin_output_wait(fin_solver* s);
/* Restart: a q%04d.dat file (this library's or the reference's) becomes the
 * state, its header the time; alpha and the hybrid flags as fin_set_state. */
int fin_read_frame(fin_solver* s, const char* path);
/* conservation.dat (void ConSoln(const StateVars&), lib/2d/ConSoln.cpp:
 * 34-93): with a directory set, fin_advance / fin_solve append a line after
 * every accepted step, as FinSolveRK.cpp:362 (FinSolveMD.cpp:284,
 * FinSolveLxW.cpp:229) calls ConSoln: "%24.16e " for t and for each total
 * dx*dy*sum q (magnitudes below 1e-99 printed as 0), then a newline; the
 * file is truncated when t == 0.  The totals are summed on the device with
 * compensation (the reference sums in order), so they agree with the
 * reference's to its rounding error.  NULL switches it off.
 * fin_write_conservation appends the line of the current state now
 * (RunFinpack.cpp:89 at t = 0). */
int fin_set_conservation_file(fin_solver* s, const char* outdir);
int fin_write_conservation(fin_solver* s);
/* qhelp.dat (void WriteQhelp(), lib/2d/WriteQhelp.cpp:20-43) under outdir. */
int fin_write_qhelp(const fin_params* p, const char* outdir);

/* Device time of the last fin_solve/fin_advance/fin_step_fixed call in
 * milliseconds (CUDA events on the solver's stream around the whole call). */
int fin_last_kernel_ms(fin_solver* s, double* ms);

/* With timing on, every stage-kernel launch is bracketed by CUDA events and
 * its duration accumulated; fin_kernel_time returns the sum and the count
 * since fin_set_kernel_timing was last called. */
int fin_set_kernel_timing(fin_solver* s, int on);
int fin_kernel_time(fin_solver* s, double* ms, long long* launches);
/* The same for the hybrid form's indicator launches. */
int fin_indicator_time(fin_solver* s, double* ms, long long* launches);

/* Measured FMA throughput of the current device in TFLOP/s (FMA = 2 flops),
 * FP64 (fp64 != 0) or FP32: the denominators of pipe-utilisation figures. */
int fin_fma_peak(int fp64, double* tflops);

/* Counts of kernel launches issued by this solver since creation. */
int fin_launch_count(fin_solver* s, long long* launches);

/* ---- device-resident interface ---------------------------------------- */
/* The device keeps each component as its own plane of mx*my values,
 * j (y) fastest then i (x): plane m starts at m*plane_stride elements. */
int fin_device_layout(fin_solver* s, size_t* plane_stride, size_t* row_stride);
/* Device pointer to the solver's current state planes (FP64). */
int fin_state_device_ptr(fin_solver* s, double** q_dev);

/* ---- troubled-cell indicator network ---------------------------------- */
/* No counterpart in the reference (its WENO weights are the labels the
 * network learns, lib/WenoReconstruct.cpp:131-134 against :104).  A
 * 20 -> 32 -> 32 -> 1 GELU network with BF16 weights and activations and FP32
 * accumulation, run and trained on tcgen05 tensor cores.  Parameters (FP32,
 * fin_mlp_nparam() values): W1[32][20], b1[32], W2[32][32], b2[32], w3[32], b3. */
typedef struct fin_mlp fin_mlp;
int fin_mlp_nparam(void);
const char* fin_mlp_last_error(void);
/* params == NULL: He-uniform initialisation from seed. */
int fin_mlp_create(const float* params, unsigned long long seed, fin_mlp** out);
int fin_mlp_destroy(fin_mlp* m);
int fin_mlp_get_params(fin_mlp* m, float* out);
int fin_mlp_set_params(fin_mlp* m, const float* in);
int fin_mlp_device_params(fin_mlp* m, const float** P);
/* Logits z[n] of the n x 20 feature rows X (host arrays). */
int fin_mlp_forward(fin_mlp* m, const float* X_host, long long n, float* z_host);
/* Gradient of the weighted binary cross-entropy (mean over the n rows; label
 * rows weigh pos_weight when y = 1) with respect to the parameters. */
int fin_mlp_gradients(fin_mlp* m, const float* X_host, const unsigned char* y_host, long long n, float pos_weight,
                      float* grad_host, float* loss);
/* Adam training: epochs over the n rows in shuffled batches; epoch_loss
 * (may be NULL) receives the mean loss of each epoch. */
int fin_mlp_train(fin_mlp* m, const float* X_host, const unsigned char* y_host, long long n, int epochs, int batch,
                  float lr, float pos_weight, unsigned long long seed, float* epoch_loss);

/* ---- hybrid form (precision FIN_PREC_HYBRID) --------------------------- */
/* Network parameters (fin_mlp_nparam() floats) for the solver's troubled-face
 * indicator; faces whose logit exceeds z_threshold (and their 3 x 3
 * same-direction neighbours) take full WENO, all others the linear FD5
 * weights.  Every judge_every-th step is recomputed with full WENO from the
 * same state; a relative L-infinity difference above judge_tol reverts the
 * step to the full result and switches the indicator off for judge_every
 * steps (judge_every = 0: no judge).  Without this call the hybrid form runs
 * full WENO in FP32. */
int fin_set_indicator(fin_solver* s, const float* params, float z_threshold, int judge_every, double judge_tol);
/* The indicator's period: it runs on q^n of every `every`-th accepted step
 * (default 1) and its flags serve the steps in between; the 3 x 3 dilation of
 * the flags covers the one face a feature can travel at CFL <= 0.5 per step
 * over two steps.  FIN_ERR_ARG for every < 1. */
int fin_set_indicator_every(fin_solver* s, int every);
/* Troubled faces flagged in the last indicator pass, faces per pass, judge
 * steps run and steps reverted. */
int fin_hybrid_stats(fin_solver* s, long long* troubled_faces, long long* faces, long long* judges, long long* reverts);
/* The troubled-face bit masks of the last indicator pass (no reference
 * counterpart): x faces (rows 0..mx, ceil(my/32) words per row, bit b of word
 * k = column 32k+b), then y faces (rows 0..mx-1, ceil((my+1)/32) words per
 * row); nwords must be at least that total. */
int fin_hybrid_flags(fin_solver* s, unsigned* words_host, size_t nwords);
/* Training samples of the current state: features (20 floats) and labels of
 * faces offset, offset + stride, ... (x faces, then y faces), at most max_n. */
int fin_face_samples(fin_solver* s, long long offset, long long stride, long long max_n, float* X_host,
                     unsigned char* y_host, long long* n_out);

/* ---- batches of independent problems ---------------------------------- */
/* No single counterpart in the reference (an application would run
 * FinSolveRK, lib/2d/FinSolveRK.cpp:13, once per problem).  A batch holds
 * nprob independent 2D Euler problems of any grid sizes (params[k]: grid,
 * domain, boundaries, CFL numbers and nv per problem; precision (FP64, FP32
 * or hybrid), WENO version, power, epsilon, gamma, alpha_scaling and
 * global_alpha shared; SSP-RK3) and advances all of them to one end time,
 * each with its own adaptive dt: per problem the arithmetic and the step
 * control are fin_solve's (in the hybrid form also the indicator's period,
 * the judge step and the revert), so the results agree with separate runs to
 * rounding; the stages of all problems run as one launch each, from a work
 * queue of tiles.  States are passed in the reference's ghosted layout of
 * each problem, as fin_set_state. */
typedef struct fin_batch fin_batch;
int fin_batch_create(const fin_params* params, int nprob, fin_batch** out);
int fin_batch_destroy(fin_batch* b);
int fin_batch_set_state(fin_batch* b, int k, const double* q_host, double t);
int fin_batch_get_state(fin_batch* b, int k, double* q_host, double* t);
/* dtv1[k]: problem k's dt on entry and on exit (dtv[1] of RunFinpack.cpp:62);
 * steps[k] (may be NULL): its accepted steps.  Fails with the first failing
 * problem's code (FIN_ERR_NSTEPS, FIN_ERR_DT_BOUNDS, FIN_ERR_CFL_BOUNDS,
 * FIN_ERR_NONFINITE). */
int fin_batch_solve(fin_batch* b, double tend, double* dtv1, int* steps);
/* Device time of the last solve, graph replays (each one step of every
 * active problem), the tile shape the autotuner chose (0: 15x16, 1: 7x32)
 * and its stage-1 times for both (tune_ms[2]). */
int fin_batch_stats(fin_batch* b, double* device_ms, long long* replays, int* tile_cfg, double* tune_ms);
/* Hybrid form (a batch created with precision FIN_PREC_HYBRID): as
 * fin_set_indicator / fin_set_indicator_every, for every problem of the
 * batch.  Until fin_batch_set_indicator the batch runs the plain FP32 form;
 * after it the tile shape is the hybrid kernels' 15x16. */
int fin_batch_set_indicator(fin_batch* b, const float* params, float z_threshold, int judge_every, double judge_tol);
int fin_batch_set_indicator_every(fin_batch* b, int every);
/* Troubled faces the indicator flagged and faces it ran on (summed over
 * its runs), judge steps and reverts, summed over the problems. */
int fin_batch_hybrid_stats(fin_batch* b, long long* troubled_faces, long long* faces, long long* judges,
                           long long* reverts);
/* Kernel timing: with on != 0 the solves launch each step on its own with
 * CUDA events between the launch groups (no graph), and accumulate the
 * device time of each group since the call: ms[5] = control (prep, work
 * queues, control), indicator, hybrid stages, plain stages, judge
 * difference. */
int fin_batch_set_kernel_timing(fin_batch* b, int on);
int fin_batch_kernel_times(fin_batch* b, double* ms);
const char* fin_batch_last_error(void);

/* ---- for callers that cannot allocate device memory ------------------- */
/* No counterpart in the reference.  For callers that must not call
 * cudaMalloc (an application whose own allocator owns the device, or a loop
 * that may not allocate once running): ConstructL, as fin_construct_l, but on
 * device pointers in the reference's ghosted layout (q_dev read, L_dev's
 * interior written, its ghosts untouched), enqueued on `stream` (a
 * cudaStream_t; NULL = default stream) and returning without waiting.  All
 * scratch lives in a static device array of this library (about 21 MB,
 * held on every GPU that loads it until exit): no allocation of any kind.
 *   - FP64 plain form only; mx*my must not exceed 262144 cells, larger
 *     grids return FIN_ERR_SIZE.
 *   - The first call on each device looks up the array's device address and
 *     sets the kernels' shared-memory limit; make that first call before any
 *     stream capture.
 *   - Calls share the one array: calls that overlap on the GPU (other
 *     streams, other threads) race; serialise them.
 *   - check == 0: the call returns once its kernels are enqueued, and a
 *     non-finite wave speed or state goes unreported.  check != 0: the call
 *     waits for `stream` and returns FIN_ERR_NONFINITE when the stage met a
 *     non-finite speed (what fin_construct_l reports).
 *   - An error already pending from the caller's own CUDA work is left in
 *     place and the call returns FIN_ERR_CUDA without launching anything.
 *   - Errors are reported by the return code only (fin_last_error does not
 *     describe them). */
int fin_construct_l_noalloc(const fin_params* p, const double* q_dev, double* L_dev, void* stream, int check);

/* ---- ideal MHD (physics FIN_PHYS_MHD) ---------------------------------- */
/* The reference's apps/2d/mhd application path: lib/2d's ConstructL with the
 * MHD callbacks (apps/2d/mhd/lib/FluxFunc.cpp, SetWaveSpd.cpp,
 * ProjectLeftEig.cpp, ProjectRightEig.cpp), the potential A3 advanced by the
 * Hamilton-Jacobi step (ConstructHJ_L.cpp:29-113), constrained transport
 * (AfterStep.cpp:13-60) and the application's FinSolveRK (SSP-RK3,
 * FinSolveRK.cpp:17-395) with its CFL number (GetCFL.cpp:31-73); doubly
 * periodic boundaries (apps/2d/mhd/orszag_tang/SetBndValues.cpp).
 * fin_params: physics FIN_PHYS_MHD, meqn 8, maux 1, mbc >= 5, time_order 3,
 * precision FIN_PREC_FP64, FIN_PREC_FP32 or FIN_PREC_HYBRID.  q arrays are the ghosted
 * (mx, my, 8) layout above, aux arrays the ghosted (mx, my, 1) layout.
 * Errors: fin_mhd_last_error(). */
typedef struct fin_mhd fin_mhd;
const char* fin_mhd_last_error(void);
int fin_mhd_create(const fin_params* p, fin_mhd** out);
int fin_mhd_destroy(fin_mhd* s);
/* State (interior read; ghosts come from the periodic remap) and its time. */
int fin_mhd_set_state(fin_mhd* s, const double* q_host, const double* aux_host, double t);
/* aux_host may be NULL; ghosts are written with the periodic images. */
int fin_mhd_get_state(fin_mhd* s, double* q_host, double* aux_host, double* t);
/* ConstructL (lib/2d/ConstructL.cpp:13-408 with the MHD callbacks) on a host
 * state: L interior written, ghosts untouched; smax_host optional, ghosted
 * (mx+1, my+1, 2), max-accumulated. */
int fin_mhd_construct_l(fin_mhd* s, const double* q_host, const double* aux_host, double* L_host,
                        double* smax_host);
/* ConstructHJ_L_Order1 (ConstructHJ_L.cpp:29-113): Laux interior written. */
int fin_mhd_construct_hj_l(fin_mhd* s, const double* q_host, const double* aux_host, double* Laux_host);
/* AfterStep (AfterStep.cpp:13-60): B1, B2 of q_host rebuilt from aux_host. */
int fin_mhd_after_step(fin_mhd* s, double* q_host, const double* aux_host);
/* FinSolveRK of the MHD application from the state's t to tend; dtv as
 * fin_solve's.  fin_mhd_advance stops after max_steps accepted steps. */
int fin_mhd_solve(fin_mhd* s, double tend, double* dtv, int* nsteps_out);
int fin_mhd_advance(fin_mhd* s, double tend, double* dtv, int max_steps, int* nsteps_out);
/* One step of exactly dt with no CFL control; cfl_out receives GetCFL's value. */
int fin_mhd_step_fixed(fin_mhd* s, double dt, double* cfl_out);
/* max over interior cells of |D_x B1 + D_y B2|, D the 4th-order central
 * difference of the constrained transport (zero to rounding when B is the
 * transport's curl of A3). */
int fin_mhd_div_b(fin_mhd* s, double* max_div);
/* Device time of the last solve/advance/step_fixed call (ms); stage-kernel
 * times when timing is on; launches since creation; the device state (9
 * planes: q then A3) and its plane stride. */
int fin_mhd_last_kernel_ms(fin_mhd* s, double* ms);
int fin_mhd_set_kernel_timing(fin_mhd* s, int on);
int fin_mhd_kernel_time(fin_mhd* s, double* ms, long long* launches);
int fin_mhd_launch_count(fin_mhd* s, long long* launches);
int fin_mhd_device_state(fin_mhd* s, double** q_dev, size_t* plane_stride);
/* Hybrid form (precision FIN_PREC_HYBRID): the troubled-face network
 * (fin_mlp_nparam() floats; trained on MHD labels: the WENO5-JS weights of
 * any of the eight characteristic fields departing from the linear weights
 * by more than 10 %), its logit threshold, and the judge step (every
 * judge_every-th hybrid step is recomputed with full WENO from the same
 * state; a relative L-infinity difference above judge_tol takes the full
 * result and switches the indicator off for judge_every steps).  Faces with a
 * troubled flag in their 3 x 3 same-direction window take the full
 * characteristic WENO flux, all others the linear FD5 weights.  Without this
 * call the hybrid form runs full WENO in FP32. */
int fin_mhd_set_indicator(fin_mhd* s, const float* params, float z_threshold, int judge_every, double judge_tol);
int fin_mhd_set_indicator_every(fin_mhd* s, int every);
int fin_mhd_hybrid_stats(fin_mhd* s, long long* troubled_faces, long long* faces, long long* judges,
                         long long* reverts);
int fin_mhd_indicator_time(fin_mhd* s, double* ms, long long* launches);
/* Training samples of the current state: 20 features and a label per face
 * for faces offset, offset + stride, ... (x faces, then y faces), at most max_n. */
int fin_mhd_face_samples(fin_mhd* s, long long offset, long long stride, long long max_n, float* X_host,
                         unsigned char* y_host, long long* n_out);

#ifdef __cplusplus
}
#endif

#endif /* FINESS_B200_H */
