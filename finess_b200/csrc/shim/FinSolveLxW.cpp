// void FinSolveLxW(StateVars& Qnew, double tend, double dtv[])
// (lib/2d/RunFinpack.h:19, lib/2d/FinSolveLxW.cpp:16) over fin_solve: the
// Lax-Wendroff step (FinSolveLxW.cpp:120-176), with the MPP limiter when
// the application's parameters switch it on (:126-158).
#include "fin_shim.h"

void FinSolveLxW(StateVars& Qnew, double tend, double dtv[]) { fin_shim_finsolve(Qnew, tend, dtv, "FinSolveLxW"); }
