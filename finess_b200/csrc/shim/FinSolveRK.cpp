// void FinSolveRK(StateVars& Qnew, double tend, double dtv[])
// (lib/2d/RunFinpack.h:18, lib/2d/FinSolveRK.cpp:13) over fin_solve.
#include "fin_shim.h"

void FinSolveRK(StateVars& Qnew, double tend, double dtv[]) { fin_shim_finsolve(Qnew, tend, dtv, "FinSolveRK"); }
