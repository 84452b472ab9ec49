// void FinSolveMD(StateVars& Qnew, double tend, double dtv[])
// (lib/2d/RunFinpack.h:20, lib/2d/FinSolveMD.cpp:21) over fin_solve: the
// two-stage multiderivative steps (time_order 4, FinSolveMD.cpp:116-170) or
// the fifth-order ones (:172-226) on the device.
#include "fin_shim.h"

void FinSolveMD(StateVars& Qnew, double tend, double dtv[]) { fin_shim_finsolve(Qnew, tend, dtv, "FinSolveMD"); }
