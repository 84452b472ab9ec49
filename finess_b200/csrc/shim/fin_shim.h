// Relink shim: the reference's own C++ entry points (ConstructL,
// GlobalWaveSpd, FinSolveRK, FinSolveMD, FinSolveLxW, UpdateSoln, GetCFL,
// ConstructIntegratedR, ConstructLxWL) implemented over the C ABI of
// libfinb200.so, one object per reference object file, so
// an unmodified FINESS application relinks against this library by naming
// these objects in its Makefile (lib/2d/Makefile.defs:79-109 lists the names
// an application may override).  Compiled inside the application's build,
// against the reference's headers (StateVars.h, tensors.h) and the
// application's generated IniParams.h.
#ifndef FIN_SHIM_H
#define FIN_SHIM_H

#include <vector>
#include "StateVars.h"
#include "finess_b200.h"

// The solver for the application's grid, created on first use from
// global_ini_params; boundary conditions are read off the application's own
// SetBndValues (see fin_shim_common.cpp).
fin_solver* fin_shim_solver();

// The fin_params fields held by global_ini_params, and the boundary
// conditions read off the application's SetBndValues.
void fin_shim_params(fin_params* out);
void fin_shim_probe_bc(int mx, int my, int mbc, int meqn, int maux, int* bc);

// dTensorBC3 <-> contiguous ghosted buffer in the same (i, j, m) order.
void fin_shim_pack(const dTensorBC3& t, std::vector<double>& buf);
void fin_shim_unpack_interior(const std::vector<double>& buf, dTensorBC3& t);
void fin_shim_unpack_all(const std::vector<double>& buf, dTensorBC3& t);

// Reference-style failure: print and exit(1), as lib/2d/GetCFL.cpp:43-48 and
// FinSolveRK.cpp:84-92 do.
void fin_shim_check(int rc, const char* where);

// One FinSolveRK / FinSolveMD / FinSolveLxW call on the device; the solver's
// stepper is the one global_ini_params names.
void fin_shim_finsolve(StateVars& Qnew, double tend, double dtv[], const char* name);

#endif
