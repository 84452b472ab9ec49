// void FinSolveRK(StateVars& Qnew, double tend, double dtv[])
// (lib/2d/RunFinpack.h:18, lib/2d/FinSolveRK.cpp:13) over fin_solve: the state
// goes to the device once per call (one output frame of RunFinpack.cpp:95-130),
// every step runs there, and the frame's result comes back with its ghost
// frame filled as SetBndValues would fill it.  conservation.dat gets its line
// after every accepted step (FinSolveRK.cpp:362 calls ConSoln there) from
// totals summed on the device; where the output directory does not exist the
// lines are dropped, as the reference's ofstream drops them.  The per-stage
// hooks (BeforeStep/AfterStep, hooks.h) are not called on the device path.
#include "IniParams.h"
#include "fin_shim.h"

void FinSolveRK(StateVars& Qnew, double tend, double dtv[])
{
    fin_solver* s = fin_shim_solver();
    std::vector<double> q;
    fin_shim_pack(Qnew.const_ref_q(), q);
    fin_shim_check(fin_set_state(s, q.data(), Qnew.get_t()), "FinSolveRK");
    fin_set_conservation_file(s, global_ini_params.get_output_dir().c_str());
    int nsteps = 0;
    fin_shim_check(fin_solve(s, tend, dtv, &nsteps), "FinSolveRK");
    double t = 0.0;
    fin_shim_check(fin_get_state(s, q.data(), &t), "FinSolveRK");
    fin_shim_unpack_all(q, Qnew.ref_q());
    Qnew.set_t(t);
}
