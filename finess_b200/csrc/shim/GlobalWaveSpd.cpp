// void GlobalWaveSpd(const StateVars&, double&, double&)
// (lib/2d/ConstructL.h:26, lib/2d/GlobalWaveSpd.cpp:20) over fin_global_wave_spd.
#include "fin_shim.h"

void GlobalWaveSpd(const StateVars& Q, double& alpha1, double& alpha2)
{
    fin_solver* s = fin_shim_solver();
    std::vector<double> q;
    fin_shim_pack(Q.const_ref_q(), q);
    fin_shim_check(fin_global_wave_spd(s, q.data(), &alpha1, &alpha2), "GlobalWaveSpd");
}
