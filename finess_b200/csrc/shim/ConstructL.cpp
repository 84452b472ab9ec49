// void ConstructL(StateVars&, dTensorBC3& Lstar, dTensorBC3& smax)
// (lib/2d/FinSolveRK.h:18, lib/2d/ConstructL.cpp:13) over fin_construct_l.
#include "fin_shim.h"

void ConstructL(StateVars& Q, dTensorBC3& Lstar, dTensorBC3& smax)
{
    fin_solver* s = fin_shim_solver();
    std::vector<double> q, L, sm;
    fin_shim_pack(Q.const_ref_q(), q);
    fin_shim_pack(Lstar, L);
    fin_shim_pack(smax, sm);
    fin_shim_check(fin_construct_l(s, q.data(), L.data(), sm.data()), "ConstructL");
    fin_shim_unpack_interior(L, Lstar);
    fin_shim_unpack_all(sm, smax);
}
