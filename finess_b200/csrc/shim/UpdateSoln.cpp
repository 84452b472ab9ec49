// Both UpdateSoln overloads of lib/2d/UpdateSoln.cpp (declared
// lib/2d/FinSolveRK.h:21-29), over fin_update_soln and fin_update_soln5.
// One object file holds both, as the reference's does, so an application
// that names UpdateSoln.o in its Makefile replaces both.
#include "fin_shim.h"

// orders 1-4: qnew = alpha1 qstar + alpha2 qnew + beta dt L (UpdateSoln.cpp:14-38)
void UpdateSoln(double alpha1, double alpha2, double beta, double dt, const StateVars& Qstar,
                const dTensorBC3& Lstar, StateVars& Qnew)
{
    fin_solver* s = fin_shim_solver();
    std::vector<double> qs, L, qn;
    fin_shim_pack(Qstar.const_ref_q(), qs);
    fin_shim_pack(Lstar, L);
    fin_shim_pack(Qnew.const_ref_q(), qn);
    double t = Qnew.get_t();
    fin_shim_check(fin_update_soln(s, alpha1, alpha2, beta, dt, qs.data(), Qstar.get_t(), L.data(), qn.data(), &t),
                   "UpdateSoln");
    fin_shim_unpack_all(qn, Qnew.ref_q());
    Qnew.set_t(t);
}

// the fifth-order stepper's form (UpdateSoln.cpp:43-80)
void UpdateSoln(double g1, double g2, double g3, double delta, double beta, double dt, const StateVars& Qold,
                const dTensorBC3& Lstar, StateVars& Q1, StateVars& Q2)
{
    fin_solver* s = fin_shim_solver();
    std::vector<double> qo, L, q1, q2;
    fin_shim_pack(Qold.const_ref_q(), qo);
    fin_shim_pack(Lstar, L);
    fin_shim_pack(Q1.const_ref_q(), q1);
    fin_shim_pack(Q2.const_ref_q(), q2);
    fin_shim_check(fin_update_soln5(s, g1, g2, g3, delta, beta, dt, qo.data(), L.data(), q1.data(), q2.data()),
                   "UpdateSoln");
    fin_shim_unpack_all(q1, Q1.ref_q());
    fin_shim_unpack_all(q2, Q2.ref_q());
}
