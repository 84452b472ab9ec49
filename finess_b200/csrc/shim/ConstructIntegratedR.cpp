// The three ConstructIntegratedR overloads of lib/2d/ConstructIntegratedR.cpp
// (declared lib/2d/constructs.h:16-31) over fin_construct_integrated_r,
// fin_construct_integrated_r2 and fin_construct_integrated_r3.  F and G get
// the interior and the 3-cell ghost frame the reference computes
// (ConstructIntegratedR.cpp:97-98: i, j from 1-3 to m+3); smax is not
// written (the reference does not write it either).
#include "fin_shim.h"

void ConstructIntegratedR(double dt, const StateVars& Q, dTensorBC3& smax, dTensorBC3& F, dTensorBC3& G)
{
    (void)smax;
    fin_solver* s = fin_shim_solver();
    std::vector<double> q, f, g;
    fin_shim_pack(Q.const_ref_q(), q);
    fin_shim_pack(F, f);
    fin_shim_pack(G, g);
    fin_shim_check(fin_construct_integrated_r(s, dt, q.data(), f.data(), g.data()), "ConstructIntegratedR");
    fin_shim_unpack_all(f, F);
    fin_shim_unpack_all(g, G);
}

void ConstructIntegratedR(double dt, double alpha1, double beta1, const StateVars& Q1, double alpha2, double beta2,
                          const StateVars& Q2, dTensorBC3& smax, dTensorBC3& F, dTensorBC3& G)
{
    (void)smax;
    fin_solver* s = fin_shim_solver();
    std::vector<double> q1, q2, f, g;
    fin_shim_pack(Q1.const_ref_q(), q1);
    fin_shim_pack(Q2.const_ref_q(), q2);
    fin_shim_pack(F, f);
    fin_shim_pack(G, g);
    fin_shim_check(fin_construct_integrated_r2(s, dt, alpha1, beta1, q1.data(), alpha2, beta2, q2.data(), f.data(),
                                               g.data()),
                   "ConstructIntegratedR");
    fin_shim_unpack_all(f, F);
    fin_shim_unpack_all(g, G);
}

void ConstructIntegratedR(double dt, double alpha1, double beta1, double charlie1, const StateVars& Q1,
                          double alpha2, double beta2, double charlie2, const StateVars& Q2, dTensorBC3& smax,
                          dTensorBC3& F, dTensorBC3& G)
{
    (void)smax;
    fin_solver* s = fin_shim_solver();
    std::vector<double> q1, q2, f, g;
    fin_shim_pack(Q1.const_ref_q(), q1);
    fin_shim_pack(Q2.const_ref_q(), q2);
    fin_shim_pack(F, f);
    fin_shim_pack(G, g);
    fin_shim_check(fin_construct_integrated_r3(s, dt, alpha1, beta1, charlie1, q1.data(), alpha2, beta2, charlie2,
                                               q2.data(), f.data(), g.data()),
                   "ConstructIntegratedR");
    fin_shim_unpack_all(f, F);
    fin_shim_unpack_all(g, G);
}
