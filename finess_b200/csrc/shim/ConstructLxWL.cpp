// Both ConstructLxWL overloads of lib/2d/ConstructLxWL.cpp (declared
// lib/2d/constructs.h:44-51) over fin_construct_lxwl: L's interior, smax
// max-accumulated, and (second overload) the face fluxes Fhat, Ghat.
#include "fin_shim.h"

void ConstructLxWL(const StateVars& Q, const dTensorBC3& F, const dTensorBC3& G, dTensorBC3* pFhat,
                   dTensorBC3* pGhat, dTensorBC3& Lstar, dTensorBC3& smax)
{
    fin_solver* s = fin_shim_solver();
    std::vector<double> q, f, g, L, sm, fh, gh;
    fin_shim_pack(Q.const_ref_q(), q);
    fin_shim_pack(F, f);
    fin_shim_pack(G, g);
    fin_shim_pack(Lstar, L);
    fin_shim_pack(smax, sm);
    if (pFhat) fin_shim_pack(*pFhat, fh);
    if (pGhat) fin_shim_pack(*pGhat, gh);
    fin_shim_check(fin_construct_lxwl(s, q.data(), f.data(), g.data(), L.data(), sm.data(),
                                      pFhat ? fh.data() : nullptr, pGhat ? gh.data() : nullptr),
                   "ConstructLxWL");
    fin_shim_unpack_interior(L, Lstar);
    fin_shim_unpack_all(sm, smax);
    if (pFhat) fin_shim_unpack_all(fh, *pFhat);
    if (pGhat) fin_shim_unpack_all(gh, *pGhat);
}

void ConstructLxWL(const StateVars& Q, const dTensorBC3& F, const dTensorBC3& G, dTensorBC3& Lstar,
                   dTensorBC3& smax)
{
    ConstructLxWL(Q, F, G, nullptr, nullptr, Lstar, smax);
}
