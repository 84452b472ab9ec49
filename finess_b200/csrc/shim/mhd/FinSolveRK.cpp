// void FinSolveRK(StateVars& Qnew, double tend, double dtv[]) of the ideal-MHD
// application (apps/2d/mhd/lib/FinSolveRK.cpp:17, named in
// apps/2d/mhd/lib/Makefile.defs:37) over fin_mhd_solve: q and the potential
// A3 (aux) go to the device once per call, every step (the three stages with
// ConstructHJ_L, UpdateSolnWithAux and AfterStep's constrained transport)
// runs there, and the frame comes back with its ghost cells filled by the
// periodic remap.  The device applies boundaries as an index remap, so the
// application's SetBndValues must be doubly periodic (checked on first use);
// the per-stage hooks and the per-step ConSoln file are not called.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "IniParams.h"
#include "fin_shim.h"

namespace {

fin_mhd* g_mhd = nullptr;
fin_params g_mkey;

void check(int rc, const char* where)
{
    if (rc == FIN_OK) return;
    printf(" Error in %s: %s (finess_b200 status %d)\n", where, fin_mhd_last_error(), rc);
    exit(1);
}

fin_mhd* mhd_solver()
{
    fin_params p;
    fin_shim_params(&p);
    p.physics = FIN_PHYS_MHD;
    p.constrained_transport = global_ini_params.get_constrained_transport() ? 1 : 0;
    if (g_mhd && memcmp(&p, &g_mkey, sizeof(p)) == 0) return g_mhd;
    g_mkey = p;
    int bc[4];
    fin_shim_probe_bc(p.mx, p.my, p.mbc, p.meqn, p.maux, bc);
    for (int k = 0; k < 4; k++)
        if (bc[k] != FIN_BC_PERIODIC) {
            printf(" Error: the MHD path remaps doubly periodic boundaries only (SetBndValues side %d)\n", k);
            exit(1);
        }
    if (g_mhd) fin_mhd_destroy(g_mhd);
    g_mhd = nullptr;
    check(fin_mhd_create(&p, &g_mhd), "fin_mhd_create");
    return g_mhd;
}

}  // namespace

void FinSolveRK(StateVars& Qnew, double tend, double dtv[])
{
    fin_mhd* m = mhd_solver();
    std::vector<double> q, aux;
    fin_shim_pack(Qnew.const_ref_q(), q);
    fin_shim_pack(Qnew.const_ref_aux(), aux);
    check(fin_mhd_set_state(m, q.data(), aux.data(), Qnew.get_t()), "FinSolveRK");
    int nsteps = 0;
    check(fin_mhd_solve(m, tend, dtv, &nsteps), "FinSolveRK");
    double t = 0.0;
    check(fin_mhd_get_state(m, q.data(), aux.data(), &t), "FinSolveRK");
    fin_shim_unpack_all(q, Qnew.ref_q());
    fin_shim_unpack_all(aux, Qnew.ref_aux());
    Qnew.set_t(t);
}
