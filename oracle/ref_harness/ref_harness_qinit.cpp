// The reference's own SampleFunction (lib/2d/SampleFunction.cpp:62-125) with
// one of its applications' QinitFunc (apps/2d/euler/riemann_test or
// test_exact2, compiled by oracle/Makefile into its own library), through a
// small extern "C" API.  TEST INFRASTRUCTURE ONLY: the checker of the
// device's initial-data sampling.
#include <algorithm>
#include "IniParams.h"
#include "tensors.h"
#include "finess_b200.h"

IniParams global_ini_params;

void QinitFunc(const dTensor2& xpts, dTensor2& qvals);   // the application's (app_defined.h:7)
void SampleFunction(int istart, int iend, int jstart, int jend, const dTensorBC3& qin, const dTensorBC3& auxin,
                    dTensorBC3& Fout, void (*Func)(const dTensor2&, const dTensor2&, const dTensor2&, dTensor2&));

// The four-argument form SampleFunction calls, as lib/2d/RunFinpack.cpp:144-149 wraps it.
static void qinit_wrapper(const dTensor2& xpts, const dTensor2&, const dTensor2&, dTensor2& qvals)
{
    QinitFunc(xpts, qvals);
}

extern "C" {

// RunFinpack.cpp:72-80: a zeroed state of the ghosted grid, sampled over
// i = 1-mbc .. mx+mbc, j = 1-mbc .. my+mbc into the ghosted array q.
int ref_qinit(const fin_params* p, int opt, double* q)
{
    IniParams& g = global_ini_params;
    g.meqn = p->meqn; g.maux = 0;
    g.mx = p->mx; g.my = p->my; g.mbc = p->mbc;
    g.xlow = p->xlow; g.xhigh = p->xhigh; g.ylow = p->ylow; g.yhigh = p->yhigh;
    g.gamma = p->gamma;
    g.OPT = opt;
    dTensorBC3 qn(g.mx, g.my, g.meqn, g.mbc), aux(g.mx, g.my, 1, g.mbc);
    qn.setall(0.);
    aux.setall(0.);
    SampleFunction(1 - g.mbc, g.mx + g.mbc, 1 - g.mbc, g.my + g.mbc, qn, aux, qn, &qinit_wrapper);
    const int n = qn.numel();
    for (int k = 0; k < n; k++) q[k] = qn.vget(k);
    return 0;
}

}  // extern "C"
