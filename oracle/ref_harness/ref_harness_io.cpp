// Harness that links the reference's own, unmodified output routines
// (lib/2d/Output.cpp, lib/2d/WriteQhelp.cpp, lib/2d/ConSoln.cpp) into
// oracle/_ref/libfinref_io.so and drives them through a small extern "C"
// API, so the files this library writes from device state can be compared
// byte for byte with the reference's.  TEST INFRASTRUCTURE ONLY.
#include <string>
#include "IniParams.h"
#include "tensors.h"
#include "StateVars.h"
#include "finess_b200.h"

IniParams global_ini_params;

void Output(const StateVars& Q, int nframe);
void WriteQhelp();
void ConSoln(const StateVars& Q);

static void load(dTensorBC3& t, const double* src)
{
    const int n = t.numel();
    for (int k = 0; k < n; k++) t.vset(k, src[k]);
}

extern "C" {

// The parameters the three routines read, and the output directory.
int ref_io_setup(const fin_params* p, const char* outdir)
{
    IniParams& g = global_ini_params;
    g.ndims = 2;
    g.meqn = p->meqn;
    g.maux = p->maux;
    g.nout = p->nout;
    g.mcapa = 0;
    g.mx = p->mx;
    g.my = p->my;
    g.mbc = p->mbc;
    g.xlow = p->xlow;
    g.xhigh = p->xhigh;
    g.ylow = p->ylow;
    g.yhigh = p->yhigh;
    g.output_dir = outdir;
    return 0;
}

// q, aux: the reference's ghosted layout ((mx+2mbc) x (my+2mbc) x meqn / maux).
int ref_io_output(const double* q, const double* aux, double t, int nframe)
{
    const IniParams& g = global_ini_params;
    StateVars Q(t, g.mx, g.my, g.meqn, g.maux, g.mbc);
    load(Q.ref_q(), q);
    if (g.maux > 0) load(Q.ref_aux(), aux);
    Output(Q, nframe);
    return 0;
}

int ref_io_qhelp(void)
{
    WriteQhelp();
    return 0;
}

int ref_io_consoln(const double* q, const double* aux, double t)
{
    const IniParams& g = global_ini_params;
    StateVars Q(t, g.mx, g.my, g.meqn, g.maux, g.mbc);
    load(Q.ref_q(), q);
    if (g.maux > 0) load(Q.ref_aux(), aux);
    ConSoln(Q);
    return 0;
}

}  // extern "C"
