// Both GetCFL overloads of lib/2d/GetCFL.cpp (declared lib/2d/misc2d.h:7-8),
// over fin_get_cfl and fin_get_cfl_alpha.  Out-of-bounds dt or CFL numbers
// print the reference's messages and exit(1), as GetCFL.cpp:43-48,61-66 do.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include "fin_shim.h"

namespace {

double finish(int rc, double dt, double cfl)
{
    if (rc == FIN_ERR_DT_BOUNDS) {
        std::cout << std::endl << " Error: dt is out of bounds ... " << std::endl;
        std::cout << "     dt = " << dt << std::endl << std::endl;
        exit(1);
    }
    if (rc == FIN_ERR_CFL_BOUNDS) {
        std::cout << std::endl << " Error: CFL number is out of bounds ... " << std::endl;
        std::cout << "     CFL = " << cfl << std::endl << std::endl;
        exit(1);
    }
    fin_shim_check(rc, "GetCFL");
    return cfl;
}

}  // namespace

double GetCFL(double dt, double dtmax, const dTensorBC3& aux, const dTensorBC3& smax)
{
    (void)aux;
    fin_solver* s = fin_shim_solver();
    std::vector<double> sm;
    fin_shim_pack(smax, sm);
    double cfl = 0.0;
    const int rc = fin_get_cfl(s, dt, dtmax, sm.data(), &cfl);
    return finish(rc, dt, cfl);
}

double GetCFL(double dt, double dtmax, double alpha1, double alpha2)
{
    fin_params p;
    fin_shim_params(&p);
    double cfl = 0.0;
    const int rc = fin_get_cfl_alpha(&p, dt, dtmax, alpha1, alpha2, &cfl);
    return finish(rc, dt, cfl);
}
