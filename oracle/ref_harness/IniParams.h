// Parameter accessor for building the reference's hot-path sources as a test
// oracle.  TEST INFRASTRUCTURE ONLY: nothing in the product links this.
//
// The reference generates its IniParams class from Python specs
// (python/finess/params/params.py:358-497; specs in finess.py, weno.py,
// dim2.py, euler.py, mhd.py).  That generator is Python-2 only, so the
// harness supplies this hand-written class instead.  It exposes the same
// accessor names and the same WenoVersion enumerators the library sources
// call (lib/WenoReconstruct.cpp:44-64), with values set by the harness's
// extern "C" setup function rather than by parsing parameters.ini.
#ifndef FIN_REF_HARNESS_INIPARAMS_H
#define FIN_REF_HARNESS_INIPARAMS_H

#include <string>

class IniParams {
public:
    struct WenoVersion { enum enum_type { FD, JS, Z, DEFAULT }; };
    struct TimeSteppingMethod { enum enum_type { RK, SDC, LxW, MD, USER_DEFINED, DEFAULT }; };

    // [finess]
    int ndims = 2, nout = 1, nv = 500000, space_order = 5, time_order = 3;
    int verbosity = 0, mcapa = 0, maux = 1, meqn = 5;
    bool source_term = false, global_alpha = true, mpp_limiter = false;
    double tfinal = 1.0, initial_dt = 1e-3, max_dt = 1e10, max_cfl = 0.45, desired_cfl = 0.4;
    TimeSteppingMethod::enum_type time_stepping_method = TimeSteppingMethod::RK;
    std::string output_dir = "output";
    // [grid]
    int mx = 10, my = 10, mbc = 3;
    double xlow = 0, xhigh = 1, ylow = 0, yhigh = 1;
    // [weno]
    WenoVersion::enum_type weno_version = WenoVersion::JS;
    double power_param = 2.0, alpha_scaling = 1.1, epsilon = 1e-6;
    // [euler] / [mhd]
    double gamma = 1.4;
    bool constrained_transport = true;
    // [initial] of apps/2d/euler/riemann_test (its this_app_params.py): the
    // shock tube's direction
    int OPT = 1;

    int get_ndims() const { return ndims; }
    int get_nout() const { return nout; }
    int get_nv() const { return nv; }
    int get_space_order() const { return space_order; }
    int get_time_order() const { return time_order; }
    int get_verbosity() const { return verbosity; }
    int get_mcapa() const { return mcapa; }
    int get_maux() const { return maux; }
    int get_meqn() const { return meqn; }
    bool get_source_term() const { return source_term; }
    bool get_global_alpha() const { return global_alpha; }
    bool get_mpp_limiter() const { return mpp_limiter; }
    double get_tfinal() const { return tfinal; }
    double get_initial_dt() const { return initial_dt; }
    double get_max_dt() const { return max_dt; }
    double get_max_cfl() const { return max_cfl; }
    double get_desired_cfl() const { return desired_cfl; }
    TimeSteppingMethod::enum_type get_time_stepping_method() const { return time_stepping_method; }
    std::string get_output_dir() const { return output_dir; }
    int get_mx() const { return mx; }
    int get_my() const { return my; }
    int get_mbc() const { return mbc; }
    double get_xlow() const { return xlow; }
    double get_xhigh() const { return xhigh; }
    double get_ylow() const { return ylow; }
    double get_yhigh() const { return yhigh; }
    // Derived exactly as python/finess/params/dim2.py:57-66 does: (high-low)/m.
    double get_dx() const { return (xhigh - xlow) / mx; }
    double get_dy() const { return (yhigh - ylow) / my; }
    WenoVersion::enum_type get_weno_version() const { return weno_version; }
    double get_power_param() const { return power_param; }
    double get_alpha_scaling() const { return alpha_scaling; }
    double get_epsilon() const { return epsilon; }
    double get_gamma() const { return gamma; }
    bool get_constrained_transport() const { return constrained_transport; }
    int get_OPT() const { return OPT; }
};

extern IniParams global_ini_params;

#endif
