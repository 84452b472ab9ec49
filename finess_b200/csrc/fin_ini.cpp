// parameters.ini reader: the same file an unmodified FINESS application
// ships.  Keys, defaults, enumerations and checks follow the reference's
// parameter specs (python/finess/params/finess.py, dim2.py, weno.py,
// euler.py, mhd.py), which its build turns into the IniParams class
// (python/finess/params/params.py:358-497) read by lib/sys/IniParser.h.
// Booleans parse as true/false like stringToAny<bool> (lib/sys/util.h:9).
//
// This library adds one optional section, [finess_b200]:
//   bc_xlow, bc_xhigh, bc_ylow, bc_yhigh = periodic | transmissive
//   precision = fp64 | fp32 | hybrid
// (boundary conditions are application code in the reference; here they are
// an index remap applied on load).
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include "finess_b200.h"

namespace {

thread_local std::string g_ini_err;

std::string trim(const std::string& s)
{
    size_t a = 0, b = s.size();
    while (a < b && isspace((unsigned char)s[a])) a++;
    while (b > a && isspace((unsigned char)s[b - 1])) b--;
    return s.substr(a, b - a);
}

std::string lower(std::string s)
{
    for (auto& c : s) c = (char)tolower((unsigned char)c);
    return s;
}

struct Ini {
    std::map<std::string, std::string> kv;   // "section.key" -> value
    bool has(const std::string& k) const { return kv.count(k) != 0; }
    const std::string& get(const std::string& k) const { return kv.at(k); }
};

bool parse_int(const std::string& s, int* out)
{
    char* end = nullptr;
    long v = strtol(s.c_str(), &end, 10);
    if (end == s.c_str() || *end != '\0') return false;
    *out = (int)v;
    return true;
}

bool parse_double(const std::string& s, double* out)
{
    char* end = nullptr;
    double v = strtod(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0') return false;
    *out = v;
    return true;
}

bool parse_bool(const std::string& s, int* out)
{
    const std::string l = lower(s);
    if (l == "true" || l == "1") { *out = 1; return true; }
    if (l == "false" || l == "0") { *out = 0; return true; }
    return false;
}

int fail(const std::string& msg)
{
    g_ini_err = msg;
    return FIN_ERR_ARG;
}

}  // namespace

extern "C" const char* fin_ini_last_error(void) { return g_ini_err.c_str(); }

extern "C" int fin_params_from_ini(const char* path, fin_params* p)
{
    if (!path || !p) return fail("null argument");
    std::ifstream f(path);
    if (!f) return fail(std::string("cannot open ") + path);
    Ini ini;
    std::string line, section;
    int lineno = 0;
    while (std::getline(f, line)) {
        lineno++;
        const size_t c = line.find_first_of(";#");
        if (c != std::string::npos) line = line.substr(0, c);
        line = trim(line);
        if (line.empty()) continue;
        if (line[0] == '[') {
            const size_t e = line.find(']');
            if (e == std::string::npos) return fail("line " + std::to_string(lineno) + ": bad section header");
            section = lower(trim(line.substr(1, e - 1)));
            continue;
        }
        const size_t eq = line.find('=');
        if (eq == std::string::npos) return fail("line " + std::to_string(lineno) + ": expected key = value");
        ini.kv[section + "." + lower(trim(line.substr(0, eq)))] = trim(line.substr(eq + 1));
    }

    fin_params_default(p);
    int ndims = 2, verbosity = 0, mcapa = 0;
    double tfinal = 0.0;
    struct IntKey { const char* k; int* dst; bool required; };
    struct DblKey { const char* k; double* dst; bool required; };
    const IntKey ints[] = {
        {"finess.ndims", &ndims, true}, {"finess.nout", &p->nout, false}, {"finess.nv", &p->nv, true},
        {"finess.space_order", &p->space_order, true}, {"finess.time_order", &p->time_order, true},
        {"finess.verbosity", &verbosity, true}, {"finess.mcapa", &mcapa, true}, {"finess.maux", &p->maux, true},
        {"finess.meqn", &p->meqn, true},
        {"grid.mx", &p->mx, true}, {"grid.my", &p->my, true}, {"grid.mbc", &p->mbc, true},
    };
    const DblKey dbls[] = {
        {"finess.tfinal", &tfinal, true}, {"finess.initial_dt", &p->initial_dt, true},
        {"finess.max_dt", &p->max_dt, true}, {"finess.max_cfl", &p->max_cfl, true},
        {"finess.desired_cfl", &p->desired_cfl, true},
        {"grid.xlow", &p->xlow, true}, {"grid.xhigh", &p->xhigh, true},
        {"grid.ylow", &p->ylow, true}, {"grid.yhigh", &p->yhigh, true},
        {"weno.power_param", &p->power_param, false}, {"weno.alpha_scaling", &p->alpha_scaling, false},
        {"weno.epsilon", &p->epsilon, false}, {"euler.gamma", &p->gamma, false},
        {"mhd.gamma", &p->gamma, false},
    };
    for (const auto& k : ints) {
        if (!ini.has(k.k)) {
            if (k.required) return fail(std::string("missing parameter ") + k.k);
            continue;
        }
        if (!parse_int(ini.get(k.k), k.dst)) return fail(std::string("not an integer: ") + k.k);
    }
    for (const auto& k : dbls) {
        if (!ini.has(k.k)) {
            if (k.required) return fail(std::string("missing parameter ") + k.k);
            continue;
        }
        if (!parse_double(ini.get(k.k), k.dst)) return fail(std::string("not a number: ") + k.k);
    }
    p->tfinal = tfinal;
    p->verbosity = verbosity;
    if (!ini.has("finess.source_term")) return fail("missing parameter finess.source_term");
    if (!parse_bool(ini.get("finess.source_term"), &p->source_term)) return fail("not a bool: finess.source_term");
    if (ini.has("finess.global_alpha") && !parse_bool(ini.get("finess.global_alpha"), &p->global_alpha))
        return fail("not a bool: finess.global_alpha");
    int mpp = 0;
    if (ini.has("finess.mpp_limiter") && !parse_bool(ini.get("finess.mpp_limiter"), &mpp))
        return fail("not a bool: finess.mpp_limiter");
    if (!ini.has("finess.time_stepping_method")) return fail("missing parameter finess.time_stepping_method");
    {
        const std::string m = ini.get("finess.time_stepping_method");
        if (m == "Runge-Kutta") p->time_stepping_method = FIN_TS_RK;
        else if (m == "Lax-Wendroff") p->time_stepping_method = FIN_TS_LXW;
        else if (m == "Multiderivative") p->time_stepping_method = FIN_TS_MD;
        else if (m == "SDC" || m == "User-Defined") return fail("time_stepping_method " + m + " is not built here");
        else return fail("unknown time_stepping_method " + m);
    }
    // [mhd] (python/finess/params/mhd.py): its presence selects the MHD callbacks
    if (ini.has("mhd.gamma")) {
        p->physics = FIN_PHYS_MHD;
        if (ini.has("mhd.constrained_transport") &&
            !parse_bool(ini.get("mhd.constrained_transport"), &p->constrained_transport))
            return fail("not a bool: mhd.constrained_transport");
    }
    if (ini.has("weno.weno_version")) {
        const std::string v = ini.get("weno.weno_version");
        if (v == "JS") p->weno_version = FIN_WENO_JS;
        else if (v == "Z") p->weno_version = FIN_WENO_Z;
        else if (v == "FD") p->weno_version = FIN_WENO_FD;
        else return fail("unknown weno_version " + v);
    }
    const char* bck[4] = {"finess_b200.bc_xlow", "finess_b200.bc_xhigh", "finess_b200.bc_ylow", "finess_b200.bc_yhigh"};
    int* bcd[4] = {&p->bc_xlow, &p->bc_xhigh, &p->bc_ylow, &p->bc_yhigh};
    for (int k = 0; k < 4; k++) {
        if (!ini.has(bck[k])) continue;
        const std::string v = lower(ini.get(bck[k]));
        if (v == "periodic") *bcd[k] = FIN_BC_PERIODIC;
        else if (v == "transmissive") *bcd[k] = FIN_BC_TRANSMISSIVE;
        else return fail(std::string("unknown boundary condition for ") + bck[k]);
    }
    if (ini.has("finess_b200.precision")) {
        const std::string v = lower(ini.get("finess_b200.precision"));
        if (v == "fp64") p->precision = FIN_PREC_FP64;
        else if (v == "fp32") p->precision = FIN_PREC_FP32;
        else if (v == "hybrid") p->precision = FIN_PREC_HYBRID;
        else return fail("unknown precision " + v);
    }

    // Checks of finess.py, dim2.py and weno.py, with their messages.
    if (!(ndims == 1 || ndims == 2 || ndims == 3)) return fail("finess.ndims should be one of 1, 2, 3.");
    if (ndims != 2) return fail("finess.ndims: this library implements the 2D path");
    if (!(p->nout > 0)) return fail("finess.nout should > 0.");
    if (!(tfinal >= 0.0)) return fail("finess.tfinal should >= 0.");
    if (!(p->initial_dt > 0.0)) return fail("finess.initial_dt should > 0.");
    if (!(p->max_dt >= p->initial_dt)) return fail("finess.max_dt should >= finess.initial_dt.");
    if (!(p->desired_cfl > 0.0)) return fail("finess.desired_cfl should > 0.");
    if (!(p->max_cfl >= p->desired_cfl)) return fail("finess.max_cfl should >= finess.desired_cfl.");
    if (!(p->nv > 0)) return fail("finess.nv should > 0.");
    {
        const int so = p->space_order;
        if (!(so == 1 || so == 3 || so == 5 || so == 7 || so == 9 || so == 11))
            return fail("finess.space_order should be one of 1, 3, 5, 7, 9, 11.");
    }
    if (!(p->time_order >= 1 && p->time_order <= 5)) return fail("finess.time_order should be one of 1, 2, 3, 4, 5.");
    if (!(verbosity == 0 || verbosity == 1)) return fail("finess.verbosity should be one of 0, 1.");
    if (!(mcapa >= 0)) return fail("finess.mcapa should >= 0.");
    if (!(p->maux >= mcapa)) return fail("finess.maux should >= finess.mcapa.");
    if (!(p->meqn >= 1)) return fail("finess.meqn should >= 1.");
    if (!(p->xhigh > p->xlow)) return fail("grid.xhigh should > grid.xlow.");
    if (!(p->yhigh > p->ylow)) return fail("grid.yhigh should > grid.ylow.");
    if (!(p->alpha_scaling >= 1.0)) return fail("weno.alpha_scaling should >= 1.");
    if (!(p->epsilon > 0.0)) return fail("weno.epsilon should > 0.");
    p->mpp_limiter = mpp;
    return FIN_OK;
}
