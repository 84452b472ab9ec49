"""ctypes mirror of include/finess_b200.h (struct layout and enums)."""
import ctypes as C

FIN_OK = 0
FIN_ERR_ARG = 1
FIN_ERR_CUDA = 2
FIN_ERR_NO_DEVICE = 3
FIN_ERR_NSTEPS = 4
FIN_ERR_DT_BOUNDS = 5
FIN_ERR_CFL_BOUNDS = 6
FIN_ERR_NONFINITE = 7
FIN_ERR_UNSUPPORTED = 8
FIN_ERR_SIZE = 9

FIN_WENO_FD, FIN_WENO_JS, FIN_WENO_Z = 0, 1, 2
FIN_TS_RK, FIN_TS_LXW, FIN_TS_MD = 0, 2, 3
FIN_BC_PERIODIC, FIN_BC_TRANSMISSIVE = 0, 1
FIN_PHYS_EULER = 0
FIN_PHYS_MHD = 1
FIN_PREC_FP64, FIN_PREC_FP32, FIN_PREC_HYBRID = 0, 1, 2
# initial data sampled on the device (fin_set_state_qinit)
FIN_QINIT_VORTEX, FIN_QINIT_RIEMANN4, FIN_QINIT_SHOCK_ENTROPY, FIN_QINIT_SHOCK_TUBE, FIN_QINIT_VORTEX_EXACT2 = 1, 2, 3, 4, 5

WENO_NAMES = {"FD": FIN_WENO_FD, "JS": FIN_WENO_JS, "Z": FIN_WENO_Z}


class FinParams(C.Structure):
    _fields_ = [
        ("meqn", C.c_int), ("maux", C.c_int),
        ("space_order", C.c_int), ("time_order", C.c_int),
        ("time_stepping_method", C.c_int),
        ("global_alpha", C.c_int), ("source_term", C.c_int),
        ("nv", C.c_int), ("verbosity", C.c_int),
        ("initial_dt", C.c_double), ("max_dt", C.c_double),
        ("max_cfl", C.c_double), ("desired_cfl", C.c_double),
        ("mx", C.c_int), ("my", C.c_int), ("mbc", C.c_int),
        ("xlow", C.c_double), ("xhigh", C.c_double),
        ("ylow", C.c_double), ("yhigh", C.c_double),
        ("weno_version", C.c_int),
        ("epsilon", C.c_double), ("power_param", C.c_double), ("alpha_scaling", C.c_double),
        ("gamma", C.c_double),
        ("bc_xlow", C.c_int), ("bc_xhigh", C.c_int), ("bc_ylow", C.c_int), ("bc_yhigh", C.c_int),
        ("physics", C.c_int),
        ("precision", C.c_int),
        ("tfinal", C.c_double),
        ("nout", C.c_int),
        ("constrained_transport", C.c_int),
        ("mpp_limiter", C.c_int),
    ]

    def copy(self):
        other = FinParams()
        C.pointer(other)[0] = self
        return other

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


def default_params(**overrides):
    """Defaults of the reference's parameter specs (python/finess/params/
    finess.py, weno.py, euler.py); fields can be overridden by keyword."""
    p = FinParams()
    p.meqn, p.maux = 5, 0
    p.space_order, p.time_order = 5, 3
    p.time_stepping_method = FIN_TS_RK
    p.global_alpha, p.source_term = 0, 0
    p.nv, p.verbosity = 500000, 0
    p.initial_dt, p.max_dt, p.max_cfl, p.desired_cfl = 1e-3, 1e10, 0.45, 0.4
    p.mx, p.my, p.mbc = 10, 10, 3
    p.xlow, p.xhigh, p.ylow, p.yhigh = 0.0, 1.0, 0.0, 1.0
    p.weno_version = FIN_WENO_JS
    p.epsilon, p.power_param, p.alpha_scaling = 1e-6, 2.0, 1.1
    p.gamma = 1.4
    p.bc_xlow = p.bc_xhigh = p.bc_ylow = p.bc_yhigh = FIN_BC_PERIODIC
    p.physics = FIN_PHYS_EULER
    p.precision = FIN_PREC_FP64
    p.tfinal, p.nout = 0.0, 1
    p.mpp_limiter = 0
    p.constrained_transport = 1
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(f"fin_params has no field {k!r}")
        setattr(p, k, v)
    return p


def ghosted_shape(p):
    """numpy shape of a reference dTensorBC3(mx, my, meqn, mbc): (i, j, m)."""
    return (p.mx + 2 * p.mbc, p.my + 2 * p.mbc, p.meqn)


def aux_shape(p):
    """numpy shape of the auxiliary dTensorBC3(mx, my, maux, mbc)."""
    return (p.mx + 2 * p.mbc, p.my + 2 * p.mbc, p.maux)


def smax_shape(p):
    return (p.mx + 1 + 2 * p.mbc, p.my + 1 + 2 * p.mbc, 2)
