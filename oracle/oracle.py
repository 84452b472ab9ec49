"""ctypes front end of the two CPU checkers.  TEST INFRASTRUCTURE ONLY.

* ``Oracle``: oracle/liboracle.so, the plain-C restatement of the reference's
  hot path (finess_oracle.c).
* ``RefLib``: oracle/_ref/libfinref.so, the reference's own sources
  (lib/2d/ConstructL.cpp, lib/WenoReconstruct.cpp, lib/2d/FinSolveRK.cpp, ...)
  compiled in place by oracle/Makefile with the harness in ref_harness/.
* ``MhdRefLib``: oracle/_ref/libfinref_mhd.so, the same for the ideal-MHD
  path (lib/2d/ConstructL.cpp with apps/2d/mhd/lib and the Orszag-Tang case).
  The MHD arrays are q (mx+2mbc, my+2mbc, 8) and aux (mx+2mbc, my+2mbc, 1).
* ``IoRefLib``: oracle/_ref/libfinref_io.so, the reference's output routines
  (lib/2d/Output.cpp, WriteQhelp.cpp, ConSoln.cpp) writing their files.
* ``RefQinit``: oracle/_ref/libfinref_qinit_<app>.so, the reference's
  SampleFunction with an application's own QinitFunc.

All take and return numpy arrays in the reference's ghosted dTensorBC3 layout
(lib/tensors.h:267-273), shape (mx+2mbc, my+2mbc, meqn).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from finess_b200._abi import FinParams, aux_shape, ghosted_shape, smax_shape  # noqa: E402

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfinref.so")
# the same reference objects relinked against libfinb200.so through the shim
REF_SHIM_SO = os.path.join(HERE, "_ref", "libfinref_shim.so")
# the reference's own steppers with their building blocks relinked against libfinb200.so
REF_SHIM_PARTS_SO = os.path.join(HERE, "_ref", "libfinref_shim_parts.so")
REF_MHD_SO = os.path.join(HERE, "_ref", "libfinref_mhd.so")
# the MHD application's objects relinked against libfinb200.so (its FinSolveRK replaced)
REF_MHD_SHIM_SO = os.path.join(HERE, "_ref", "libfinref_mhd_shim.so")


def build_oracle():
    """Compile liboracle.so (seconds, gcc only) if it is missing or stale."""
    srcs = [os.path.join(HERE, f) for f in ("finess_oracle.c", "mhd_oracle.c", "finess_oracle.h")]
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < max(os.path.getmtime(f) for f in srcs):
        subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)


class Oracle:
    def __init__(self):
        build_oracle()
        lib = C.CDLL(ORACLE_SO)
        P = C.POINTER(FinParams)
        lib.oracle_set_bnd.argtypes = [P, _dp]
        lib.oracle_global_wave_spd.argtypes = [P, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.oracle_construct_l.argtypes = [P, _dp, _dp, _dp]
        lib.oracle_construct_l.restype = C.c_int
        lib.oracle_construct_lxwl.argtypes = [P, _dp, _dp, _dp, _dp, _dp]
        lib.oracle_construct_lxwl.restype = C.c_int
        lib.oracle_construct_integrated_r.argtypes = [P, C.c_double, _dp, _dp, _dp]
        lib.oracle_construct_integrated_r.restype = C.c_int
        lib.oracle_weno5.argtypes = [C.c_int, C.c_double, C.c_double, _dp]
        lib.oracle_weno5.restype = C.c_double
        lib.oracle_weno_js5_weights.argtypes = [C.c_double, C.c_double, _dp, _dp]
        lib.oracle_finsolve.argtypes = [P, _dp, C.POINTER(C.c_double), C.c_double, _dp, C.POINTER(C.c_int)]
        lib.oracle_finsolve.restype = C.c_int
        lib.oracle_step_fixed.argtypes = [P, _dp, C.c_double, C.POINTER(C.c_double)]
        lib.oracle_step_fixed.restype = C.c_int
        lib.oracle_conservation_totals.argtypes = [P, _dp, _dp]
        lib.oracle_face_samples.argtypes = [P, _dp, _dp, np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")]
        lib.oracle_mhd_set_bnd.argtypes = [P, _dp, _dp]
        lib.oracle_mhd_global_wave_spd.argtypes = [P, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.oracle_mhd_construct_l.argtypes = [P, _dp, _dp, _dp]
        lib.oracle_mhd_construct_l.restype = C.c_int
        lib.oracle_mhd_construct_hj_l.argtypes = [P, _dp, _dp, _dp]
        lib.oracle_mhd_construct_hj_l.restype = C.c_int
        lib.oracle_mhd_after_step.argtypes = [P, _dp, _dp]
        lib.oracle_mhd_step_fixed.argtypes = [P, _dp, _dp, C.c_double, C.POINTER(C.c_double)]
        lib.oracle_mhd_step_fixed.restype = C.c_int
        lib.oracle_mhd_finsolve.argtypes = [P, _dp, _dp, C.POINTER(C.c_double), C.c_double, _dp,
                                            C.POINTER(C.c_int)]
        lib.oracle_mhd_finsolve.restype = C.c_int
        lib.oracle_orszag_tang.argtypes = [P, _dp, _dp]
        lib.oracle_mhd_face_samples.argtypes = [P, _dp, _dp, np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")]
        self.lib = lib

    def set_bnd(self, p, q):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        self.lib.oracle_set_bnd(C.byref(p), q)
        return q

    def global_wave_spd(self, p, q):
        a1, a2 = C.c_double(), C.c_double()
        self.lib.oracle_global_wave_spd(C.byref(p), np.ascontiguousarray(q), C.byref(a1), C.byref(a2))
        return a1.value, a2.value

    def construct_l(self, p, q, smax=None):
        L = np.zeros(ghosted_shape(p))
        sm = np.zeros(smax_shape(p)) if smax is None else np.ascontiguousarray(smax).copy()
        rc = self.lib.oracle_construct_l(C.byref(p), np.ascontiguousarray(q), L, sm)
        if rc:
            raise ValueError(f"oracle_construct_l failed: {rc}")
        return L, sm

    def construct_integrated_r(self, p, dt, q):
        F = np.zeros(ghosted_shape(p))
        G = np.zeros(ghosted_shape(p))
        rc = self.lib.oracle_construct_integrated_r(C.byref(p), dt, np.ascontiguousarray(q), F, G)
        if rc:
            raise ValueError(f"oracle_construct_integrated_r failed: {rc}")
        return F, G

    def construct_lxwl(self, p, q, F, G):
        L = np.zeros(ghosted_shape(p))
        sm = np.zeros(smax_shape(p))
        rc = self.lib.oracle_construct_lxwl(C.byref(p), np.ascontiguousarray(q), np.ascontiguousarray(F),
                                            np.ascontiguousarray(G), L, sm)
        if rc:
            raise ValueError(f"oracle_construct_lxwl failed: {rc}")
        return L, sm

    def weno5(self, version, eps, pw, u):
        return self.lib.oracle_weno5(version, eps, pw, np.ascontiguousarray(u, dtype=np.float64))

    def js5_weights(self, eps, pw, u):
        w = np.zeros(3)
        self.lib.oracle_weno_js5_weights(eps, pw, np.ascontiguousarray(u, dtype=np.float64), w)
        return w

    def finsolve(self, p, q, t, tend, dt):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        tt = C.c_double(t)
        dtv = np.array([0.0, dt, p.max_dt])
        n = C.c_int(0)
        rc = self.lib.oracle_finsolve(C.byref(p), q, C.byref(tt), tend, dtv, C.byref(n))
        return rc, q, tt.value, dtv[1], n.value

    def step_fixed(self, p, q, dt):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        cfl = C.c_double(0.0)
        rc = self.lib.oracle_step_fixed(C.byref(p), q, dt, C.byref(cfl))
        if rc:
            raise ValueError(f"oracle_step_fixed failed: {rc}")
        return q, cfl.value

    def face_samples(self, p, q):
        nf = (p.mx + 1) * p.my + p.mx * (p.my + 1)
        X = np.zeros((nf, 20))
        y = np.zeros(nf, dtype=np.uint8)
        self.lib.oracle_face_samples(C.byref(p), np.ascontiguousarray(q), X, y)
        return X, y

    def conservation_totals(self, p, q):
        out = np.zeros(p.meqn)
        self.lib.oracle_conservation_totals(C.byref(p), np.ascontiguousarray(q), out)
        return out

    # ---- ideal MHD (mhd_oracle.c) ----
    def mhd_set_bnd(self, p, q, aux):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        aux = np.ascontiguousarray(aux, dtype=np.float64).copy()
        self.lib.oracle_mhd_set_bnd(C.byref(p), q, aux)
        return q, aux

    def mhd_global_wave_spd(self, p, q):
        a1, a2 = C.c_double(), C.c_double()
        self.lib.oracle_mhd_global_wave_spd(C.byref(p), np.ascontiguousarray(q), C.byref(a1), C.byref(a2))
        return a1.value, a2.value

    def mhd_construct_l(self, p, q, smax=None):
        L = np.zeros(ghosted_shape(p))
        sm = np.zeros(smax_shape(p)) if smax is None else np.ascontiguousarray(smax).copy()
        rc = self.lib.oracle_mhd_construct_l(C.byref(p), np.ascontiguousarray(q), L, sm)
        if rc:
            raise ValueError(f"oracle_mhd_construct_l failed: {rc}")
        return L, sm

    def mhd_construct_hj_l(self, p, q, aux):
        La = np.zeros(aux_shape(p))
        rc = self.lib.oracle_mhd_construct_hj_l(C.byref(p), np.ascontiguousarray(q), np.ascontiguousarray(aux), La)
        if rc:
            raise ValueError(f"oracle_mhd_construct_hj_l failed: {rc}")
        return La

    def mhd_after_step(self, p, q, aux):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        self.lib.oracle_mhd_after_step(C.byref(p), q, np.ascontiguousarray(aux))
        return q

    def mhd_step_fixed(self, p, q, aux, dt):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        aux = np.ascontiguousarray(aux, dtype=np.float64).copy()
        cfl = C.c_double(0.0)
        rc = self.lib.oracle_mhd_step_fixed(C.byref(p), q, aux, dt, C.byref(cfl))
        if rc:
            raise ValueError(f"oracle_mhd_step_fixed failed: {rc}")
        return q, aux, cfl.value

    def mhd_finsolve(self, p, q, aux, t, tend, dt):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        aux = np.ascontiguousarray(aux, dtype=np.float64).copy()
        tt = C.c_double(t)
        dtv = np.array([0.0, dt, p.max_dt])
        n = C.c_int(0)
        rc = self.lib.oracle_mhd_finsolve(C.byref(p), q, aux, C.byref(tt), tend, dtv, C.byref(n))
        return rc, q, aux, tt.value, dtv[1], n.value

    def mhd_face_samples(self, p, q):
        nf = (p.mx + 1) * p.my + p.mx * (p.my + 1)
        X = np.zeros((nf, 20))
        y = np.zeros(nf, dtype=np.uint8)
        self.lib.oracle_mhd_face_samples(C.byref(p), np.ascontiguousarray(q), X, y)
        return X, y

    def orszag_tang(self, p):
        q = np.zeros(ghosted_shape(p))
        aux = np.zeros(aux_shape(p))
        self.lib.oracle_orszag_tang(C.byref(p), q, aux)
        return q, aux


class RefLib:
    """The reference's own compiled sources; available where oracle/_ref was built."""

    @staticmethod
    def available(path=REF_SO):
        return os.path.exists(path)

    def __init__(self, path=REF_SO):
        lib = C.CDLL(path)
        P = C.POINTER(FinParams)
        lib.ref_setup.argtypes = [P]
        lib.ref_set_bnd.argtypes = [_dp]
        lib.ref_construct_l.argtypes = [_dp, _dp, _dp]
        lib.ref_construct_l.restype = C.c_int
        lib.ref_global_wave_spd.argtypes = [_dp, _dp]
        lib.ref_construct_integrated_r.argtypes = [C.c_double, _dp, _dp, _dp]
        lib.ref_finsolve.argtypes = [C.c_int, _dp, C.POINTER(C.c_double), C.c_double, _dp]
        lib.ref_finsolve.restype = C.c_int
        lib.ref_last_steps.restype = C.c_longlong
        self.lib = lib
        self.last_steps = None

    def setup(self, p):
        self.lib.ref_setup(C.byref(p))

    def set_bnd(self, p, q):
        self.setup(p)
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        self.lib.ref_set_bnd(q)
        return q

    def global_wave_spd(self, p, q):
        self.setup(p)
        out = np.zeros(2)
        self.lib.ref_global_wave_spd(np.ascontiguousarray(q), out)
        return out[0], out[1]

    def construct_l(self, p, q, smax=None):
        self.setup(p)
        L = np.zeros(ghosted_shape(p))
        sm = np.zeros(smax_shape(p)) if smax is None else np.ascontiguousarray(smax).copy()
        rc = self.lib.ref_construct_l(np.ascontiguousarray(q), L, sm)
        if rc:
            raise ValueError(f"ref_construct_l failed: {rc}")
        return L, sm

    def construct_integrated_r(self, p, dt, q):
        self.setup(p)
        F = np.zeros(ghosted_shape(p))
        G = np.zeros(ghosted_shape(p))
        self.lib.ref_construct_integrated_r(dt, np.ascontiguousarray(q), F, G)
        return F, G

    def finsolve(self, p, q, t, tend, dt):
        self.setup(p)
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        tt = C.c_double(t)
        dtv = np.array([0.0, dt, p.max_dt])
        rc = self.lib.ref_finsolve(p.time_stepping_method, q, C.byref(tt), tend, dtv)
        self.last_steps = int(self.lib.ref_last_steps())   # accepted steps of this run
        return rc, q, tt.value, dtv[1]


class MhdRefLib:
    """The reference's own ideal-MHD sources; available where oracle/_ref was built."""

    @staticmethod
    def available(path=REF_MHD_SO):
        return os.path.exists(path)

    def __init__(self, path=REF_MHD_SO):
        lib = C.CDLL(path)
        lib.ref_mhd_setup.argtypes = [C.POINTER(FinParams)]
        lib.ref_mhd_qinit.argtypes = [_dp, _dp]
        lib.ref_mhd_set_bnd.argtypes = [_dp, _dp]
        lib.ref_mhd_construct_l.argtypes = [_dp, _dp, _dp, _dp]
        lib.ref_mhd_construct_l.restype = C.c_int
        lib.ref_mhd_global_wave_spd.argtypes = [_dp, _dp, _dp]
        lib.ref_mhd_construct_hj_l.argtypes = [_dp, _dp, _dp]
        lib.ref_mhd_after_step.argtypes = [_dp, _dp]
        lib.ref_mhd_finsolve.argtypes = [_dp, _dp, C.POINTER(C.c_double), C.c_double, _dp]
        lib.ref_mhd_finsolve.restype = C.c_int
        self.lib = lib

    def setup(self, p):
        self.lib.ref_mhd_setup(C.byref(p))

    def qinit(self, p):
        self.setup(p)
        q = np.zeros(ghosted_shape(p))
        aux = np.zeros(aux_shape(p))
        self.lib.ref_mhd_qinit(q, aux)
        return q, aux

    def set_bnd(self, p, q, aux):
        self.setup(p)
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        aux = np.ascontiguousarray(aux, dtype=np.float64).copy()
        self.lib.ref_mhd_set_bnd(q, aux)
        return q, aux

    def global_wave_spd(self, p, q, aux):
        self.setup(p)
        out = np.zeros(2)
        self.lib.ref_mhd_global_wave_spd(np.ascontiguousarray(q), np.ascontiguousarray(aux), out)
        return out[0], out[1]

    def construct_l(self, p, q, aux, smax=None):
        self.setup(p)
        L = np.zeros(ghosted_shape(p))
        sm = np.zeros(smax_shape(p)) if smax is None else np.ascontiguousarray(smax).copy()
        rc = self.lib.ref_mhd_construct_l(np.ascontiguousarray(q), np.ascontiguousarray(aux), L, sm)
        if rc:
            raise ValueError(f"ref_mhd_construct_l failed: {rc}")
        return L, sm

    def construct_hj_l(self, p, q, aux):
        self.setup(p)
        La = np.zeros(aux_shape(p))
        self.lib.ref_mhd_construct_hj_l(np.ascontiguousarray(q), np.ascontiguousarray(aux), La)
        return La

    def after_step(self, p, q, aux):
        self.setup(p)
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        self.lib.ref_mhd_after_step(q, np.ascontiguousarray(aux))
        return q

    def finsolve(self, p, q, aux, t, tend, dt):
        self.setup(p)
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        aux = np.ascontiguousarray(aux, dtype=np.float64).copy()
        tt = C.c_double(t)
        dtv = np.array([0.0, dt, p.max_dt])
        rc = self.lib.ref_mhd_finsolve(q, aux, C.byref(tt), tend, dtv)
        return rc, q, aux, tt.value, dtv[1]


class RefQinit:
    """The reference's SampleFunction with one application's own QinitFunc
    (app "riemann_test" or "test_exact2"); available where oracle/_ref was
    built.  sample(p, opt) returns the ghosted (mx+2mbc, my+2mbc, 5) array
    RunFinpack.cpp:80 fills (ghosts sampled too)."""

    @staticmethod
    def path(app):
        return os.path.join(HERE, "_ref", f"libfinref_qinit_{app}.so")

    @staticmethod
    def available(app):
        return os.path.exists(RefQinit.path(app))

    def __init__(self, app):
        lib = C.CDLL(RefQinit.path(app))
        lib.ref_qinit.argtypes = [C.POINTER(FinParams), C.c_int, _dp]
        lib.ref_qinit.restype = C.c_int
        self.lib = lib

    def sample(self, p, opt=1):
        q = np.zeros(ghosted_shape(p))
        rc = self.lib.ref_qinit(C.byref(p), opt, q)
        if rc:
            raise ValueError(f"ref_qinit failed: {rc}")
        return q


REF_IO_SO = os.path.join(HERE, "_ref", "libfinref_io.so")


class IoRefLib:
    """The reference's own output routines (lib/2d/Output.cpp, WriteQhelp.cpp,
    ConSoln.cpp); available where oracle/_ref was built."""

    @staticmethod
    def available(path=REF_IO_SO):
        return os.path.exists(path)

    def __init__(self, path=REF_IO_SO):
        lib = C.CDLL(path)
        lib.ref_io_setup.argtypes = [C.POINTER(FinParams), C.c_char_p]
        lib.ref_io_output.argtypes = [_dp, _dp, C.c_double, C.c_int]
        lib.ref_io_consoln.argtypes = [_dp, _dp, C.c_double]
        self.lib = lib

    def _aux(self, p, aux):
        if aux is None:
            return np.zeros((p.mx + 2 * p.mbc, p.my + 2 * p.mbc, max(p.maux, 1)))
        return np.ascontiguousarray(aux, dtype=np.float64)

    def output(self, p, outdir, q, t, nframe, aux=None):
        self.lib.ref_io_setup(C.byref(p), os.fsencode(outdir))
        self.lib.ref_io_output(np.ascontiguousarray(q, dtype=np.float64), self._aux(p, aux), t, nframe)

    def qhelp(self, p, outdir):
        self.lib.ref_io_setup(C.byref(p), os.fsencode(outdir))
        self.lib.ref_io_qhelp()

    def consoln(self, p, outdir, q, t, aux=None):
        self.lib.ref_io_setup(C.byref(p), os.fsencode(outdir))
        self.lib.ref_io_consoln(np.ascontiguousarray(q, dtype=np.float64), self._aux(p, aux), t)
