"""Python front end of libfinb200.so (the C ABI in include/finess_b200.h).

The product is the CUDA library; this module loads it with ctypes and mirrors
the reference's entry points with the same names and argument meaning:

* ``ConstructL(q)``      -> lib/2d/ConstructL.cpp:13 (returns L and smax)
* ``GlobalWaveSpd(q)``   -> lib/2d/GlobalWaveSpd.cpp:20
* ``FinSolveRK(tend, dtv)`` -> lib/2d/FinSolveRK.cpp:13 (advances the device state)

Arrays are numpy float64 in the reference's ghosted (i, j, m) layout.  There
is no CPU fallback: if the library or a B200 is missing, construction raises.
"""
import ctypes as C
import os

import numpy as np

from ._abi import FIN_OK, FinParams, ghosted_shape, smax_shape

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libfinb200.so")
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_lib = None


class FinError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"finess_b200 error {code}: {msg}")
        self.code = code


def load_library(path=LIB_PATH):
    """Load libfinb200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with __graft_entry__.build()")
    lib = C.CDLL(path)
    P = C.POINTER(FinParams)
    vp = C.c_void_p
    lib.fin_params_default.argtypes = [P]
    lib.fin_last_error.restype = C.c_char_p
    lib.fin_abi_version.restype = C.c_int
    lib.fin_create.argtypes = [P, C.POINTER(vp)]
    lib.fin_destroy.argtypes = [vp]
    lib.fin_set_state.argtypes = [vp, _dp, C.c_double]
    lib.fin_get_state.argtypes = [vp, _dp, C.POINTER(C.c_double)]
    lib.fin_construct_l.argtypes = [vp, _dp, _dp, C.c_void_p]
    lib.fin_global_wave_spd.argtypes = [vp, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.fin_solve.argtypes = [vp, C.c_double, _dp, C.POINTER(C.c_int)]
    lib.fin_step_fixed.argtypes = [vp, C.c_double, C.POINTER(C.c_double)]
    lib.fin_conservation_totals.argtypes = [vp, _dp]
    lib.fin_last_kernel_ms.argtypes = [vp, C.POINTER(C.c_double)]
    lib.fin_launch_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    lib.fin_device_layout.argtypes = [vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    lib.fin_state_device_ptr.argtypes = [vp, C.POINTER(C.c_void_p)]
    lib.fin_advance.argtypes = [vp, C.c_double, _dp, C.c_int, C.POINTER(C.c_int)]
    lib.fin_set_kernel_timing.argtypes = [vp, C.c_int]
    lib.fin_kernel_time.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
    lib.fin_indicator_time.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
    lib.fin_indicator_time.restype = C.c_int
    lib.fin_fma_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    lib.fin_set_indicator.argtypes = [vp, np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"), C.c_float,
                                      C.c_int, C.c_double]
    lib.fin_set_indicator.restype = C.c_int
    lib.fin_set_indicator_every.argtypes = [vp, C.c_int]
    lib.fin_set_indicator_every.restype = C.c_int
    lib.fin_hybrid_stats.argtypes = [vp] + [C.POINTER(C.c_longlong)] * 4
    lib.fin_hybrid_stats.restype = C.c_int
    lib.fin_face_samples.argtypes = [vp, C.c_longlong, C.c_longlong, C.c_longlong,
                                     np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"),
                                     np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS"), C.POINTER(C.c_longlong)]
    lib.fin_face_samples.restype = C.c_int
    lib.fin_construct_integrated_r.argtypes = [vp, C.c_double, _dp, _dp, _dp]
    lib.fin_construct_integrated_r.restype = C.c_int
    lib.fin_params_from_ini.argtypes = [C.c_char_p, P]
    lib.fin_params_from_ini.restype = C.c_int
    lib.fin_ini_last_error.restype = C.c_char_p
    lib.fin_output_frame.argtypes = [vp, C.c_int, C.c_char_p]
    lib.fin_output_wait.argtypes = [vp]
    lib.fin_read_frame.argtypes = [vp, C.c_char_p]
    lib.fin_set_conservation_file.argtypes = [vp, C.c_char_p]
    lib.fin_write_conservation.argtypes = [vp]
    lib.fin_write_qhelp.argtypes = [P, C.c_char_p]
    lib.fin_set_state_qinit.argtypes = [vp, C.c_int, C.c_void_p, C.c_int, C.c_double]
    lib.fin_set_state_qinit.restype = C.c_int
    for name in ("fin_output_frame", "fin_output_wait", "fin_read_frame", "fin_set_conservation_file",
                 "fin_write_conservation", "fin_write_qhelp"):
        getattr(lib, name).restype = C.c_int
    for name in ("fin_create", "fin_destroy", "fin_set_state", "fin_get_state", "fin_construct_l",
                 "fin_global_wave_spd", "fin_solve", "fin_step_fixed", "fin_conservation_totals",
                 "fin_last_kernel_ms", "fin_launch_count", "fin_device_layout", "fin_state_device_ptr",
                 "fin_advance", "fin_set_kernel_timing", "fin_kernel_time", "fin_fma_peak"):
        getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def write_qhelp(p, outdir):
    """qhelp.dat of the parameters under outdir."""
    lib = load_library()
    _check(lib.fin_write_qhelp(C.byref(p), os.fsencode(outdir)))


def params_from_ini(path):
    """parameters.ini -> FinParams through the library's reader."""
    lib = load_library()
    p = FinParams()
    rc = lib.fin_params_from_ini(os.fsencode(path), C.byref(p))
    if rc != FIN_OK:
        raise FinError(rc, lib.fin_ini_last_error().decode())
    return p


def fma_peak_tflops(fp64=True):
    lib = load_library()
    v = C.c_double()
    _check(lib.fin_fma_peak(1 if fp64 else 0, C.byref(v)))
    return v.value


def _check(rc):
    if rc != FIN_OK:
        raise FinError(rc, _lib.fin_last_error().decode())


class Solver:
    """One problem resident on the current CUDA device."""

    def __init__(self, params: FinParams):
        self.lib = load_library()
        self.p = params.copy()
        h = C.c_void_p()
        _check(self.lib.fin_create(C.byref(self.p), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.fin_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state -------------------------------------------------------------
    def set_state(self, q, t=0.0):
        q = np.ascontiguousarray(q, dtype=np.float64)
        assert q.shape == ghosted_shape(self.p), (q.shape, ghosted_shape(self.p))
        _check(self.lib.fin_set_state(self.h, q, t))

    def set_state_qinit(self, problem, prm=(), t=0.0):
        """Initial data sampled on the device (SampleFunction with a built-in
        QinitFunc functor; problem = FIN_QINIT_*, prm its parameters)."""
        a = np.ascontiguousarray(prm, dtype=np.float64)
        _check(self.lib.fin_set_state_qinit(self.h, int(problem), a.ctypes.data_as(C.c_void_p) if a.size else None,
                                            int(a.size), t))

    def get_state(self, out=None):
        """(q, t): the state in the reference's ghosted layout, into `out`
        (a C-contiguous float64 array of that shape, e.g. in pinned host
        memory) when given."""
        if out is not None:
            assert out.shape == ghosted_shape(self.p) and out.dtype == np.float64 and out.flags["C_CONTIGUOUS"]
            q = out
        else:
            q = np.zeros(ghosted_shape(self.p))
        t = C.c_double()
        _check(self.lib.fin_get_state(self.h, q, C.byref(t)))
        return q, t.value

    # -- reference entry points -------------------------------------------
    def ConstructL(self, q, smax=None):
        q = np.ascontiguousarray(q, dtype=np.float64)
        L = np.zeros(ghosted_shape(self.p))
        sm = np.zeros(smax_shape(self.p)) if smax is None else np.ascontiguousarray(smax, dtype=np.float64).copy()
        _check(self.lib.fin_construct_l(self.h, q, L, sm.ctypes.data_as(C.c_void_p)))
        return L, sm

    def GlobalWaveSpd(self, q):
        a1, a2 = C.c_double(), C.c_double()
        _check(self.lib.fin_global_wave_spd(self.h, np.ascontiguousarray(q, dtype=np.float64), C.byref(a1),
                                            C.byref(a2)))
        return a1.value, a2.value

    def FinSolveRK(self, tend, dtv):
        """Advance the device state to tend; dtv = [_, dt, max_dt] is updated in place."""
        dtv = np.ascontiguousarray(dtv, dtype=np.float64)
        n = C.c_int()
        _check(self.lib.fin_solve(self.h, tend, dtv, C.byref(n)))
        return dtv, n.value

    # FinSolveMD (lib/2d/FinSolveMD.cpp:21) and FinSolveLxW (FinSolveLxW.cpp:16)
    # run through the same driver; the solver's time_stepping_method picks the steps.
    FinSolveMD = FinSolveRK
    FinSolveLxW = FinSolveRK

    def ConstructIntegratedR(self, dt, q):
        """1-state ConstructIntegratedR; returns ghosted F, G (interior + 3 ghost layers set)."""
        F = np.zeros(ghosted_shape(self.p))
        G = np.zeros(ghosted_shape(self.p))
        _check(self.lib.fin_construct_integrated_r(self.h, dt, np.ascontiguousarray(q, dtype=np.float64), F, G))
        return F, G

    def set_indicator(self, params, z_threshold=0.0, judge_every=20, judge_tol=1e-3, every=1):
        """Hybrid form: the troubled-face network's parameters, the judge step,
        and the indicator's period in accepted steps."""
        _check(self.lib.fin_set_indicator(self.h, np.ascontiguousarray(params, dtype=np.float32), z_threshold,
                                          judge_every, judge_tol))
        _check(self.lib.fin_set_indicator_every(self.h, every))

    def hybrid_stats(self):
        v = [C.c_longlong() for _ in range(4)]
        _check(self.lib.fin_hybrid_stats(self.h, *[C.byref(x) for x in v]))
        return {"troubled_faces": v[0].value, "faces": v[1].value, "judges": v[2].value, "reverts": v[3].value}

    def hybrid_flags(self):
        """Troubled-face flags of the last indicator pass, one bool per face:
        x faces (mx+1) x my (i-major), then y faces mx x (my+1)."""
        p = self.p
        wx, wy = (p.my + 31) >> 5, (p.my + 32) >> 5
        n = (p.mx + 1) * wx + p.mx * wy
        w = np.zeros(n, dtype=np.uint32)
        self.lib.fin_hybrid_flags.argtypes = [C.c_void_p, np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS"),
                                              C.c_size_t]
        self.lib.fin_hybrid_flags.restype = C.c_int
        _check(self.lib.fin_hybrid_flags(self.h, w, n))
        bits = np.unpackbits(w.view(np.uint8), bitorder="little")
        fx = bits[:(p.mx + 1) * wx * 32].reshape(p.mx + 1, wx * 32)[:, :p.my]
        fy = bits[(p.mx + 1) * wx * 32:].reshape(p.mx, wy * 32)[:, :p.my + 1]
        return np.concatenate([fx.ravel(), fy.ravel()]).astype(bool)

    def face_samples(self, offset=0, stride=1, max_n=None):
        """Indicator features (n x 20) and WENO-JS labels of the current state's faces."""
        p = self.p
        nf = (p.mx + 1) * p.my + p.mx * (p.my + 1)
        n = (nf - offset + stride - 1) // stride
        if max_n is not None:
            n = min(n, max_n)
        X = np.zeros((n, 20), dtype=np.float32)
        y = np.zeros(n, dtype=np.uint8)
        nout = C.c_longlong()
        _check(self.lib.fin_face_samples(self.h, offset, stride, n, X, y, C.byref(nout)))
        return X[:nout.value], y[:nout.value]

    def advance(self, tend, dtv, max_steps):
        """FinSolveRK stopping after max_steps accepted steps; returns (dtv, nsteps)."""
        dtv = np.ascontiguousarray(dtv, dtype=np.float64)
        n = C.c_int()
        _check(self.lib.fin_advance(self.h, tend, dtv, max_steps, C.byref(n)))
        return dtv, n.value

    def set_kernel_timing(self, on=True):
        _check(self.lib.fin_set_kernel_timing(self.h, 1 if on else 0))

    def kernel_time(self):
        ms, n = C.c_double(), C.c_longlong()
        _check(self.lib.fin_kernel_time(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def indicator_time(self):
        ms, n = C.c_double(), C.c_longlong()
        _check(self.lib.fin_indicator_time(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def step_fixed(self, dt):
        cfl = C.c_double()
        _check(self.lib.fin_step_fixed(self.h, dt, C.byref(cfl)))
        return cfl.value

    # -- output files (lib/2d/Output.cpp, ConSoln.cpp, WriteQhelp.cpp) -----
    def output_frame(self, nframe, outdir):
        """Starts writing q%04d.dat / a%04d.dat of the current state under
        outdir (asynchronous; output_wait() returns when they are on disk)."""
        _check(self.lib.fin_output_frame(self.h, nframe, os.fsencode(outdir)))

    def output_wait(self):
        _check(self.lib.fin_output_wait(self.h))

    def read_frame(self, path):
        """Restart from a q%04d.dat file: its values become the state, its header t."""
        _check(self.lib.fin_read_frame(self.h, os.fsencode(path)))

    def set_conservation_file(self, outdir):
        """conservation.dat under outdir, a line per accepted step (None: off)."""
        _check(self.lib.fin_set_conservation_file(self.h, None if outdir is None else os.fsencode(outdir)))

    def write_conservation(self):
        _check(self.lib.fin_write_conservation(self.h))

    def conservation_totals(self):
        out = np.zeros(self.p.meqn)
        _check(self.lib.fin_conservation_totals(self.h, out))
        return out

    def last_kernel_ms(self):
        ms = C.c_double()
        _check(self.lib.fin_last_kernel_ms(self.h, C.byref(ms)))
        return ms.value

    def launch_count(self):
        n = C.c_longlong()
        _check(self.lib.fin_launch_count(self.h, C.byref(n)))
        return n.value
