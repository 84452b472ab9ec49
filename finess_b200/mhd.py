"""Ideal MHD (fin_mhd_* of the C ABI): the reference's apps/2d/mhd path.

``MhdSolver`` mirrors the MHD application's entry points with the same names
and argument meaning:

* ``ConstructL(q, aux)``   -> lib/2d/ConstructL.cpp:13 with the MHD callbacks
* ``ConstructHJ_L(q, aux)`` -> apps/2d/mhd/lib/ConstructHJ_L.cpp:29 (Order1)
* ``AfterStep(q, aux)``    -> apps/2d/mhd/lib/AfterStep.cpp:13 (constrained transport)
* ``FinSolveRK(tend, dtv)`` -> apps/2d/mhd/lib/FinSolveRK.cpp:17

Arrays are numpy float64 in the reference's ghosted layout: q (mx+2mbc,
my+2mbc, 8), aux (mx+2mbc, my+2mbc, 1).  There is no CPU fallback.

    python -m finess_b200.mhd [--n 2048] [--tend 3.141592653589793] [--precision fp64|fp32|hybrid|both|all]

runs the Orszag-Tang vortex and prints device time, cell-updates/s, max
|div B| and the FP32 / hybrid forms' density L1/Linf error against the FP64
run when it ran too (``both``: FP64 and FP32; ``all``: FP64, FP32 and the
hybrid form with the MHD-trained network, indicator every 2 steps, judge
every 50 at 1e-3).
"""
import argparse
import ctypes as C
import json
import math

import numpy as np

from . import problems as P
from ._abi import (FIN_OK, FIN_PREC_FP32, FIN_PREC_FP64, FIN_PREC_HYBRID, FinParams, aux_shape, ghosted_shape,
                   smax_shape)
from .solver import FinError, load_library

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def _lib():
    lib = load_library()
    if not getattr(lib, "_mhd_bound", False):
        vp = C.c_void_p
        lib.fin_mhd_last_error.restype = C.c_char_p
        lib.fin_mhd_create.argtypes = [C.POINTER(FinParams), C.POINTER(vp)]
        lib.fin_mhd_destroy.argtypes = [vp]
        lib.fin_mhd_set_state.argtypes = [vp, _dp, _dp, C.c_double]
        lib.fin_mhd_get_state.argtypes = [vp, _dp, _dp, C.POINTER(C.c_double)]
        lib.fin_mhd_construct_l.argtypes = [vp, _dp, _dp, _dp, C.c_void_p]
        lib.fin_mhd_construct_hj_l.argtypes = [vp, _dp, _dp, _dp]
        lib.fin_mhd_after_step.argtypes = [vp, _dp, _dp]
        lib.fin_mhd_solve.argtypes = [vp, C.c_double, _dp, C.POINTER(C.c_int)]
        lib.fin_mhd_advance.argtypes = [vp, C.c_double, _dp, C.c_int, C.POINTER(C.c_int)]
        lib.fin_mhd_step_fixed.argtypes = [vp, C.c_double, C.POINTER(C.c_double)]
        lib.fin_mhd_div_b.argtypes = [vp, C.POINTER(C.c_double)]
        lib.fin_mhd_last_kernel_ms.argtypes = [vp, C.POINTER(C.c_double)]
        lib.fin_mhd_set_kernel_timing.argtypes = [vp, C.c_int]
        lib.fin_mhd_kernel_time.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
        lib.fin_mhd_launch_count.argtypes = [vp, C.POINTER(C.c_longlong)]
        lib.fin_mhd_device_state.argtypes = [vp, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]
        fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        u8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
        ll = C.POINTER(C.c_longlong)
        lib.fin_mhd_set_indicator.argtypes = [vp, fp, C.c_float, C.c_int, C.c_double]
        lib.fin_mhd_set_indicator_every.argtypes = [vp, C.c_int]
        lib.fin_mhd_hybrid_stats.argtypes = [vp, ll, ll, ll, ll]
        lib.fin_mhd_indicator_time.argtypes = [vp, C.POINTER(C.c_double), ll]
        lib.fin_mhd_face_samples.argtypes = [vp, C.c_longlong, C.c_longlong, C.c_longlong, fp, u8, ll]
        for n in ("fin_mhd_create", "fin_mhd_destroy", "fin_mhd_set_state", "fin_mhd_get_state",
                  "fin_mhd_construct_l", "fin_mhd_construct_hj_l", "fin_mhd_after_step", "fin_mhd_solve",
                  "fin_mhd_advance", "fin_mhd_step_fixed", "fin_mhd_div_b", "fin_mhd_last_kernel_ms",
                  "fin_mhd_set_kernel_timing", "fin_mhd_kernel_time", "fin_mhd_launch_count",
                  "fin_mhd_device_state", "fin_mhd_set_indicator", "fin_mhd_set_indicator_every",
                  "fin_mhd_hybrid_stats", "fin_mhd_indicator_time", "fin_mhd_face_samples"):
            getattr(lib, n).restype = C.c_int
        lib._mhd_bound = True
    return lib


class MhdSolver:
    """One MHD problem resident on the current device."""

    def __init__(self, params):
        self.lib = _lib()
        self.p = params.copy()
        h = C.c_void_p()
        self._check(self.lib.fin_mhd_create(C.byref(self.p), C.byref(h)))
        self.h = h

    def _check(self, rc):
        if rc != FIN_OK:
            raise FinError(rc, self.lib.fin_mhd_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.fin_mhd_destroy(self.h)
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

    def _arrays(self, q, aux):
        q = np.ascontiguousarray(q, dtype=np.float64)
        aux = np.ascontiguousarray(aux, dtype=np.float64)
        assert q.shape == ghosted_shape(self.p) and aux.shape == aux_shape(self.p)
        return q, aux

    def set_state(self, q, aux, t=0.0):
        q, aux = self._arrays(q, aux)
        self._check(self.lib.fin_mhd_set_state(self.h, q, aux, t))

    def get_state(self):
        q = np.zeros(ghosted_shape(self.p))
        aux = np.zeros(aux_shape(self.p))
        t = C.c_double()
        self._check(self.lib.fin_mhd_get_state(self.h, q, aux, C.byref(t)))
        return q, aux, t.value

    def ConstructL(self, q, aux, smax=None):
        q, aux = self._arrays(q, aux)
        L = np.zeros(ghosted_shape(self.p))
        sm = np.zeros(smax_shape(self.p)) if smax is None else np.ascontiguousarray(smax, dtype=np.float64).copy()
        self._check(self.lib.fin_mhd_construct_l(self.h, q, aux, L, sm.ctypes.data_as(C.c_void_p)))
        return L, sm

    def ConstructHJ_L(self, q, aux):
        q, aux = self._arrays(q, aux)
        La = np.zeros(aux_shape(self.p))
        self._check(self.lib.fin_mhd_construct_hj_l(self.h, q, aux, La))
        return La

    def AfterStep(self, q, aux):
        q, aux = self._arrays(q, aux)
        q = q.copy()
        self._check(self.lib.fin_mhd_after_step(self.h, q, aux))
        return q

    def FinSolveRK(self, tend, dtv):
        """Advance to tend; dtv[1] is the starting dt and receives the next one."""
        dtv = np.ascontiguousarray(dtv, dtype=np.float64)
        n = C.c_int()
        self._check(self.lib.fin_mhd_solve(self.h, tend, dtv, C.byref(n)))
        return n.value

    def advance(self, tend, dtv, max_steps):
        dtv = np.ascontiguousarray(dtv, dtype=np.float64)
        n = C.c_int()
        self._check(self.lib.fin_mhd_advance(self.h, tend, dtv, max_steps, C.byref(n)))
        return n.value

    def step_fixed(self, dt):
        cfl = C.c_double()
        self._check(self.lib.fin_mhd_step_fixed(self.h, dt, C.byref(cfl)))
        return cfl.value

    def div_b(self):
        d = C.c_double()
        self._check(self.lib.fin_mhd_div_b(self.h, C.byref(d)))
        return d.value

    def last_kernel_ms(self):
        ms = C.c_double()
        self._check(self.lib.fin_mhd_last_kernel_ms(self.h, C.byref(ms)))
        return ms.value

    def set_kernel_timing(self, on=True):
        self._check(self.lib.fin_mhd_set_kernel_timing(self.h, int(on)))

    def kernel_time(self):
        ms, n = C.c_double(), C.c_longlong()
        self._check(self.lib.fin_mhd_kernel_time(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def launch_count(self):
        n = C.c_longlong()
        self._check(self.lib.fin_mhd_launch_count(self.h, C.byref(n)))
        return n.value

    # ---- hybrid form ----
    def set_indicator(self, params, z_threshold=0.0, judge_every=50, judge_tol=1e-3, every=1):
        """The troubled-face network (MHD-trained parameters), the judge step
        and the indicator's period in accepted steps."""
        self._check(self.lib.fin_mhd_set_indicator(self.h, np.ascontiguousarray(params, dtype=np.float32),
                                                   z_threshold, judge_every, judge_tol))
        self._check(self.lib.fin_mhd_set_indicator_every(self.h, every))

    def hybrid_stats(self):
        v = [C.c_longlong() for _ in range(4)]
        self._check(self.lib.fin_mhd_hybrid_stats(self.h, *[C.byref(x) for x in v]))
        return {"troubled_faces": v[0].value, "faces": v[1].value, "judges": v[2].value, "reverts": v[3].value}

    def indicator_time(self):
        ms, n = C.c_double(), C.c_longlong()
        self._check(self.lib.fin_mhd_indicator_time(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def face_samples(self, offset=0, stride=1, max_n=None):
        """Indicator features (n x 20) and labels of the current state's faces."""
        p = self.p
        nf = (p.mx + 1) * p.my + p.mx * (p.my + 1)
        n = (nf - offset + stride - 1) // stride
        if max_n is not None:
            n = min(n, max_n)
        X = np.zeros((n, 20), dtype=np.float32)
        y = np.zeros(n, dtype=np.uint8)
        nout = C.c_longlong()
        self._check(self.lib.fin_mhd_face_samples(self.h, offset, stride, n, X, y, C.byref(nout)))
        return X[:nout.value], y[:nout.value]


def first_dt(p, q):
    """desired_cfl / (max fast speed * (1/dx + 1/dy)) of a state: the MHD CFL
    number (apps/2d/mhd/lib/GetCFL.cpp:58) at the desired value."""
    mb = p.mbc
    Q = q[mb:mb + p.mx, mb:mb + p.my]
    g = p.gamma
    rho = Q[..., 0]
    u1, u2, u3 = Q[..., 1] / rho, Q[..., 2] / rho, Q[..., 3] / rho
    Bsq = (Q[..., 5:8] ** 2).sum(-1)
    pr = (g - 1) * (Q[..., 4] - 0.5 * rho * (u1 * u1 + u2 * u2 + u3 * u3) - 0.5 * Bsq)
    a2 = np.abs(g * pr / rho)
    t = a2 + Bsq / rho
    cf = np.sqrt(0.5 * (t + np.sqrt(np.abs(t * t - 4 * a2 * Q[..., 5] ** 2 / rho))))
    s = max(float(np.max(np.abs(u1) + cf)), float(np.max(np.abs(u2) + cf)))
    dx = (p.xhigh - p.xlow) / p.mx
    dy = (p.yhigh - p.ylow) / p.my
    return p.desired_cfl / (s * (1.0 / dx + 1.0 / dy))


def run_orszag_tang(n=2048, tend=math.pi, precisions=("fp64",), max_steps=None):
    """Orszag-Tang vortex on the device in the requested forms: steps, device
    seconds, cell-updates/s, max |div B|, and the FP32 form's density errors
    against the FP64 run when both ran."""
    out = {"problem": "orszag_tang", "n": n, "tend": tend}
    finals = {}
    forms = {"fp64": FIN_PREC_FP64, "fp32": FIN_PREC_FP32, "hybrid": FIN_PREC_HYBRID}
    for prec in precisions:
        p = P.orszag_tang_params(n=n)
        p.precision = forms[prec]
        q0, aux0 = P.orszag_tang_init(p)
        with MhdSolver(p) as s:
            s.set_state(q0, aux0)
            if prec == "hybrid":
                from .indicator import DEFAULT_MHD_WEIGHTS
                z = np.load(DEFAULT_MHD_WEIGHTS)
                s.set_indicator(z["params"], float(z["z_threshold"]), 50, 1e-3, 2)
                s.set_kernel_timing(True)
            dtv = np.array([0.0, first_dt(p, q0), p.max_dt])
            steps = s.advance(tend, dtv, max_steps if max_steps else 0x7fffffff)
            ms = s.last_kernel_ms()
            q, aux, t = s.get_state()
            out[prec] = {"steps": steps, "t": t, "device_s": ms * 1e-3,
                         "cell_updates_per_s": float(n) * n * steps / (ms * 1e-3),
                         "max_div_b": s.div_b(), "dt_last": float(dtv[1])}
            if prec == "hybrid":
                st = s.hybrid_stats()
                ims, il = s.indicator_time()
                kms, kl = s.kernel_time()
                out[prec].update({"hybrid": st, "troubled_fraction_last": st["troubled_faces"] / max(st["faces"], 1),
                                  "indicator_ms_mean": ims / max(il, 1), "stage_ms_mean": kms / max(kl, 1)})
            finals[prec] = q
    for prec in ("fp32", "hybrid"):
        if "fp64" in finals and prec in finals:
            l1, linf = P.density_errors(p, finals[prec], finals["fp64"])
            out[prec + "_vs_fp64_density"] = {"l1": l1, "linf": linf}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--tend", type=float, default=math.pi)
    ap.add_argument("--precision", default="both", choices=["fp64", "fp32", "hybrid", "both", "all"])
    ap.add_argument("--max-steps", type=int, default=0)
    a = ap.parse_args()
    precs = {"both": ("fp64", "fp32"), "all": ("fp64", "fp32", "hybrid")}.get(a.precision, (a.precision,))
    print(json.dumps(run_orszag_tang(a.n, a.tend, precs, a.max_steps or None)))


if __name__ == "__main__":
    main()
