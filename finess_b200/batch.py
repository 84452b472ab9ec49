"""Batches of independent problems (fin_batch_* of the C ABI).

``Batch`` advances many 2D Euler problems of uneven grid sizes to one end
time, each with its own adaptive SSP-RK3 dt; per problem the results agree
with a separate ``Solver.FinSolveRK`` of it to rounding.  ``sweep_problem``
builds problem k of the uneven four-quadrant Riemann sweep (grid N x N per problem, N
log-uniform in [64, 1024]; quadrant states rho ~ U[0.1, 2], u, v ~
U[-1.5, 1.5], p ~ U[0.02, 2]; interface ~ U[0.3, 0.7]^2; transmissive
boundaries; CFL 0.4) from a seed.

    python -m finess_b200.batch [--n 1024] [--tend 0.25] [--seed 0] [--precision fp32|fp64|hybrid] [--separate]
"""
import argparse
import ctypes as C
import json
import math

import numpy as np

from . import problems as P
from ._abi import FIN_OK, FIN_PREC_FP32, FIN_PREC_FP64, FIN_PREC_HYBRID, FIN_WENO_Z, FinParams, ghosted_shape
from .solver import FinError, Solver, load_library

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def _lib():
    lib = load_library()
    if not getattr(lib, "_batch_bound", False):
        vp = C.c_void_p
        lib.fin_batch_create.argtypes = [C.POINTER(FinParams), C.c_int, C.POINTER(vp)]
        lib.fin_batch_destroy.argtypes = [vp]
        lib.fin_batch_set_state.argtypes = [vp, C.c_int, _dp, C.c_double]
        lib.fin_batch_get_state.argtypes = [vp, C.c_int, _dp, C.POINTER(C.c_double)]
        lib.fin_batch_solve.argtypes = [vp, C.c_double, _dp, np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")]
        lib.fin_batch_stats.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                        np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")]
        lib.fin_batch_set_indicator.argtypes = [vp, np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"),
                                                C.c_float, C.c_int, C.c_double]
        lib.fin_batch_set_indicator_every.argtypes = [vp, C.c_int]
        lib.fin_batch_hybrid_stats.argtypes = [vp] + [C.POINTER(C.c_longlong)] * 4
        lib.fin_batch_set_kernel_timing.argtypes = [vp, C.c_int]
        lib.fin_batch_kernel_times.argtypes = [vp, np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")]
        lib.fin_batch_last_error.restype = C.c_char_p
        for n in ("fin_batch_create", "fin_batch_destroy", "fin_batch_set_state", "fin_batch_get_state",
                  "fin_batch_solve", "fin_batch_stats", "fin_batch_set_indicator", "fin_batch_set_indicator_every",
                  "fin_batch_hybrid_stats", "fin_batch_set_kernel_timing", "fin_batch_kernel_times"):
            getattr(lib, n).restype = C.c_int
        lib._batch_bound = True
    return lib


def _check(lib, rc):
    if rc != FIN_OK:
        raise FinError(rc, lib.fin_batch_last_error().decode())


class Batch:
    """nprob problems (a list of FinParams) resident on the current device."""

    def __init__(self, params):
        self.lib = _lib()
        self.p = [q.copy() for q in params]
        arr = (FinParams * len(self.p))(*self.p)
        h = C.c_void_p()
        _check(self.lib, self.lib.fin_batch_create(arr, len(self.p), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.fin_batch_destroy(self.h)
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

    def set_state(self, k, q, t=0.0):
        q = np.ascontiguousarray(q, dtype=np.float64)
        assert q.shape == ghosted_shape(self.p[k])
        _check(self.lib, self.lib.fin_batch_set_state(self.h, k, q, t))

    def get_state(self, k):
        q = np.zeros(ghosted_shape(self.p[k]))
        t = C.c_double()
        _check(self.lib, self.lib.fin_batch_get_state(self.h, k, q, C.byref(t)))
        return q, t.value

    def solve(self, tend, dt):
        """Every problem to tend; dt: per-problem dt on entry. Returns (dt, steps)."""
        dtv = np.ascontiguousarray(dt, dtype=np.float64).copy()
        steps = np.zeros(len(self.p), dtype=np.int32)
        _check(self.lib, self.lib.fin_batch_solve(self.h, tend, dtv, steps))
        return dtv, steps

    def set_indicator(self, params, z_threshold=0.0, judge_every=20, judge_tol=1e-3, every=1):
        """Hybrid form: the troubled-face network, the judge step and the
        indicator's period in accepted steps, for every problem (as
        ``Solver.set_indicator``)."""
        _check(self.lib, self.lib.fin_batch_set_indicator(self.h, np.ascontiguousarray(params, dtype=np.float32),
                                                          z_threshold, judge_every, judge_tol))
        _check(self.lib, self.lib.fin_batch_set_indicator_every(self.h, every))

    def hybrid_stats(self):
        v = [C.c_longlong() for _ in range(4)]
        _check(self.lib, self.lib.fin_batch_hybrid_stats(self.h, *[C.byref(x) for x in v]))
        return {"troubled_faces": v[0].value, "faces": v[1].value, "judges": v[2].value, "reverts": v[3].value}

    def set_kernel_timing(self, on=True):
        """Launch steps one by one with events between the launch groups
        (diagnostic: no graph) and accumulate each group's device time."""
        _check(self.lib, self.lib.fin_batch_set_kernel_timing(self.h, 1 if on else 0))

    def kernel_times(self):
        ms = np.zeros(5)
        _check(self.lib, self.lib.fin_batch_kernel_times(self.h, ms))
        return dict(zip(("control_ms", "indicator_ms", "hybrid_stages_ms", "plain_stages_ms", "judge_diff_ms"),
                        map(float, ms)))

    def stats(self):
        ms, reps, cfg = C.c_double(), C.c_longlong(), C.c_int()
        tune = np.zeros(2)
        _check(self.lib, self.lib.fin_batch_stats(self.h, C.byref(ms), C.byref(reps), C.byref(cfg), tune))
        return {"device_ms": ms.value, "replays": reps.value, "tile_shape": ["15x16", "7x32"][cfg.value]
                if cfg.value >= 0 else None, "tune_stage_ms": {"15x16": tune[0], "7x32": tune[1]}}


def sweep_problem(seed, k, nmin=64, nmax=1024, precision=FIN_PREC_FP32, weno=FIN_WENO_Z):
    """Problem k of the uneven Riemann sweep of a seed: (params, initial state).
    Each problem draws from its own stream (SeedSequence(seed).spawn), so any
    problem can be rebuilt alone."""
    rng = np.random.default_rng(np.random.SeedSequence([seed, k]))
    N = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
    p = P.riemann_params(n=N, weno=weno)
    p.precision = precision
    return p, P.random_riemann_state(p, rng)


def _sweep_grid(seed, k, nmin=64, nmax=1024, precision=FIN_PREC_FP32, weno=FIN_WENO_Z):
    rng = np.random.default_rng(np.random.SeedSequence([seed, k]))
    N = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
    p = P.riemann_params(n=N, weno=weno)
    p.precision = precision
    return p


def first_dt(p, q):
    """desired_cfl * min(dx, dy) / max wave speed of q (as bench.py's first dt)."""
    g = p.gamma
    mb = p.mbc
    qi = q[mb:mb + p.mx, mb:mb + p.my]
    rho = qi[..., 0]
    u, v = qi[..., 1] / rho, qi[..., 2] / rho
    pr = (g - 1.0) * (qi[..., 4] - 0.5 * rho * (u * u + v * v))
    c = np.sqrt(np.abs(g * pr / rho))
    a = max(float(np.max(np.abs(u) + c)), float(np.max(np.abs(v) + c)))
    return p.desired_cfl * min((p.xhigh - p.xlow) / p.mx, (p.yhigh - p.ylow) / p.my) / a


# Hybrid-form schedule of the sweep (as the single-problem benchmark's): the
# indicator every 2nd accepted step, every 50th hybrid step judged against a
# full-WENO step with tolerance 1e-3.
HYB_EVERY, HYB_JUDGE_EVERY, HYB_JUDGE_TOL = 2, 50, 1e-3
PRECISIONS = {"fp64": FIN_PREC_FP64, "fp32": FIN_PREC_FP32, "hybrid": FIN_PREC_HYBRID}


def load_indicator(path=None):
    """(network parameters, z threshold) of the trained troubled-face network."""
    from .indicator import DEFAULT_WEIGHTS
    W = np.load(path or DEFAULT_WEIGHTS)
    return W["params"], float(W["z_threshold"])


def run_sweep(n=1024, tend=0.25, seed=0, precision=FIN_PREC_FP32, separate=False, indicator=None,
              kernel_times=False):
    """The sweep batched (one persistent launch per stage over all problems)
    and, optionally, every problem run on its own; device times and
    cell-updates/s of both.  The hybrid form takes indicator = (params,
    z threshold), by default the trained network.  kernel_times: the batch
    runs without its graph, with the device time of each launch group."""
    hyb = precision == FIN_PREC_HYBRID
    if hyb and indicator is None:
        indicator = load_indicator()
    params = [_sweep_grid(seed, k, precision=precision) for k in range(n)]
    cells = np.array([p.mx * p.my for p in params], dtype=np.float64)
    dts = np.zeros(n)
    name = {v: k for k, v in PRECISIONS.items()}[precision]
    out = {"problems": n, "seed": seed, "tend": tend, "precision": name,
           "grid_min": int(min(p.mx for p in params)), "grid_max": int(max(p.mx for p in params)),
           "cells_total": float(cells.sum())}
    with Batch(params) as b:
        if hyb:
            b.set_indicator(indicator[0], indicator[1], HYB_JUDGE_EVERY, HYB_JUDGE_TOL, HYB_EVERY)
        for k in range(n):
            p, q = sweep_problem(seed, k, precision=precision)
            dts[k] = first_dt(p, q)
            b.set_state(k, q)
        if kernel_times:
            b.set_kernel_timing(True)
        _, steps = b.solve(tend, dts)
        st = b.stats()
        hst = b.hybrid_stats() if hyb else None
        kt = b.kernel_times() if kernel_times else None
    cu = float(np.sum(cells * steps))
    out["batched"] = {"cell_updates": cu, "device_s": st["device_ms"] * 1e-3,
                      "cell_updates_per_s": cu / (st["device_ms"] * 1e-3), "steps_max": int(steps.max()),
                      "graph_replays": st["replays"], "tile_shape": st["tile_shape"],
                      "autotune_stage1_ms": st["tune_stage_ms"]}
    if kt:
        out["batched"]["graph"] = False
        out["batched"]["kernel_times_ms"] = kt
    if hyb:
        out["batched"]["hybrid"] = dict(hst, troubled_fraction=hst["troubled_faces"] / max(hst["faces"], 1),
                                        indicator_every=HYB_EVERY, judge_every=HYB_JUDGE_EVERY,
                                        judge_tol=HYB_JUDGE_TOL)
    if separate:
        tot = 0.0
        for k in range(n):
            p, q = sweep_problem(seed, k, precision=precision)
            with Solver(p) as s:
                if hyb:
                    s.set_indicator(indicator[0], indicator[1], HYB_JUDGE_EVERY, HYB_JUDGE_TOL, HYB_EVERY)
                s.set_state(q)
                s.FinSolveRK(tend, np.array([0.0, dts[k], p.max_dt]))
                tot += s.last_kernel_ms() * 1e-3
        out["separate"] = {"device_s": tot, "cell_updates_per_s": cu / tot}
        out["batched_over_separate"] = out["batched"]["cell_updates_per_s"] / out["separate"]["cell_updates_per_s"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--tend", type=float, default=0.25)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", default="fp32", choices=sorted(PRECISIONS))
    ap.add_argument("--separate", action="store_true", help="also run every problem on its own")
    ap.add_argument("--kernel-times", action="store_true",
                    help="run the batch without its graph and report each launch group's device time")
    a = ap.parse_args()
    print(json.dumps(run_sweep(a.n, a.tend, a.seed, PRECISIONS[a.precision], a.separate,
                               kernel_times=a.kernel_times)))


if __name__ == "__main__":
    main()
