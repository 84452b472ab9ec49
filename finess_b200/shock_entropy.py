"""The learned-indicator workload: 2D Euler shock / entropy-wave interaction.

[-5, 5] x [0, 1], 8192 x 1024 cells, transmissive in x and periodic in y;
a Mach-3 shock at x = -4 runs into the density wave
rho = 1 + 0.2 sin(5x) + 0.1 sin(2 pi y) (problems.shock_entropy_init);
WENO5-JS, global Lax-Friedrichs, SSP-RK3 at CFL 0.4 to t = 1.8.  The plain
FP64 and FP32 forms and the hybrid form (FP32 bulk, the trained troubled-face
network every 2nd step, every 50th hybrid step judged against full WENO with
tolerance 1e-3) run the same frame; the report gives each form's steps,
device time and cell-updates/s, and the FP32 and hybrid density errors
against the FP64 run.

    python -m finess_b200.shock_entropy [--nx 8192] [--ny 1024] [--tend 1.8] [--precision all]
"""
import argparse
import json

import numpy as np

from . import problems as P
from ._abi import FIN_PREC_FP32, FIN_PREC_FP64, FIN_PREC_HYBRID, FIN_WENO_JS
from .batch import HYB_EVERY, HYB_JUDGE_EVERY, HYB_JUDGE_TOL, first_dt, load_indicator
from .solver import Solver

FORMS = {"fp64": FIN_PREC_FP64, "fp32": FIN_PREC_FP32, "hybrid": FIN_PREC_HYBRID}


def run_shock_entropy(nx=8192, ny=1024, tend=1.8, precisions=("fp64", "fp32", "hybrid"), max_steps=None):
    out = {"problem": "shock_entropy", "nx": nx, "ny": ny, "tend": tend, "weno": "JS"}
    finals = {}
    p = None
    for prec in precisions:
        p = P.shock_entropy_params(nx=nx, ny=ny, weno=FIN_WENO_JS)
        p.precision = FORMS[prec]
        q0 = P.shock_entropy_init(p)
        with Solver(p) as s:
            if prec == "hybrid":
                W, z = load_indicator()
                s.set_indicator(W, z, HYB_JUDGE_EVERY, HYB_JUDGE_TOL, HYB_EVERY)
                s.set_kernel_timing(True)
            s.set_state(q0)
            dtv = np.array([0.0, first_dt(p, q0), p.max_dt])
            dtv, steps = s.advance(tend, dtv, max_steps if max_steps else 0x7fffffff)
            ms = s.last_kernel_ms()
            q, t = s.get_state()
            out[prec] = {"steps": steps, "t": t, "device_s": ms * 1e-3,
                         "cell_updates_per_s": float(nx) * ny * steps / (ms * 1e-3), "dt_last": float(dtv[1])}
            if prec == "hybrid":
                st = s.hybrid_stats()
                ims, il = s.indicator_time()
                kms, kl = s.kernel_time()
                out[prec].update({"hybrid": st, "troubled_fraction_last": st["troubled_faces"] / max(st["faces"], 1),
                                  "indicator_ms_mean": ims / max(il, 1), "stage_ms_mean": kms / max(kl, 1),
                                  "schedule": {"indicator_every": HYB_EVERY, "judge_every": HYB_JUDGE_EVERY,
                                               "judge_tol": HYB_JUDGE_TOL}})
            finals[prec] = q
    for prec in ("fp32", "hybrid"):
        if "fp64" in finals and prec in finals:
            l1, linf = P.density_errors(p, finals[prec], finals["fp64"])
            out[prec + "_vs_fp64_density"] = {"l1": l1, "linf": linf}
    if "fp64" in out and "hybrid" in out:
        out["hybrid_over_fp64_speed"] = out["hybrid"]["cell_updates_per_s"] / out["fp64"]["cell_updates_per_s"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=8192)
    ap.add_argument("--ny", type=int, default=1024)
    ap.add_argument("--tend", type=float, default=1.8)
    ap.add_argument("--precision", default="all", choices=["fp64", "fp32", "hybrid", "all"])
    ap.add_argument("--max-steps", type=int, default=0)
    a = ap.parse_args()
    precs = ("fp64", "fp32", "hybrid") if a.precision == "all" else (a.precision,)
    print(json.dumps(run_shock_entropy(a.nx, a.ny, a.tend, precs, a.max_steps or None)))


if __name__ == "__main__":
    main()
