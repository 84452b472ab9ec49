"""RunFinpack's frame loop on the device (lib/2d/RunFinpack.cpp:57-130):
qhelp.dat, frame 0 and its conservation line, then per frame FinSolveRK to
t = n tfinal / nout and Output(n), with conservation.dat appended after
every accepted step.  The frame files are written asynchronously (the next
frame's steps run while the previous frame is formatted and written); with
--sync each frame waits for its files, as the reference's loop does.

    python -m finess_b200.frames --problem riemann --n 4096 --nout 4 --tfinal 0.02 --outdir /tmp/out [--sync]
        [--precision fp64|fp32|hybrid]

run_frames returns the last frame's state (``q_last``, ``t_last``) beside the
figures, so a checker can write the same frame with another implementation.
"""
import argparse
import json
import os
import time

import numpy as np

from . import problems as P
from ._abi import FIN_PREC_FP32, FIN_PREC_FP64, FIN_PREC_HYBRID
from .batch import HYB_EVERY, HYB_JUDGE_EVERY, HYB_JUDGE_TOL, first_dt, load_indicator
from .solver import Solver, write_qhelp

PRECISIONS = {"fp64": FIN_PREC_FP64, "fp32": FIN_PREC_FP32, "hybrid": FIN_PREC_HYBRID}


def problem(name, n):
    if name == "riemann":
        p = P.riemann_params(n=n)
        return p, P.riemann_init(p)
    if name == "vortex":
        p = P.vortex_params(n=n)
        return p, P.vortex_exact(p)
    if name == "shock_entropy":
        p = P.shock_entropy_params(nx=2 * n, ny=n // 4)
        return p, P.shock_entropy_init(p)
    raise ValueError(name)


def run_frames(name="riemann", n=4096, nout=4, tfinal=0.02, outdir="output", precision="fp64", sync=False):
    p, q0 = problem(name, n)
    p.precision = PRECISIONS[precision]
    p.nout, p.tfinal = nout, tfinal
    os.makedirs(outdir, exist_ok=True)
    out = {"problem": name, "mx": p.mx, "my": p.my, "nout": nout, "tfinal": tfinal, "precision": precision,
           "async_output": not sync}
    with Solver(p) as s:
        if precision == "hybrid":
            W, z = load_indicator()
            s.set_indicator(W, z, HYB_JUDGE_EVERY, HYB_JUDGE_TOL, HYB_EVERY)
        t0 = time.perf_counter()
        write_qhelp(p, outdir)
        s.set_state(q0, 0.0)
        s.set_conservation_file(outdir)
        s.write_conservation()
        s.output_frame(0, outdir)
        dtv = np.array([0.0, first_dt(p, q0), p.max_dt])
        steps, device_ms, wait_s = 0, 0.0, 0.0
        for k in range(1, nout + 1):
            if sync:
                w = time.perf_counter()
                s.output_wait()
                wait_s += time.perf_counter() - w
            dtv, m = s.advance(k * tfinal / nout, dtv, 0x7fffffff)
            steps += m
            device_ms += s.last_kernel_ms()
            s.output_frame(k, outdir)
        w = time.perf_counter()
        s.output_wait()
        wait_s += time.perf_counter() - w
        wall = time.perf_counter() - t0
        q_last, t_last = s.get_state()
    frame_bytes = os.path.getsize(os.path.join(outdir, "q%04d.dat" % nout))
    out.update({"steps": steps, "wall_s": wall, "device_s": device_ms * 1e-3, "output_wait_s": wait_s,
                "frames_written": nout + 1, "frame_file_bytes": frame_bytes,
                "cell_updates_per_s_wall": float(p.mx) * p.my * steps / wall})
    out["q_last"], out["t_last"] = q_last, t_last
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--problem", default="riemann", choices=["riemann", "vortex", "shock_entropy"])
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--nout", type=int, default=4)
    ap.add_argument("--tfinal", type=float, default=0.02)
    ap.add_argument("--outdir", default="output")
    ap.add_argument("--precision", default="fp64", choices=sorted(PRECISIONS))
    ap.add_argument("--sync", action="store_true", help="wait for each frame's files before the next frame")
    a = ap.parse_args()
    out = run_frames(a.problem, a.n, a.nout, a.tfinal, a.outdir, a.precision, a.sync)
    out.pop("q_last")
    print(json.dumps(out))


if __name__ == "__main__":
    main()
