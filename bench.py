"""Benchmark of the B200 WENO right-hand side + SSP-RK3 stepper.

Workload (one "step" = one full SSP-RK3 time step with FinSolveRK's adaptive
dt and CFL check): the 2D Euler four-quadrant Riemann problem on [0,1]^2,
4096 x 4096 cells, transmissive boundaries, interface (0.8, 0.8), WENO5-Z,
global LLF with characteristic projection, CFL 0.4, to t = 0.8.  Synthetic
closed-form initial data; the state (673 MB per FP64 array) is far larger
than the 126 MB L2, so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--forms fp64,fp32,hybrid]
    python bench.py --whole-runs [--n N]                  # every form to t = 0.8, errors against FP64
    python bench.py --space-orders [--n N] [--steps K]    # LLF, WENO7/9/11 beside WENO5 (FP64)
    python bench.py --mpp [--n N] [--steps K]             # Lax-Wendroff with / without the MPP limiter
    python bench.py --frames [--n N]                      # frame files, and the reference's Output beside them
    python bench.py --sweep [--gpus N]                    # the 1024-problem uneven sweep split across N GPUs

The headline form is the hybrid (FP32 bulk + troubled-face network run every
HYB_EVERY accepted steps, judge step every HYB_JUDGE_EVERY steps) when trained
weights are present (finess_b200/data/), else FP64.  The hybrid's cost per
step grows as the flow develops (more troubled faces), so the headline run is
one whole hybrid run from t = 0 to t = 0.8: the W warm-up and K timed steps
are taken in its middle (from t = WINDOW_T), and the run's total device time
gives the whole-run throughput.  `value` is the K-step window with the judge
step's cost amortised over its period (one full-WENO FP32 step every
HYB_JUDGE_EVERY steps); `speedup_vs_fp64` is the whole hybrid run against the
plain FP64 form (whose cost per step does not depend on the state: every
face takes full WENO).  The line also carries every form's throughput and an
"equal L1 error" block (each form's density L1 error on two reduced problems,
the hybrid with the same settings).  --whole-runs runs every form to t = 0.8
at the full size and states the FP32 and hybrid errors against the FP64 run.

N > 1 runs as N independent replicas (one per GPU, launched by torchrun); the
path has no exchange between problems.  Prints one JSON line on rank 0.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "2D Euler WENO5 cell-updates/s, hybrid FP32 vs plain FP64 GPU at equal L1 err"
UNIT = "cell-updates/s"
N_CELLS = 4096
# Algorithmic HBM bytes per cell-update of a perfectly fused SSP-RK3 step with
# FP64 state, meqn 5: stage 1 reads q and writes q1 (80 B), stages 2 and 3
# each read two arrays and write one (120 B each).
# Every form keeps the state in FP64, so the bytes are the same for all.
BYTES_PER_CELL_UPDATE = 320.0
# Hybrid-form schedule: the indicator runs on q^n of every 2nd accepted step
# (its flags, dilated by one face, serve the next step too: at CFL 0.4 a wave
# moves at most 0.8 cells in two steps), and every 50th hybrid step is judged
# against a full-WENO step from the same state.
HYB_EVERY = 2
HYB_JUDGE_EVERY = 50
# the end of the headline run and the start of its timed window
T_END = 0.8
WINDOW_T = 0.4


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"fin_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic_bytes_per_cell(form):
    """Per-cell DRAM traffic of an average stage launch from the committed ncu
    summary (profiles/stage_kernel_*.txt, line 'dram_bytes_per_cell_<form>: X A'
    with X measured on one launch whose algorithmic bytes per cell are A):
    X scaled to the stage average of 320/3 algorithmic bytes per cell."""
    import glob
    for f in sorted(glob.glob(os.path.join(ROOT, "profiles", "stage_kernel_*.txt"))):
        for line in open(f):
            if line.startswith(f"dram_bytes_per_cell_{form}:"):
                try:
                    x, alg = (float(v) for v in line.split(":", 1)[1].split()[:2])
                    return x * (BYTES_PER_CELL_UPDATE / 3.0) / alg
                except ValueError:
                    pass
    return None


FORMS = ("fp64", "fp32", "hybrid")


def load_indicator():
    from finess_b200.indicator import DEFAULT_WEIGHTS
    if not os.path.exists(DEFAULT_WEIGHTS):
        return None
    W = np.load(DEFAULT_WEIGHTS)
    return W["params"], float(W["z_threshold"])


def make_solver(p, form, indicator, judge_every=HYB_JUDGE_EVERY, judge_tol=1e-3, every=HYB_EVERY):
    from finess_b200.solver import Solver
    from finess_b200._abi import FIN_PREC_FP32, FIN_PREC_FP64, FIN_PREC_HYBRID
    p = p.copy()
    p.precision = {"fp64": FIN_PREC_FP64, "fp32": FIN_PREC_FP32, "hybrid": FIN_PREC_HYBRID}[form]
    s = Solver(p)
    if form == "hybrid":
        s.set_indicator(indicator[0], indicator[1], judge_every, judge_tol, every)
    return s


def ghosted_shape_of(p):
    from finess_b200._abi import ghosted_shape
    return ghosted_shape(p)


def first_dt(p, s, q0):
    a1, a2 = s.GlobalWaveSpd(q0)
    return p.desired_cfl * min((p.xhigh - p.xlow) / p.mx, (p.yhigh - p.ylow) / p.my) / max(a1, a2)


def accuracy_block(indicator, forms):
    """Density L1 (area-normalised) of each form: the isentropic vortex (200^2,
    one period, against the exact solution) and the four-quadrant Riemann
    problem (512^2 to t = 0.8, against the FP64 run at 1024^2 averaged onto
    the 512^2 cells)."""
    from finess_b200 import problems as P

    def run(p, q0, tend, form):
        s = make_solver(p, form, indicator)
        s.set_state(q0, 0.0)
        dtv = np.array([0.0, first_dt(p, s, q0), p.max_dt])
        s.FinSolveRK(tend, dtv)
        q, _ = s.get_state()
        st = s.hybrid_stats() if form == "hybrid" else None
        s.close()
        return q, st

    out = {}
    p = P.vortex_params(n=200)
    q0, qe = P.vortex_exact(p), P.vortex_exact(p, t=10.0)
    for f in forms:
        q, st = run(p, q0, 10.0, f)
        out[f"vortex200_{f}_L1"] = P.density_errors(p, q, qe)[0]
    pf = P.riemann_params(n=1024)
    qf, _ = run(pf, P.riemann_init(pf), 0.8, "fp64")
    mb = pf.mbc
    fi = qf[mb:mb + 1024, mb:mb + 1024]
    p = P.riemann_params(n=512)
    q0 = P.riemann_init(p)
    qr = np.zeros_like(q0)
    qr[p.mbc:p.mbc + 512, p.mbc:p.mbc + 512] = 0.25 * (fi[0::2, 0::2] + fi[1::2, 0::2] + fi[0::2, 1::2] + fi[1::2, 1::2])
    for f in forms:
        q, st = run(p, q0, 0.8, f)
        out[f"riemann512_{f}_L1"] = P.density_errors(p, q, qr)[0]
        if st:
            out["riemann512_hybrid_judges"] = st["judges"]
            out["riemann512_hybrid_reverts"] = st["reverts"]
    for k in ("vortex200", "riemann512"):
        if f"{k}_hybrid_L1" in out:
            out[f"{k}_hybrid_over_fp64"] = out[f"{k}_hybrid_L1"] / out[f"{k}_fp64_L1"]
    return out


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def reference_impl():
    """The reference's own CPU code (oracle/_ref, all host threads through
    OpenMP) where it was built, else the C restatement (one thread)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle, RefLib
    if RefLib.available():
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        return RefLib(), "reference", int(os.environ["OMP_NUM_THREADS"])
    return Oracle(), "port", 1


def reference_steps(impl, p, q, steps):
    """`steps` fixed-dt SSP-RK3 steps of the reference's FinSolveRK in one
    call (its arrays allocated once, as in a run); returns (seconds, q)."""
    a1, a2 = impl.global_wave_spd(p, q)
    dt = 0.5 * p.desired_cfl * min((p.xhigh - p.xlow) / p.mx, (p.yhigh - p.ylow) / p.my) / max(a1, a2)
    p = p.copy()
    p.max_dt = dt          # FinSolveRK keeps dt = min(max_dt, ...) = dt: `steps` steps to the end time
    t0 = time.perf_counter()
    out = impl.finsolve(p, q, 0.0, (steps - 0.5) * dt, dt)
    el = time.perf_counter() - t0
    return el, out[1]


def cpu_baseline(n=N_CELLS, steps=2):
    """The reference's CPU code on a bounded sample of the workload: `steps`
    SSP-RK3 steps of the same problem at its full size."""
    from finess_b200 import problems as P
    from finess_b200._abi import FIN_WENO_Z
    impl, kind, cores = reference_impl()
    p = P.riemann_params(n=n, weno=FIN_WENO_Z)
    q = impl.set_bnd(p, P.riemann_init(p))
    el, _ = reference_steps(impl, p, q, steps)
    return {"value": n * n * steps / el, "unit": UNIT, "cores": cores, "kind": kind, "cpu_model": cpu_model(),
            "sample": f"{steps} SSP-RK3 steps of the same problem (WENO5-Z, 4-quadrant Riemann) at {n}x{n} in one "
                      f"FinSolveRK call, {el:.1f} s"}


def run_reference_arm(args):
    """The reference's own CPU code (oracle/_ref) on the workload's full size:
    W warm-up steps on a 512^2 sample (threads and caches), then K SSP-RK3
    steps at 4096^2 in one FinSolveRK call, timed by the host clock."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from finess_b200 import problems as P
    from finess_b200._abi import FIN_WENO_Z
    impl, kind, cores = reference_impl()
    pw = P.riemann_params(n=512, weno=FIN_WENO_Z)
    reference_steps(impl, pw, impl.set_bnd(pw, P.riemann_init(pw)), args.warmup)
    n = args.n
    p = P.riemann_params(n=n, weno=FIN_WENO_Z)
    q = impl.set_bnd(p, P.riemann_init(p))
    el, _ = reference_steps(impl, p, q, args.steps)
    value = n * n * args.steps / el
    sample = (f"{args.steps} SSP-RK3 steps of the workload at its full size ({n}x{n}) in one FinSolveRK call "
              f"(warm-up: {args.warmup} steps at 512x512)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "euler2d_riemann4q_wenoz_rk3", "grid": f"{n}x{n}", "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "cpu_model": cpu_model(),
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


SPACE_ORDERS = ((5, "JS"), (1, "JS"), (7, "JS"), (7, "Z"), (7, "FD"), (9, "JS"), (9, "Z"), (9, "FD"), (11, "JS"))


def run_space_orders(args):
    """The other spatial orders of ConstructL (LLF, JS7/9/11, Z7/9, FD7/9,
    FP64, SSP-RK3) beside WENO5-JS: the isentropic vortex on [0,10]^2 at
    n x n, periodic, CFL 0.4, one JSON line per scheme with the device time
    per step (fin_advance, CUDA events) and, where oracle/_ref exists, the
    reference's own FinSolveRK on a bounded 256^2 sample (3 steps, all host
    threads)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from finess_b200 import problems as P
    from finess_b200._abi import FIN_WENO_FD, FIN_WENO_JS, FIN_WENO_Z
    from finess_b200.batch import first_dt as batch_first_dt
    from finess_b200.solver import Solver
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefLib
    ref = RefLib() if (RefLib.available() and not args.no_cpu_baseline) else None
    ver = {"JS": FIN_WENO_JS, "Z": FIN_WENO_Z, "FD": FIN_WENO_FD}
    n = args.n if args.n != N_CELLS else 2048
    for so, vn in SPACE_ORDERS:
        mbc = max(3, (so + 1) // 2)
        p = P.vortex_params(n=n, weno=ver[vn], space_order=so, mbc=mbc)
        q0 = P.vortex_exact(p)
        dt0 = batch_first_dt(p, q0)
        with Solver(p) as s:
            s.set_state(q0)
            s.advance(1.0, np.array([0.0, dt0, p.max_dt]), args.warmup)
            _, k = s.advance(1.0, np.array([0.0, dt0, p.max_dt]), args.steps)
            ms = s.last_kernel_ms()
        line = {"metric": f"2D Euler space_order {so} ({vn}) cell-updates/s, FP64 SSP-RK3", "value": n * n * k / (ms * 1e-3),
                "unit": UNIT, "n_gpus": 1, "steps": k, "warmup": args.warmup, "ms_per_step": ms / k,
                "higher_is_better": True, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "euler2d_vortex_periodic_rk3", "grid": f"{n}x{n}", "space_order": so,
                           "weno": vn, "mbc": mbc, "cfl": 0.4}}
        if ref is not None:
            m = 256
            pr = P.vortex_params(n=m, weno=ver[vn], space_order=so, mbc=mbc)
            qr = P.vortex_exact(pr)
            dtr = batch_first_dt(pr, qr)
            qr = ref.set_bnd(pr, qr)
            t0 = time.perf_counter()
            rc, _, _, _ = ref.finsolve(pr, qr, 0.0, 2.5 * dtr, dtr)   # three steps
            el = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": m * m * 3 / el, "unit": UNIT, "kind": "reference",
                                    "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                                    "sample": f"3 SSP-RK3 steps at {m}x{m}, {el:.2f} s", "rc": rc}
        print(json.dumps(line), flush=True)


def run_mpp(args):
    """Lax-Wendroff (time_order 3, mbc 5, WENO5-Z, FP64) with and without the
    MPP positivity limiter on the four-quadrant Riemann problem at 2048^2 and
    4096^2: device time per step through fin_advance (CUDA events), one JSON
    line per case."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from finess_b200 import problems as P
    from finess_b200._abi import FIN_TS_LXW, FIN_TS_MD, FIN_WENO_Z
    from finess_b200.batch import first_dt as batch_first_dt
    from finess_b200.solver import Solver
    for n in ((args.n,) if args.n != N_CELLS else (2048, 4096)):
        for mpp in (0, 1):
            p = P.riemann_params(n=n, weno=FIN_WENO_Z, method=FIN_TS_MD, time_stepping_method=FIN_TS_LXW,
                                 time_order=3, mpp_limiter=mpp)
            q0 = P.riemann_init(p)
            dt0 = batch_first_dt(p, q0)
            with Solver(p) as s:
                s.set_state(q0)
                s.advance(1.0, np.array([0.0, dt0, p.max_dt]), args.warmup)
                _, k = s.advance(1.0, np.array([0.0, dt0, p.max_dt]), args.steps)
                ms = s.last_kernel_ms()
            print(json.dumps({"metric": "2D Euler Lax-Wendroff cell-updates/s" + (" with the MPP limiter" if mpp else ""),
                              "value": n * n * k / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": k,
                              "warmup": args.warmup, "ms_per_step": ms / k, "higher_is_better": True,
                              "dtype": "f64", "data": "synthetic",
                              "config": {"workload": "euler2d_riemann4q_wenoz_lxw", "grid": f"{n}x{n}",
                                         "mpp_limiter": mpp, "mbc": 5}}), flush=True)


def run_whole_runs(args):
    """Every form from t = 0 to T_END at the full size (one JSON line): device
    time of each whole run (CUDA events around fin_advance), its steps, and
    the FP32 and hybrid density L1 (area-normalised) and L-infinity against
    the FP64 run (the plain method, itself pinned to the reference)."""
    ws, rank, local = dist_env()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    from finess_b200 import problems as P
    indicator = load_indicator()
    forms = [f for f in (args.forms.split(",") if args.forms else FORMS) if f != "hybrid" or indicator]
    p = P.riemann_params(n=args.n)
    q0 = P.riemann_init(p)
    cells = p.mx * p.my
    runs, states = {}, {}
    for form in forms:
        s = make_solver(p, form, indicator)
        s.set_state(q0, 0.0)
        dtv = np.array([0.0, first_dt(p, s, q0), p.max_dt])
        ms, steps = 0.0, 0
        while True:
            dtv, k = s.advance(T_END, dtv, 2000)
            ms += s.last_kernel_ms()
            steps += k
            if k < 2000:
                break
        q, t = s.get_state()
        runs[form] = {"device_s": ms * 1e-3, "steps": steps, "t_end": t,
                      "value": cells * steps / (ms * 1e-3), "ms_per_step": ms / steps}
        if form == "hybrid":
            runs[form]["indicator"] = s.hybrid_stats()
        states[form] = q
        s.close()
    if "fp64" in states:
        for form in forms:
            if form == "fp64":
                continue
            l1, linf = P.density_errors(p, states[form], states["fp64"])
            runs[form]["density_L1_vs_fp64"] = l1
            runs[form]["density_Linf_vs_fp64"] = linf
            runs[form]["speedup_vs_fp64"] = runs[form]["value"] / runs["fp64"]["value"]
    print(json.dumps({"metric": METRIC + " (whole runs to t = 0.8)", "unit": UNIT, "n_gpus": 1,
                      "config": {"workload": "euler2d_riemann4q_wenoz_rk3", "grid": f"{p.mx}x{p.my}", "t_end": T_END,
                                 "hybrid_schedule": {"indicator_every": HYB_EVERY, "judge_every": HYB_JUDGE_EVERY,
                                                     "judge_tol": 1e-3}},
                      "runs": runs}), flush=True)


def run_segments(args):
    """The hybrid whole run to T_END in segments of 0.1 (one JSON line per
    segment): steps, ms per step, the mean stage and indicator launch times
    (CUDA events per launch), and the indicator's flagged fraction of the
    faces at the segment's end, raw and after the stage kernel's 3 x 3
    dilation of same-direction faces."""
    import torch
    torch.cuda.set_device(0)
    from finess_b200 import problems as P
    indicator = load_indicator()
    p = P.riemann_params(n=args.n)
    q0 = P.riemann_init(p)
    s = make_solver(p, "hybrid", indicator)
    s.set_state(q0, 0.0)
    dtv = np.array([0.0, first_dt(p, s, q0), p.max_dt])

    def dilate(a):
        d = a.copy()
        d[1:, :] |= a[:-1, :]
        d[:-1, :] |= a[1:, :]
        e = d.copy()
        e[:, 1:] |= d[:, :-1]
        e[:, :-1] |= d[:, 1:]
        return e
    nx = (p.mx + 1) * p.my
    nseg = int(round(T_END / 0.1))
    for k in range(1, nseg + 1):
        s.set_kernel_timing(True)
        dtv, m = s.advance(0.1 * k if k < nseg else T_END, dtv, 1 << 30)
        ms = s.last_kernel_ms()
        kms, kl = s.kernel_time()
        ims, il = s.indicator_time()
        s.set_kernel_timing(False)
        f = s.hybrid_flags()
        fx, fy = f[:nx].reshape(p.mx + 1, p.my), f[nx:].reshape(p.mx, p.my + 1)
        st = s.hybrid_stats()
        print(json.dumps({"t": round(0.1 * k, 3), "steps": m, "ms_per_step": ms / max(m, 1),
                          "stage_kernel_ms": kms / max(kl, 1), "indicator_kernel_ms": ims / max(il, 1),
                          "flagged_raw": float((fx.sum() + fy.sum()) / f.size),
                          "flagged_dilated": float((dilate(fx).sum() + dilate(fy).sum()) / f.size),
                          "judges": st["judges"], "reverts": st["reverts"]}), flush=True)
    s.close()


def run_small(args):
    """Small single problems (config 1's isentropic vortex, FP64, WENO5-JS,
    SSP-RK3, to t = 10) through fin_advance, whose step control reads the
    CFL back to the host every step, and through a batch of one problem
    (step control on the device, each step one CUDA graph replay, the host
    polled every few steps); both must give the same state bit for bit."""
    import torch
    torch.cuda.set_device(0)
    from finess_b200 import problems as P
    from finess_b200.batch import Batch
    from finess_b200._abi import FIN_PREC_FP64
    for n in (64, 200, 512):
        p = P.vortex_params(n=n)
        p.precision = FIN_PREC_FP64
        q0 = P.vortex_exact(p, 0.0)
        s = make_solver(p, "fp64", None)
        s.set_state(q0, 0.0)
        dt0 = first_dt(p, s, q0)
        dtv, k = s.advance(10.0, np.array([0.0, dt0, p.max_dt]), 1 << 30)
        adv_ms = s.last_kernel_ms()
        qa, _ = s.get_state()
        s.close()
        with Batch([p]) as b:
            b.set_state(0, q0, 0.0)
            _, steps = b.solve(10.0, np.array([dt0]))
            bat_ms = b.stats()["device_ms"]
            qb, _ = b.get_state(0)
        print(json.dumps({"grid": f"{n}x{n}", "steps": int(k), "batch_steps": int(steps[0]),
                          "fin_advance_ms": adv_ms, "fin_advance_us_per_step": 1e3 * adv_ms / k,
                          "batch_of_one_ms": bat_ms, "batch_us_per_step": 1e3 * bat_ms / max(int(steps[0]), 1),
                          "bitwise_equal": bool(np.array_equal(qa, qb))}), flush=True)


def run_frames_bench(args):
    """RunFinpack's frame loop on the device (finess_b200.frames), then the
    reference's own Output (oracle/_ref/libfinref_io.so, one host thread) on
    the last frame's state: its time, and whether its file is byte-identical
    to the one this library wrote."""
    ws, rank, local = dist_env()
    if rank != 0:
        return
    import tempfile
    from finess_b200.frames import run_frames
    n = args.n if args.n != N_CELLS else 2048
    outdir = tempfile.mkdtemp(prefix="fin_frames_")
    out = run_frames("riemann", n, 4, 0.02, outdir, "fp64", False)
    q_last, t_last = out.pop("q_last"), out.pop("t_last")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import IoRefLib
    from finess_b200 import problems as P
    if IoRefLib.available():
        p = P.riemann_params(n=n)
        refdir = os.path.join(outdir, "reference")
        os.makedirs(refdir, exist_ok=True)
        w = time.perf_counter()
        IoRefLib().output(p, refdir, q_last, t_last, 4)
        out["reference_output_s"] = time.perf_counter() - w
        with open(os.path.join(outdir, "q%04d.dat" % 4), "rb") as a, \
                open(os.path.join(refdir, "q%04d.dat" % 4), "rb") as b:
            out["reference_frame_identical"] = a.read() == b.read()
    print(json.dumps(out), flush=True)


def run_sweep_bench(args):
    """The batched uneven sweep (1024 four-quadrant Riemann problems, N
    log-uniform in [64, 1024], FP32, SSP-RK3 to t = 0.25) with its problems
    split across the ranks by estimated work (finess_b200/sweep_ranks.py):
    no exchange between ranks; whole-job cell-updates/s over the slowest
    rank's device time (strong scaling)."""
    ws, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    from finess_b200 import replicas
    from finess_b200.batch import PRECISIONS
    from finess_b200.sweep_ranks import batch_solve, run_sweep_ranks
    replicas.init(ws, backend="nccl", timeout_s=300)
    out = run_sweep_ranks(1024, 0, rank, ws, batch_solve(0, PRECISIONS["fp32"], 0.25))
    if rank == 0:
        print(json.dumps({"metric": "2D Euler batched uneven sweep cell-updates/s (1024 problems, FP32)",
                          "value": out["cell_updates_per_s"], "unit": UNIT, "n_gpus": ws, "scaling": "strong",
                          "higher_is_better": True, "data": "synthetic", "dtype": "f32 (f64 state)",
                          "config": {"workload": "euler2d_riemann_sweep1024_rk3", "tend": 0.25, "seed": 0,
                                     "parallelism": f"problems split over {ws} ranks"},
                          "detail": out}), flush=True)
    replicas.finish()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--forms", default=None, help="comma list of fp64,fp32,hybrid (default: all available)")
    ap.add_argument("--n", type=int, default=N_CELLS)
    ap.add_argument("--window-t", type=float, default=WINDOW_T,
                    help="time of the headline run at which the warm-up and timed steps start")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-md", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--space-orders", action="store_true",
                    help="time the other spatial orders (LLF, WENO7/9/11) instead of the headline workload")
    ap.add_argument("--mpp", action="store_true",
                    help="time Lax-Wendroff with and without the MPP limiter instead of the headline workload")
    ap.add_argument("--whole-runs", action="store_true",
                    help="every form to t = 0.8 at full size, with the errors against the FP64 run")
    ap.add_argument("--frames", action="store_true",
                    help="frame files from device state, and the reference's Output on the last frame")
    ap.add_argument("--sweep", action="store_true",
                    help="the uneven 1024-problem sweep (FP32, to t = 0.25), its problems split across the ranks")
    ap.add_argument("--small", action="store_true",
                    help="small single problems (200^2 vortex and others) through fin_advance and a batch of one")
    ap.add_argument("--segments", action="store_true",
                    help="the hybrid whole run in segments of 0.1: per-segment cost and flagged fractions")
    ap.add_argument("--save-state", default=None, metavar="PATH",
                    help="profiling case: run the headline problem (first form of --forms) from t = 0 to "
                         "--window-t and save its state to PATH (.npz)")
    ap.add_argument("--load-state", default=None, metavar="PATH",
                    help="profiling case: W + K steps of the first form of --forms from the state saved at PATH "
                         "(few launches before a captured one)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.mpp:
        if args.steps == 50:
            args.steps = 20
        run_mpp(args)
        return
    if args.space_orders:
        if args.steps == 50:
            args.steps = 10
        run_space_orders(args)
        return
    if args.whole_runs:
        run_whole_runs(args)
        return
    if args.frames:
        run_frames_bench(args)
        return
    if args.sweep:
        run_sweep_bench(args)
        return
    if args.segments:
        run_segments(args)
        return
    if args.small:
        run_small(args)
        return
    if args.save_state or args.load_state:
        run_state_case(args)
        return
    if args.impl == "reference":
        run_reference_arm(args)
        return

    ws, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    from finess_b200 import replicas
    from finess_b200.replicas import barrier, max_over_ranks
    replicas.init(ws, backend="nccl", timeout_s=120)

    from finess_b200 import problems as P
    from finess_b200.solver import fma_peak_tflops
    indicator = load_indicator()
    forms = [f for f in (args.forms.split(",") if args.forms else FORMS) if f != "hybrid" or indicator]
    headline = "hybrid" if "hybrid" in forms else forms[0]
    p = P.riemann_params(n=args.n)
    q0 = P.riemann_init(p)
    cells = p.mx * p.my

    def window(s, dtv, tag):
        """W warm-up steps, then K timed steps (barrier + device sync on both
        sides, device time by CUDA events, max over ranks)."""
        dtv, nw = s.advance(T_END, dtv, args.warmup)
        warm_ms = s.last_kernel_ms()
        st0 = s.hybrid_stats() if tag == "hybrid" else None
        s.set_kernel_timing(True)
        l0 = s.launch_count()
        barrier()
        torch.cuda.nvtx.range_push(f"timed {tag}")   # lets a profiler select the timed launches
        dtv, nst = s.advance(T_END, dtv, args.steps)
        torch.cuda.nvtx.range_pop()
        dev_ms = s.last_kernel_ms()
        barrier()
        if nst != args.steps:
            raise RuntimeError(f"{tag}: only {nst} steps taken")
        dev_ms = max_over_ranks(dev_ms)
        kms, kl = s.kernel_time()
        ims, il = s.indicator_time() if tag == "hybrid" else (0.0, 0)
        s.set_kernel_timing(False)
        r = {"value": ws * cells * args.steps / (dev_ms * 1e-3), "ms_per_step": dev_ms / args.steps,
             "stage_kernel_ms": kms / kl, "launches": s.launch_count() - l0, "kernel_stats": (kms, kl),
             "warmup_steps": nw, "warmup_ms": warm_ms}
        if tag == "hybrid":
            st = s.hybrid_stats()
            r["indicator"] = {**st, "kernel_ms": ims / il if il else None, "launches_in_window": il,
                              "every": HYB_EVERY, "judge_every": HYB_JUDGE_EVERY,
                              "judges_in_window": st["judges"] - st0["judges"]}
        return dtv, r

    # ---- plain forms: K-step windows from t = 0 (their cost per step does
    # not depend on the state: every face takes full WENO) ----
    results, clocks, whole = {}, None, None
    for form in forms:
        if form == "hybrid":
            continue
        s = make_solver(p, form, indicator)
        s.set_state(q0, 0.0)
        _, results[form] = window(s, np.array([0.0, first_dt(p, s, q0), p.max_dt]), form)
        s.close()

    # ---- the hybrid: one whole run from t = 0 to T_END, with the warm-up and
    # the timed window starting at t = window_t; the segments before and after
    # the window are timed by CUDA events too, which gives the whole-run rate ----
    q_mid = None
    if "hybrid" in forms:
        s = make_solver(p, "hybrid", indicator)
        s.set_state(q0, 0.0)
        sampler = ClockSampler(local)
        sampler.start()
        dtv = np.array([0.0, first_dt(p, s, q0), p.max_dt])
        dtv, n1 = s.advance(args.window_t, dtv, 1 << 30)
        ms1 = s.last_kernel_ms()
        q_mid = torch.empty(ghosted_shape_of(p), dtype=torch.float64, pin_memory=True).numpy()
        _, t_mid = s.get_state(out=q_mid)
        dtv, r = window(s, dtv, "hybrid")
        n_w, ms_w = r.pop("warmup_steps"), r.pop("warmup_ms")
        ms_k = r["ms_per_step"] * args.steps
        dtv, n3 = s.advance(T_END, dtv, 1 << 30)
        ms3 = s.last_kernel_ms()
        clocks = sampler.stop()
        st = s.hybrid_stats()
        s.close()
        r["window_start_t"] = t_mid + 0.0
        results["hybrid"] = r
        steps_all = n1 + n_w + args.steps + n3
        ms_all = max_over_ranks(ms1 + ms_w + ms_k + ms3)
        whole = {"steps": steps_all, "device_s": ms_all * 1e-3, "t_end": T_END,
                 "value": ws * cells * steps_all / (ms_all * 1e-3), "judges": st["judges"], "reverts": st["reverts"],
                 "troubled_faces_last_indicator": st["troubled_faces"], "faces": st["faces"]}
        if "fp32" in results:
            # the judge step's cost is one full-WENO FP32 step (the fp32 form)
            jw = r["indicator"]["judges_in_window"]
            t_amort = r["ms_per_step"] * args.steps + (args.steps / HYB_JUDGE_EVERY - jw) * results["fp32"]["ms_per_step"]
            r["value_judge_amortized"] = ws * cells * args.steps / (t_amort * 1e-3)
    hr = results[headline]
    value = hr.get("value_judge_amortized", hr["value"])
    ms_per_step = ws * cells / value * 1e3
    launches = hr["launches"]
    kernel_stats = hr.pop("kernel_stats")
    for r in results.values():
        r.pop("kernel_stats", None)
        r.pop("warmup_steps", None)
        r.pop("warmup_ms", None)

    # ---- roofline of the headline form's stage kernel ----
    hbm, peak_kind = measured_peaks()
    avg_launch_ms = kernel_stats[0] / kernel_stats[1]
    alg_bytes_launch = cells * BYTES_PER_CELL_UPDATE / 3.0
    achieved = alg_bytes_launch / (avg_launch_ms * 1e-3) / 1e9
    tr = profile_traffic_bytes_per_cell(headline)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": (tr * cells) if tr is not None else None,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "kernel": ("k_stage_hyb (hybrid form" if headline == "hybrid" else f"k_stage ({headline} form")
                          + ": fused ConstructL + UpdateSoln + wave-speed maxima)",
                "avg_launch_ms": avg_launch_ms, "launches": kernel_stats[1]}
    try:
        pipe = {"fp64_fma_peak_tflops": fma_peak_tflops(True), "fp32_fma_peak_tflops": fma_peak_tflops(False)}
    except Exception:
        pipe = None

    # ---- e2e: host state in, K steps, host state out, through the C ABI,
    # from the same mid-run state as the timed window ----
    # The host state lives in pinned memory (allocated and filled before the
    # timed region); the first dt is an input of the frame, as dtv[1] is in
    # the reference's RunFinpack, so it is worked out before the timed region.
    s = make_solver(p, headline, indicator)
    q_in = q_mid
    if q_in is None:
        q_in = torch.empty(q0.shape, dtype=torch.float64, pin_memory=True).numpy()
        q_in[...] = q0
    t_in = results[headline].get("window_start_t", 0.0)
    q_out = torch.empty(q0.shape, dtype=torch.float64, pin_memory=True).numpy()
    dt0 = first_dt(p, s, q_in)
    barrier()
    t0 = time.perf_counter()
    s.set_state(q_in, t_in)
    s.advance(T_END, np.array([0.0, dt0, p.max_dt]), args.steps)
    s.get_state(out=q_out)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    s.close()
    state_bytes = q0.nbytes
    e2e = {"value": ws * cells * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": state_bytes / args.steps, "d2h_bytes_per_step": state_bytes / args.steps,
           "api": "fin_set_state + fin_advance(K steps) + fin_get_state on pinned host arrays in the reference's "
                  "ghosted layout (one FinSolveRK frame from the window's mid-run state)"}

    # ---- the same problem with the two-stage multiderivative stepper (FP64) ----
    md = None
    if not args.no_md:
        from finess_b200._abi import FIN_TS_MD
        pm = p.copy()
        pm.time_stepping_method, pm.time_order, pm.mbc = FIN_TS_MD, 4, 5
        qm = P.riemann_init(pm)
        sm = make_solver(pm, "fp64", None)
        sm.set_state(qm, 0.0)
        dtvm, _ = sm.advance(T_END, np.array([0.0, first_dt(pm, sm, qm), pm.max_dt]), args.warmup)
        barrier()
        dtvm, nm = sm.advance(T_END, dtvm, args.steps)
        md_ms = max_over_ranks(sm.last_kernel_ms())
        sm.close()
        md = {"value": ws * cells * nm / (md_ms * 1e-3), "unit": UNIT, "ms_per_step": md_ms / nm,
              "stepper": "FinSolveMD time_order 4 (two-stage Lax-Wendroff/PIF), FP64"}

    accuracy = None
    if rank == 0 and not args.no_accuracy:
        accuracy = accuracy_block(indicator, forms)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(n=args.n)
        except Exception as e:  # report, never fail the bench line
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": None, "sample": f"failed: {e}"}

    if rank == 0:
        fp64v = results["fp64"]["value"] if "fp64" in results else None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "fp32": "f32 (f64 state)", "hybrid": "f32 (f64 state) + bf16 indicator"}[headline],
            "data": "synthetic",
            "config": {"workload": "euler2d_riemann4q_wenoz_rk3", "grid": f"{p.mx}x{p.my}", "form": headline,
                       "weno": "Z", "time": "SSP-RK3", "cfl": 0.4, "t_end": T_END, "parallelism": f"replicas{ws}",
                       "window": (f"steps from t = {results[headline]['window_start_t']:.4f} of a whole hybrid "
                                  f"run to t = {T_END}; value has the judge step amortised over its period"
                                  if headline == "hybrid" else "steps from t = 0"),
                       "l2": "inputs larger than L2 (673 MB per state array)",
                       "hybrid_schedule": {"indicator_every": HYB_EVERY, "judge_every": HYB_JUDGE_EVERY,
                                           "judge_tol": 1e-3}},
            "forms": results,
            "whole_run": whole,
            "speedup_vs_fp64": (whole["value"] / fp64v) if (whole and fp64v) else
                               ((value / fp64v) if fp64v else None),
            "speedup_vs_fp64_window": (value / fp64v) if fp64v else None,
            "accuracy": accuracy,
            "roofline": roofline, "pipe": pipe, "cpu_baseline": cpu, "e2e": e2e, "md_stepper": md,
            "clocks": clocks, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    replicas.finish()


def run_state_case(args):
    """Profiling cases from a mid-run state: --save-state runs the headline
    problem from t = 0 to --window-t in one form and saves the state;
    --load-state takes W + K steps from such a state, so a profiler capture
    of a stage or indicator launch at that state follows only a few launches
    (the whole run to --window-t happens in another process)."""
    import torch
    torch.cuda.set_device(0)
    from finess_b200 import problems as P
    indicator = load_indicator()
    form = (args.forms or "hybrid").split(",")[0]
    p = P.riemann_params(n=args.n)
    s = make_solver(p, form, indicator)
    if args.save_state:
        q0 = P.riemann_init(p)
        s.set_state(q0, 0.0)
        dtv, k = s.advance(args.window_t, np.array([0.0, first_dt(p, s, q0), p.max_dt]), 1 << 30)
        q, t = s.get_state()
        np.savez(args.save_state, q=q, t=t, n=args.n)
        out = {"saved": args.save_state, "form": form, "grid": f"{p.mx}x{p.my}", "t": t, "steps": k}
    else:
        z = np.load(args.load_state)
        if int(z["n"]) != args.n:
            raise SystemExit(f"{args.load_state} holds a {int(z['n'])}^2 state; pass --n {int(z['n'])}")
        q, t = z["q"], float(z["t"])
        s.set_state(q, t)
        dtv = np.array([0.0, first_dt(p, s, q), p.max_dt])
        dtv, nw = s.advance(T_END + 1.0, dtv, args.warmup)
        s.set_kernel_timing(True)
        dtv, k = s.advance(T_END + 1.0, dtv, args.steps)
        kms, kl = s.kernel_time()
        out = {"loaded": args.load_state, "form": form, "grid": f"{p.mx}x{p.my}", "t_start": t, "steps": k,
               "ms_per_step": s.last_kernel_ms() / max(k, 1), "stage_kernel_ms": kms / max(kl, 1)}
        if form == "hybrid":
            ims, il = s.indicator_time()
            out["indicator_kernel_ms"] = ims / il if il else None
            out["hybrid_stats"] = s.hybrid_stats()
        s.set_kernel_timing(False)
    s.close()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
