"""Benchmark of the B200 WENO right-hand side + SSP-RK3 stepper.

Workload (one "step" = one full SSP-RK3 time step with FinSolveRK's adaptive
dt and CFL check): the 2D Euler four-quadrant Riemann problem on [0,1]^2,
4096 x 4096 cells, transmissive boundaries, interface (0.8, 0.8), WENO5-Z,
global LLF with characteristic projection, CFL 0.4.  Synthetic closed-form
initial data; the state (673 MB per FP64 array) is far larger than the 126 MB
L2, so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form fp64|fp32]

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
BYTES_PER_CELL_UPDATE = {"fp64": 320.0, "fp32": 320.0}
BYTES_PER_CELL_PER_LAUNCH = {1: 80.0, 2: 120.0, 3: 120.0}


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
    """Per-cell DRAM traffic of one stage launch from the committed ncu summary
    (profiles/stage_kernel_*.txt, line 'dram_bytes_per_cell_<form>: X')."""
    import glob
    for f in sorted(glob.glob(os.path.join(ROOT, "profiles", "stage_kernel_*.txt"))):
        for line in open(f):
            if line.startswith(f"dram_bytes_per_cell_{form}:"):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    pass
    return None


def build_problem(n, form):
    from finess_b200 import problems as P
    from finess_b200._abi import FIN_PREC_FP32, FIN_PREC_FP64, FIN_WENO_Z
    p = P.riemann_params(n=n, weno=FIN_WENO_Z)
    p.precision = FIN_PREC_FP32 if form == "fp32" else FIN_PREC_FP64
    q0 = P.riemann_init(p)
    return p, q0


def cpu_baseline(seconds_target=15.0, n=512):
    """The reference's own CPU code (oracle/_ref, all host threads) -- or the C
    restatement when oracle/_ref is absent -- on a bounded sample: SSP-RK3
    steps of the same problem at n x n."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle, RefLib
    from finess_b200 import problems as P
    from finess_b200._abi import FIN_WENO_Z
    p = P.riemann_params(n=n, weno=FIN_WENO_Z)
    q = P.riemann_init(p)
    if RefLib.available():
        impl, kind = RefLib(), "reference"
        q = impl.set_bnd(p, q)
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    else:
        impl, kind = Oracle(), "port"
        q = impl.set_bnd(p, q)
        cores = 1
    t = 0.0
    dt = 0.4 * (1.0 / n) / 3.0
    steps, elapsed = 0, 0.0
    while elapsed < seconds_target and steps < 200:
        t0 = time.perf_counter()
        out = impl.finsolve(p, q, t, t + dt, dt)   # one step (tend = t + dt)
        elapsed += time.perf_counter() - t0
        q, t = out[1], out[2]
        steps += 1
    value = n * n * steps / elapsed
    return {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{steps} SSP-RK3 steps of the same problem (WENO5-Z, 4-quadrant Riemann) at {n}x{n}, "
                      f"{elapsed:.1f} s"}


def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle, RefLib
    from finess_b200 import problems as P
    from finess_b200._abi import FIN_WENO_Z
    n = 512
    p = P.riemann_params(n=n, weno=FIN_WENO_Z)
    q = P.riemann_init(p)
    if RefLib.available():
        impl, kind, cores = RefLib(), "reference", int(os.environ["OMP_NUM_THREADS"])
    else:
        impl, kind, cores = Oracle(), "port", 1
    q = impl.set_bnd(p, q)
    t = 0.0
    dtv1 = 0.4 * (1.0 / n) / 3.0
    for _ in range(args.warmup):
        out = impl.finsolve(p, q, t, t + dtv1, dtv1)
        q, t = out[1], out[2]
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out = impl.finsolve(p, q, t, t + dtv1, dtv1)
        q, t = out[1], out[2]
    el = time.perf_counter() - t0
    value = n * n * args.steps / el
    sample = f"{args.steps} SSP-RK3 steps of the same problem at {n}x{n} (bounded sample of the 4096^2 workload)"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "euler2d_riemann4q_wenoz_rk3", "grid": f"{n}x{n}", "sample_of": "4096x4096",
                   "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--n", type=int, default=N_CELLS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-md", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference_arm(args)
        return

    ws, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from finess_b200.solver import Solver, fma_peak_tflops
    p, q0 = build_problem(args.n, args.form)
    cells = p.mx * p.my
    s = Solver(p)
    s.set_state(q0, 0.0)
    tend = 0.8
    # initial_dt of parameters.ini chosen for this grid: desired CFL at the
    # initial maximum wave speed
    a1, a2 = s.GlobalWaveSpd(q0)
    dt0 = p.desired_cfl * min((p.xhigh - p.xlow) / p.mx, (p.yhigh - p.ylow) / p.my) / max(a1, a2)
    s.set_state(q0, 0.0)
    dtv = np.array([0.0, dt0, p.max_dt])
    dtv, _ = s.advance(tend, dtv, args.warmup)

    # ---- timed region: K steps, device-resident state ----
    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    s.set_kernel_timing(True)
    l0 = s.launch_count()
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    dtv, nst = s.advance(tend, dtv, args.steps)
    dev_ms = s.last_kernel_ms()
    barrier()
    clocks = sampler.stop()
    launches = s.launch_count() - l0
    kms, klaunches = s.kernel_time()
    s.set_kernel_timing(False)
    if nst != args.steps:
        raise RuntimeError(f"only {nst} steps taken")
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([dev_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = float(t.item())
    value = ws * cells * args.steps / (dev_ms * 1e-3)
    ms_per_step = dev_ms / args.steps

    # ---- roofline of the stage kernel ----
    hbm, peak_kind = measured_peaks()
    avg_launch_ms = kms / klaunches
    alg_bytes_launch = cells * BYTES_PER_CELL_UPDATE[args.form] / 3.0
    achieved = alg_bytes_launch / (avg_launch_ms * 1e-3) / 1e9
    tr = profile_traffic_bytes_per_cell(args.form)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": (tr * cells) if tr is not None else None,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "kernel": "k_stage (fused ConstructL + UpdateSoln + wave-speed maxima)",
                "avg_launch_ms": avg_launch_ms, "launches": klaunches}
    # FP64 / FP32 pipe: measured FMA peak of this GPU
    try:
        pk64 = fma_peak_tflops(True)
        pk32 = fma_peak_tflops(False)
    except Exception:
        pk64 = pk32 = None
    pipe = {"fp64_fma_peak_tflops": pk64, "fp32_fma_peak_tflops": pk32}

    # ---- e2e: host state in, K steps, host state out, through the C ABI ----
    qh = q0
    e2e_s = None
    if True:
        qbuf = np.empty_like(q0)
        barrier()
        t0 = time.perf_counter()
        s.set_state(qh, 0.0)
        dtv2, n2 = s.advance(tend, np.array([0.0, dt0, p.max_dt]), args.steps)
        qout, _ = s.get_state()
        barrier()
        e2e_s = time.perf_counter() - t0
        if ws > 1:
            import torch.distributed as dist
            t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        del qbuf
    state_bytes = q0.nbytes
    e2e = {"value": ws * cells * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": state_bytes / args.steps, "d2h_bytes_per_step": state_bytes / args.steps,
           "api": "fin_set_state + fin_advance(K steps) + fin_get_state on host arrays (one FinSolveRK frame)"}

    # ---- the same problem with the two-stage multiderivative (Lax-Wendroff /
    # PIF) stepper, FP64 (device-resident, same K) ----
    md = None
    if args.form == "fp64" and not args.no_md:
        from finess_b200._abi import FIN_TS_MD
        pm = p.copy()
        pm.time_stepping_method, pm.time_order, pm.mbc = FIN_TS_MD, 4, 5
        from finess_b200 import problems as P
        qm = P.riemann_init(pm)
        sm = Solver(pm)
        sm.set_state(qm, 0.0)
        dtvm, _ = sm.advance(tend, np.array([0.0, dt0, pm.max_dt]), args.warmup)
        barrier()
        dtvm, nm = sm.advance(tend, dtvm, args.steps)
        md_ms = sm.last_kernel_ms()
        sm.close()
        md = {"value": cells * nm / (md_ms * 1e-3), "unit": UNIT, "ms_per_step": md_ms / nm,
              "stepper": "FinSolveMD time_order 4 (two-stage Lax-Wendroff/PIF)"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline()
        except Exception as e:  # report, never fail the bench line
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": None, "sample": f"failed: {e}"}
    s.close()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": "euler2d_riemann4q_wenoz_rk3", "grid": f"{p.mx}x{p.my}", "form": args.form,
                       "weno": "Z", "time": "SSP-RK3", "cfl": 0.4, "parallelism": f"replicas{ws}",
                       "l2": "inputs larger than L2 (673 MB per state array)"},
            "roofline": roofline, "pipe": pipe, "cpu_baseline": cpu, "e2e": e2e, "md_stepper": md,
            "clocks": clocks, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
