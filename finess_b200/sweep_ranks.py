"""The uneven batch sweep split across the GPUs of one node.

The sweep's problems are independent, so the split needs no exchange on the
data path: each rank (one process per GPU) runs its share of the problems in
its own batch (one persistent launch per stage, fin_batch_*), and the ranks
share only the replica timing protocol (a barrier and device synchronise on
both sides, the maximum of the per-rank device times; finess_b200/replicas.py).

The problems are dealt out by estimated cost with the longest-processing-time
rule (largest first, each to the rank with the least work so far): a problem
of N x N cells run to a fixed end time at a fixed CFL number takes a number
of steps proportional to N, so its work is proportional to N^3.  Whole-job
throughput is all ranks' cell-updates over the slowest rank's device time
(strong scaling: the total work is fixed).

    python -m torch.distributed.run --nproc-per-node N -m finess_b200.sweep_ranks [--n 1024] [--precision fp32]
"""
import argparse
import json

import numpy as np

from . import replicas
from .batch import PRECISIONS, _sweep_grid


def problem_sizes(n, seed, nmin=64, nmax=1024):
    """Grid size N of each of the n problems of the sweep of a seed."""
    return [_sweep_grid(seed, k, nmin, nmax).mx for k in range(n)]


def partition(costs, world):
    """Problem indices per rank, by the longest-processing-time rule; ties go
    to the lower rank and, within a rank, indices are sorted."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for k in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda w: (load[w], w))
        parts[r].append(k)
        load[r] += costs[k]
    return [sorted(p) for p in parts], load


def batch_solve(seed, precision, tend, nmin=64, nmax=1024):
    """The default per-rank solve: this rank's problems in one batch on the
    current GPU.  Returns f(indices) -> (device seconds, steps per problem,
    final states per problem)."""
    def solve(indices, keep_states=False):
        from .batch import HYB_EVERY, HYB_JUDGE_EVERY, HYB_JUDGE_TOL, Batch, first_dt, load_indicator, sweep_problem
        if not indices:   # the same collectives as the other ranks, no work
            replicas.barrier()
            replicas.barrier()
            return 0.0, [], []
        probs = [sweep_problem(seed, k, nmin, nmax, precision=precision) for k in indices]
        with Batch([p for p, _ in probs]) as b:
            if precision == PRECISIONS["hybrid"]:
                W, z = load_indicator()
                b.set_indicator(W, z, HYB_JUDGE_EVERY, HYB_JUDGE_TOL, HYB_EVERY)
            dts = np.zeros(len(probs))
            for i, (p, q) in enumerate(probs):
                dts[i] = first_dt(p, q)
                b.set_state(i, q)
            replicas.barrier()
            _, steps = b.solve(tend, dts)
            replicas.barrier()
            dev_s = b.stats()["device_ms"] * 1e-3
            states = [b.get_state(i)[0] for i in range(len(probs))] if keep_states else []
        return dev_s, [int(s) for s in steps], states
    return solve


def run_sweep_ranks(n, seed, rank, world, solve, sizes=None, keep_states=False):
    """This rank's share of the sweep through solve(indices, keep_states).
    Returns a dict of the whole job's figures (the same on every rank) and,
    with keep_states, every problem's final state gathered on every rank
    (outside the timed region; a check of the split, not part of a run)."""
    import torch.distributed as dist
    sizes = problem_sizes(n, seed) if sizes is None else sizes
    parts, load = partition([float(N) ** 3 for N in sizes], world)
    mine = parts[rank]
    dev_s, steps, states = solve(mine, keep_states)
    cu = float(sum(sizes[k] * sizes[k] * s for k, s in zip(mine, steps)))
    out = {"problems": n, "ranks": world, "problems_this_rank": len(mine),
           "cell_updates": replicas.sum_over_ranks(cu), "device_s_max": replicas.max_over_ranks(dev_s),
           "load_imbalance": max(load) / (sum(load) / world) if sum(load) > 0 else 1.0}
    out["cell_updates_per_s"] = out["cell_updates"] / out["device_s_max"] if out["device_s_max"] > 0 else None
    if keep_states:
        mine_res = {k: (st, s) for k, st, s in zip(mine, states, steps)}
        if world > 1:
            allres = [None] * world
            dist.all_gather_object(allres, mine_res)
        else:
            allres = [mine_res]
        merged = {}
        for d in allres:
            merged.update(d)
        out["results"] = merged
    return out


def main():
    import os
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--tend", type=float, default=0.25)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", default="fp32", choices=sorted(PRECISIONS))
    a = ap.parse_args()
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    replicas.init(ws, backend="nccl", timeout_s=300)
    out = run_sweep_ranks(a.n, a.seed, rank, ws, batch_solve(a.seed, PRECISIONS[a.precision], a.tend))
    if rank == 0:
        print(json.dumps(dict(out, precision=a.precision, tend=a.tend, seed=a.seed, scaling="strong")))
    replicas.finish()


if __name__ == "__main__":
    main()
