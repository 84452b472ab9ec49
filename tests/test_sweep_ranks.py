"""The uneven sweep split across ranks (finess_b200/sweep_ranks.py) on the
CPU: the longest-processing-time split covers every problem once and
balances the estimated work, and two gloo ranks, each solving its share,
give exactly the results of one rank solving everything.  The per-rank solve
here is the oracle's FinSolveRK on small grids (the split and the timing
protocol are what is tested; the GPU batch is tested in test_gpu_batch.py)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from finess_b200.sweep_ranks import partition, problem_sizes

SEED, N_PROB, NMIN, NMAX, TEND = 3, 7, 8, 20, 0.02


def test_partition_covers_every_problem_once_and_balances():
    sizes = problem_sizes(1024, 0)
    assert min(sizes) >= 64 and max(sizes) <= 1024
    costs = [float(N) ** 3 for N in sizes]
    for world in (1, 2, 3, 4, 8):
        parts, load = partition(costs, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(1024))
        assert max(load) / (sum(load) / world) <= 1.02
        assert np.isclose(sum(load), sum(costs))


def test_partition_more_ranks_than_problems():
    parts, load = partition([8.0, 1.0], 4)
    assert parts == [[0], [1], [], []]


def oracle_solve(indices, keep_states=False):
    """FinSolveRK of the oracle (the C restatement) on problems of the small sweep."""
    import time
    from oracle import Oracle
    from finess_b200.batch import first_dt, sweep_problem
    from finess_b200._abi import FIN_PREC_FP64
    o = Oracle()
    t0 = time.perf_counter()
    states, steps = [], []
    for k in indices:
        p, q = sweep_problem(SEED, k, nmin=NMIN, nmax=NMAX, precision=FIN_PREC_FP64)
        q = o.set_bnd(p, q)
        rc, q1, t1, dt1, n = o.finsolve(p, q, 0.0, TEND, first_dt(p, q))
        assert rc == 0
        states.append(q1)
        steps.append(n)
    from finess_b200 import replicas
    replicas.barrier(device_sync=False)
    return time.perf_counter() - t0, steps, states if keep_states else []


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    from finess_b200 import replicas
    from finess_b200.sweep_ranks import run_sweep_ranks
    try:
        replicas.init(ws, backend="gloo", timeout_s=60)
        sizes = problem_sizes(N_PROB, SEED, NMIN, NMAX)
        out = run_sweep_ranks(N_PROB, SEED, rank, ws, oracle_solve, sizes=sizes, keep_states=True)
        q.put((rank, out))
    except Exception as e:
        q.put((rank, "error: " + repr(e)))
    finally:
        replicas.finish()


def test_two_gloo_ranks_equal_one_rank():
    from finess_b200 import replicas
    from finess_b200.sweep_ranks import run_sweep_ranks
    replicas.init(1, backend="gloo")
    sizes = problem_sizes(N_PROB, SEED, NMIN, NMAX)
    one = run_sweep_ranks(N_PROB, SEED, 0, 1, oracle_solve, sizes=sizes, keep_states=True)
    replicas.finish()
    ctx = mp.get_context("spawn")
    qq = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, qq)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(qq.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    for r in (0, 1):
        assert not isinstance(res[r], str), res[r]
        two = res[r]
        assert two["ranks"] == 2 and one["ranks"] == 1
        assert two["cell_updates"] == one["cell_updates"]
        assert sorted(two["results"]) == list(range(N_PROB))
        for k in range(N_PROB):
            assert two["results"][k][1] == one["results"][k][1]              # steps
            assert np.array_equal(two["results"][k][0], one["results"][k][0])   # final state, bit for bit
    assert res[0]["problems_this_rank"] + res[1]["problems_this_rank"] == N_PROB
