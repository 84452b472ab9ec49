"""The replica timing protocol of bench.py --gpus N (finess_b200/replicas.py)
with two ranks over gloo on the CPU: barrier, max over ranks, whole-job
throughput, and a rank that never arrives ending the other's wait with an
error instead of a hang."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q, absent):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    from finess_b200 import replicas
    try:
        replicas.init(ws, backend="gloo", timeout_s=5 if absent is not None else 60)
        if absent is not None and rank == absent:
            q.put((rank, "left"))
            return                       # leaves between steps: no collective of its own in flight
        replicas.barrier(device_sync=False)
        t = 0.25 * (rank + 1)            # rank-dependent "device time"
        out = (replicas.max_over_ranks(t), replicas.throughput(1000.0 * (rank + 1), t))
        replicas.barrier(device_sync=False)
        q.put((rank, out))
    except Exception as e:              # the collective ran out of time
        q.put((rank, "error: " + type(e).__name__))
    finally:
        if absent is None:
            replicas.finish()


def _run(ws, absent=None):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q, absent)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return res


def test_two_ranks_max_and_throughput():
    res = _run(2)
    for r in (0, 1):
        mx, thr = res[r]
        assert mx == 0.5                                # max(0.25, 0.5)
        assert thr == pytest.approx(3000.0 / 0.5)       # (1000 + 2000) units / slowest time


def test_absent_rank_ends_the_wait_with_an_error():
    res = _run(2, absent=1)
    assert res[1] == "left"
    assert isinstance(res[0], str) and res[0].startswith("error")


def test_single_rank_needs_no_process_group():
    from finess_b200 import replicas
    replicas.init(1, backend="gloo")
    assert replicas.max_over_ranks(0.3) == 0.3
    assert replicas.throughput(600.0, 0.3) == pytest.approx(2000.0)
    replicas.finish()
