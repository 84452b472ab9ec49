"""Replica plumbing for runs on several GPUs of one node.

One process per GPU, each stepping its own copy of the problem: the path has
no exchange between problems (a single problem split across GPUs would need
a halo exchange and a max-allreduce per stage, which is not built).  What the
ranks share is the timing protocol: a barrier and a device synchronise on
both sides of the timed region, the maximum of the per-rank times, and a
whole-job throughput of (units all ranks processed) / (that maximum).

The backend is NCCL on GPUs; the same functions run over gloo on the CPU.
"""
import datetime

import torch
import torch.distributed as dist

_state = {"ws": 1, "device": "cpu"}


def init(world_size, backend="nccl", timeout_s=120):
    """Join the process group (rendezvous from MASTER_ADDR / MASTER_PORT /
    RANK / WORLD_SIZE) when there is more than one rank.  A short timeout
    makes a rank that never arrives end the others' next collective with an
    error instead of a hang."""
    _state["ws"] = world_size
    _state["device"] = "cuda" if backend == "nccl" else "cpu"
    if world_size > 1:
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def barrier(device_sync=True):
    """All ranks arrive, then this rank's device work is finished."""
    if _state["ws"] > 1:
        dist.barrier()
    if device_sync and torch.cuda.is_available():
        torch.cuda.synchronize()


def _reduce(v, op):
    if _state["ws"] == 1:
        return float(v)
    t = torch.tensor([float(v)], device=_state["device"], dtype=torch.float64)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(v):
    """The largest value over all ranks (the job's time for a timed region)."""
    return _reduce(v, dist.ReduceOp.MAX)


def sum_over_ranks(v):
    return _reduce(v, dist.ReduceOp.SUM)


def throughput(units_this_rank, seconds_this_rank):
    """Whole-job units per second: every rank's units over the slowest
    rank's time."""
    return sum_over_ranks(units_this_rank) / max_over_ranks(seconds_this_rank)


def finish():
    if _state["ws"] > 1 and dist.is_initialized():
        dist.destroy_process_group()
    _state["ws"] = 1
