"""Replica runs over several GPUs of one node (one process per GPU).

The circuit workloads fit one B200 (<= 33 qubits complex128, 34 complex64),
so multi-GPU runs are replicas: every rank runs its own copy of the step on
its own GPU, with no data-path collective.  The only exchanges are a barrier
around the timed region and the maximum of the ranks' device times, from
which the whole-job throughput is units of all ranks / that maximum.

`init` reads RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* (torchrun's
environment) and uses NCCL when CUDA is available, gloo otherwise (the CPU
tests of this module run two gloo ranks).
"""
from __future__ import annotations

import datetime
import os


def init(backend: str | None = None, timeout_s: int = 120):
    """(world_size, rank, local_rank); joins the process group when
    world_size > 1 (short timeout, so a missing rank ends in an error)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def _device():
    import torch
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x: float, ws: int) -> float:
    """The maximum of x over all ranks (every rank gets it)."""
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        if dist.get_backend() == "nccl":
            import torch
            dist.barrier(device_ids=[torch.cuda.current_device()])
        else:
            dist.barrier()


def done(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def job_throughput(units_per_rank: float, ws: int, seconds_max: float) -> float:
    """Whole-job rate: every rank processed units_per_rank in at most
    seconds_max (the slowest rank's device time)."""
    return units_per_rank * ws / seconds_max
