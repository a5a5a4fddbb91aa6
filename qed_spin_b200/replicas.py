"""Replica plumbing for runs on several GPUs of one node: the path has no cross-GPU exchange (each replica
solves its own sector), so N processes, one per GPU, run independent replicas; the only collectives are a
barrier around the timed region and the max over ranks of the measured times.

The backend is NCCL on GPUs and gloo on CPU (the tests drive the same code with gloo ranks). The rendezvous
reads RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT (torchrun sets them).
"""
from __future__ import annotations

import datetime
import os


def world() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 300) -> tuple[int, int, int]:
    """Joins the process group when the world has more than one rank; NCCL ranks bind their local GPU."""
    size, rank, local = world()
    if size > 1:
        import torch
        import torch.distributed as dist
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return size, rank, local


def barrier(size: int) -> None:
    if size > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, size: int) -> float:
    """The maximum of a per-rank time over all ranks (every rank gets it)."""
    if size == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, size: int, seconds_max: float) -> float:
    """Units per second of the whole job: every rank's units over the slowest rank's time (weak scaling)."""
    return size * units_per_rank / seconds_max


def finish(size: int) -> None:
    if size > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
