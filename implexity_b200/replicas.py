"""Independent replicas over torch.distributed.

The solver does not shard (no domain decomposition): with N GPUs every rank
runs its own replica of the workload, and only the timing is combined -- the
slowest rank's device time bounds the job.  One process per GPU; the process
group carries the barrier and the max-reduction of the per-rank times.
"""
from __future__ import annotations

import os
from datetime import timedelta


def env_rank() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0) -> tuple[int, int, int]:
    """Joins the process group when WORLD_SIZE > 1 (env:// rendezvous)."""
    rank, world, local = env_rank()
    if world > 1:
        import torch
        import torch.distributed as dist

        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
    return rank, world, local


def _device(backend: str):
    import torch

    return torch.device("cuda") if backend == "nccl" else torch.device("cpu")


def max_over_ranks(value: float) -> float:
    """Maximum of a per-rank scalar (times are taken as the slowest rank)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device(dist.get_backend()))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist

    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def finalize() -> None:
    import torch.distributed as dist

    if dist.is_initialized():
        dist.destroy_process_group()
