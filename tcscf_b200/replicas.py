"""Replica plumbing for multi-GPU runs: one process per GPU, each running the same Fock build on its
own device with no data-path collective (the build's r1 rows are independent, but one build is not
split across GPUs here), timed as the maximum over ranks.

The reference has no MPI or collective call site (one process, one device per SCF in
src/HartreeFock.cpp); N processes under torchrun are N independent builds, so the whole-job figure
is the slowest rank's time divided by the builds all ranks completed.
"""
from __future__ import annotations

import datetime
import os


def env_ranks() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment; (0, 1, 0) without it."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def init(world: int, local_rank: int, timeout_s: float = 600.0, backend: str | None = None) -> str | None:
    """Join the process group when world > 1: NCCL on a GPU node, gloo where no GPU is visible.
    Returns the backend used (None for a single process)."""
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist

    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local_rank)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return backend


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The largest `value` over all ranks (every rank takes this step, in the same order)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_seconds_per_build(max_total_ms: float, steps: int, world: int) -> float:
    """Seconds per build for the whole job: the slowest rank's time for its `steps` builds, divided
    by the steps x world builds all ranks completed (weak scaling: work per rank is fixed)."""
    return max_total_ms / 1e3 / (steps * world)


def finalize(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        if dist.is_initialized():
            dist.destroy_process_group()
