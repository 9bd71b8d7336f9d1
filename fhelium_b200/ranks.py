"""Rank plumbing of multi-GPU runs: one process per GPU.

Ciphertexts are independent and keys are read-only, so a batch splits across
ranks with no exchange on the data path (weak scaling when every rank keeps
its own batch, strong when a global batch is sharded).  The only collectives
are a barrier on each side of a timed region and a max-reduction of the
per-rank device times; every rank issues them in the same order.  The
process group is created with a short timeout so that ranks waiting on one
that died end with an error instead of waiting for good.
"""

from __future__ import annotations

import datetime
import os

import torch


def init(backend: str | None = None, timeout_s: float = 300.0) -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment; joins the
    process group when the world size is above one (NCCL on GPUs unless
    `backend` says otherwise)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        backend = backend or "nccl"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def barrier(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, ws: int, device: torch.device | str = "cpu") -> float:
    """The largest `x` over all ranks (the job's time is its slowest rank's)."""
    if ws == 1:
        return float(x)
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(total: int, ws: int, rank: int) -> tuple[int, int]:
    """[start, end) of rank's share of `total` items: contiguous, disjoint,
    covering, sizes differing by at most one."""
    if ws < 1 or not 0 <= rank < ws:
        raise ValueError("need 0 <= rank < world size")
    base, extra = divmod(total, ws)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def job_rate(items_per_rank: int, ws: int, max_ms: float) -> float:
    """Whole-job throughput: all ranks' items over the slowest rank's time."""
    return ws * items_per_rank / (max_ms / 1000.0)


def finish(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
