"""Multi-GPU plumbing for independent scenes: one process per GPU, no collective on the data
path. Scenes shard across ranks (each rank owns its own seeded scenes: weak scaling, or a
contiguous slice of a fixed list: strong scaling); ranks meet only at barriers and at the
max/sum reductions of the timings and counts (`torch.distributed`, NCCL on GPUs, gloo on
CPU)."""
from __future__ import annotations

import datetime
import os


def init(backend: str | None = None, timeout_s: float = 300.0):
    """(world_size, rank, local_rank); joins the process group when world_size > 1."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return ws, rank, local


def rank_seed(base: int, rank: int) -> int:
    """Seed of a rank's own scenes under weak scaling (distinct per rank)."""
    return base + 1000 * rank


def shard(n_total: int, rank: int, world: int) -> range:
    """Contiguous slice of a fixed scene list owned by `rank` (strong scaling)."""
    per, extra = divmod(n_total, world)
    lo = rank * per + min(rank, extra)
    return range(lo, lo + per + (1 if rank < extra else 0))


def _reduce(x: float, op: str) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def reduce_max(x: float) -> float:
    return _reduce(x, "max")


def reduce_sum(x: float) -> float:
    return _reduce(x, "sum")


def barrier():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def finalize():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
