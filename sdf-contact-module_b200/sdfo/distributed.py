"""Multi-GPU plumbing for the SDF hot path: replicas and independent shards.

Every unit of work here is independent -- a query point, a contact pose, a
mesh to build -- so N GPUs run N replicas of the grid (it is small next to
180 GB of HBM) and split the batch; nothing crosses NVLink on the data path.
The only collective is a scalar reduction used to time a step as the slowest
rank (``max_over_ranks``), or to gather per-shard results when a caller wants
them on one rank (``gather_rows``).  torch.distributed provides the process
group (NCCL on GPUs, Gloo on CPU).
"""
from __future__ import annotations


def shard_range(n: int, rank: int, world: int):
    """Contiguous [start, stop) slice of n units owned by `rank` of `world`
    (sizes differ by at most one; every unit is owned exactly once)."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(int(n), world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _device_for_backend():
    import torch
    import torch.distributed as dist

    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """All-reduce MAX of a Python float (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(local, total_rows: int):
    """All-gather per-rank row blocks of a 2-D tensor sharded with shard_range
    into the full (total_rows, ...) tensor on every rank."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return local
    world = dist.get_world_size()
    dev = _device_for_backend()
    spans = [shard_range(total_rows, r, world) for r in range(world)]
    rows = max(b - a for a, b in spans)
    width = tuple(local.shape[1:])
    # equal-size blocks (padded to the largest shard), trimmed after the gather
    pad = torch.zeros((rows,) + width, dtype=local.dtype, device=dev)
    pad[: local.shape[0]] = local.to(dev)
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    return torch.cat([p[: b - a] for p, (a, b) in zip(parts, spans)], 0)
