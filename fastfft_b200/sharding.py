"""Template sharding across GPUs (one process per GPU, torch.distributed for plumbing).

Templates are independent units: rank r of W correlates templates [start, stop) of the
batch against its own copy of the image spectrum (prepared locally from the replicated
image, so the data path has no collective).  Only the per-template results that a search
keeps -- here (peak value, peak index) pairs -- are gathered, which is a few bytes per
template.
"""
from __future__ import annotations


def shard_range(n_items: int, world_size: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced [start, stop) of n_items for rank (sizes differ by at most one)."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("bad world_size / rank")
    base, extra = divmod(n_items, world_size)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _dist():
    import torch.distributed as dist

    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(value: float, device=None) -> float:
    """Max of a scalar over all ranks (the elapsed-time rule for multi-GPU timing)."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_peaks(values, indices, n_total: int, device=None):
    """Gather per-template (peak value, peak index) of every rank's shard, in template order.

    values/indices: 1D tensors for this rank's shard_range(n_total, W, rank) templates.
    Returns two tensors of length n_total (on `device`).
    """
    import torch

    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return values, indices
    world = dist.get_world_size()
    cap = shard_range(n_total, world, 0)[1]  # largest shard
    v = torch.zeros(cap, dtype=torch.float64, device=device)
    i = torch.full((cap,), -1, dtype=torch.int64, device=device)
    v[: values.numel()] = values.to(torch.float64)
    i[: indices.numel()] = indices.to(torch.int64)
    vs = [torch.empty_like(v) for _ in range(world)]
    is_ = [torch.empty_like(i) for _ in range(world)]
    dist.all_gather(vs, v)
    dist.all_gather(is_, i)
    out_v, out_i = [], []
    for r in range(world):
        a, b = shard_range(n_total, world, r)
        out_v.append(vs[r][: b - a])
        out_i.append(is_[r][: b - a])
    return torch.cat(out_v), torch.cat(out_i)
