"""Query partitioning across GPUs: one process per GPU, each holding its own
committed copy of the volume (a replica) and sampling a contiguous slice of
the query points.  Sampling has no exchange step, so the data path needs no
collective; `gather` is only for callers that want every result on every
rank (an all-gather over the process group: NCCL over NVLink on GPUs, gloo
on CPU).
"""
from __future__ import annotations


def query_slice(n: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of rank's share of n queries: contiguous, in rank order,
    sizes differing by at most one (the first n % world ranks take one
    more)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of size {world}")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def gather(local, n: int, group=None):
    """All-gathers the ranks' result slices (tensors of shape (count, ...)
    laid out by query_slice) into one tensor of n rows on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rows = max(query_slice(n, r, world)[1] - query_slice(n, r, world)[0] for r in range(world))
    pad = torch.zeros((rows,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([parts[r][:query_slice(n, r, world)[1] - query_slice(n, r, world)[0]]
                      for r in range(world)])


def sample_sharded(sample_fn, points, rank: int, world: int, gather_results: bool = False, group=None):
    """Runs sample_fn (e.g. Sampler.sample or Sampler.gradient) on this rank's
    slice of `points`; returns the slice's results, or all results when
    gather_results is set."""
    start, stop = query_slice(points.shape[0], rank, world)
    local = sample_fn(points[start:stop])
    return gather(local, points.shape[0], group) if gather_results else local
