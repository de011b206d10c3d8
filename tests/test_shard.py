"""Host logic of query partitioning across ranks (openvkl_b200/shard.py):
slices cover the queries exactly once in order, and the all-gather of the
ranks' results equals the single-process result.  The multi-rank case runs
as two gloo processes on the CPU; the sampler stands in as a host function
(the GPU sampling itself is covered by the -m gpu tests)."""
import os

import numpy as np
import pytest

from openvkl_b200.shard import query_slice


@pytest.mark.parametrize("n,world", [(0, 1), (1, 2), (7, 3), (1000, 8), (1 << 20, 5)])
def test_slices_partition_in_order(n, world):
    bounds = [query_slice(n, r, world) for r in range(world)]
    assert bounds[0][0] == 0 and bounds[-1][1] == n
    for (a, b), (c, d) in zip(bounds, bounds[1:]):
        assert b == c
    sizes = [b - a for a, b in bounds]
    assert max(sizes) - min(sizes) <= 1


def test_bad_rank_rejected():
    with pytest.raises(ValueError):
        query_slice(10, 2, 2)


def _field(p):
    import torch
    return torch.sin(p[:, 0]) * p[:, 1] + p[:, 2]


def _worker(rank, world, port, n, q):
    import torch
    import torch.distributed as dist
    from openvkl_b200.shard import sample_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        g = torch.Generator().manual_seed(5)
        pts = torch.rand((n, 3), generator=g)
        full = sample_sharded(_field, pts, rank, world, gather_results=True)
        q.put((rank, bool(torch.equal(full, _field(pts)))))
    finally:
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, 10001, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    results = dict(q.get(timeout=10) for _ in procs)
    assert results == {0: True, 1: True}
