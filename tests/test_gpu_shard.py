"""Query partitioning (openvkl_b200/shard.py) on the device's own sampler.

Each rank of a world of 2 or 3 samples its contiguous slice of the points
through vklComputeSampleN / vklComputeGradientN; here the ranks run one after
another on one GPU (sampling has no exchange step, so a rank's result does
not depend on the others running).  The concatenation in rank order must
equal the single call bit for bit, for a dense volume with the texture atlas
and for a sparse VDB, samples and gradients."""
import numpy as np
import pytest

from openvkl_b200.fields import shell_leaves, sinusoid_field_torch
from openvkl_b200.shard import query_slice, sample_sharded
from tests.conftest import bits

pytestmark = pytest.mark.gpu


def _volumes(vkl, device):
    dense = vkl.structured_regular(device, sinusoid_field_torch((200, 180, 160), seed=4), shared=True)
    origins, values = shell_leaves(domain=128, shells=2, thickness=0.06, seed=8)
    L = len(origins)
    sparse = vkl.vdb_volume(device, np.full(L, 3), origins, np.ones(L), packed_dense=values)
    return [(dense, (200, 180, 160)), (sparse, (128, 128, 128))]


@pytest.mark.parametrize("world", [2, 3])
def test_rank_slices_concatenate_to_single_call(vkl, device, world):
    import torch
    for vol, dims in _volumes(vkl, device):
        smp = vkl.Sampler(vol, filter=100, gradient_filter=100)
        g = torch.Generator(device="cuda").manual_seed(world)
        n = (1 << 22) + 13
        hi = torch.tensor(dims, dtype=torch.float32, device="cuda")
        pts = (torch.rand((n, 3), generator=g, device="cuda") * (hi + 2) - 1).contiguous()
        for fn in (smp.sample, smp.gradient):
            whole = fn(pts)
            parts = [sample_sharded(fn, pts, r, world) for r in range(world)]
            assert sum(p.shape[0] for p in parts) == n
            assert [query_slice(n, r, world)[1] - query_slice(n, r, world)[0] for r in range(world)] == \
                [p.shape[0] for p in parts]
            got = torch.cat(parts)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(bits(got.cpu().numpy()), bits(whole.cpu().numpy()))
