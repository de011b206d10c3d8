"""Batched multi-volume sampling (vklCudaNewSampleBatch; an extension).

A batch of jobs over many volumes must give, bit for bit, the samples and
gradients of the per-job vklComputeSampleN / vklComputeGradientN calls:
fused classes (dense voxel types, plain sparse leaves, trilinear) and the
jobs that fall back to plain launches inside the graph (tricubic, nearest,
compressed leaves), uneven point counts including 0 and 1, points outside
the volumes, outputs of only one kind, repeated runs and autotuned
configurations.
"""
import numpy as np
import pytest

from openvkl_b200.fields import shell_leaves, sinusoid_field
from tests.conftest import bits

pytestmark = pytest.mark.gpu


def _volumes(vkl, device):
    rng = np.random.default_rng(4)
    vols = []
    for i in range(14):
        dims = tuple(int(d) for d in np.exp(rng.uniform(np.log(9), np.log(70), 3)).round())
        f = sinusoid_field(dims, seed=30 + i)
        dtype = [np.float32, np.float32, np.float16, np.uint8, np.int16, np.float64, np.uint16][i % 7]
        if np.issubdtype(dtype, np.integer):
            info = np.iinfo(dtype)
            f = np.clip(f * 40 + (0 if info.min < 0 else 60), info.min, info.max)
        vols.append((vkl.structured_regular(device, f.astype(dtype), cell_centered=(i % 5 == 3)), dims))
    origins, values = shell_leaves(domain=96, shells=2, thickness=0.06, seed=8)
    L = len(origins)
    for comp in (None, "fp16"):
        v = vkl.vdb_volume(device, np.full(L, 3), origins, np.ones(L), packed_dense=values, compression=comp)
        vols.append((v, (96, 96, 96)))
    return vols


def _jobs(vkl, vols, seed):
    import torch
    rng = np.random.default_rng(seed)
    jobs, refs = [], []
    filters = [100] * 12 + [200, 0, 100, 100]
    for i, (vol, dims) in enumerate(vols):
        n = int(np.exp(rng.uniform(0, np.log(60000)))) if i % 6 else [0, 1, 7, 5000][i % 4]
        lo = -2.0
        hi = np.array(dims, np.float64) + 1.0
        pts = torch.from_numpy((lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)).cuda()
        smp = vkl.Sampler(vol, filter=filters[i], gradient_filter=filters[i])
        want_s = i % 4 != 1
        want_g = i % 4 != 2
        s = torch.full((n,), 7.0, device="cuda") if want_s else None
        g = torch.full((n, 3), 7.0, device="cuda") if want_g else None
        jobs.append((smp, pts, s, g))
        refs.append((smp.sample(pts).cpu().numpy() if want_s else None,
                     smp.gradient(pts).cpu().numpy() if want_g else None))
    return jobs, refs


def _check(jobs, refs):
    for (smp, pts, s, g), (rs, rg) in zip(jobs, refs):
        if s is not None:
            np.testing.assert_array_equal(bits(s.cpu().numpy()), bits(rs))
        if g is not None:
            np.testing.assert_array_equal(bits(g.cpu().numpy()), bits(rg))


@pytest.mark.parametrize("autotune", [False, True])
def test_batch_equals_per_job_calls(vkl, device, autotune):
    import torch
    vols = _volumes(vkl, device)
    jobs, refs = _jobs(vkl, vols, seed=1)
    batch = vkl.SampleBatch(device, jobs, autotune=autotune)
    cfg = batch.config()
    assert cfg["fused_jobs"] >= 8
    for rep in range(2):
        for _, _, s, g in jobs:
            if s is not None:
                s.fill_(7.0)
            if g is not None:
                g.fill_(7.0)
        batch.run()
        torch.cuda.synchronize()
        _check(jobs, refs)
    batch.release()


def test_batch_rejects_host_memory_and_bad_attributes(vkl, device):
    import torch
    vol = vkl.structured_regular(device, sinusoid_field((16, 16, 16), seed=2))
    smp = vkl.Sampler(vol)
    pts = torch.zeros((10, 3), device="cuda")
    out = torch.zeros(10, device="cuda")
    host = np.zeros((10, 3), np.float32)

    class HostArray:  # a host buffer dressed as a tensor for the binding
        shape = host.shape

        def data_ptr(self):
            return host.ctypes.data

    with pytest.raises(vkl.VKLError) as e:
        vkl.SampleBatch(device, [(smp, HostArray(), out, None)])
    assert e.value.code == 2 and "device memory" in e.value.msg
    with pytest.raises(vkl.VKLError) as e:
        vkl.SampleBatch(device, [(smp, pts, out, None, 3)])
    assert e.value.code == 2 and "attribute" in e.value.msg


def test_batch_jobs_on_mixed_type_attributes(vkl, device):
    """A job's fused class follows the voxel type of the attribute it samples:
    jobs on the float (texture atlas), half and int16 attributes of one
    multi-attribute volume equal the per-call samples and gradients."""
    import torch
    dims = (37, 29, 23)
    f = sinusoid_field(dims, seed=51)
    attrs = [f, sinusoid_field(dims, seed=52).astype(np.float16),
             np.clip(sinusoid_field(dims, seed=53) * 40, -32768, 32767).astype(np.int16)]
    vol = vkl.structured_regular(device, attrs)
    smp = vkl.Sampler(vol)
    rng = np.random.default_rng(54)
    jobs, refs = [], []
    for attr in (2, 0, 1, 0):
        pts = torch.from_numpy((rng.random((3000, 3)) * (np.array(dims) + 2) - 1.5).astype(np.float32)).cuda()
        s = torch.full((3000,), 7.0, device="cuda")
        g = torch.full((3000, 3), 7.0, device="cuda")
        jobs.append((smp, pts, s, g, attr))
        refs.append((smp.sample(pts, attr=attr).cpu().numpy(), smp.gradient(pts, attr=attr).cpu().numpy()))
    batch = vkl.SampleBatch(device, jobs)
    assert batch.config()["fused_jobs"] == 4
    batch.run()
    torch.cuda.synchronize()
    _check([j[:4] for j in jobs], refs)
    batch.release()
