"""Temporally varying (motion-blur) structuredRegular volumes against the
oracle: structured data (temporallyStructuredNumTimesteps values per voxel)
and unstructured data (per-voxel temporallyUnstructuredIndices into the data
and temporallyUnstructuredTimes), every voxel type, the three filters,
samples and gradients at per-point times (host and device arrays, the
1-wide and 4-wide calls), multi-attribute sampling, value ranges over all
time samples, interval iteration, and the reference's validation errors.
Results are compared bit for bit (the taps interpolate in time with the
reference's expressions, then the spatial filter runs on them)."""
import numpy as np
import pytest

from openvkl_b200.fields import sinusoid_field, uniform_points, random_rays
from tests.conftest import bits

pytestmark = pytest.mark.gpu

DIMS = (23, 19, 17)


def _structured(dtype, n_t=4, seed=1):
    base = sinusoid_field(DIMS, seed=seed)
    steps = [base * (1.0 + 0.5 * k) + 0.1 * k for k in range(n_t)]
    data = np.stack(steps, -1)  # (Z, Y, X, T): each voxel's samples consecutive
    if np.issubdtype(dtype, np.integer):
        info = np.iinfo(dtype)
        data = np.clip(data * 30 + (0 if info.min < 0 else 80), info.min, info.max)
    return data.astype(dtype).reshape(-1)


def _unstructured(seed=3, idx_dtype=np.uint32):
    rng = np.random.default_rng(seed)
    nv = DIMS[0] * DIMS[1] * DIMS[2]
    cnt = rng.integers(1, 6, nv)
    idx = np.concatenate([[0], np.cumsum(cnt)]).astype(idx_dtype)
    times = np.concatenate([np.sort(rng.choice(np.linspace(0, 1, 97, dtype=np.float32), k, replace=False))
                            for k in cnt]).astype(np.float32)
    vals = rng.uniform(-2, 3, int(idx[-1])).astype(np.float32)
    return vals, idx, times


def _points(n, seed):
    pts = uniform_points(n, (-1.5, -1.5, -1.5), tuple(d + 0.5 for d in DIMS), seed)
    t = np.random.default_rng(seed + 7).uniform(0, 1, n).astype(np.float32)
    t[:50] = 0.0
    t[50:100] = 1.0
    return pts, t


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.float16, np.float32, np.float64])
def test_structured_all_filters(vkl, device, oracle, dtype):
    data = _structured(dtype)
    ref = oracle.OracleVolume.dense_temporal(data, DIMS, num_timesteps=4)
    vol = vkl.structured_regular(device, data, dims=DIMS, num_timesteps=4)
    np.testing.assert_array_equal(vol.value_range(), ref.value_range())
    pts, t = _points(20000, 2)
    for f in (0, 100, 200):
        smp = vkl.Sampler(vol, filter=f, gradient_filter=f)
        np.testing.assert_array_equal(bits(smp.sample(pts, times=t)), bits(ref.sample_times(pts, t, filter=f)))
        np.testing.assert_array_equal(bits(smp.gradient(pts, times=t)),
                                      bits(ref.gradient_times(pts, t, filter=f)))


@pytest.mark.parametrize("idx_dtype", [np.uint32, np.uint64])
def test_unstructured_all_filters(vkl, device, oracle, idx_dtype):
    vals, idx, times = _unstructured(idx_dtype=idx_dtype)
    ref = oracle.OracleVolume.dense_temporal(vals, DIMS, indices=idx, times=times)
    vol = vkl.structured_regular(device, vals, dims=DIMS, time_indices=idx, times=times)
    np.testing.assert_array_equal(vol.value_range(), ref.value_range())
    pts, t = _points(20000, 4)
    # times on the samples' own time grid too (exact matches in the search)
    t[100:400] = np.linspace(0, 1, 97, dtype=np.float32)[np.arange(300) % 97]
    for f in (0, 100, 200):
        smp = vkl.Sampler(vol, filter=f, gradient_filter=f)
        np.testing.assert_array_equal(bits(smp.sample(pts, times=t)), bits(ref.sample_times(pts, t, filter=f)))
        np.testing.assert_array_equal(bits(smp.gradient(pts, times=t)),
                                      bits(ref.gradient_times(pts, t, filter=f)))


def test_times_on_device_scalar_wide_and_multi_attribute(vkl, device, oracle):
    import torch
    a0 = _structured(np.float32, n_t=3, seed=5)
    a1 = _structured(np.float16, n_t=3, seed=6)
    ref0 = oracle.OracleVolume.dense_temporal(a0, DIMS, num_timesteps=3)
    ref1 = oracle.OracleVolume.dense_temporal(a1, DIMS, num_timesteps=3)
    vol = vkl.structured_regular(device, [a0, a1], dims=DIMS, num_timesteps=3)
    smp = vkl.Sampler(vol)
    pts, t = _points(5000, 8)
    got = smp.sample(torch.from_numpy(pts).cuda(), times=torch.from_numpy(t).cuda()).cpu().numpy()
    np.testing.assert_array_equal(bits(got), bits(ref0.sample_times(pts, t)))
    m = smp.sample_m(pts, [1, 0], times=t)
    np.testing.assert_array_equal(bits(m[:, 0]), bits(ref1.sample_times(pts, t)))
    np.testing.assert_array_equal(bits(m[:, 1]), bits(ref0.sample_times(pts, t)))
    for i in range(3):
        want = ref0.sample_times(pts[i:i + 1], t[i:i + 1])[0]
        assert bits(np.float32(smp.sample_one(pts[i], time=t[i])))[()] == bits(want)[()]
    # time 0 is the default
    np.testing.assert_array_equal(bits(smp.sample(pts)), bits(ref0.sample_times(pts, None)))


def test_intervals_and_hits_at_time_zero(vkl, device, oracle):
    data = _structured(np.float32, n_t=3, seed=9)
    ref = oracle.OracleVolume.dense_temporal(data, DIMS, num_timesteps=3)
    vol = vkl.structured_regular(device, data, dims=DIMS, num_timesteps=3)
    b = ref.info()["bounds"]
    o, d, tr = random_rays(2000, b[:3], b[3:], seed=11)
    lo, hi = ref.value_range()
    vr = [[lo, lo + 0.3 * (hi - lo)]]
    ctx = vkl.IntervalIteratorContext(vkl.Sampler(vol), value_ranges=vr)
    got, gcnt = ctx.iterate_n(o, d, tr, max_per_ray=256)
    want, wcnt = ref.intervals(o, d, tr, value_ranges=vr, max_intervals=256)
    np.testing.assert_array_equal(gcnt, wcnt)
    mask = np.arange(256)[None, :] < gcnt[:, None]
    np.testing.assert_array_equal(bits(got[mask]), bits(want[mask]))
    isos = np.array([0.0, 1.0], np.float32)
    hctx = vkl.HitIteratorContext(vkl.Sampler(vol), isos)
    hg, hc = hctx.iterate_n(o, d, tr, max_per_ray=32)
    hw, hwc = ref.hits(o, d, tr, isos, max_hits=32)
    np.testing.assert_array_equal(hc, hwc)
    k = np.minimum(hc, 32)
    mask = np.arange(32)[None, :] < k[:, None]
    np.testing.assert_array_equal(bits(hg[mask]), bits(hw[mask]))
    assert hc.sum() > 0


def test_validation_errors(vkl, device):
    data = _structured(np.float32, n_t=3)
    with pytest.raises(vkl.VKLError, match="elements, but expected"):
        vkl.structured_regular(device, data[:-3], dims=DIMS, num_timesteps=3)
    vals, idx, times = _unstructured()
    bad = idx.copy()
    bad[5] = bad[4]
    with pytest.raises(vkl.VKLError, match="increase strictly monotonically"):
        vkl.structured_regular(device, vals, dims=DIMS, time_indices=bad, times=times)
    bt = times.copy()
    bt[int(idx[1]) - 1] = 1.5  # the first voxel's last time: still increasing, out of [0, 1]
    with pytest.raises(vkl.VKLError, match="bounded by 0.0 and 1.0"):
        vkl.structured_regular(device, vals, dims=DIMS, time_indices=idx, times=bt)
    with pytest.raises(vkl.VKLError, match="should not have"):
        vkl.structured_regular(device, vals, dims=DIMS, num_timesteps=2, time_indices=idx, times=times)
