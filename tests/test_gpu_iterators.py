"""GPU parity of the interval and hit iterators against the oracle: interval
counts and hit counts bit-exact, interval bounds / value ranges /
nominalDeltaT and hit t / sample / epsilon bit-exact, for dense and sparse
volumes, several value-range filters and interval resolution hints; the
per-ray C API (vklInitIntervalIterator / vklIterateInterval, hit analogues)
returns the same records as the batched extension."""
import numpy as np
import pytest

from openvkl_b200.fields import random_rays, shell_leaves, sinusoid_field
from tests.conftest import bits

pytestmark = pytest.mark.gpu


def _dense(vkl, device, oracle, dims=(48, 40, 56)):
    vox = sinusoid_field(dims, seed=21)
    return vox, oracle.OracleVolume.dense_volume(vox), vkl.structured_regular(device, vox)


def _sparse(vkl, device, oracle):
    origins, values = shell_leaves(domain=128, shells=2, thickness=0.06, seed=8)
    L = len(origins)
    ref = oracle.OracleVolume.vdb_volume(np.full(L, 3), origins, np.ones(L), values)
    vol = vkl.vdb_volume(device, np.full(L, 3), origins, np.ones(L), packed_dense=values)
    return ref, vol


def _compare_intervals(got, gcnt, want, wcnt):
    np.testing.assert_array_equal(gcnt, wcnt)
    for r in range(len(gcnt)):
        k = min(int(gcnt[r]), got.shape[1])
        np.testing.assert_array_equal(bits(got[r, :k]), bits(want[r, :k]), err_msg=f"ray {r}")


@pytest.mark.parametrize("hint", [0.0, 0.3, 0.5, 0.9, 1.0])
def test_dense_intervals(vkl, device, oracle, hint):
    vox, ref, vol = _dense(vkl, device, oracle)
    b = ref.info()["bounds"]
    o, d, t = random_rays(3000, b[:3], b[3:], seed=1)
    lo, hi = float(vox.min()), float(vox.max())
    q = np.linspace(lo, hi, 9)
    ranges = np.array([[q[0], q[1]], [q[3], q[4]], [q[5], q[6]], [q[7], q[8]]], np.float32)
    for vr in (None, ranges):
        smp = vkl.Sampler(vol)
        ctx = vkl.IntervalIteratorContext(smp, value_ranges=vr, hint=hint)
        got, gcnt = ctx.iterate_n(o, d, t, max_per_ray=512)
        want, wcnt = ref.intervals(o, d, t, value_ranges=vr, hint=hint, max_intervals=512)
        _compare_intervals(got, gcnt, want, wcnt)


def test_sparse_intervals(vkl, device, oracle):
    ref, vol = _sparse(vkl, device, oracle)
    b = ref.info()["bounds"]
    o, d, t = random_rays(3000, b[:3], b[3:], seed=2)
    for hint, vr in ((0.5, None), (1.0, [[0.4, 0.6]]), (0.1, [[0.0, 0.1], [0.9, 1.0]])):
        ctx = vkl.IntervalIteratorContext(vkl.Sampler(vol), value_ranges=vr, hint=hint)
        got, gcnt = ctx.iterate_n(o, d, t, max_per_ray=1024)
        want, wcnt = ref.intervals(o, d, t, value_ranges=vr, hint=hint, max_intervals=1024)
        _compare_intervals(got, gcnt, want, wcnt)


@pytest.mark.parametrize("filt", [100, 200])
def test_dense_hits(vkl, device, oracle, filt):
    vox, ref, vol = _dense(vkl, device, oracle)
    b = ref.info()["bounds"]
    o, d, t = random_rays(2000, b[:3], b[3:], seed=3)
    isos = np.array([-0.5, 0.25, 0.5], np.float32)
    ctx = vkl.HitIteratorContext(vkl.Sampler(vol, filter=filt), isos)
    got, gcnt = ctx.iterate_n(o, d, t, max_per_ray=64)
    want, wcnt = ref.hits(o, d, t, isos, filter=filt, max_hits=64)
    _compare_intervals(got, gcnt, want, wcnt)
    assert gcnt.sum() > 0


def test_sparse_hits(vkl, device, oracle):
    ref, vol = _sparse(vkl, device, oracle)
    b = ref.info()["bounds"]
    o, d, t = random_rays(1500, b[:3], b[3:], seed=4)
    isos = np.array([0.25, 0.5], np.float32)
    ctx = vkl.HitIteratorContext(vkl.Sampler(vol), isos)
    got, gcnt = ctx.iterate_n(o, d, t, max_per_ray=64)
    want, wcnt = ref.hits(o, d, t, isos, max_hits=64)
    _compare_intervals(got, gcnt, want, wcnt)
    assert gcnt.sum() > 0


def test_zramp_hits_through_per_ray_api(vkl, device):
    n = 64
    sp = 1.0 / (n - 1)
    z = (np.arange(n, dtype=np.float32) * np.float32(sp))
    vox = np.broadcast_to(z[:, None, None], (n, n, n)).copy()
    vol = vkl.structured_regular(device, vox, grid_origin=(0, 0, 0), grid_spacing=(sp, sp, sp))
    isos = []
    f = np.float32(0.1)
    while f < 1:
        isos.append(f)
        f = np.float32(f + np.float32(0.1))
    ctx = vkl.HitIteratorContext(vkl.Sampler(vol), isos)
    hits = ctx.iterate_one((0.5, 0.5, -1.0), (0.0, 0.0, 1.0), (0.0, np.inf))
    assert len(hits) == len(isos)
    for h, iso in zip(hits, isos):
        assert h[1] == iso
        assert abs(h[0] - (float(iso) + 1.0)) <= 1e-3


def test_per_ray_api_equals_batched(vkl, device, oracle):
    vox, ref, vol = _dense(vkl, device, oracle, dims=(24, 24, 24))
    b = ref.info()["bounds"]
    o, d, t = random_rays(6, b[:3], b[3:], seed=5)
    smp = vkl.Sampler(vol)
    ictx = vkl.IntervalIteratorContext(smp, value_ranges=[[-0.3, 0.3]], hint=0.5)
    got, gcnt = ictx.iterate_n(o, d, t, max_per_ray=128)
    hctx = vkl.HitIteratorContext(smp, [0.0, 0.4])
    hgot, hcnt = hctx.iterate_n(o, d, t, max_per_ray=32)
    for r in range(len(o)):
        one = ictx.iterate_one(o[r], d[r], t[r])
        assert len(one) == gcnt[r]
        np.testing.assert_array_equal(bits(one), bits(got[r, :gcnt[r]]))
        h1 = hctx.iterate_one(o[r], d[r], t[r])
        assert len(h1) == hcnt[r]
        np.testing.assert_array_equal(bits(h1), bits(hgot[r, :hcnt[r]]))


def test_macrocell_intervals(vkl, device, oracle):
    """16^3-voxel macrocell intervals (context parameter "macrocells", the
    interval walk of the reference's legacy structuredRegular volume; an
    extension here): dims that are not multiples of 16, a grid origin and
    anisotropic spacing, rays from all sides, with and without value-range
    filters; counts and intervals bit-exact against the oracle."""
    dims = (53, 40, 37)
    vox = sinusoid_field(dims, seed=23)
    kw = dict(grid_origin=(-3.0, 2.5, 1.0), grid_spacing=(0.5, 1.25, 0.75))
    ref = oracle.OracleVolume.dense_volume(vox, **kw)
    vol = vkl.structured_regular(device, vox, **kw)
    b = ref.info()["bounds"]
    o, d, t = random_rays(4000, b[:3], b[3:], seed=7)
    # axis-aligned rays, rays starting inside, and a bounded t range
    o[:200] = (b[:3] + b[3:]) / 2
    d[:200] = np.eye(3, dtype=np.float32)[np.arange(200) % 3] * np.where(np.arange(200) % 2, 1, -1)[:, None]
    t[200:400] = [[5.0, 20.0]]
    lo, hi = float(vox.min()), float(vox.max())
    for vr in (None, [[lo, lo + 0.2 * (hi - lo)]], [[lo, lo + 0.1], [hi - 0.3, hi]]):
        ctx = vkl.IntervalIteratorContext(vkl.Sampler(vol), value_ranges=vr, macrocells=True)
        got, gcnt = ctx.iterate_n(o, d, t, max_per_ray=32)
        want, wcnt = ref.macrocell_intervals(o, d, t, value_ranges=vr, max_intervals=32)
        _compare_intervals(got, gcnt, want, wcnt)
        assert gcnt.sum() > 0


def test_macrocell_intervals_reject_unsupported(vkl, device):
    """The legacy walk covers vertex-centered volumes given by gridOrigin /
    gridSpacing: a rotated or cell-centered volume is rejected at the
    context's commit, and the per-ray API refuses macrocell contexts."""
    vox = sinusoid_field((20, 20, 20), seed=2)
    i2o = np.array([0, 1, 0, -1, 0, 0, 0, 0, 1, 0, 0, 0], np.float32)
    for kw in (dict(index_to_object=i2o), dict(cell_centered=True)):
        vol = vkl.structured_regular(device, vox, **kw)
        with pytest.raises(vkl.VKLError):
            vkl.IntervalIteratorContext(vkl.Sampler(vol), macrocells=True)
    vol = vkl.structured_regular(device, vox)
    ctx = vkl.IntervalIteratorContext(vkl.Sampler(vol), macrocells=True)
    with pytest.raises(vkl.VKLError):
        ctx.iterate_one((0.5, 0.5, -1.0), (0.0, 0.0, 1.0), (0.0, np.inf))
