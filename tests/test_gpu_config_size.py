"""GPU parity at the sizes the benchmark times.

The other parity tests use small shapes.  Here the device is compared with
the oracle on the benchmark's own volumes and query sets, where layouts and
addresses change with size:

* the 1024^3 float32 volume (4 GiB): texture-atlas rows of 64 z-planes with
  a seam at every 64th plane, byte offsets of the bricked copy up to 2^32;
  coherent points from the benchmark's orbit-camera generator (every 30th
  image row, 17.7M points), points on both sides of every atlas row seam, on
  the faces and outside them, and in the last z-slabs; trilinear samples and
  gradients through the atlas and through bricked loads, tricubic on a
  subset;
* the interval iterator over the same volume: the benchmark's 1920x1080
  camera rays, every 16th row, 4 quartile value ranges;
* the 4096^3 shell VDB (about 6.7M float leaves, 13.7 GB): 2^20 points in
  active leaves and 2^16 hit-iterator rays at isovalues 0.25 / 0.5;
* a 64-volume slice of the batched workload (edges 16-256, 1k-1M points
  per volume) through one batched launch.

Each result is compared bit for bit with the oracle's parity build and,
where the arithmetic differs, checked against the oracle's FP-contraction
build within 4 ULP or 1e-6 x max(|v|, 1) (tests/parity.py).  Interval and
hit counts must be equal to both builds.
"""
import math
import os

import numpy as np
import pytest

from tests.conftest import bits
from tests.parity import assert_within_contraction

pytestmark = pytest.mark.gpu

DIMS = (1024, 1024, 1024)
WIDTH, HEIGHT, SPP = 1920, 1080, 256


def _threads():
    return os.cpu_count() or 1


@pytest.fixture(scope="module")
def dense1024(vkl, oracle):
    import torch
    from openvkl_b200.fields import sinusoid_volume
    vox = sinusoid_volume(DIMS, seed=1)
    ref = oracle.OracleVolume.dense_volume(vox)
    fma = oracle.OracleVolume.dense_volume(vox, fma=True)
    tvox = torch.from_numpy(vox).cuda()
    dev_lsu = vkl.Device("cuda")
    dev_lsu.set_int("textureSampling", 0)
    dev_atlas = vkl.Device("cuda")
    vol_atlas = vkl.structured_regular(dev_atlas, tvox, shared=True)
    vol_lsu = vkl.structured_regular(dev_lsu, tvox, shared=True)
    yield {"vox": vox, "ref": ref, "fma": fma, "atlas": vol_atlas, "lsu": vol_lsu, "tvox": tvox}
    del vol_atlas, vol_lsu
    torch.cuda.empty_cache()


def _coherent_rows(step=32):
    """The benchmark's coherent points (orbit camera, 256 jittered samples
    per ray, generated on the GPU by the same generator and seed), every
    `step`-th image row."""
    import torch
    from openvkl_b200.fields import orbit_camera_samples_torch
    hi = tuple(d - 1 for d in DIMS)
    allp = orbit_camera_samples_torch(WIDTH, HEIGHT, SPP, (0, 0, 0), hi, seed=3)
    rows = torch.arange(0, HEIGHT, step, device="cuda")
    pix = (rows[:, None] * WIDTH + torch.arange(WIDTH, device="cuda")[None, :]).reshape(-1)
    idx = (pix[:, None] * SPP + torch.arange(SPP, device="cuda")[None, :]).reshape(-1)
    out = allp[idx].cpu().numpy()
    del allp
    torch.cuda.empty_cache()
    return out


def _edge_points(seed=11):
    """Points on both sides of every texture-atlas row seam (z-planes 64k-1
    and 64k), on and just outside each face, and in the last z-slabs (byte
    offsets of the bricked copy above 2^31)."""
    rng = np.random.default_rng(seed)
    X, Y, Z = DIMS
    parts = []
    seams = np.arange(64, Z, 64)
    for zc in np.concatenate([seams - 1, seams]):
        n = 512
        p = np.stack([rng.uniform(-1, X, n), rng.uniform(-1, Y, n), zc + rng.uniform(0, 1, n)], 1)
        parts.append(p)
    # exactly on the seam planes and on integer voxel positions
    for zc in (63.0, 64.0, 127.0, 128.0, 1023.0):
        g = rng.integers(0, 1023, (256, 2)).astype(np.float64)
        parts.append(np.stack([g[:, 0], g[:, 1], np.full(256, zc)], 1))
    # faces: on, just inside, just outside (background taps)
    for axis in range(3):
        for v in (-1.0, -0.5, -1e-3, 0.0, 1e-3, 1022.999, 1023.0, 1023.001, 1023.5, 1024.0):
            n = 256
            p = rng.uniform(0, 1023, (n, 3))
            p[:, axis] = v
            parts.append(p)
    # the last z-slabs (highest addresses)
    parts.append(np.stack([rng.uniform(0, 1023, 20000), rng.uniform(0, 1023, 20000),
                           rng.uniform(1015, 1023.5, 20000)], 1))
    return np.concatenate(parts).astype(np.float32)


def _compare(got, want, what):
    got, want = np.asarray(got), np.asarray(want)
    eq = bits(got).reshape(len(got), -1) == bits(want).reshape(len(want), -1)
    rows = np.nonzero(~eq.all(1))[0]
    assert rows.size == 0, f"{what}: {rows.size} mismatches, first at {rows[:5]}"


def test_dense_1024_trilinear_atlas_and_bricked(vkl, dense1024):
    """2^24 coherent points + seam / face / high-offset points, trilinear
    samples through the texture atlas and through bricked loads."""
    import torch
    ref, fma = dense1024["ref"], dense1024["fma"]
    pts = np.concatenate([_coherent_rows(30), _edge_points()])
    assert len(pts) > (1 << 24)
    want = ref.sample_parallel(pts, threads=_threads())
    tp = torch.from_numpy(pts).cuda()
    for path in ("atlas", "lsu"):
        smp = vkl.Sampler(dense1024[path])
        got = smp.sample(tp).cpu().numpy()
        _compare(got, want, f"trilinear sample ({path})")
    assert_within_contraction(got, fma.sample_parallel(pts, threads=_threads()), "trilinear sample vs fma")


def test_dense_1024_gradient_and_tricubic(vkl, dense1024):
    import torch
    ref, fma = dense1024["ref"], dense1024["fma"]
    rng = np.random.default_rng(5)
    coh = _coherent_rows(64)
    edge = _edge_points(seed=12)
    pts = np.concatenate([coh[rng.choice(len(coh), 1 << 21, replace=False)], edge])
    tp = torch.from_numpy(pts).cuda()
    wg = ref.gradient_parallel(pts, threads=_threads())
    for path in ("atlas", "lsu"):
        got = vkl.Sampler(dense1024[path]).gradient(tp).cpu().numpy()
        _compare(got, wg, f"trilinear gradient ({path})")
    assert_within_contraction(got, fma.gradient_parallel(pts, threads=_threads()), "trilinear gradient vs fma")
    sub = np.concatenate([pts[:1 << 18], edge])
    ts = torch.from_numpy(sub).cuda()
    smp = vkl.Sampler(dense1024["atlas"], filter=200, gradient_filter=200)
    ws = ref.sample_parallel(sub, filter=200, threads=_threads())
    _compare(smp.sample(ts).cpu().numpy(), ws, "tricubic sample")
    wgc = ref.gradient_parallel(sub, filter=200, threads=_threads())
    gc = smp.gradient(ts).cpu().numpy()
    _compare(gc, wgc, "tricubic gradient")
    assert_within_contraction(gc, fma.gradient_parallel(sub, filter=200, threads=_threads()),
                              "tricubic gradient vs fma")


def test_dense_1024_intervals_camera_rows(vkl, dense1024):
    """Interval iterator: the benchmark's 1920x1080 orbit-camera rays, every
    16th row, 4 quartile value ranges, default hint; every interval of every
    ray compared."""
    from openvkl_b200.fields import camera_rays
    ref, fma, vol = dense1024["ref"], dense1024["fma"], dense1024["atlas"]
    o, d, t = camera_rays(WIDTH, HEIGHT, (0, 0, 0), tuple(x - 1 for x in DIMS))
    rows = np.arange(0, HEIGHT, 16)
    sel = (rows[:, None] * WIDTH + np.arange(WIDTH)[None, :]).reshape(-1)
    o, d, t = o[sel], d[sel], t[sel]
    lo, hi = vol.value_range()
    q = np.linspace(lo, hi, 5, dtype=np.float32)
    vr = np.stack([q[:-1], q[1:]], 1)
    ctx = vkl.IntervalIteratorContext(vkl.Sampler(vol), value_ranges=vr)
    _, cnt = ctx.iterate_n(o, d, t, max_per_ray=0)
    m = int(np.max(cnt))
    got, gcnt = ctx.iterate_n(o, d, t, max_per_ray=m)
    want, wcnt = ref.intervals(o, d, t, value_ranges=vr, max_intervals=m)
    np.testing.assert_array_equal(gcnt, wcnt)
    assert int(gcnt.sum()) > 100 * len(o)
    mask = np.arange(m)[None, :] < gcnt[:, None]
    np.testing.assert_array_equal(bits(got[mask]), bits(want[mask]))
    fw, fcnt = fma.intervals(o, d, t, value_ranges=vr, max_intervals=m)
    np.testing.assert_array_equal(gcnt, fcnt)
    assert_within_contraction(got[mask], fw[mask], "intervals vs fma")


@pytest.fixture(scope="module")
def vdb4096(vkl, oracle):
    """The benchmark's sparse VDB: 4096^3 domain shells, float leaves.  The
    oracle needs the leaves in host memory (13.7 GB)."""
    import psutil
    import torch
    from openvkl_b200.fields import shell_vdb_torch
    if psutil.virtual_memory().available < 48 << 30:
        pytest.skip("the 4096^3 VDB oracle needs about 30 GB of free host memory")
    origins, values, _, _ = shell_vdb_torch(domain=4096, seed=5)
    L = origins.shape[0]
    host = values.cpu().numpy()
    dev = vkl.Device("cuda")
    vol = vkl.vdb_volume(dev, np.full(L, 3), origins, np.ones(L), packed_dense=values, shared=True)
    ref = oracle.OracleVolume.vdb_volume(np.full(L, 3), origins, np.ones(L), host)
    fma = oracle.OracleVolume.vdb_volume(np.full(L, 3), origins, np.ones(L), host, fma=True)
    yield {"origins": origins, "vol": vol, "ref": ref, "fma": fma, "values": values}
    del vol
    torch.cuda.empty_cache()


def test_vdb_4096_interior_points(vkl, vdb4096):
    import torch
    origins, ref = vdb4096["origins"], vdb4096["ref"]
    rng = np.random.default_rng(13)
    pick = rng.integers(0, len(origins), 1 << 20)
    pts = (origins[pick] + rng.uniform(0, 8, (1 << 20, 3))).astype(np.float32)
    tp = torch.from_numpy(pts).cuda()
    smp = vkl.Sampler(vdb4096["vol"], filter=100, gradient_filter=100)
    _compare(smp.sample(tp).cpu().numpy(), ref.sample_parallel(pts, threads=_threads()), "vdb trilinear")
    sub = pts[:1 << 17]
    ts = torch.from_numpy(sub).cuda()
    _compare(smp.gradient(ts).cpu().numpy(), ref.gradient_parallel(sub, threads=_threads()), "vdb gradient")
    cub = vkl.Sampler(vdb4096["vol"], filter=200)
    _compare(cub.sample(ts).cpu().numpy(), ref.sample_parallel(sub, filter=200, threads=_threads()),
             "vdb tricubic")
    got = smp.sample(tp).cpu().numpy()
    assert_within_contraction(got, vdb4096["fma"].sample_parallel(pts, threads=_threads()), "vdb vs fma")


def test_vdb_4096_hits(vkl, vdb4096):
    from openvkl_b200.fields import random_rays
    ref = vdb4096["ref"]
    o, d, t = random_rays(1 << 16, (0, 0, 0), (4096,) * 3, seed=4)
    ctx = vkl.HitIteratorContext(vkl.Sampler(vdb4096["vol"]), [0.25, 0.5])
    got, gcnt = ctx.iterate_n(o, d, t, max_per_ray=16)
    want, wcnt = ref.hits(o, d, t, np.array([0.25, 0.5], np.float32), max_hits=16)
    np.testing.assert_array_equal(gcnt, wcnt)
    assert int(gcnt.sum()) > len(o) // 4
    k = np.minimum(gcnt, 16)
    mask = np.arange(16)[None, :] < k[:, None]
    np.testing.assert_array_equal(bits(got[mask]), bits(want[mask]))
    # Against the FP-contraction build the hit counts are not exact: a march
    # sample within rounding of an isovalue can change sides and add or drop
    # a pair of hits (measured: 6 of these 65,536 rays, by 2).  The bound
    # stated here is 0.05 % of the rays.
    fw, fcnt = vdb4096["fma"].hits(o, d, t, np.array([0.25, 0.5], np.float32), max_hits=16)
    assert np.count_nonzero(gcnt != fcnt) <= len(o) // 2000


def test_batched_64_volume_slice(vkl, device, oracle):
    """The first 64 volumes of the batched workload (same generator and
    seeds), sample + gradient of every point in one batched launch."""
    import torch
    from openvkl_b200.fields import sinusoid_field_torch, uniform_points_torch
    rng = np.random.default_rng(7)
    jobs, refs = [], []
    for i in range(64):
        dims = tuple(int(round(math.exp(rng.uniform(math.log(16), math.log(256))))) for _ in range(3))
        n = int(round(math.exp(rng.uniform(math.log(1e3), math.log(1e6)))))
        vox = sinusoid_field_torch(dims, seed=100 + i)
        vol = vkl.structured_regular(device, vox, shared=True)
        smp = vkl.Sampler(vol, filter=100, gradient_filter=100)
        pts = uniform_points_torch(n, (0, 0, 0), tuple(d - 1 for d in dims), seed=200 + i)
        jobs.append((smp, pts, torch.empty(n, device="cuda"), torch.empty((n, 3), device="cuda")))
        refs.append((vox.cpu().numpy(), pts.cpu().numpy(), vol))
    batch = vkl.SampleBatch(device, jobs)
    batch.run()
    torch.cuda.synchronize()
    total = 0
    for (smp, pts, s, g), (vox, hp, _) in zip(jobs, refs):
        r = oracle.OracleVolume.dense_volume(vox)
        _compare(s.cpu().numpy(), r.sample_parallel(hp, threads=_threads()), "batched sample")
        _compare(g.cpu().numpy(), r.gradient_parallel(hp, threads=_threads()), "batched gradient")
        total += len(hp)
    assert total > 1 << 22
    batch.release()


def test_dense_1024_macrocell_intervals_camera_rows(vkl, dense1024):
    """16^3-voxel macrocell intervals (the legacy structuredRegular iterator,
    an extension here) on the same volume and rays as the default-iterator
    test above: counts and every interval bit-exact against the oracle's
    restatement of the same walk."""
    from openvkl_b200.fields import camera_rays
    ref, vol = dense1024["ref"], dense1024["atlas"]
    o, d, t = camera_rays(WIDTH, HEIGHT, (0, 0, 0), tuple(x - 1 for x in DIMS))
    rows = np.arange(0, HEIGHT, 16)
    sel = (rows[:, None] * WIDTH + np.arange(WIDTH)[None, :]).reshape(-1)
    o, d, t = o[sel], d[sel], t[sel]
    lo, hi = vol.value_range()
    q = np.linspace(lo, hi, 5, dtype=np.float32)
    vr = np.stack([q[:-1], q[1:]], 1)
    ctx = vkl.IntervalIteratorContext(vkl.Sampler(vol), value_ranges=vr, macrocells=True)
    _, cnt = ctx.iterate_n(o, d, t, max_per_ray=0)
    m = int(np.max(cnt))
    got, gcnt = ctx.iterate_n(o, d, t, max_per_ray=m)
    want, wcnt = ref.macrocell_intervals(o, d, t, value_ranges=vr, max_intervals=m)
    np.testing.assert_array_equal(gcnt, wcnt)
    assert int(gcnt.sum()) > 50 * len(o)
    mask = np.arange(m)[None, :] < gcnt[:, None]
    np.testing.assert_array_equal(bits(got[mask]), bits(want[mask]))
