"""GPU parity of the cuda device's structuredRegular sampling and gradients
against the oracle, through the C-ABI.

The device arithmetic restates the reference's float expressions operation by
operation, so results are compared bit for bit (uint32 patterns, NaN
backgrounds included).  The same inputs are also scored against the FP64
evaluation of the same filters (documented tolerance 1e-5 relative to the
field's magnitude) to state the FP32 error.
"""
import numpy as np
import pytest

from openvkl_b200.fields import sinusoid_field, uniform_points
from tests.conftest import bits

pytestmark = pytest.mark.gpu

FILTERS = {"nearest": 0, "linear": 100, "cubic": 200}


def _pts_around(dims, n, seed, pad=1.5):
    lo = np.array([-pad] * 3)
    hi = np.array(dims, np.float64) - 1 + pad
    return uniform_points(n, lo, hi, seed)


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.uint16, np.float16, np.float32, np.float64])
@pytest.mark.parametrize("filt", list(FILTERS))
def test_dense_types_and_filters_bit_exact(vkl, device, oracle, dtype, filt):
    dims = (21, 17, 13)  # not multiples of the 8^3 leaf
    f = sinusoid_field(dims, seed=3)
    if np.issubdtype(dtype, np.integer):
        info = np.iinfo(dtype)
        f = np.clip(f * 40 + (0 if info.min < 0 else 60), info.min, info.max)
    vox = f.astype(dtype)
    pts = _pts_around(dims, 20000, seed=4)
    ref = oracle.OracleVolume.dense_volume(vox)
    vol = vkl.structured_regular(device, vox)
    smp = vkl.Sampler(vol, filter=FILTERS[filt], gradient_filter=FILTERS[filt])
    s = smp.sample(pts)
    np.testing.assert_array_equal(bits(s), bits(ref.sample(pts, filter=FILTERS[filt])))
    g = smp.gradient(pts)
    np.testing.assert_array_equal(bits(g), bits(ref.gradient(pts, filter=FILTERS[filt])))


@pytest.mark.parametrize("cell", [False, True])
def test_transform_background_and_origin(vkl, device, oracle, cell):
    dims = (16, 24, 20)
    vox = sinusoid_field(dims, seed=7)
    ang = 0.3
    c, s_ = np.cos(ang), np.sin(ang)
    # column-major [vx vy vz p]: rotation about z, anisotropic scale, offset
    i2o = np.array([0.5 * c, 0.5 * s_, 0, -0.7 * s_, 0.7 * c, 0, 0, 0, 0.25, 3.0, -2.0, 1.5], np.float32)
    kw = dict(cell_centered=cell, index_to_object=i2o, index_origin=(-3, 5, 2), background=[0.125])
    ref = oracle.OracleVolume.dense_volume(vox, **kw)
    vol = vkl.structured_regular(device, vox, **kw)
    np.testing.assert_array_equal(vol.bounding_box(), ref.info()["bounds"])
    b = ref.info()["bounds"]
    pts = uniform_points(30000, b[:3] - 0.5, b[3:] + 0.5, seed=9)
    for name, fv in FILTERS.items():
        smp = vkl.Sampler(vol, filter=fv, gradient_filter=fv)
        np.testing.assert_array_equal(bits(smp.sample(pts)), bits(ref.sample(pts, filter=fv)), err_msg=name)
        np.testing.assert_array_equal(bits(smp.gradient(pts)), bits(ref.gradient(pts, filter=fv)), err_msg=name)
    np.testing.assert_array_equal(vol.value_range(), ref.value_range())


def test_config1_full_size_linear_and_gradient(vkl, device, oracle):
    """structuredRegular 128^3 float32 vertex-centered, seeded sinusoid field,
    2^20 uniform points: vklComputeSampleN + vklComputeGradientN."""
    dims = (128, 128, 128)
    vox = sinusoid_field(dims, seed=1)
    pts = uniform_points(1 << 20, (0, 0, 0), (127, 127, 127), seed=2)
    ref = oracle.OracleVolume.dense_volume(vox)
    vol = vkl.structured_regular(device, vox)
    smp = vkl.Sampler(vol)
    s = smp.sample(pts)
    np.testing.assert_array_equal(bits(s), bits(ref.sample(pts)))
    np.testing.assert_array_equal(bits(smp.gradient(pts)), bits(ref.gradient(pts)))
    # error vs the FP64 evaluation of the same trilinear filter
    d = ref.sample_fp64(pts[:100000])
    rel = np.abs(s[:100000].astype(np.float64) - d) / np.maximum(np.abs(d), 1.0)
    assert rel.max() < 1e-5


def test_device_pointers_and_multi_attribute(vkl, device, oracle):
    import torch
    dims = (32, 32, 32)
    a0 = sinusoid_field(dims, seed=1)
    a1 = sinusoid_field(dims, seed=2).astype(np.float16)
    a2 = (sinusoid_field(dims, seed=3) * 100).astype(np.int16)
    ref = oracle.OracleVolume.dense_volume([a0, a1, a2])
    vol = vkl.structured_regular(device, [a0, a1, a2])
    assert vol.num_attributes() == 3
    smp = vkl.Sampler(vol)
    pts = _pts_around(dims, 5000, seed=5)
    out = smp.sample_m(pts, [2, 0, 1])
    for j, a in enumerate([2, 0, 1]):
        np.testing.assert_array_equal(bits(out[:, j]), bits(ref.sample(pts, attr=a)))
    # device-resident inputs / outputs are used in place
    tp = torch.from_numpy(pts).cuda()
    ts = smp.sample(tp, attr=1)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(bits(ts.cpu().numpy()), bits(ref.sample(pts, attr=1)))


def test_scalar_and_wide_entry_points(vkl, device, oracle):
    dims = (16, 16, 16)
    vox = sinusoid_field(dims, seed=11)
    ref = oracle.OracleVolume.dense_volume(vox)
    vol = vkl.structured_regular(device, vox)
    smp = vkl.Sampler(vol, filter=200, gradient_filter=200)
    pts = _pts_around(dims, 16, seed=6, pad=-1.0)
    want = ref.sample(pts, filter=200)
    for i in range(4):
        assert bits(np.float32(smp.sample_one(pts[i])))[()] == bits(want[i])[()]
    np.testing.assert_array_equal(bits(smp.gradient_one(pts[0])), bits(ref.gradient(pts[:1], filter=200)[0]))
    for w in (4, 8, 16):
        valid = (np.arange(w) % 3 != 1).astype(np.int32)
        got = smp.sample_w(pts[:w], valid=valid)
        np.testing.assert_array_equal(bits(got[valid == 1]), bits(want[:w][valid == 1]))
        g = smp.gradient_w(pts[:w], valid=valid)
        gw = ref.gradient(pts[:w], filter=200)
        np.testing.assert_array_equal(bits(g[valid == 1]), bits(gw[valid == 1]))
        assert np.isnan(g[valid == 0]).all()  # invalid lanes are not written


def test_wide_multi_attribute_entry_points(vkl, device, oracle):
    """vklComputeSampleM4/8/16: samples[m * W + lane] is attribute
    attributeIndices[m] at that lane (the layout the reference tutorial
    prints, examples/vklTutorialCPU.c:212-231)."""
    dims = (20, 12, 10)
    vox = [sinusoid_field(dims, seed=s) for s in (21, 22, 23)]
    ref = oracle.OracleVolume.dense_volume(vox)
    vol = vkl.structured_regular(device, vox)
    smp = vkl.Sampler(vol)
    pts = _pts_around(dims, 16, seed=9, pad=-1.0)
    attrs = [2, 0, 1, 2]
    for w in (4, 8, 16):
        valid = (np.arange(w) % 4 != 2).astype(np.int32)
        got = smp.sample_m_w(pts[:w], attrs, valid=valid)
        for m, a in enumerate(attrs):
            np.testing.assert_array_equal(bits(got[m][valid == 1]), bits(ref.sample(pts[:w], attr=a)[valid == 1]))
        assert np.isnan(got[:, valid == 0]).all()


def test_shared_device_buffer_and_strided_host_data(vkl, device, oracle):
    import torch
    dims = (24, 16, 8)
    vox = sinusoid_field(dims, seed=13)
    ref = oracle.OracleVolume.dense_volume(vox)
    tvox = torch.from_numpy(vox).cuda()
    vol = vkl.structured_regular(device, tvox, shared=True)
    pts = _pts_around(dims, 4000, seed=8)
    np.testing.assert_array_equal(bits(vkl.Sampler(vol).sample(pts)), bits(ref.sample(pts)))
    # strided host source: every other float of an interleaved buffer
    inter = np.stack([vox, np.zeros_like(vox)], -1)
    v2 = vkl.Volume(device, "structuredRegular")
    v2.set_vec3i("dimensions", dims)
    v2.set_data("data", vkl.Data(device, inter, vkl_type=vkl.VKL_FLOAT, num_items=vox.size, byte_stride=8))
    v2.commit()
    np.testing.assert_array_equal(bits(vkl.Sampler(v2).sample(pts)), bits(ref.sample(pts)))


def test_error_paths(vkl, device):
    v = vkl.Volume(device, "structuredRegular")
    v.set_vec3i("dimensions", (4, 4, 4))
    with pytest.raises(vkl.VKLError, match="missing required 'data'"):
        v.commit()
    v.set_data("data", vkl.Data(device, np.zeros(10, np.float32)))
    with pytest.raises(vkl.VKLError, match="has 10 elements, but expected 64"):
        v.commit()
    with pytest.raises(vkl.VKLError):
        vkl.Volume(device, "unstructured")


@pytest.mark.parametrize("where", ["pinned", "pageable", "host_in_device_out", "device_in_host_out"])
def test_chunked_host_pointer_calls(vkl, device, where):
    """Host-pointer calls above the pipelining threshold are cut into
    8M-point chunks that cycle through three staging slots; results must equal
    the all-device call bit for bit (here 4 chunks: every slot reused once)."""
    import torch
    dims = (40, 33, 27)
    vox = sinusoid_field(dims, seed=17)
    vol = vkl.structured_regular(device, vox)
    smp = vkl.Sampler(vol, filter=100, gradient_filter=100)
    n = 3 * (1 << 23) + 4099
    pts_d = torch.rand((n, 3), device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    pts_d = (pts_d * torch.tensor([d + 1.0 for d in dims], device="cuda") - 1.0).contiguous()
    want_s = smp.sample(pts_d)
    want_g = smp.gradient(pts_d)
    if where == "pinned":
        pin = pts_d.cpu().pin_memory()
        out_s, out_g = torch.empty(n).pin_memory(), torch.empty((n, 3)).pin_memory()
        got_s, got_g = smp.sample(pin, out=out_s), smp.gradient(pin, out=out_g)
    elif where == "pageable":
        host = pts_d.cpu().numpy()
        got_s, got_g = smp.sample(host), smp.gradient(host)
    elif where == "host_in_device_out":
        host = pts_d.cpu().numpy()
        got_s = smp.sample(host, out=torch.empty(n, device="cuda"))
        got_g = smp.gradient(host, out=torch.empty((n, 3), device="cuda"))
    else:
        got_s = smp.sample(pts_d, out=np.empty(n, np.float32))
        got_g = smp.gradient(pts_d, out=np.empty((n, 3), np.float32))
    as_np = lambda t: t.cpu().numpy() if hasattr(t, "cpu") else t
    np.testing.assert_array_equal(bits(as_np(got_s)), bits(want_s.cpu().numpy()))
    np.testing.assert_array_equal(bits(as_np(got_g)), bits(want_g.cpu().numpy()))


def _atlas_cases(vkl, device_on, device_off, oracle, vox, **kw):
    """Samples and gradients of one float volume committed with the texture
    atlas (device_on) and without it (device_off), against the oracle."""
    ref = oracle.OracleVolume.dense_volume(vox, **kw)
    on = vkl.structured_regular(device_on, vox, **kw)
    off = vkl.structured_regular(device_off, vox, **kw)
    return ref, on, off


@pytest.mark.parametrize("case", ["plain", "index_origin", "cell_centered", "transform"])
def test_texture_atlas_bit_exact(vkl, oracle, case):
    """Trilinear samples and gradients of dense float volumes read through
    the z-plane texture atlas (tld4 footprint gathers) equal the bricked
    loads' and the oracle's bit for bit, inside, on the faces and outside
    the domain, for odd dims, index origins, cell-centered data, background
    values and a rotated transform."""
    on, off = vkl.Device("cuda"), vkl.Device("cuda")
    off.set_int("textureSampling", 0)
    dims = (67, 45, 33)
    vox = sinusoid_field(dims, seed=31)
    kw = {"plain": {}, "index_origin": {"index_origin": (-3, 2, 5), "background": [-1.5]},
          "cell_centered": {"cell_centered": True, "background": [0.25]},
          "transform": {"index_to_object": [0.8, 0.6, 0, -0.6, 0.8, 0, 0, 0, 1.25, 3.0, -2.0, 1.0]}}[case]
    ref, von, voff = _atlas_cases(vkl, on, off, oracle, vox, **kw)
    b = np.array(von.bounding_box(), np.float64)
    pts = uniform_points(200000, b[:3] - 2, b[3:] + 2, seed=32)
    for fv in (100,):
        son, soff = vkl.Sampler(von, filter=fv, gradient_filter=fv), vkl.Sampler(voff, filter=fv, gradient_filter=fv)
        want = ref.sample(pts, filter=fv)
        np.testing.assert_array_equal(bits(son.sample(pts)), bits(want))
        np.testing.assert_array_equal(bits(soff.sample(pts)), bits(want))
        gw = ref.gradient(pts, filter=fv)
        np.testing.assert_array_equal(bits(son.gradient(pts)), bits(gw))
        np.testing.assert_array_equal(bits(soff.gradient(pts)), bits(gw))


def test_texture_atlas_skipped_for_denormals(vkl, oracle):
    """The texture path flushes denormals to zero, so a float attribute with
    denormal voxels is sampled from the bricked copy: results stay the
    oracle's.  A second, denormal-free attribute of the same volume keeps
    its atlas."""
    on = vkl.Device("cuda")
    dims = (40, 36, 30)
    a = sinusoid_field(dims, seed=33) * np.float32(1e-37)  # many results below FLT_MIN
    a.reshape(-1)[::7] = np.float32(3e-39)  # denormal voxels
    b = sinusoid_field(dims, seed=34)
    ref = oracle.OracleVolume.dense_volume([a, b])
    vol = vkl.structured_regular(on, [a, b])
    smp = vkl.Sampler(vol)
    pts = uniform_points(100000, (-1, -1, -1), (40, 36, 30), seed=35)
    for attr in (0, 1):
        np.testing.assert_array_equal(bits(smp.sample(pts, attr=attr)), bits(ref.sample(pts, attr=attr)))
    assert (np.abs(ref.sample(pts, attr=0)) < np.float32(1.1754944e-38)).any()


def test_device_released_before_its_objects(vkl, oracle):
    """vklReleaseDevice frees the device only once its objects are gone, as
    in the reference (API.cpp:298-303, objects hold a reference to their
    device): a volume and sampler keep working after the device's release,
    and releasing them last frees it."""
    dev = vkl.Device("cuda")
    vox = sinusoid_field((40, 24, 20), seed=41)
    ref = oracle.OracleVolume.dense_volume(vox)
    vol = vkl.structured_regular(dev, vox)
    smp = vkl.Sampler(vol)
    pts = uniform_points(20000, (-1, -1, -1), (40, 24, 20), seed=42)
    handle, dev.handle = dev.handle, None
    dev.lib.vklReleaseDevice(handle)  # the application's handle goes first
    np.testing.assert_array_equal(bits(smp.sample(pts)), bits(ref.sample(pts)))
    np.testing.assert_array_equal(bits(smp.gradient(pts)), bits(ref.gradient(pts)))
    smp.release()
    vol.release()  # the last object: the device (and its atlas pool) go here
