"""vklCudaDenseValueRangeNoAlloc, the allocation-free value-range entry point.

Its result is compared with the existing path, vklGetValueRange of a
structuredRegular volume committed over the same voxels, on two calls in a
row (the second runs on scratch left by the first).  Tolerance: exact; both
paths take min/max over the same voxel windows of NaN-free data.  This file
sorts last so it also runs after every other GPU test in one process.
"""
import numpy as np
import pytest

from openvkl_b200.fields import sinusoid_field

pytestmark = pytest.mark.gpu


def _voxels(dims, dtype, seed):
    f = sinusoid_field(dims, seed=seed)
    if np.issubdtype(dtype, np.integer):
        info = np.iinfo(dtype)
        f = np.clip(f * 40 + (0 if info.min < 0 else 60), info.min, info.max)
    return f.astype(dtype)


def _as_cuda(vox):
    import torch
    if vox.dtype == np.uint16:  # passed as raw 16-bit words with an explicit type
        return torch.from_numpy(vox.view(np.int16)).cuda()
    return torch.from_numpy(vox).cuda()


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.uint16, np.float16, np.float32, np.float64])
@pytest.mark.parametrize("dims,background", [((21, 17, 13), None), ((64, 64, 64), None),
                                             ((40, 9, 33), -7.5), ((1, 1, 1), 3.0)])
def test_matches_committed_volume(vkl, device, dtype, dims, background):
    import torch
    vox = _voxels(dims, dtype, seed=11)
    vol = vkl.structured_regular(device, vox, background=background)
    expected = vol.value_range()
    d = _as_cuda(vox)
    out = torch.full((2,), float("nan"), dtype=torch.float32, device="cuda")
    t = vkl.VKL_USHORT if dtype == np.uint16 else None
    bg = float("nan") if background is None else background
    for _ in range(2):
        out.fill_(float("nan"))
        vkl.dense_value_range_no_alloc(device, d, out, background=bg, vkl_type=t)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_array_equal(got, expected)  # tolerance: exact


def test_large_volume_many_blocks(vkl, device):
    # 256 x 256 x 512 voxels = 65536 leaves = 256 blocks: exercises the
    # last-block reduction over many partials and the counter re-arm.
    import torch
    g = torch.Generator(device="cuda").manual_seed(5)
    d = torch.rand((512, 256, 256), generator=g, device="cuda", dtype=torch.float32) * 8 - 3
    d[300, 17, 200] = -11.25
    d[5, 250, 3] = 42.5
    vol = vkl.structured_regular(device, d.cpu().numpy())
    expected = vol.value_range()
    out = torch.empty(2, dtype=torch.float32, device="cuda")
    for _ in range(2):
        vkl.dense_value_range_no_alloc(device, d, out)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), expected)
    assert expected[0] == np.float32(-11.25) and expected[1] == np.float32(42.5)


def test_no_device_memory_taken_after_setup(vkl, device):
    import torch
    d = torch.from_numpy(_voxels((48, 40, 56), np.float32, seed=2)).cuda()
    out = torch.empty(2, dtype=torch.float32, device="cuda")
    vkl.dense_value_range_no_alloc(device, d, out)  # set-up call
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    torch0 = torch.cuda.memory_allocated()
    for _ in range(5):
        vkl.dense_value_range_no_alloc(device, d, out)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == torch0


def test_rejects_volumes_beyond_scratch(vkl, device):
    import ctypes
    import torch
    d = torch.zeros(8, dtype=torch.float32, device="cuda")
    out = torch.empty(2, dtype=torch.float32, device="cuda")
    lib = device.lib
    # 2049 x 2048 x 2048 voxels = 257 * 256 * 256 leaves > 16,777,216: rejected
    # on the host before anything is launched (the buffer is never read).
    code = lib.vklCudaDenseValueRangeNoAlloc(device.handle, ctypes.c_void_p(d.data_ptr()),
                                             vkl.VKL_FLOAT, 2049, 2048, 2048, 0.0,
                                             ctypes.c_void_p(out.data_ptr()))
    device.pending = None
    assert code == 2  # VKL_INVALID_ARGUMENT
    assert "exceed the maximum of 16777216" in device.last_error()[1]
    code = lib.vklCudaDenseValueRangeNoAlloc(device.handle, None, vkl.VKL_FLOAT, 8, 8, 8, 0.0,
                                             ctypes.c_void_p(out.data_ptr()))
    device.pending = None
    assert code == 2
    code = lib.vklCudaDenseValueRangeNoAlloc(device.handle, ctypes.c_void_p(d.data_ptr()),
                                             vkl.VKL_INT, 2, 2, 2, 0.0,
                                             ctypes.c_void_p(out.data_ptr()))
    device.pending = None
    assert code == 2


@pytest.mark.parametrize("dtype", [np.float16, np.float32, np.float64])
def test_signed_zero_bounds_compare_by_value(vkl, device, dtype):
    # A volume whose minimum is zero with both +0.0 and -0.0 voxels present:
    # the two paths fold them in different orders, so the zero bound may come
    # back with either sign bit; the ranges must be equal by value.
    import torch
    dims = (24, 20, 18)
    vox = np.abs(_voxels(dims, np.float32, seed=3)).astype(dtype) + dtype(0.5)
    vox[2:9, 3:7, 1:12] = dtype(0.0)
    vox[4:6, 4:6, 2:10] = -dtype(0.0)
    vox[15, 11, 20] = -dtype(0.0)
    vol = vkl.structured_regular(device, vox)
    expected = vol.value_range()
    assert expected[0] == 0.0
    d = _as_cuda(vox)
    out = torch.empty(2, dtype=torch.float32, device="cuda")
    for _ in range(2):
        vkl.dense_value_range_no_alloc(device, d, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[0] == expected[0] and got[1] == expected[1]  # by value: -0.0 == +0.0
