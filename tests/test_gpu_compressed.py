"""Compressed VDB leaves (FP16 / BF16 / FP8-E4M3 codes with a per-leaf scale
and offset, decoded in FP32; an extension of the cuda device).

Parity: the device's compressed volume equals, bit for bit, the oracle's
volume built from the decoded leaves (the oracle restates the quantizer):
tree and value ranges, samples and gradients for every filter, intervals
and hits.  Error: samples against the FP64 trilinear evaluation of the
original float leaves, as max |error| relative to the volume's value range.
The bound written per format is the code rounding (2^-11, 2^-8, 2^-4 of a
leaf's half range; a leaf's half range is at most half the value range) on
top of the FP32 path's own error.
"""
import numpy as np
import pytest

from openvkl_b200.fields import random_rays, shell_leaves
from tests.conftest import bits

pytestmark = pytest.mark.gpu

FORMATS = {"fp16": 2.0 ** -11, "bf16": 2.0 ** -8, "fp8": 2.0 ** -4}


def _shells(domain=128, seed=5):
    origins, values = shell_leaves(domain=domain, shells=2, thickness=0.06, seed=seed)
    L = len(origins)
    # level-2 and level-1 tiles away from the leaves: tiles stay float
    t_orig = np.array([[domain + 4096, 0, 0], [0, domain + 128, 0], [8192, 8192, 8192]], np.int32)
    origins = np.concatenate([origins, t_orig])
    levels = np.concatenate([np.full(L, 3, np.uint32), np.array([2, 2, 1], np.uint32)])
    formats = np.concatenate([np.ones(L, np.uint32), np.zeros(3, np.uint32)])
    tiles = np.array([0.25, 0.75, 0.5], np.float32)
    return origins, levels, formats, values.astype(np.float32), tiles


def _points(origins, n_leaf, b, seed):
    rng = np.random.default_rng(seed)
    leaf = (origins[:n_leaf][rng.integers(0, n_leaf, 20000)] + rng.uniform(-2, 10, (20000, 3)))
    far = rng.uniform(b[:3] - 4, b[3:] + 4, (5000, 3))
    return np.concatenate([leaf, far]).astype(np.float32)


@pytest.mark.parametrize("fmt", list(FORMATS))
def test_compressed_vdb_bit_exact_vs_decoded_oracle(vkl, device, oracle, fmt):
    origins, levels, formats, vals, tiles = _shells()
    dec, _ = oracle.quantize_leaves(fmt, vals)
    ref = oracle.OracleVolume.vdb_volume(levels, origins, formats, dec, tiles)
    vol = vkl.vdb_volume(device, levels, origins, formats, packed_dense=vals, packed_tile=tiles,
                         compression=fmt)
    for level in range(3):
        vox, rng, org = vol.tree_level(level)
        rvox, rrng, rorg = ref.level(level, 1)
        np.testing.assert_array_equal(vox, rvox)
        np.testing.assert_array_equal(org, rorg)
        np.testing.assert_array_equal(bits(rng), bits(rrng))
    np.testing.assert_array_equal(vol.value_range(), ref.value_range())
    b = ref.info()["bounds"]
    pts = _points(origins, len(vals) // 512, b, seed=3)
    for fv in (0, 100, 200):
        smp = vkl.Sampler(vol, filter=fv, gradient_filter=fv)
        np.testing.assert_array_equal(bits(smp.sample(pts)), bits(ref.sample(pts, filter=fv)))
        np.testing.assert_array_equal(bits(smp.gradient(pts)), bits(ref.gradient(pts, filter=fv)))
    o, d, t = random_rays(1500, b[:3], b[3:], seed=4)
    ctx = vkl.IntervalIteratorContext(vkl.Sampler(vol), value_ranges=[[0.4, 0.6]], hint=0.5)
    got, gcnt = ctx.iterate_n(o, d, t, max_per_ray=1024)
    want, wcnt = ref.intervals(o, d, t, value_ranges=[[0.4, 0.6]], hint=0.5, max_intervals=1024)
    np.testing.assert_array_equal(gcnt, wcnt)
    for r in range(len(gcnt)):
        np.testing.assert_array_equal(bits(got[r, :gcnt[r]]), bits(want[r, :wcnt[r]]))
    hctx = vkl.HitIteratorContext(vkl.Sampler(vol), np.array([0.25, 0.5], np.float32))
    got, gcnt = hctx.iterate_n(o, d, t, max_per_ray=64)
    want, wcnt = ref.hits(o, d, t, np.array([0.25, 0.5], np.float32), max_hits=64)
    np.testing.assert_array_equal(gcnt, wcnt)
    for r in range(len(gcnt)):
        np.testing.assert_array_equal(bits(got[r, :gcnt[r]]), bits(want[r, :wcnt[r]]))
    assert gcnt.sum() > 0


@pytest.mark.parametrize("fmt", list(FORMATS))
def test_compressed_error_vs_fp64(vkl, device, oracle, fmt):
    origins, levels, formats, vals, tiles = _shells(seed=6)
    ref = oracle.OracleVolume.vdb_volume(levels, origins, formats, vals, tiles)
    vol = vkl.vdb_volume(device, levels, origins, formats, packed_dense=vals, packed_tile=tiles,
                         compression=fmt)
    n_leaf = len(vals) // 512
    rng = np.random.default_rng(9)
    # interior points: every trilinear tap inside active leaves' neighbourhood
    pts = (origins[:n_leaf][rng.integers(0, n_leaf, 50000)] + rng.uniform(0.5, 7.5, (50000, 3))).astype(np.float32)
    exact = ref.sample_fp64(pts, filter=100)
    got = vkl.Sampler(vol, filter=100).sample(pts).astype(np.float64)
    plain = vkl.Sampler(vkl.vdb_volume(device, levels, origins, formats, packed_dense=vals,
                                       packed_tile=tiles), filter=100).sample(pts).astype(np.float64)
    ok = ~np.isnan(exact)
    vrange = float(vals.max() - vals.min())
    err = np.abs(got[ok] - exact[ok]).max() / vrange
    err_plain = np.abs(plain[ok] - exact[ok]).max() / vrange
    assert err_plain <= 1e-6  # the FP32 path
    assert err <= FORMATS[fmt] * 0.5 + 1e-6, (fmt, err)
    print(f"{fmt}: max |error| / value range = {err:.3e} (FP32 path {err_plain:.3e})")


# Stencil-block leaves ("<fmt>_blocks"): each dense leaf is stored as 8
# blocks of 5^3 codes holding its voxels plus the next voxel on the +x/+y/+z
# side, with one scale and offset over that 9^3 window; a trilinear stencil
# whose base voxel lies in a dense leaf reads its 8 corners from one block.
# The oracle restates the window, the quantizer and that corner rule.
@pytest.mark.parametrize("fmt", list(FORMATS))
def test_blocked_vdb_bit_exact_vs_oracle(vkl, device, oracle, fmt):
    origins, levels, formats, vals, tiles = _shells()
    ref, _ = oracle.vdb_blocked_volume(fmt, levels, origins, formats, vals, tiles)
    vol = vkl.vdb_volume(device, levels, origins, formats, packed_dense=vals, packed_tile=tiles,
                         compression=fmt + "_blocks")
    for level in range(3):
        vox, rng, org = vol.tree_level(level)
        rvox, rrng, rorg = ref.level(level, 1)
        np.testing.assert_array_equal(vox, rvox)
        np.testing.assert_array_equal(bits(rng), bits(rrng))
    np.testing.assert_array_equal(vol.value_range(), ref.value_range())
    b = ref.info()["bounds"]
    pts = _points(origins, len(vals) // 512, b, seed=3)
    for fv in (0, 100, 200):
        smp = vkl.Sampler(vol, filter=fv, gradient_filter=fv)
        np.testing.assert_array_equal(bits(smp.sample(pts)), bits(ref.sample(pts, filter=fv)))
        np.testing.assert_array_equal(bits(smp.gradient(pts)), bits(ref.gradient(pts, filter=fv)))
    # a depth-limited walk never reaches a leaf: the per-corner path
    for depth in (1, 2):
        smp = vkl.Sampler(vol, filter=100, max_sampling_depth=depth)
        np.testing.assert_array_equal(bits(smp.sample(pts)),
                                      bits(ref.sample(pts, filter=100, max_sampling_depth=depth)))
    o, d, t = random_rays(1500, b[:3], b[3:], seed=4)
    ctx = vkl.IntervalIteratorContext(vkl.Sampler(vol), value_ranges=[[0.4, 0.6]], hint=0.5)
    got, gcnt = ctx.iterate_n(o, d, t, max_per_ray=1024)
    want, wcnt = ref.intervals(o, d, t, value_ranges=[[0.4, 0.6]], hint=0.5, max_intervals=1024)
    np.testing.assert_array_equal(gcnt, wcnt)
    for r in range(len(gcnt)):
        np.testing.assert_array_equal(bits(got[r, :gcnt[r]]), bits(want[r, :wcnt[r]]))
    hctx = vkl.HitIteratorContext(vkl.Sampler(vol), np.array([0.25, 0.5], np.float32))
    got, gcnt = hctx.iterate_n(o, d, t, max_per_ray=64)
    want, wcnt = ref.hits(o, d, t, np.array([0.25, 0.5], np.float32), max_hits=64)
    np.testing.assert_array_equal(gcnt, wcnt)
    for r in range(len(gcnt)):
        np.testing.assert_array_equal(bits(got[r, :gcnt[r]]), bits(want[r, :wcnt[r]]))
    assert gcnt.sum() > 0


@pytest.mark.parametrize("fmt", list(FORMATS))
def test_blocked_error_vs_fp64(vkl, device, oracle, fmt):
    """Same bound as the per-leaf codes: a window's half range is at most half
    the value range of these volumes (no background inside the windows)."""
    origins, levels, formats, vals, tiles = _shells(seed=6)
    ref = oracle.OracleVolume.vdb_volume(levels, origins, formats, vals, tiles)
    vol = vkl.vdb_volume(device, levels, origins, formats, packed_dense=vals, packed_tile=tiles,
                         compression=fmt + "_blocks")
    n_leaf = len(vals) // 512
    rng = np.random.default_rng(9)
    pts = (origins[:n_leaf][rng.integers(0, n_leaf, 50000)] + rng.uniform(0.5, 7.5, (50000, 3))).astype(np.float32)
    exact = ref.sample_fp64(pts, filter=100)
    got = vkl.Sampler(vol, filter=100).sample(pts).astype(np.float64)
    ok = ~np.isnan(exact)
    vrange = float(vals.max() - vals.min())
    err = np.abs(got[ok] - exact[ok]).max() / vrange
    assert err <= FORMATS[fmt] * 0.5 + 1e-6, (fmt, err)
    print(f"{fmt}_blocks: max |error| / value range = {err:.3e}")
