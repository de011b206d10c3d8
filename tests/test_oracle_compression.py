"""Pins the oracle's restatement of compressed leaf storage (the cuda
device's FP16 / BF16 / FP8-E4M3 codes with a per-leaf scale and offset; an
extension without a reference counterpart).

The format rounding is checked against torch's independent float16,
bfloat16 and float8_e4m3fn conversions (round to nearest, ties to even) on
values inside each format's range; torch's E4M3 conversion turns overflow
into NaN where the device saturates (its SATFINITE conversion), so overflow
is checked against the saturation rule directly.  The leaf quantizer is
checked against its stated error bound.
"""
import numpy as np
import pytest

from oracle import pyoracle as O


def _values(n, seed):
    rng = np.random.default_rng(seed)
    mag = np.exp2(rng.uniform(-12, 9, n))
    x = (rng.choice([-1.0, 1.0], n) * mag).astype(np.float32)
    # exact ties of the coarsest format and a few specials
    ties = np.array([1.0625, 17.0, 2.0 ** -9 * 2.5, 2.0 ** -9 * 1.5, -3.25, 0.0, -0.0, 1.0 + 2.0 ** -11,
                     1.0 + 3 * 2.0 ** -11, 1.0 + 2.0 ** -8], np.float32)
    return np.concatenate([x, ties])


@pytest.mark.parametrize("fmt", ["fp16", "bf16", "fp8"])
def test_round_format_matches_torch(fmt):
    import torch
    tdt = {"fp16": torch.float16, "bf16": torch.bfloat16, "fp8": torch.float8_e4m3fn}[fmt]
    x = _values(200000, seed=1)
    if fmt == "fp8":
        x = x[np.abs(x) <= 448]
    got = O.round_format(fmt, x)
    want = torch.from_numpy(x).to(tdt).float().numpy()
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_fp8_saturates_and_keeps_nan():
    x = np.array([448, 463.9, 464, 500, 1e30, np.inf, -1e9, np.nan], np.float32)
    got = O.round_format("fp8", x)
    np.testing.assert_array_equal(got[:7], [448, 448, 448, 448, 448, 448, -448])
    assert np.isnan(got[7])


def test_fp16_overflow_rounds_to_inf():
    got = O.round_format("fp16", np.array([65504, 65519.9, 65520, -1e6], np.float32))
    assert got[0] == 65504 and got[1] == 65504 and np.isinf(got[2]) and got[3] == -np.inf


@pytest.mark.parametrize("fmt,rel", [("fp16", 2.0 ** -11), ("bf16", 2.0 ** -8), ("fp8", 2.0 ** -4)])
def test_quantize_leaves_error_bound(fmt, rel):
    rng = np.random.default_rng(7)
    leaves = rng.normal(size=(64, 512)).astype(np.float32) * rng.uniform(0.01, 100, (64, 1)).astype(np.float32)
    leaves += rng.uniform(-50, 50, (64, 1)).astype(np.float32)
    dec, so = O.quantize_leaves(fmt, leaves)
    dec = dec.reshape(64, 512)
    half = 0.5 * (leaves.max(1) - leaves.min(1))
    err = np.abs(dec.astype(np.float64) - leaves).max(1)
    # code rounding (rel * half) plus the float decode roundings
    bound = rel * half + 4 * np.finfo(np.float32).eps * np.abs(leaves).max(1)
    assert np.all(err <= bound)
    np.testing.assert_allclose(so[:, 1], 0.5 * leaves.min(1) + 0.5 * leaves.max(1), rtol=0, atol=0)


def test_quantize_constant_and_nan_leaves():
    leaves = np.zeros((3, 512), np.float32)
    leaves[0] = 0.375
    leaves[1, :] = np.nan
    leaves[2] = np.linspace(-1, 1, 512, dtype=np.float32)
    leaves[2, 17] = np.nan
    for fmt in ("fp16", "bf16", "fp8"):
        dec, so = O.quantize_leaves(fmt, leaves)
        dec = dec.reshape(3, 512)
        assert np.all(dec[0] == np.float32(0.375)) and so[0, 0] == 1.0  # constant leaf is exact
        assert np.all(np.isnan(dec[1]))
        assert np.isnan(dec[2, 17]) and not np.isnan(np.delete(dec[2], 17)).any()
        assert dec[2, 0] == -1 and dec[2, -1] == 1  # the extremes decode exactly


@pytest.mark.parametrize("fmt", ["fp16", "bf16", "fp8"])
def test_blocked_windows_and_corner_rule(fmt):
    """Stencil-block leaves in the oracle: each dense leaf's 9^3 window holds
    its own voxels in [0, 8)^3 and the neighbours' (or empty space's) on the
    +x/+y/+z side; groups of 512 quantize as whole leaves do; a stencil inside
    one leaf reads the same decoded values through the window as through the
    leaf, and a stencil crossing into a neighbour reads this leaf's window."""
    from openvkl_b200.fields import shell_leaves
    origins, values = shell_leaves(domain=64, shells=1, thickness=0.1, seed=4)
    L = len(origins)
    lv, fm = np.full(L, 3, np.uint32), np.ones(L, np.uint32)
    flt = O.OracleVolume.vdb_volume(lv, origins, fm, values)
    w = flt.leaf_windows()
    np.testing.assert_array_equal(w[:, :8, :8, :8].reshape(L, -1), values.reshape(L, -1))
    # the +x face of leaf 0 equals the float volume's samples at those voxels
    face = origins[0] + np.stack(np.meshgrid([8], np.arange(9), np.arange(9), indexing="ij"), -1).reshape(-1, 3)
    np.testing.assert_array_equal(w[0, 8].reshape(-1), flt.sample(face.astype(np.float32), filter=0))
    d1, s1 = O.quantize_groups(fmt, values, 512)
    d2, s2 = O.quantize_leaves(fmt, values)
    np.testing.assert_array_equal(d1, d2)
    np.testing.assert_array_equal(s1, s2)
    vol, sos = O.vdb_blocked_volume(fmt, lv, origins, fm, values)
    dec, so = O.quantize_groups(fmt, w, 729)
    np.testing.assert_array_equal(so, sos[0])
    dec = dec.reshape(L, 9, 9, 9)
    rng = np.random.default_rng(2)
    leaf = rng.integers(0, L, 4000)
    inner = (origins[leaf] + rng.uniform(0, 7, (4000, 3))).astype(np.float32)
    plain = O.OracleVolume.vdb_volume(lv, origins, fm, np.ascontiguousarray(dec[:, :8, :8, :8]).reshape(-1))
    np.testing.assert_array_equal(vol.sample(inner), plain.sample(inner))
    # base voxel on a leaf's last voxel in x: the corners come from the window
    edge = origins[leaf].astype(np.float32) + np.float32([7.5, 3.25, 2.75])
    f = np.float32(0.5)
    lo, hi = dec[leaf, 7, 3:5, 2:4], dec[leaf, 8, 3:5, 2:4]

    def lerp(t, a, b):
        return (np.float32(1) - t) * a + t * b

    def plane(p):
        return lerp(np.float32(0.25), lerp(np.float32(0.75), p[:, 0, 0], p[:, 0, 1]),
                    lerp(np.float32(0.75), p[:, 1, 0], p[:, 1, 1]))
    np.testing.assert_array_equal(vol.sample(edge), lerp(f, plane(lo), plane(hi)))
