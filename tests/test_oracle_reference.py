"""Pins the oracle (C++ restatement of the reference CPU device) against the
reference's own test assertions and fixtures.

The reference CPU device cannot be built here (ISPC / rkcommon / Embree are
absent), so these checks restate the reference's Catch2 tests with their
fields, tolerances and expected values:

* tricubic coefficient map == the reference's expanded table
  (VdbSampler_tricubic.ih:34-389 -> tests/golden/tricubic_coeff_map.json)
* vertex sampling == procedural value within 1e-4, all voxel types
  (testing/apps/tests/structured_regular_volume.h:10-55)
* gradients of the wavelet within 0.1 of the analytic gradient away from the
  boundary (structured_volume_gradients.cpp:15-70)
* nearest gradients are exactly 0 (vdb_volume.cpp:523-525)
* dense <-> sparse equivalence: structuredRegular(cellCentered) and vdb over
  the same voxels give identical boxes, samples, gradients and intervals
  (vdb_volume_dense.cpp:115-349)
* interval continuity: first interval at the box entry, shared endpoints,
  last at the exit (interval_iterator.cpp:42-133)
* Z-ramp hits at t = iso + 1 within 1e-3, one hit per isovalue
  (hit_iterator.cpp:13-135)
* InnerNode observer: node boxes contain their voxels and ranges contain the
  voxel values (vdb_volume_inner_node_observer.cpp:78-132)
* commit errors of malformed VDB input (vdb_volume.cpp:17-79)
* dense leaf value ranges equal a direct restatement of the reference's fold
  order on volumes with NaN and -0.0 voxels (VdbSampler.ispc:460-557,
  VdbSampler_dense.ih:35-105)
"""
import json
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def wavelet(p):
    p = np.asarray(p, np.float64)
    return np.sin(3 * p[..., 0]) + np.sin(3 * p[..., 1]) + np.cos(3 * p[..., 2])


def wavelet_grad(p):
    p = np.asarray(p, np.float64)
    return np.stack([3 * np.cos(3 * p[..., 0]), 3 * np.cos(3 * p[..., 1]), -3 * np.sin(3 * p[..., 2])], -1)


def object_coords(dims, origin, spacing):
    X, Y, Z = dims
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    o = np.asarray(origin, np.float32)
    s = np.asarray(spacing, np.float32)
    return np.stack([o[0] + x.astype(np.float32) * s[0], o[1] + y.astype(np.float32) * s[1],
                     o[2] + z.astype(np.float32) * s[2]], -1).astype(np.float32)


def sanitize(v, dtype):
    """Procedural value stored as the voxel type (testing/volume/procedural_functions.h)."""
    if np.issubdtype(dtype, np.integer):
        info = np.iinfo(dtype)
        return np.clip(v, info.min, info.max).astype(dtype)
    return v.astype(dtype)


def test_tricubic_map_matches_reference_table(oracle):
    ref = json.load(open(os.path.join(HERE, "golden", "tricubic_coeff_map.json")))["rows"]
    start, cols, w = oracle.tricubic_map()
    assert len(cols) == sum(len(r) for r in ref) == 1000
    for r in range(64):
        mine = [(float(w[e]), int(cols[e])) for e in range(start[r], start[r + 1])]
        assert mine == [(float(a), int(b)) for a, b in ref[r]], f"row {r}"


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.uint16, np.float16, np.float32, np.float64])
def test_vertex_sampling_all_types(oracle, dtype):
    dims = (32, 32, 32)
    oc = object_coords(dims, (0, 0, 0), (1, 1, 1))
    vox = sanitize(wavelet(oc) * (50 if np.issubdtype(dtype, np.integer) else 1), dtype)
    v = oracle.OracleVolume.dense_volume(vox, grid_origin=(0, 0, 0), grid_spacing=(1, 1, 1))
    # step 2, never touching the upper boundary (structured_regular_volume.h:60-77)
    pts = oc[::2, ::2, ::2].reshape(-1, 3)
    truth = vox[::2, ::2, ::2].reshape(-1).astype(np.float32)
    for f in (oracle.FILTER_NEAREST, oracle.FILTER_LINEAR):
        s = v.sample(pts, filter=f)
        np.testing.assert_allclose(s, truth, rtol=0, atol=1e-4 * max(1.0, float(np.abs(truth).max())))
    # cubic interpolates the vertex values too, away from the filter support edge
    inner = oc[2:-2:2, 2:-2:2, 2:-2:2].reshape(-1, 3)
    tin = vox[2:-2:2, 2:-2:2, 2:-2:2].reshape(-1).astype(np.float32)
    s = v.sample(inner, filter=oracle.FILTER_CUBIC)
    np.testing.assert_allclose(s, tin, rtol=0, atol=1e-4 * max(1.0, float(np.abs(tin).max())))


def test_upper_boundary_vertex_reads_background(oracle):
    # taps beyond the last vertex read the undefined (NaN) background
    vox = np.ones((8, 8, 8), np.float32)
    v = oracle.OracleVolume.dense_volume(vox)
    assert np.isnan(v.sample(np.array([[7, 7, 7]], np.float32))[0])
    v2 = oracle.OracleVolume.dense_volume(vox, background=[0.25])
    assert v2.sample(np.array([[7.5, 3, 3]], np.float32))[0] == np.float32(0.5 * 1 + 0.5 * 0.25)


def test_xyz_field_is_reproduced_by_trilinear(oracle):
    dims = (16, 16, 16)
    sp = 1.0 / 15
    oc = object_coords(dims, (0, 0, 0), (sp, sp, sp))
    vox = (oc[..., 0] * oc[..., 1] * oc[..., 2]).astype(np.float32)
    v = oracle.OracleVolume.dense_volume(vox, grid_origin=(0, 0, 0), grid_spacing=(sp, sp, sp))
    rng = np.random.default_rng(0)
    pts = rng.uniform(0.0, 0.999, size=(2000, 3)).astype(np.float32)
    s = v.sample(pts)
    # trilinear of a trilinear field is exact up to rounding
    np.testing.assert_allclose(s, pts[:, 0] * pts[:, 1] * pts[:, 2], atol=1e-4)


@pytest.mark.parametrize("filt", ["linear", "cubic"])
def test_wavelet_gradients_within_reference_tolerance(oracle, filt):
    # 128^3 over a box of size 2, boundaries skipped (structured_volume_gradients.cpp:15-70)
    n = 128
    sp = 2.0 / (n - 1)
    oc = object_coords((n, n, n), (-1, -1, -1), (sp, sp, sp))
    v = oracle.OracleVolume.dense_volume(wavelet(oc).astype(np.float32), grid_origin=(-1, -1, -1),
                                         grid_spacing=(sp, sp, sp))
    f = oracle.FILTER_LINEAR if filt == "linear" else oracle.FILTER_CUBIC
    # the cubic stencil reaches one voxel further (vdb_volume.cpp:249-270 skips it)
    lo = 1 if filt == "linear" else 2
    pts = oc[lo:-lo:5, lo:-lo:5, lo:-lo:5].reshape(-1, 3)
    g = v.gradient(pts, filter=f)
    np.testing.assert_allclose(g, wavelet_grad(pts), atol=0.1)
    assert np.all(v.gradient(pts[:100], filter=oracle.FILTER_NEAREST) == 0)


def _dense_and_sparse(oracle, dims, seed=0):
    rng = np.random.default_rng(seed)
    X, Y, Z = dims
    oc = object_coords(dims, (0, 0, 0), (0.1, 0.1, 0.1))
    vox = (wavelet(oc) + rng.uniform(-0.01, 0.01, size=oc.shape[:3])).astype(np.float32)
    dense = oracle.OracleVolume.dense_volume(vox, cell_centered=True)
    origins, packed = [], []
    for z in range(0, Z, 8):
        for y in range(0, Y, 8):
            for x in range(0, X, 8):
                origins.append((x, y, z))
                packed.append(vox[z:z + 8, y:y + 8, x:x + 8].transpose(2, 1, 0).reshape(-1))
    L = len(origins)
    sparse = oracle.OracleVolume.vdb_volume(np.full(L, 3), np.array(origins), np.ones(L),
                                            np.concatenate(packed))
    return vox, dense, sparse


def test_dense_sparse_equivalence(oracle):
    vox, dense, sparse = _dense_and_sparse(oracle, (24, 16, 32))
    di, si = dense.info(), sparse.info()
    np.testing.assert_array_equal(di["bounds"], si["bounds"])
    np.testing.assert_array_equal(di["domain"], si["domain"])
    np.testing.assert_array_equal(dense.value_range(), sparse.value_range())
    rng = np.random.default_rng(1)
    pts = rng.uniform(-0.5, [24.5, 16.5, 32.5], size=(5000, 3)).astype(np.float32)
    for f in (oracle.FILTER_NEAREST, oracle.FILTER_LINEAR, oracle.FILTER_CUBIC):
        a, b = dense.sample(pts, filter=f), sparse.sample(pts, filter=f)
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
        ga, gb = dense.gradient(pts, filter=f), sparse.gradient(pts, filter=f)
        np.testing.assert_array_equal(ga.view(np.uint32), gb.view(np.uint32))
    o = rng.uniform(-5, 40, size=(300, 3)).astype(np.float32)
    d = rng.normal(size=(300, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = np.tile(np.array([[0, 1e30]], np.float32), (300, 1))
    for hint in (0.0, 0.5):
        ia, ca = dense.intervals(o, d, t, hint=hint)
        ib, cb = sparse.intervals(o, d, t, hint=hint)
        np.testing.assert_array_equal(ca, cb)
        np.testing.assert_array_equal(ia, ib)


def test_interval_continuity(oracle):
    n = 64
    vox = np.random.default_rng(0).random((n, n, n)).astype(np.float32)
    v = oracle.OracleVolume.dense_volume(vox)
    rng = np.random.default_rng(2)
    o = np.tile(np.array([[-10.0, 31.3, 31.7]], np.float32), (200, 1)) + rng.uniform(-2, 2, (200, 3)).astype(np.float32)
    d = np.tile(np.array([[1.0, 0.0, 0.0]], np.float32), (200, 1)) + rng.uniform(-0.2, 0.2, (200, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = np.tile(np.array([[0, 1e30]], np.float32), (200, 1))
    iv, cnt = v.intervals(o, d, t, hint=0.5, max_intervals=256)
    dom = v.info()["domain"]
    for r in range(200):
        k = int(cnt[r])
        assert k > 0
        ints = iv[r, :k]
        # consecutive intervals share endpoints exactly
        assert np.all(ints[1:, 0] == ints[:-1, 1])
        # first starts at the box entry, last ends at the exit
        inv = 1.0 / d[r].astype(np.float64)
        ta = (dom[:3] - o[r]) * inv
        tb = (dom[3:] - o[r]) * inv
        t0, t1 = np.max(np.minimum(ta, tb)), np.min(np.maximum(ta, tb))
        assert ints[0, 0] == pytest.approx(t0, abs=1e-3)
        assert ints[-1, 1] == pytest.approx(t1, abs=1e-3)
        # nominalDeltaT = min_i 1/|dir_i| in index space (spacing 1)
        assert ints[0, 4] == pytest.approx(1.0 / np.max(np.abs(d[r])), rel=1e-6)


def test_interval_value_range_filtering(oracle):
    n = 32
    z = np.arange(n, dtype=np.float32)
    vox = np.broadcast_to(z[:, None, None], (n, n, n)).copy()  # value = z index
    v = oracle.OracleVolume.dense_volume(vox)
    o = np.array([[5.5, 5.5, -5.0]], np.float32)
    d = np.array([[0.0, 0.0, 1.0]], np.float32)
    t = np.array([[0, 1e30]], np.float32)
    all_iv, all_c = v.intervals(o, d, t, hint=0.5)
    sel_iv, sel_c = v.intervals(o, d, t, value_ranges=[[10.0, 12.0]], hint=0.5)
    assert 0 < sel_c[0] < all_c[0]
    for iv in sel_iv[0, :sel_c[0]]:
        assert iv[3] >= 10.0 and iv[2] <= 12.0


def test_zramp_hits(oracle):
    n = 128
    sp = 1.0 / (n - 1)
    oc = object_coords((n, n, n), (0, 0, 0), (sp, sp, sp))
    v = oracle.OracleVolume.dense_volume(oc[..., 2].astype(np.float32), grid_origin=(0, 0, 0),
                                         grid_spacing=(sp, sp, sp))
    isos = []
    f = np.float32(0.1)
    while f < 1:
        isos.append(f)
        f = np.float32(f + np.float32(0.1))
    hits, cnt = v.hits(np.array([[0.5, 0.5, -1]], np.float32), np.array([[0, 0, 1]], np.float32),
                       np.array([[0, np.inf]], np.float32), np.array(isos, np.float32))
    assert cnt[0] == len(isos)
    for i, iso in enumerate(isos):
        assert hits[0, i, 1] == iso
        assert hits[0, i, 0] == pytest.approx(float(iso) + 1.0, abs=1e-3)


def test_inner_node_observer(oracle):
    vox, dense, sparse = _dense_and_sparse(oracle, (40, 24, 16))
    for vol in (dense, sparse):
        nodes = vol.inner_nodes(max_depth=2)
        assert len(nodes) == (40 // 8) * (24 // 8) * (16 // 8)
        for b in nodes:
            lo = np.floor(b[:3] / 0.1 + 0.5).astype(int) if False else b[:3].astype(int)
            x0, y0, z0 = [int(round(c)) for c in b[:3]]
            blk = vox[z0:z0 + 8, y0:y0 + 8, x0:x0 + 8]
            assert b[6] <= blk.min() and b[7] >= blk.max()


def test_vdb_commit_errors(oracle):
    data = np.zeros(512, np.float32)
    with pytest.raises(RuntimeError, match="^invalid node level 4 for this vdb configuration$"):
        oracle.OracleVolume.vdb_volume([4], [[0, 0, 0]], [1], data)
    with pytest.raises(RuntimeError, match="there must not be any leaf nodes on level 0"):
        oracle.OracleVolume.vdb_volume([0], [[0, 0, 0]], [0], np.zeros(0, np.float32),
                                       packed_tile=np.zeros(1, np.float32))
    with pytest.raises(RuntimeError, match="leaf nodes are only supported on the lowest level"):
        oracle.OracleVolume.vdb_volume([2], [[0, 0, 0]], [1], data)


def _reference_fold_leaf_range(vox, ox, oy, oz, bg):
    """One leaf's value range in the reference's own fold order, restated in
    Python: the 27 neighbour windows [7,8) | [0,8) | [0,2) per axis in
    neighbour order (x, y, z), voxels x outer / z inner, extend() as
    (a < b ? a : b, a > b ? a : b) (so a NaN voxel resets the running
    bound), a neighbour outside the domain contributing (bg, bg), and
    neighbour bounds that are NaN skipped (VdbSampler.ispc:460-557,
    VdbSampler_dense.ih:35-105)."""
    Z, Y, X = vox.shape
    win = [(7, 8), (0, 8), (0, 2)]
    fmin = lambda a, b: a if a < b else b
    fmax = lambda a, b: a if a > b else b
    lo, hi = np.float32(np.inf), np.float32(-np.inf)
    for ix in range(3):
        for iy in range(3):
            for iz in range(3):
                nx, ny, nz = ox + (ix - 1) * 8, oy + (iy - 1) * 8, oz + (iz - 1) * 8
                if not (0 <= nx < X and 0 <= ny < Y and 0 <= nz < Z):
                    nlo = nhi = np.float32(bg)
                else:
                    nlo, nhi = np.float32(np.inf), np.float32(-np.inf)
                    for x in range(*win[ix]):
                        for y in range(*win[iy]):
                            for z in range(*win[iz]):
                                px, py, pz = nx + x, ny + y, nz + z
                                if px < X and py < Y and pz < Z:
                                    v = np.float32(vox[pz, py, px])
                                    nlo, nhi = fmin(nlo, v), fmax(nhi, v)
                if not np.isnan(nlo):
                    lo = fmin(lo, nlo)
                if not np.isnan(nhi):
                    hi = fmax(hi, nhi)
    return lo, hi


@pytest.mark.parametrize("background", [float("nan"), -0.0, 0.5])
def test_leaf_ranges_follow_reference_fold_order(oracle, background):
    """The oracle's dense leaf ranges (the parity target of the GPU commit)
    equal the reference's fold order bit for bit on a volume with NaN and
    -0.0 voxels, where the order decides the result."""
    rng = np.random.default_rng(17)
    dims = (19, 17, 13)
    vox = rng.uniform(-1, 1, dims[::-1]).astype(np.float32)
    flat = vox.reshape(-1)
    flat[rng.choice(flat.size, flat.size // 40, replace=False)] = np.nan
    flat[rng.choice(flat.size, flat.size // 20, replace=False)] = -0.0
    flat[rng.choice(flat.size, flat.size // 20, replace=False)] = 0.0
    vox[4:9] = np.where(rng.random(vox[4:9].shape) < 0.5, np.float32(0.0), np.float32(-0.0))
    ref = oracle.OracleVolume.dense_volume(vox, background=[background])
    v2, rng2, _ = ref.level(2, 1)
    leaf = (v2 & 3) == 3
    got = rng2[leaf]
    # one level-2 node; its voxels index leaves as x * 256 + y * 16 + z
    want = []
    for lx in range((dims[0] + 7) // 8):
        for ly in range((dims[1] + 7) // 8):
            for lz in range((dims[2] + 7) // 8):
                want.append(_reference_fold_leaf_range(vox, 8 * lx, 8 * ly, 8 * lz, background))
    want = np.array(want, np.float32)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_macrocell_interval_continuity_and_ranges(oracle):
    """The 16^3-voxel macrocell walk (the reference's legacy structuredRegular
    iterator, GridAccelerator.ispc:146-240): the interval continuity assertion
    of interval_iterator.cpp:108 (consecutive intervals share endpoints), the
    first and last intervals at the box's entry and exit, nominalDeltaT =
    min_i spacing_i / |dir_i| (GridAcceleratorIterator.ispc:76-78), and every
    macrocell range equal to the min / max over its 17^3 clamped vertices."""
    n = 70
    vox = np.random.default_rng(0).random((n, n, n)).astype(np.float32)
    v = oracle.OracleVolume.dense_volume(vox, grid_origin=(1.0, -2.0, 0.5), grid_spacing=(0.5, 0.5, 0.5))
    rng = np.random.default_rng(2)
    o = np.tile(np.array([[-10.0, 15.3, 17.7]], np.float32), (200, 1)) + rng.uniform(-2, 2, (200, 3)).astype(np.float32)
    d = np.tile(np.array([[1.0, 0.0, 0.0]], np.float32), (200, 1)) + rng.uniform(-0.3, 0.3, (200, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = np.tile(np.array([[0, 1e30]], np.float32), (200, 1))
    iv, cnt = v.macrocell_intervals(o, d, t, max_intervals=64)
    lo = np.array([1.0, -2.0, 0.5])
    hi = lo + (n - 1) * 0.5
    for r in range(200):
        k = int(cnt[r])
        assert k > 0
        ints = iv[r, :k]
        assert np.all(ints[1:, 0] == ints[:-1, 1])
        inv = 1.0 / d[r].astype(np.float64)
        ta, tb = (lo - o[r]) * inv, (hi - o[r]) * inv
        t0, t1 = np.max(np.minimum(ta, tb)), np.min(np.maximum(ta, tb))
        assert ints[0, 0] == pytest.approx(t0, abs=1e-3)
        assert ints[-1, 1] == pytest.approx(t1, abs=1e-3)
        assert ints[0, 4] == pytest.approx(0.5 / np.max(np.abs(d[r])), rel=1e-6)
    mr = v.macrocell_ranges()
    assert mr.shape == (5, 5, 5, 2)
    for cz, cy, cx in [(0, 0, 0), (4, 4, 4), (2, 3, 1), (4, 0, 2)]:
        blk = vox[cz * 16:min(n, cz * 16 + 17), cy * 16:min(n, cy * 16 + 17), cx * 16:min(n, cx * 16 + 17)]
        assert mr[cz, cy, cx, 0] == blk.min() and mr[cz, cy, cx, 1] == blk.max()
