"""GPU parity of the cuda device's VDB path against the oracle: tree
construction (node / leaf indexing and per-voxel value ranges bit-exact),
sparse sampling and gradients for all filters, FP16 leaves, tiles on upper
levels, maxSamplingDepth, node.data input, and the dense tree."""
import numpy as np
import pytest

from openvkl_b200.fields import shell_leaves, sinusoid_field, uniform_points
from tests.conftest import bits

pytestmark = pytest.mark.gpu


def _shell_vdb(domain=128, seed=5, dtype=np.float32, tiles=True):
    origins, values = shell_leaves(domain=domain, shells=2, thickness=0.06, seed=seed)
    L = len(origins)
    levels = np.full(L, 3, np.uint32)
    formats = np.ones(L, np.uint32)
    tile_vals = np.zeros(0, np.float32)
    if tiles:
        # level-2 tiles (128^3) and level-1 tiles (4096^3) away from the leaves
        t_orig = np.array([[domain + 4096, 0, 0], [0, domain + 128, 0], [8192, 8192, 8192]], np.int32)
        t_lvl = np.array([2, 2, 1], np.uint32)
        origins = np.concatenate([origins, t_orig])
        levels = np.concatenate([levels, t_lvl])
        formats = np.concatenate([formats, np.zeros(3, np.uint32)])
        tile_vals = np.array([0.25, 0.75, 0.5], np.float32)
    return origins, levels, formats, values.astype(dtype), tile_vals.astype(dtype)


def _check_tree(vol, ref, num_attr=1):
    for level in range(3):
        vox, rng, org = vol.tree_level(level)
        rvox, rrng, rorg = ref.level(level, num_attr)
        assert len(org) == ref.num_nodes(level)
        np.testing.assert_array_equal(vox, rvox)
        np.testing.assert_array_equal(org, rorg)
        np.testing.assert_array_equal(bits(rng), bits(rrng))
    assert vol.tree_level(3) == ref.num_nodes(3)


@pytest.mark.parametrize("dtype", [np.float32, np.float16])
def test_sparse_tree_and_sampling_bit_exact(vkl, device, oracle, dtype):
    origins, levels, formats, vals, tvals = _shell_vdb(dtype=dtype)
    ref = oracle.OracleVolume.vdb_volume(levels, origins, formats, vals, tvals)
    vol = vkl.vdb_volume(device, levels, origins, formats, packed_dense=vals, packed_tile=tvals)
    _check_tree(vol, ref)
    np.testing.assert_array_equal(vol.bounding_box(), ref.info()["bounds"])
    np.testing.assert_array_equal(vol.value_range(), ref.value_range())
    rng = np.random.default_rng(3)
    # points near active leaves and anywhere in the (large) domain
    leaf_pts = (origins[:len(vals) // 512][rng.integers(0, len(vals) // 512, 30000)]
                + rng.uniform(-2, 10, (30000, 3))).astype(np.float32)
    b = ref.info()["bounds"]
    far = uniform_points(10000, b[:3] - 4, b[3:] + 4, seed=4)
    pts = np.concatenate([leaf_pts, far])
    for fv in (0, 100, 200):
        smp = vkl.Sampler(vol, filter=fv, gradient_filter=fv)
        np.testing.assert_array_equal(bits(smp.sample(pts)), bits(ref.sample(pts, filter=fv)))
        np.testing.assert_array_equal(bits(smp.gradient(pts)), bits(ref.gradient(pts, filter=fv)))


def test_tree_walk_equals_leaf_map(vkl, device, oracle):
    # sampling normally reads the flat leaf map; with it turned off every tap
    # walks the tree: both must give the oracle's results
    origins, levels, formats, vals, tvals = _shell_vdb(domain=96, seed=12)
    ref = oracle.OracleVolume.vdb_volume(levels, origins, formats, vals, tvals)
    pts = (origins[np.random.default_rng(2).integers(0, len(origins), 20000)]
           + np.random.default_rng(3).uniform(-3, 11, (20000, 3))).astype(np.float32)
    for leaf_map in (True, False):
        vol = vkl.vdb_volume(device, levels, origins, formats, packed_dense=vals, packed_tile=tvals,
                             leaf_map=leaf_map)
        _check_tree(vol, ref)
        for fv in (0, 100, 200):
            smp = vkl.Sampler(vol, filter=fv, gradient_filter=fv)
            np.testing.assert_array_equal(bits(smp.sample(pts)), bits(ref.sample(pts, filter=fv)))
            np.testing.assert_array_equal(bits(smp.gradient(pts)), bits(ref.gradient(pts, filter=fv)))


@pytest.mark.parametrize("depth", [0, 1, 2])
def test_max_sampling_depth(vkl, device, oracle, depth):
    origins, levels, formats, vals, tvals = _shell_vdb(domain=64, seed=9)
    ref = oracle.OracleVolume.vdb_volume(levels, origins, formats, vals, tvals)
    vol = vkl.vdb_volume(device, levels, origins, formats, packed_dense=vals, packed_tile=tvals)
    smp = vkl.Sampler(vol, max_sampling_depth=depth)
    rng = np.random.default_rng(1)
    pts = (origins[rng.integers(0, len(origins), 5000)] + rng.uniform(0, 8, (5000, 3))).astype(np.float32)
    np.testing.assert_array_equal(bits(smp.sample(pts)),
                                  bits(ref.sample(pts, max_sampling_depth=depth)))


def test_node_data_input_matches_packed(vkl, device, oracle):
    origins, levels, formats, vals, tvals = _shell_vdb(domain=64, seed=2)
    n_dense = len(vals) // 512
    node_data = [vals[i * 512:(i + 1) * 512] for i in range(n_dense)] + [tvals[i:i + 1] for i in range(len(tvals))]
    ref = oracle.OracleVolume.vdb_volume(levels, origins, formats, vals, tvals)
    vol = vkl.vdb_volume(device, levels, origins, formats, node_data=node_data)
    rng = np.random.default_rng(7)
    pts = (origins[rng.integers(0, len(origins), 8000)] + rng.uniform(-1, 9, (8000, 3))).astype(np.float32)
    np.testing.assert_array_equal(bits(vkl.Sampler(vol).sample(pts)), bits(ref.sample(pts)))


def test_dense_tree_bit_exact(vkl, device, oracle):
    dims = (300, 140, 36)  # several level-2 nodes, partial leaves
    vox = sinusoid_field(dims, seed=5)
    ref = oracle.OracleVolume.dense_volume(vox, background=[-2.0])
    vol = vkl.structured_regular(device, vox, background=[-2.0])
    _check_tree(vol, ref)
    np.testing.assert_array_equal(vol.value_range(), ref.value_range())


def _planted_field(dims, dtype, seed):
    """A sinusoid field with NaN voxels, scattered -0.0 / +0.0 voxels, one
    slab of mixed-sign zeros (whole leaf windows whose range is zero) and one
    all-NaN block (leaf windows with no number at all)."""
    X, Y, Z = dims
    rng = np.random.default_rng(seed)
    v = sinusoid_field(dims, seed=seed).astype(np.float64)
    flat = v.reshape(-1)
    n = flat.size
    if np.issubdtype(dtype, np.floating):
        flat[rng.choice(n, n // 200, replace=False)] = np.nan
        flat[rng.choice(n, n // 200, replace=False)] = -0.0
    flat[rng.choice(n, n // 200, replace=False)] = 0.0
    v[Z // 3:Z // 3 + 12, :, :] = np.where(rng.random((min(12, Z - Z // 3), Y, X)) < 0.5, 0.0, -0.0)
    if np.issubdtype(dtype, np.floating):
        v[:10, :10, :10] = np.nan
    if dtype == np.uint8:
        return np.clip((v + 2.5) * 50, 0, 255).astype(np.uint8)
    return v.astype(dtype)


@pytest.mark.parametrize("dims", [(300, 140, 36), (320, 40, 24), (77, 45, 19), (9, 8, 17)])
@pytest.mark.parametrize("dtype", [np.float32, np.float16, np.float64, np.uint8])
@pytest.mark.parametrize("background", [None, -2.0, -0.0, 0.0])
def test_dense_leaf_ranges_nan_and_signed_zero(vkl, device, oracle, dims, dtype, background):
    """Leaf ranges of dense volumes with NaN and -0.0 voxels: a NaN voxel
    resets the running bound of the reference's fold (VdbSampler_dense.ih:
    35-105), and a zero bound takes the sign of the zero the fold meets
    last, so these windows depend on the fold order.  Compared bit for bit
    on the leaves' parent level (one leaf per voxel).  Upper levels and the
    volume range are compared by value: where +0.0 and -0.0 bounds of
    different leaves tie, the sign follows the tie rule of rkcommon's
    range1f::extend, which is not part of the reference tree."""
    vox = _planted_field(dims, dtype, seed=11)
    bg = None if background is None else [background]
    ref = oracle.OracleVolume.dense_volume(vox, background=bg)
    vol = vkl.structured_regular(device, vox, background=bg)
    for level in range(3):
        _, rng, org = vol.tree_level(level)
        _, rrng, rorg = ref.level(level, 1)
        np.testing.assert_array_equal(org, rorg)
        if level == 2:
            np.testing.assert_array_equal(bits(rng), bits(rrng))
        else:
            np.testing.assert_array_equal(rng, rrng)
    np.testing.assert_array_equal(vol.value_range(), ref.value_range())
    # the planted cases reach the reference-order path: some leaf ranges
    # differ from the NaN-ignoring min / max of their windows
    if np.issubdtype(dtype, np.floating) and background is None and dims[0] == 300:
        X, Y, Z = dims
        f = vox.astype(np.float32)
        vox2, rng, _ = vol.tree_level(2)
        leaf = (vox2 & 3) == 3
        got = rng[leaf]
        plain = []
        for lz in range((Z + 7) // 8):
            for ly in range((Y + 7) // 8):
                for lx in range((X + 7) // 8):
                    w = f[max(8 * lz - 1, 0):8 * lz + 10, max(8 * ly - 1, 0):8 * ly + 10,
                          max(8 * lx - 1, 0):8 * lx + 10]
                    w = w[~np.isnan(w)]
                    plain.append((w.min(), w.max()) if w.size else (np.inf, -np.inf))
        # leaves are x-fastest, level-2 voxels z-fastest within a node
        plain = np.array(plain, np.float32)
        assert len(plain) == len(got)
        assert not np.array_equal(np.sort(bits(plain[:, 0])), np.sort(bits(got[:, 0])))


def test_inner_node_observer_matches_oracle(vkl, device, oracle):
    origins, levels, formats, vals, tvals = _shell_vdb(domain=64, seed=4)
    ref = oracle.OracleVolume.vdb_volume(levels, origins, formats, vals, tvals)
    vol = vkl.vdb_volume(device, levels, origins, formats, packed_dense=vals, packed_tile=tvals)
    for depth in (0, 1, 2):
        got = vol.inner_nodes(max_depth=depth)
        want = ref.inner_nodes(max_depth=depth)
        key = lambda a: a[np.lexsort(a.T[::-1])]
        np.testing.assert_array_equal(key(got), key(want))


def test_vdb_validation_errors(vkl, device):
    data = np.zeros(512, np.float32)
    with pytest.raises(vkl.VKLError) as e:
        vkl.vdb_volume(device, [4], [[0, 0, 0]], [1], node_data=[data])
    assert e.value.code == 1 and e.value.msg == "invalid node level 4 for this vdb configuration"
    with pytest.raises(vkl.VKLError, match="Node data too small"):
        vkl.vdb_volume(device, [3], [[0, 0, 0]], [1], node_data=[data[:1]])


def _volume_buffers_style(vkl, device, levels, origins, formats, node_data, temporal_format=None,
                          structured_steps=None):
    """A vdb volume with the parameter set the reference's VdbVolumeBuffers
    utility gives every volume it creates (utility/vdb/include/openvkl/
    utility/vdb/VdbVolumeBuffers.h:668-816): node.temporalFormat, the
    per-node temporal arrays (zeros / null data handles for constant nodes),
    indexToObject, and node.data."""
    n = len(levels)
    v = vkl.Volume(device, "vdb")
    v.set_param("indexToObject", vkl.VKL_AFFINE3F, np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32))
    v.set_data("node.level", vkl.Data(device, np.ascontiguousarray(levels, np.uint32)))
    v.set_data("node.origin", vkl.Data(device, np.ascontiguousarray(origins, np.int32).reshape(-1),
                                       vkl_type=vkl.VKL_VEC3I))
    v.set_data("node.format", vkl.Data(device, np.ascontiguousarray(formats, np.uint32)))
    tf = np.zeros(n, np.uint32) if temporal_format is None else temporal_format
    v.set_data("node.temporalFormat", vkl.Data(device, tf))
    steps = np.zeros(n, np.int32) if structured_steps is None else structured_steps
    v.set_data("node.temporallyStructuredNumTimesteps", vkl.Data(device, steps))
    v.set_data("node.temporallyUnstructuredIndices", vkl.Data(device, objects=[None] * n))
    v.set_data("node.temporallyUnstructuredTimes", vkl.Data(device, objects=[None] * n))
    v.set_data("node.data", vkl.Data(device, objects=[vkl.Data(device, a) for a in node_data]))
    v.commit()
    return v


def test_vdb_volume_buffers_parameter_set(vkl, device, oracle):
    """Volumes made by the reference's VdbVolumeBuffers (the path OpenVDB
    ingestion takes) carry temporal parameters even when every node is
    temporally constant; they commit and sample like volumes without them.
    A non-constant node and mis-sized temporal arrays are rejected."""
    origins, levels, formats, vals, tvals = _shell_vdb(domain=64, seed=3)
    n_dense = len(vals) // 512
    node_data = [vals[i * 512:(i + 1) * 512] for i in range(n_dense)] + [tvals[i:i + 1] for i in range(len(tvals))]
    ref = oracle.OracleVolume.vdb_volume(levels, origins, formats, vals, tvals)
    vol = _volume_buffers_style(vkl, device, levels, origins, formats, node_data)
    plain = vkl.vdb_volume(device, levels, origins, formats, node_data=node_data)
    # node.data input: leaf pointers hold node indices (VdbVolume.cpp:306-317),
    # so the tree is compared with the same input minus the temporal arrays
    for level in range(3):
        for a, b in zip(vol.tree_level(level), plain.tree_level(level)):
            np.testing.assert_array_equal(a, b)
    rng = np.random.default_rng(8)
    pts = (origins[rng.integers(0, len(origins), 8000)] + rng.uniform(-1, 9, (8000, 3))).astype(np.float32)
    for fv in (0, 100, 200):
        got = vkl.Sampler(vol, filter=fv).sample(pts)
        np.testing.assert_array_equal(bits(got), bits(vkl.Sampler(plain, filter=fv).sample(pts)))
        np.testing.assert_array_equal(bits(got), bits(ref.sample(pts, filter=fv)))
    n = len(levels)
    moving = np.zeros(n, np.uint32)
    moving[0] = 1  # VKL_TEMPORAL_FORMAT_STRUCTURED
    with pytest.raises(vkl.VKLError, match="temporally varying"):
        _volume_buffers_style(vkl, device, levels, origins, formats, node_data, temporal_format=moving)
    with pytest.raises(vkl.VKLError, match="If node.temporallyStructuredNumTimesteps is set, it must have the "
                                           "same size as node.data"):
        _volume_buffers_style(vkl, device, levels, origins, formats, node_data,
                              structured_steps=np.zeros(n - 1, np.int32))


def test_dense_temporal_parameters(vkl, device, oracle):
    """structuredRegular: temporallyStructuredNumTimesteps = 0 means constant
    data (DenseVdbVolume.cpp:149-186) and is accepted; > 0 makes the data
    temporally structured, which needs that many values per voxel."""
    vox = sinusoid_field((20, 18, 16), seed=2)
    v = vkl.Volume(device, "structuredRegular")
    v.set_vec3i("dimensions", (20, 18, 16))
    v.set_int("temporallyStructuredNumTimesteps", 0)
    v.set_data("data", vkl.Data(device, vox))
    v.commit()
    ref = oracle.OracleVolume.dense_volume(vox)
    pts = uniform_points(4000, (0, 0, 0), (19, 17, 15), seed=5)
    np.testing.assert_array_equal(bits(vkl.Sampler(v).sample(pts)), bits(ref.sample(pts)))
    v.set_int("temporallyStructuredNumTimesteps", 2)
    with pytest.raises(vkl.VKLError, match="has 5760 elements, but expected 11520"):
        v.commit()


@pytest.mark.parametrize("fv,depth", [(0, 3), (100, 3), (200, 3), (100, 1)])
def test_leaf_access_observer(vkl, device, oracle, fv, depth):
    """vklNewSamplerObserver(sampler, "LeafNodeAccess"): after sampling, the
    observer's buffer (one uint32 per leaf) holds 1 exactly at the leaves
    the oracle's tree walks reached (VdbSampleInner.ih.in:68-74), including
    tiles and excluding voxels the maxSamplingDepth cut stops above."""
    origins, levels, formats, vals, tvals = _shell_vdb()
    ref = oracle.OracleVolume.vdb_volume(levels, origins, formats, vals, tvals)
    vol = vkl.vdb_volume(device, levels, origins, formats, packed_dense=vals, packed_tile=tvals)
    smp = vkl.Sampler(vol, filter=fv, max_sampling_depth=depth)
    obs = smp.leaf_access_observer()
    assert not obs.read_uint().any()
    rng = np.random.default_rng(11)
    n_leaves = len(vals) // 512
    pts = (origins[:n_leaves][rng.integers(0, n_leaves, 3000)] + rng.uniform(-2, 10, (3000, 3))).astype(np.float32)
    b = ref.info()["bounds"]
    pts = np.concatenate([pts, uniform_points(2000, b[:3] - 4, b[3:] + 4, seed=12)])
    smp.sample(pts)
    got = obs.read_uint()
    want_s, want = ref.sample_observed(pts, len(got), filter=fv, max_sampling_depth=depth)
    np.testing.assert_array_equal(got, want)
    if depth == 3:
        assert got.any()
    # a second observer records only what is sampled after it exists
    obs2 = smp.leaf_access_observer()
    smp.sample(pts[:50])
    _, want2 = ref.sample_observed(pts[:50], len(got), filter=fv, max_sampling_depth=depth)
    np.testing.assert_array_equal(obs2.read_uint(), want2)
    obs.release()
    np.testing.assert_array_equal(bits(smp.sample(pts)), bits(want_s))


def test_leaf_access_observer_needs_a_vdb_volume(vkl, device):
    vol = vkl.structured_regular(device, sinusoid_field((16, 16, 16), seed=1))
    with pytest.raises(vkl.VKLError, match="unsupported sampler observer type"):
        vkl.Sampler(vol).leaf_access_observer()
