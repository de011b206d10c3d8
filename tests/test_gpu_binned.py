"""GPU parity of binned sampling: large incoherent calls on dense float
volumes larger than L2 are counting-sorted by index-space cell on the
device before the tile kernel.  The binned results must equal the unbinned
path's bit for bit (device parameter "binnedSampling" 0), which the other
GPU tests pin to the oracle; a subset is also checked against the oracle
here directly.  Dense float attributes are sampled through their texture
atlas by default, which needs no binning; these tests use a device with
"textureSampling" 0, so the binned path runs for every filter, and compare
the linear results with the atlas path's too."""
import numpy as np
import pytest

from tests.conftest import bits

pytestmark = pytest.mark.gpu


def _i2o():
    ang = 0.4
    c, s_ = np.cos(ang), np.sin(ang)
    return np.array([0.9 * c, 0.9 * s_, 0, -1.1 * s_, 1.1 * c, 0, 0, 0, 1.0, 5.0, -3.0, 2.0], np.float32)


@pytest.fixture(scope="module")
def big_volume(vkl):
    """A 420^3 float volume (296 MB, above the binning threshold) with a
    rotated, scaled index-to-object transform, on a device without texture
    atlases (bricked loads, binned when incoherent)."""
    from openvkl_b200.fields import sinusoid_field_torch
    dev = vkl.Device("cuda")
    dev.set_int("textureSampling", 0)
    dims = (420, 420, 420)
    vox = sinusoid_field_torch(dims, seed=31)
    vol = vkl.structured_regular(dev, vox, shared=True, index_to_object=_i2o())
    yield vol, vox, dims, dev


def _points(vol, n, seed, pad=2.0):
    import torch
    b = np.asarray(vol.bounding_box(), np.float64)
    g = torch.Generator(device="cuda").manual_seed(seed)
    lo = torch.tensor(b[:3] - pad, device="cuda", dtype=torch.float32)
    hi = torch.tensor(b[3:] + pad, device="cuda", dtype=torch.float32)
    return (lo + torch.rand((n, 3), generator=g, device="cuda") * (hi - lo)).contiguous()


@pytest.mark.parametrize("filt", [100, 200, 0])
def test_binned_equals_unbinned(vkl, device, big_volume, filt):
    import torch
    vol, vox, _, dev = big_volume
    smp = vkl.Sampler(vol, filter=filt, gradient_filter=filt)
    n = (1 << 27) + 4099 if filt == 100 else (1 << 24) + 77  # linear: two binning passes
    pts = _points(vol, n, seed=filt + 1)
    dev.set_int("binnedSampling", 1)
    got = smp.sample(pts)
    grad = smp.gradient(pts) if filt != 0 else None
    torch.cuda.synchronize()
    dev.set_int("binnedSampling", 0)
    want = smp.sample(pts)
    np.testing.assert_array_equal(bits(got.cpu().numpy()), bits(want.cpu().numpy()))
    if grad is not None:
        wg = smp.gradient(pts)
        np.testing.assert_array_equal(bits(grad.cpu().numpy()), bits(wg.cpu().numpy()))
    dev.set_int("binnedSampling", 1)
    if filt == 100:
        # the same volume through its texture atlas (default device)
        atlas = vkl.Sampler(vkl.structured_regular(device, vox, shared=True, index_to_object=_i2o()))
        m = 1 << 24
        np.testing.assert_array_equal(bits(atlas.sample(pts[:m]).cpu().numpy()), bits(got[:m].cpu().numpy()))


def test_binned_against_oracle_subset(vkl, device, oracle, big_volume):
    vol, vox, dims, _ = big_volume
    smp = vkl.Sampler(vol, filter=100)
    pts = _points(vol, (1 << 24) + 5, seed=9)
    got = smp.sample(pts).cpu().numpy()
    host = pts.cpu().numpy()
    idx = np.random.default_rng(3).choice(len(host), 20000, replace=False)
    ref = oracle.OracleVolume.dense_volume(vox.cpu().numpy(), index_to_object=_i2o())
    np.testing.assert_array_equal(bits(got[idx]), bits(ref.sample(host[idx])))
