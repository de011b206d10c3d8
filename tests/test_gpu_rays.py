"""Ray-run sampling (k_sample_rays.cu): large trilinear calls on dense float
volumes whose points are runs of S samples per ray are computed 8 runs at a
time with a warp's lanes across neighbouring rays.  The results must equal
the oracle bit for bit whatever path runs; the device's debug log names the
run length the detector chose.  Covered: S = 64 / 128 / 256 / 512 with whole
and partial tiles, the texture-atlas and bricked-load fields, samples and
gradients, a point array that is not 16-byte aligned (no bulk copies), and
points that are not ray runs (random points: the detector declines)."""
import numpy as np
import pytest

from openvkl_b200.fields import orbit_camera_samples, sinusoid_field, uniform_points
from tests.conftest import bits

pytestmark = pytest.mark.gpu

DIMS = (200, 180, 160)


@pytest.fixture(scope="module")
def setup(vkl, oracle):
    vox = sinusoid_field(DIMS, seed=41)
    ref = oracle.OracleVolume.dense_volume(vox)
    devs = {}
    for name, tex in (("atlas", 1), ("bricked", 0)):
        d = vkl.Device("cuda")
        d.set_int("textureSampling", tex)
        log = []
        d.capture_log(log)
        d.set_int("logLevel", 1)  # debug
        devs[name] = (d, vkl.structured_regular(d, vox), log)
    return ref, devs


def _rays(S, drop=0):
    w = 64 if S >= 128 else 128
    h = (1 << 20) // (w * S) + 3
    pts = orbit_camera_samples(w, h, S, (0, 0, 0), tuple(x - 1 for x in DIMS), seed=S)
    return pts[:len(pts) - drop]


@pytest.mark.parametrize("S", [64, 128, 256, 512])
@pytest.mark.parametrize("field", ["atlas", "bricked"])
def test_ray_runs_bit_exact(vkl, setup, S, field):
    import torch
    ref, devs = setup
    dev, vol, log = devs[field]
    smp = vkl.Sampler(vol)
    pts = _rays(S, drop=5 * S + 3)  # a partial last tile
    log.clear()
    tp = torch.from_numpy(pts).cuda()
    got = smp.sample(tp).cpu().numpy()
    assert any(f"runs of {S} samples" in m for m in log), log
    np.testing.assert_array_equal(bits(got), bits(ref.sample_parallel(pts)))
    g = smp.gradient(tp).cpu().numpy()
    np.testing.assert_array_equal(bits(g), bits(ref.gradient_parallel(pts)))


def test_unaligned_points_and_random_points(vkl, setup):
    import torch
    ref, devs = setup
    dev, vol, log = devs["atlas"]
    smp = vkl.Sampler(vol)
    pts = _rays(256)
    tp = torch.from_numpy(pts).cuda()
    log.clear()
    got = smp.sample(tp[1:]).cpu().numpy()  # 12-byte offset: plain loads instead of bulk copies
    np.testing.assert_array_equal(bits(got), bits(ref.sample_parallel(pts[1:])))
    rnd = uniform_points(1 << 21, (0, 0, 0), tuple(x - 1 for x in DIMS), seed=3)
    log.clear()
    got = smp.sample(torch.from_numpy(rnd).cuda()).cpu().numpy()
    assert not any("runs of" in m for m in log), log
    np.testing.assert_array_equal(bits(got), bits(ref.sample_parallel(rnd)))


def test_host_pointer_chunks(vkl, setup):
    """Host arrays go through the chunked copy pipeline; the run length is
    detected on the first chunk and used for all."""
    ref, devs = setup
    dev, vol, log = devs["atlas"]
    smp = vkl.Sampler(vol)
    pts = orbit_camera_samples(128, 288, 256, (0, 0, 0), tuple(x - 1 for x in DIMS), seed=7)  # 9.4M points
    log.clear()
    got = smp.sample(pts)
    assert any("runs of 256 samples" in m for m in log), log
    np.testing.assert_array_equal(bits(got), bits(ref.sample_parallel(pts)))
