"""GPU parity of the __device__ API and of the example renderers built on it
(openvkl_b200/renderers/renderers.cu), through the renderer library's C ABI:

- per-point vklComputeSample / vklComputeGradient called from a user kernel
  equal the host API's vklComputeSampleN / vklComputeGradientN bit for bit;
- the ray march iterator, interval iterator debug and hit iterator renderers
  (vklInitIntervalIterator / vklIterateInterval / vklComputeSample, and
  vklInitHitIterator / vklIterateHit / vklComputeGradient in device code)
  produce the same image, bit for bit, as the oracle's restatement of the
  reference's renderers (oracle OracleVolume.render), on a dense and on a
  sparse VDB volume;
- the density path tracer (Woodcock tracking with isotropic scattering,
  progressive frames) accumulates the same RGBA and weight buffers as the
  oracle's restatement, bit for bit, on a dense, a sparse and a temporally
  varying volume with motion blur (its log / sincos are one shared source,
  openvkl_b200/renderers/pt_math.h)."""
import numpy as np
import pytest

from openvkl_b200.fields import shell_leaves, sinusoid_field
from tests.conftest import bits

pytestmark = pytest.mark.gpu

W, H = 80, 60


@pytest.fixture(scope="module")
def render():
    from openvkl_b200 import render as R
    R.load_library()
    return R


def _dense(vkl, device, oracle):
    vox = sinusoid_field((40, 36, 44), seed=23)
    i2o = np.array([0.9, 0.1, 0, -0.1, 0.9, 0, 0, 0, 1.1, 2.0, -1.0, 0.5], np.float32)
    return (oracle.OracleVolume.dense_volume(vox, index_to_object=i2o),
            vkl.structured_regular(device, vox, index_to_object=i2o))


def _sparse(vkl, device, oracle):
    origins, values = shell_leaves(domain=128, shells=2, thickness=0.06, seed=8)
    L = len(origins)
    ref = oracle.OracleVolume.vdb_volume(np.full(L, 3), origins, np.ones(L), values)
    vol = vkl.vdb_volume(device, np.full(L, 3), origins, np.ones(L), packed_dense=values)
    return ref, vol


@pytest.mark.parametrize("kind", ["dense", "sparse"])
@pytest.mark.parametrize("filt", [0, 100, 200])
def test_device_api_sampling_equals_host_api(vkl, device, oracle, render, kind, filt):
    import torch
    _, vol = (_dense if kind == "dense" else _sparse)(vkl, device, oracle)
    smp = vkl.Sampler(vol, filter=filt, gradient_filter=filt)
    b = np.asarray(vol.bounding_box(), np.float32)
    g = torch.Generator(device="cuda").manual_seed(filt + 1)
    lo, hi = torch.tensor(b[:3] - 1, device="cuda"), torch.tensor(b[3:] + 1, device="cuda")
    pts = (lo + torch.rand((30000, 3), generator=g, device="cuda") * (hi - lo)).contiguous()
    s, gr = render.sample_points(smp, pts)
    np.testing.assert_array_equal(bits(s.cpu().numpy()), bits(smp.sample(pts).cpu().numpy()))
    np.testing.assert_array_equal(bits(gr.cpu().numpy()), bits(smp.gradient(pts).cpu().numpy()))


@pytest.mark.parametrize("kind", ["dense", "sparse"])
@pytest.mark.parametrize("renderer", ["ray_march", "interval_debug", "hits"])
def test_renderers_match_oracle(vkl, device, oracle, render, kind, renderer):
    ref, vol = (_dense if kind == "dense" else _sparse)(vkl, device, oracle)
    smp = vkl.Sampler(vol, filter=100, gradient_filter=100)
    lo, hi = (float(x) for x in vol.value_range())
    ranges = np.array([[lo + 0.3 * (hi - lo), hi]], np.float32)
    isos = np.array([lo + 0.4 * (hi - lo), lo + 0.7 * (hi - lo)], np.float32)
    ictx = vkl.IntervalIteratorContext(smp, value_ranges=ranges, hint=0.5)
    hctx = vkl.HitIteratorContext(smp, isos)
    cam = render.orbit_camera(vol.bounding_box(), W, H)
    tf = render.transfer_function((lo, hi))
    kw = dict(sampling_rate=2.0, interval_color_scale=6.0, interval_opacity=0.3)
    got = render.render(renderer, smp, cam, W, H, tf=tf, interval_context=ictx, hit_context=hctx, **kw)
    want = ref.render(render.RENDERERS[renderer], cam.as_array(), render.DEFAULT_TF, (lo, hi), W, H,
                      vol.bounding_box(), filter=100, gradient_filter=100, value_ranges=ranges, hint=0.5,
                      iso_values=isos, **kw)
    got = got.cpu().numpy()
    assert np.isfinite(want).all() and (want[:, :, :3] > 0).any(), "empty or broken reference image"
    np.testing.assert_array_equal(bits(got), bits(want))


def test_image_files(vkl, device, oracle, render, tmp_path):
    _, vol = _dense(vkl, device, oracle)
    smp = vkl.Sampler(vol)
    img = render.render("ray_march", smp, render.orbit_camera(vol.bounding_box(), 32, 24), 32, 24,
                        interval_context=vkl.IntervalIteratorContext(smp))
    render.write_pfm(tmp_path / "f.pfm", img)
    render.write_ppm(tmp_path / "f.ppm", img)
    assert (tmp_path / "f.pfm").stat().st_size == len(b"PF\n32 24\n-1.0\n") + 32 * 24 * 12
    assert (tmp_path / "f.ppm").read_bytes().startswith(b"P6\n32 24\n255\n")


@pytest.mark.parametrize("kind", ["dense", "sparse", "temporal"])
def test_density_path_tracer_matches_oracle(vkl, device, oracle, render, kind):
    import torch
    if kind == "temporal":
        dims = (36, 30, 28)
        base = sinusoid_field(dims, seed=29)
        data = np.stack([base, base * 0.5 + 0.3, -base], -1).astype(np.float32).reshape(-1)
        ref = oracle.OracleVolume.dense_temporal(data, dims, num_timesteps=3)
        vol = vkl.structured_regular(device, data, dims=dims, num_timesteps=3)
        kw = dict(motion_blur=True, shutter=0.6, time=0.4)
    else:
        ref, vol = (_dense if kind == "dense" else _sparse)(vkl, device, oracle)
        kw = {}
    smp = vkl.Sampler(vol, filter=100)
    lo, hi = (float(x) for x in vol.value_range())
    cam = render.orbit_camera(vol.bounding_box(), W, H)
    tf = render.transfer_function((lo, hi))
    span = float(np.max(np.asarray(vol.bounding_box())[3:] - np.asarray(vol.bounding_box())[:3]))
    pkw = dict(sigma_t_scale=8.0 / span, sigma_s_scale=1.0, max_num_scatters=3, ambient_light_intensity=1.5,
               show_bbox=True, **kw)
    rgba, wts = render.path_trace(smp, cam, W, H, frames=(0, 1), tf=tf, **pkw)
    want, wwant = ref.path_trace(cam.as_array(), render.DEFAULT_TF, (lo, hi), W, H, vol.bounding_box(),
                                 frames=(0, 1), filter=100, **pkw)
    torch.cuda.synchronize()
    got = rgba.cpu().numpy()
    assert (want[:, :, :3] > 0).any() and np.isfinite(want).all(), "empty or broken reference image"
    np.testing.assert_array_equal(bits(wts.cpu().numpy()), bits(wwant))
    np.testing.assert_array_equal(bits(got), bits(want))
