"""Learned surrogate (hash grid + MLP on the tensor cores; an extension).

* forward: the device's surrogate samples equal the oracle's FP16-rounded
  forward pass (oracle/surrogate.py) within 2e-3 absolute + 2e-3 relative
  (FP32 accumulation order is the only difference);
* gradients: the device's table and weight gradients of sum((y - t)^2)
  equal the oracle's backward pass within 2 % of each tensor's norm, and the
  losses within 1e-3 relative;
* training gain: trained on a volume's plain samples the surrogate's error is
  far below the untrained network's and below the best constant predictor;
  after calibration against the plain sampler with threshold 1e-2, sampling
  with fallback stays within the threshold on the calibration points (a
  smooth field, so that regions can pass: per-voxel noise would flag all).
"""
import numpy as np
import pytest

from openvkl_b200.fields import sinusoid_field
from oracle import surrogate as S

pytestmark = pytest.mark.gpu


def _smooth(dims):
    X, Y, Z = dims
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    return (0.5 + 0.3 * np.sin(2 * np.pi * x / X) * np.cos(2 * np.pi * y / Y) + 0.2 * z / Z).astype(np.float32)


def _setup(vkl, device, dims=(40, 36, 44), log2_table=12, base=4.0, smooth=False):
    vox = _smooth(dims) if smooth else sinusoid_field(dims, seed=17)
    vol = vkl.structured_regular(device, vox)
    smp = vkl.Sampler(vol)
    sur = vkl.Surrogate(smp, log2_table=log2_table, base_resolution=base, growth=1.5)
    b = vol.bounding_box()
    cfg = S.Config(levels=16, log2_table=log2_table, lo=b[:3], hi=b[3:], res=sur.resolutions)
    return vol, smp, sur, cfg, b


def _params(cfg, seed, table_scale):
    p = S.init_params(cfg, seed=seed, table_scale=table_scale)
    return p, p[0].reshape(-1), np.concatenate([p[1].reshape(-1), p[2].reshape(-1), p[3].reshape(-1), p[4]])


def test_forward_matches_oracle(vkl, device):
    import torch
    vol, smp, sur, cfg, b = _setup(vkl, device)
    p, table, weights = _params(cfg, seed=3, table_scale=0.5)
    sur.set_parameters(table, weights)
    rng = np.random.default_rng(5)
    pts = (b[:3] + rng.random((3000, 3)) * (b[3:] - b[:3])).astype(np.float32)
    got = sur.sample(torch.from_numpy(pts).cuda(), fallback=False).cpu().numpy().astype(np.float64)
    want, _ = S.forward(cfg, p, pts, fp16=True)
    np.testing.assert_allclose(got, want, atol=2e-3, rtol=2e-3)
    assert np.std(want) > 1e-2  # the comparison is not trivial


def test_gradients_match_oracle(vkl, device):
    import torch
    vol, smp, sur, cfg, b = _setup(vkl, device)
    p, table, weights = _params(cfg, seed=4, table_scale=0.3)
    sur.set_parameters(table, weights)
    rng = np.random.default_rng(6)
    pts = (b[:3] + rng.random((1000, 3)) * (b[3:] - b[:3])).astype(np.float32)
    tgt = rng.random(1000).astype(np.float32)
    loss, gt, gw = sur.gradient(torch.from_numpy(pts).cuda(), torch.from_numpy(tgt).cuda())
    rl, rt, r1, r2, r3, r4 = S.backward(cfg, p, pts, tgt, fp16=True)
    assert abs(loss - rl) <= 1e-3 * rl
    offs = np.cumsum([0, 64 * 32, 64 * 64, 64 * 64, 64])
    for k, ref in enumerate((r1, r2, r3, r4)):
        g = gw[offs[k]:offs[k + 1]]
        err = np.linalg.norm(g - ref.reshape(-1)) / np.linalg.norm(ref)
        assert err < 2e-2, (k, err)
    err = np.linalg.norm(gt - rt.reshape(-1)) / np.linalg.norm(rt)
    assert err < 2e-2, err


def test_training_gains_over_untrained_and_fallback_bounds_error(vkl, device):
    import torch
    vol, smp, sur, cfg, b = _setup(vkl, device, dims=(128, 128, 128), log2_table=15, base=8.0, smooth=True)
    p, table, weights = _params(cfg, seed=7, table_scale=1e-4)
    sur.set_parameters(table, weights)
    lo, hi = torch.tensor(b[:3]).cuda(), torch.tensor(b[3:]).cuda()
    g = torch.Generator(device="cuda").manual_seed(8)
    test = lo + torch.rand((20000, 3), generator=g, device="cuda") * (hi - lo)
    ref = smp.sample(test)
    before = (sur.sample(test, fallback=False) - ref).abs().mean().item()
    loss = torch.zeros(1, device="cuda")
    first = None
    for step in range(400):
        pts = lo + torch.rand((1 << 14, 3), generator=g, device="cuda") * (hi - lo)
        sur.train_step(pts, smp.sample(pts), 1e-2, loss)
        if step == 0:
            first = loss.item()
    last = loss.item()
    after = (sur.sample(test, fallback=False) - ref).abs().mean().item()
    constant = (ref - ref.mean()).abs().mean().item()
    assert last < 0.05 * first, (first, last)
    assert after < 0.1 * before and after < 0.2 * constant, (before, after, constant)
    cal = lo + torch.rand((1 << 18, 3), generator=g, device="cuda") * (hi - lo)
    flagged = sur.calibrate(cal, 1e-2)
    err = (sur.sample(cal, fallback=True) - smp.sample(cal)).abs().max().item()
    print(f"loss {first:.4g} -> {last:.4g}; mean error {before:.3e} -> {after:.3e} (constant {constant:.3e}); "
          f"flagged regions {flagged}/{sur.num_regions}; max error with fallback {err:.3e}")
    assert err <= 1e-2, err
