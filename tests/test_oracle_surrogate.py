"""Pins the surrogate oracle (oracle/surrogate.py, the numpy restatement of
the cuda device's hash-grid + MLP surrogate): its analytic backward pass
against central finite differences in float64, and its encoding's basic
properties (partition of unity, dense vs hashed indexing)."""
import numpy as np

from oracle import surrogate as S


def test_backward_matches_finite_differences():
    cfg = S.Config(levels=4, log2_table=8, base=4, growth=1.5)
    params = S.init_params(cfg, seed=1, table_scale=0.5)
    rng = np.random.default_rng(2)
    pts = rng.random((24, 3)).astype(np.float32)
    t = rng.random(24)
    assert S.check_gradients(cfg, params, pts, t, n_probe=12) < 1e-5


def test_encoding_interpolates_table():
    cfg = S.Config(levels=3, log2_table=10, base=2, growth=2.0)
    # a table holding a linear function of the corner coordinates is
    # reproduced exactly by the trilinear weights (dense levels only)
    tab = np.zeros((3, cfg.T, 2))
    for l in range(3):
        r = cfg.res[l]
        assert cfg.dense(l)
        c = np.arange((r + 1) ** 3)
        x, y, z = c % (r + 1), (c // (r + 1)) % (r + 1), c // ((r + 1) ** 2)
        tab[l, :len(c), 0] = x / r
        tab[l, :len(c), 1] = 2 * y / r - z / r
    pts = np.random.default_rng(3).random((100, 3)).astype(np.float32)
    enc = S.encode(cfg, tab, pts)
    for l in range(3):
        np.testing.assert_allclose(enc[:, 2 * l], pts[:, 0], atol=1e-6)
        np.testing.assert_allclose(enc[:, 2 * l + 1], 2 * pts[:, 1] - pts[:, 2], atol=1e-6)


def test_hashed_levels_wrap_into_table():
    cfg = S.Config(levels=6, log2_table=7, base=4, growth=2.0)
    assert cfg.dense(0) and not cfg.dense(5)
    pts = np.random.default_rng(4).random((50, 3)).astype(np.float32)
    for e, w in S.corners(cfg, pts):
        assert e.min() >= 0 and e.max() < cfg.T
        np.testing.assert_allclose(w.sum(1), 1.0, atol=1e-6)
