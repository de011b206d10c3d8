"""Test restatement (numpy) of the cuda device's learned surrogate: a
multi-resolution hash-grid encoding followed by a 32-64-64-64-1 ReLU MLP
without biases.  Test infrastructure only: the GPU kernels are checked
against it, and `check_gradients` pins its analytic backward pass against
central finite differences in float64.

Encoding of a point p (object space) with the volume's object bounding box
[lo, hi]:
    u = clamp((p - lo) * inv_extent, 0, 1)              (float32)
    level l: res_l = floor(base * growth^l); x = u * res_l; i = min(floor(x), res_l - 1);
             f = x - i; corners c = i + {0,1}^3
             entry = c.x + c.y (res+1) + c.z (res+1)^2        if (res+1)^3 <= T
                     (c.x ^ c.y * 2654435761 ^ c.z * 805459861) mod T  otherwise
             feature_l = sum over corners of (wx * wy) * wz * table[l, entry]
with wx = f.x for the upper corner and 1 - f.x for the lower one.
MLP: h1 = relu(W1 x), h2 = relu(W2 h1), h3 = relu(W3 h2), y = W4 . h3.
Loss: sum over points of (y - target)^2 (the device divides by the batch
size when it applies the gradients).

With `fp16=True` the oracle rounds where the device stores FP16 values: the
table and weights, the encoding, the activations, and the backward signals
fed to the tensor cores.
"""
from __future__ import annotations

import numpy as np

P1, P2 = np.uint32(2654435761), np.uint32(805459861)


class Config:
    def __init__(self, levels=16, log2_table=19, base=16.0, growth=1.5, lo=(0, 0, 0), hi=(1, 1, 1), res=None):
        self.levels = levels
        self.T = 1 << log2_table
        self.res = list(res) if res is not None else \
            [int(np.floor(np.float32(base) * np.float32(growth) ** l)) for l in range(levels)]
        self.lo = np.asarray(lo, np.float32)
        ext = np.asarray(hi, np.float32) - self.lo
        self.inv = (np.float32(1) / np.where(ext > 0, ext, np.float32(1))).astype(np.float32)

    def dense(self, l):
        return (self.res[l] + 1) ** 3 <= self.T


def _h(a, fp16):
    return a.astype(np.float16).astype(np.float64) if fp16 else a


def corners(cfg, pts):
    """Per level: (entries (n,8) int64, weights (n,8) float32)."""
    u = ((np.asarray(pts, np.float32) - cfg.lo) * cfg.inv).astype(np.float32)
    u = np.clip(u, np.float32(0), np.float32(1))
    out = []
    for l in range(cfg.levels):
        r = cfg.res[l]
        x = (u * np.float32(r)).astype(np.float32)
        i = np.minimum(np.floor(x), np.float32(r - 1)).astype(np.int64)
        f = (x - i.astype(np.float32)).astype(np.float32)
        ents, ws = [], []
        for c in range(8):
            dx, dy, dz = c >> 2, (c >> 1) & 1, c & 1
            cx, cy, cz = i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz
            if cfg.dense(l):
                e = cx + cy * (r + 1) + cz * (r + 1) * (r + 1)
            else:
                h = (cx.astype(np.uint32) ^ (cy.astype(np.uint32) * P1) ^ (cz.astype(np.uint32) * P2))
                e = (h & np.uint32(cfg.T - 1)).astype(np.int64)
            wx = f[:, 0] if dx else np.float32(1) - f[:, 0]
            wy = f[:, 1] if dy else np.float32(1) - f[:, 1]
            wz = f[:, 2] if dz else np.float32(1) - f[:, 2]
            ents.append(e)
            ws.append(((wx * wy).astype(np.float32) * wz).astype(np.float32))
        out.append((np.stack(ents, 1), np.stack(ws, 1)))
    return out


def encode(cfg, table, pts, fp16=False):
    """table: (levels, T, 2).  Returns (n, 2*levels) float64."""
    tab = _h(np.asarray(table, np.float64), fp16)
    cs = corners(cfg, pts)
    feats = []
    for l, (e, w) in enumerate(cs):
        feats.append(np.einsum("nc,ncf->nf", w.astype(np.float64), tab[l][e]))
    x = np.concatenate(feats, 1)
    return _h(x, fp16)


def forward(cfg, params, pts, fp16=False):
    table, W1, W2, W3, W4 = params
    W = [_h(np.asarray(w, np.float64), fp16) for w in (W1, W2, W3)]
    w4 = _h(np.asarray(W4, np.float64), fp16)
    x = encode(cfg, table, pts, fp16)
    acts = [x]
    h = x
    for Wl in W:
        h = _h(np.maximum(h @ Wl.T, 0.0), fp16)
        acts.append(h)
    y = h @ w4
    return y, acts


def backward(cfg, params, pts, targets, fp16=False):
    """Gradients of sum((y - t)^2) over the points with a finite target
    (the others contribute nothing): (loss, dtable (levels,T,2), dW1, dW2,
    dW3, dW4)."""
    table, W1, W2, W3, W4 = params
    W = [_h(np.asarray(w, np.float64), fp16) for w in (W1, W2, W3)]
    w4 = _h(np.asarray(W4, np.float64), fp16)
    y, acts = forward(cfg, params, pts, fp16)
    t = np.asarray(targets, np.float64)
    d = np.where(np.isfinite(t), y - np.where(np.isfinite(t), t, 0.0), 0.0)
    loss = float(np.sum(d ** 2))
    dy = 2.0 * d
    dW4 = acts[3].T @ dy
    g = _h(np.outer(dy, w4) * (acts[3] > 0), fp16)
    dW = [None, None, None]
    for l in (2, 1, 0):
        dW[l] = g.T @ acts[l]
        gx = g @ W[l]
        g = _h(gx * (acts[l] > 0), fp16) if l > 0 else gx
    dX = g  # (n, 2*levels)
    dtable = np.zeros((cfg.levels, cfg.T, 2), np.float64)
    for l, (e, w) in enumerate(corners(cfg, pts)):
        for c in range(8):
            np.add.at(dtable[l], e[:, c], w[:, c:c + 1].astype(np.float64) * dX[:, 2 * l:2 * l + 2])
    return loss, dtable, dW[0], dW[1], dW[2], dW4


def init_params(cfg, seed=0, table_scale=1e-4):
    rng = np.random.default_rng(seed)
    table = rng.uniform(-table_scale, table_scale, (cfg.levels, cfg.T, 2)).astype(np.float32)
    nin = 2 * cfg.levels

    def he(o, i):
        b = np.sqrt(6.0 / i)
        return rng.uniform(-b, b, (o, i)).astype(np.float32)
    return [table, he(64, nin), he(64, 64), he(64, 64), he(1, 64).reshape(64)]


def check_gradients(cfg, params, pts, targets, n_probe=40, eps=1e-6, seed=0):
    """Max relative difference between analytic and central-difference
    gradients (float64, no FP16 rounding) over random probes of every
    parameter tensor."""
    rng = np.random.default_rng(seed)
    params = [np.asarray(p, np.float64).copy() for p in params]
    _, *grads = backward(cfg, params, pts, targets)
    worst = 0.0
    for k, (p, gk) in enumerate(zip(params, grads)):
        flat, gflat = p.reshape(-1), gk.reshape(-1)
        # probe entries with non-zero gradient where possible
        nz = np.nonzero(gflat)[0]
        idx = rng.choice(nz, min(n_probe, len(nz)), replace=False) if len(nz) else []
        for i in idx:
            old = flat[i]
            flat[i] = old + eps
            lp = backward(cfg, params, pts, targets)[0]
            flat[i] = old - eps
            lm = backward(cfg, params, pts, targets)[0]
            flat[i] = old
            fd = (lp - lm) / (2 * eps)
            worst = max(worst, abs(fd - gflat[i]) / max(1e-8, abs(fd) + abs(gflat[i])))
    return worst
