"""Seeded synthetic volumes and query sets for the benchmark workloads.

No public dataset is involved: every workload is generated from a seed with
the shapes, sizes and value distributions of the benchmark definitions.

* `sinusoid_field`: structuredRegular voxels = sum of 4 sinusoids (integer
  frequency 1-8 cycles per domain per axis, amplitude U[0.2, 1], random
  phase) plus U[-0.05, 0.05] noise.
* `uniform_points`: points uniform in a box (incoherent queries).
* `orbit_camera_samples`: width x height camera rays through the volume, S
  jittered samples each along the ray's box interval (coherent queries,
  ray-major so consecutive points march along one ray).
* `shell_leaves`: sparse VDB leaves covering seeded spherical shells with
  fractal-noise density in [0, 1].

numpy versions serve the tests; `*_torch` versions build the same
distributions directly in GPU memory for the full-size benchmark.
"""
from __future__ import annotations

import math

import numpy as np


def _sinusoid_params(seed):
    rng = np.random.default_rng(seed)
    freq = rng.integers(1, 9, size=(4, 3))
    amp = rng.uniform(0.2, 1.0, size=4)
    phase = rng.uniform(0.0, 2 * math.pi, size=4)
    return freq, amp, phase


def sinusoid_field(dims, seed=1, noise=0.05, dtype=np.float32):
    """(Z, Y, X) array, x fastest; dims = (X, Y, Z)."""
    X, Y, Z = dims
    freq, amp, phase = _sinusoid_params(seed)
    rng = np.random.default_rng(seed + 1000)
    z = np.arange(Z, dtype=np.float64)[:, None, None] / Z
    y = np.arange(Y, dtype=np.float64)[None, :, None] / Y
    x = np.arange(X, dtype=np.float64)[None, None, :] / X
    f = np.zeros((Z, Y, X), np.float64)
    for k in range(4):
        f += amp[k] * np.sin(2 * math.pi * (freq[k, 0] * x + freq[k, 1] * y + freq[k, 2] * z) + phase[k])
    f += rng.uniform(-noise, noise, size=f.shape)
    return f.astype(dtype)


def sinusoid_volume(dims, seed=1):
    """The sinusoid field of `sinusoid_field` for large volumes: generated
    z-slab by z-slab in float32 (sin(a + c) expanded per slab), so a 1024^3
    volume needs no float64 temporaries of its own size.  (Z, Y, X), x
    fastest; dims = (X, Y, Z)."""
    X, Y, Z = dims
    freq, amp, phase = _sinusoid_params(seed)
    rng = np.random.default_rng(seed + 1000)
    out = np.empty((Z, Y, X), np.float32)
    x = (np.arange(X, dtype=np.float32) / X)[None, :]
    y = (np.arange(Y, dtype=np.float32) / Y)[:, None]
    two_pi = np.float32(2 * math.pi)
    # sin(a + c) with a = 2pi(fx x + fy y) + phase per term, c = 2pi fz z
    sa, ca = [], []
    for k in range(4):
        a = two_pi * (np.float32(freq[k, 0]) * x + np.float32(freq[k, 1]) * y) + np.float32(phase[k])
        sa.append(np.sin(a).astype(np.float32))
        ca.append(np.cos(a).astype(np.float32))
    for zi in range(Z):
        acc = rng.uniform(-0.05, 0.05, size=(Y, X)).astype(np.float32)
        for k in range(4):
            c = 2 * math.pi * freq[k, 2] * zi / Z
            acc += np.float32(amp[k]) * (sa[k] * np.float32(math.cos(c)) + ca[k] * np.float32(math.sin(c)))
        out[zi] = acc
    return out


def sinusoid_field_torch(dims, seed=1, noise=0.05, device="cuda"):
    """Same distribution as sinusoid_field, generated on the GPU in slabs of
    about 2^24 voxels."""
    import torch
    X, Y, Z = dims
    freq, amp, phase = _sinusoid_params(seed)
    g = torch.Generator(device=device)
    g.manual_seed(seed + 1000)
    out = torch.empty((Z, Y, X), dtype=torch.float32, device=device)
    x = torch.arange(X, device=device, dtype=torch.float32)[None, None, :] / X
    y = torch.arange(Y, device=device, dtype=torch.float32)[None, :, None] / Y
    step = max(1, (1 << 24) // (X * Y))
    for z0 in range(0, Z, step):
        z1 = min(Z, z0 + step)
        zz = torch.arange(z0, z1, device=device, dtype=torch.float32)[:, None, None] / Z
        acc = torch.zeros((z1 - z0, Y, X), device=device, dtype=torch.float32)
        for k in range(4):
            acc += float(amp[k]) * torch.sin(2 * math.pi * (float(freq[k, 0]) * x + float(freq[k, 1]) * y
                                                           + float(freq[k, 2]) * zz) + float(phase[k]))
        acc += (torch.rand((z1 - z0, Y, X), generator=g, device=device) * 2 - 1) * noise
        out[z0:z1] = acc
    return out


def uniform_points(n, lo, hi, seed=2):
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    return (lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)


def uniform_points_torch(n, lo, hi, seed=2, device="cuda"):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    lo = torch.tensor(lo, dtype=torch.float32, device=device)
    hi = torch.tensor(hi, dtype=torch.float32, device=device)
    return lo + torch.rand((n, 3), generator=g, device=device) * (hi - lo)


def _camera_rays(width, height, lo, hi, angle):
    """Orbit camera at `angle` around the box centre, framing the middle of
    the box so every ray crosses it; returns origins, unit dirs (H*W, 3)."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    c = 0.5 * (lo + hi)
    ext = hi - lo
    r = 1.6 * np.max(ext)
    eye = c + r * np.array([math.cos(angle), 0.35, math.sin(angle)])
    fwd = c - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    # half-extent of the image plane at the box centre: 40% of the box
    half = 0.4 * np.min(ext)
    dist = np.linalg.norm(c - eye)
    sx = half / dist
    sy = sx * height / width
    return eye, fwd, right, up, sx, sy


def orbit_camera_samples(width, height, samples, lo, hi, seed=3, angle=0.7):
    """(width*height*samples, 3) float32 points, ray-major."""
    eye, fwd, right, up, sx, sy = _camera_rays(width, height, lo, hi, angle)
    rng = np.random.default_rng(seed)
    u = (np.arange(width) + 0.5) / width * 2 - 1
    v = (np.arange(height) + 0.5) / height * 2 - 1
    uu, vv = np.meshgrid(u, v)
    d = fwd[None, :] + uu.reshape(-1, 1) * sx * right[None, :] + vv.reshape(-1, 1) * sy * up[None, :]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t0, t1 = _slab(eye, d, np.asarray(lo, np.float64), np.asarray(hi, np.float64))
    j = (np.arange(samples)[None, :] + rng.random((d.shape[0], samples))) / samples
    t = t0[:, None] + j * (t1 - t0)[:, None]
    p = eye[None, None, :] + t[:, :, None] * d[:, None, :]
    return p.reshape(-1, 3).astype(np.float32)


def orbit_camera_samples_torch(width, height, samples, lo, hi, seed=3, angle=0.7, device="cuda"):
    import torch
    eye, fwd, right, up, sx, sy = _camera_rays(width, height, lo, hi, angle)
    T = lambda a: torch.tensor(np.asarray(a), dtype=torch.float32, device=device)
    u = (torch.arange(width, device=device, dtype=torch.float32) + 0.5) / width * 2 - 1
    v = (torch.arange(height, device=device, dtype=torch.float32) + 0.5) / height * 2 - 1
    vv, uu = torch.meshgrid(v, u, indexing="ij")
    d = T(fwd)[None, :] + uu.reshape(-1, 1) * sx * T(right)[None, :] + vv.reshape(-1, 1) * sy * T(up)[None, :]
    d = d / torch.linalg.norm(d, dim=1, keepdim=True)
    e = T(eye)
    lo_t, hi_t = T(lo), T(hi)
    inv = 1.0 / d
    ta = (lo_t[None] - e[None]) * inv
    tb = (hi_t[None] - e[None]) * inv
    t0 = torch.minimum(ta, tb).amax(dim=1)
    t1 = torch.maximum(ta, tb).amin(dim=1)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    nrays = d.shape[0]
    out = torch.empty((nrays * samples, 3), dtype=torch.float32, device=device)
    chunk = 1 << 16
    base = torch.arange(samples, device=device, dtype=torch.float32)[None, :]
    for s in range(0, nrays, chunk):
        e_ = min(nrays, s + chunk)
        j = (base + torch.rand((e_ - s, samples), generator=g, device=device)) / samples
        t = t0[s:e_, None] + j * (t1 - t0)[s:e_, None]
        p = e[None, None, :] + t[:, :, None] * d[s:e_, None, :]
        out[s * samples:e_ * samples] = p.reshape(-1, 3)
    return out


def _slab(o, d, lo, hi):
    with np.errstate(divide="ignore"):
        inv = 1.0 / d
    ta = (lo[None] - o[None]) * inv
    tb = (hi[None] - o[None]) * inv
    t0 = np.minimum(ta, tb).max(axis=1)
    t1 = np.maximum(ta, tb).min(axis=1)
    return t0, t1


def camera_rays(width, height, lo, hi, angle=0.7):
    """Origins, directions and [t0, t1] box intervals of the orbit camera."""
    eye, fwd, right, up, sx, sy = _camera_rays(width, height, lo, hi, angle)
    u = (np.arange(width) + 0.5) / width * 2 - 1
    v = (np.arange(height) + 0.5) / height * 2 - 1
    uu, vv = np.meshgrid(u, v)
    d = fwd[None, :] + uu.reshape(-1, 1) * sx * right[None, :] + vv.reshape(-1, 1) * sy * up[None, :]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = np.repeat(eye[None, :], d.shape[0], axis=0)
    t = np.stack([np.zeros(d.shape[0]), np.full(d.shape[0], 1e30)], 1)
    return o.astype(np.float32), d.astype(np.float32), t.astype(np.float32)


def random_rays(n, lo, hi, seed=4):
    """Rays from points outside the box towards uniform points inside it."""
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    c = 0.5 * (lo + hi)
    r = 1.5 * np.max(hi - lo)
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    target = lo + rng.random((n, 3)) * (hi - lo)
    o = c[None, :] + dirs * r
    d = target - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = np.stack([np.zeros(n), np.full(n, 1e30)], 1)
    return o.astype(np.float32), d.astype(np.float32), t.astype(np.float32)


# ---------------------------------------------------------------------------
# Sparse VDB: spherical shells with fractal noise.
# ---------------------------------------------------------------------------
def _shell_params(seed, domain, count):
    rng = np.random.default_rng(seed)
    centers = rng.uniform(0.3, 0.7, size=(count, 3)) * domain
    radii = rng.uniform(0.1, 0.45, size=count) * domain
    return centers, radii


def _value_noise(p, seed, octaves=4):
    """Fractal sum of hashed trilinear value noise in [0, 1] (numpy)."""
    total = np.zeros(p.shape[:-1], np.float64)
    norm = 0.0
    for o in range(octaves):
        freq = 2.0 ** o / 64.0
        amp = 0.5 ** o
        q = p * freq
        i = np.floor(q).astype(np.int64)
        f = q - i
        f = f * f * (3 - 2 * f)
        acc = 0
        for c in range(8):
            dx, dy, dz = c >> 2, (c >> 1) & 1, c & 1
            h = ((i[..., 0] + dx) * 73856093) ^ ((i[..., 1] + dy) * 19349663) ^ ((i[..., 2] + dz) * 83492791) ^ (seed * 2654435761 + o)
            h = (h * 0x27d4eb2d) & 0xffffffff
            val = (h >> 8) / float(1 << 24)
            w = (f[..., 0] if dx else 1 - f[..., 0]) * (f[..., 1] if dy else 1 - f[..., 1]) * (f[..., 2] if dz else 1 - f[..., 2])
            acc = acc + w * val
        total += amp * acc
        norm += amp
    return total / norm


def shell_leaves(domain=256, shells=3, thickness=0.02, seed=5, leaf_frac_target=None):
    """Leaves (level 3, dense ZYX) of a sparse VDB over [0, domain)^3 covering
    `shells` spherical shells of relative thickness `thickness`.  Returns
    origins (L,3) int32 and packed voxel values (L*512,) float32 in [0,1]
    (z fastest inside a leaf)."""
    centers, radii = _shell_params(seed, domain, shells)
    half = 0.5 * thickness * domain
    n = domain // 8
    g = (np.arange(n) * 8 + 4.0)
    lx, ly, lz = np.meshgrid(g, g, g, indexing="ij")
    pc = np.stack([lx, ly, lz], -1).reshape(-1, 3)
    active = np.zeros(pc.shape[0], bool)
    lim = half + 4 * math.sqrt(3)
    for c, r in zip(centers, radii):
        dist = np.linalg.norm(pc - c[None], axis=1)
        active |= np.abs(dist - r) <= lim
    origins = (pc[active] - 4).astype(np.int32)
    # voxel positions, z fastest inside each leaf
    off = np.stack(np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij"), -1).reshape(-1, 3)
    vox = origins[:, None, :].astype(np.float64) + off[None, :, :] + 0.5
    dens = np.zeros(vox.shape[:2], np.float64)
    for c, r in zip(centers, radii):
        dist = np.linalg.norm(vox - c[None, None], axis=2)
        inside = np.clip(1.0 - np.abs(dist - r) / half, 0.0, 1.0)
        dens = np.maximum(dens, inside)
    noise = _value_noise(vox, seed)
    values = np.clip(dens * (0.5 + noise), 0.0, 1.0).astype(np.float32)
    return origins, values.reshape(-1)


def _value_noise_torch(p, seed, octaves=4):
    """Torch twin of `_value_noise` (float32 positions, same hash)."""
    import torch
    total = torch.zeros(p.shape[:-1], dtype=torch.float32, device=p.device)
    norm = 0.0
    for o in range(octaves):
        freq = 2.0 ** o / 64.0
        amp = 0.5 ** o
        q = p * freq
        i = torch.floor(q).to(torch.int64)
        f = q - i
        f = f * f * (3 - 2 * f)
        acc = torch.zeros_like(total)
        for c in range(8):
            dx, dy, dz = c >> 2, (c >> 1) & 1, c & 1
            h = ((i[..., 0] + dx) * 73856093) ^ ((i[..., 1] + dy) * 19349663) ^ \
                ((i[..., 2] + dz) * 83492791) ^ (seed * 2654435761 + o)
            h = (h * 0x27d4eb2d) & 0xffffffff
            val = (h >> 8).to(torch.float32) / float(1 << 24)
            w = (f[..., 0] if dx else 1 - f[..., 0]) * (f[..., 1] if dy else 1 - f[..., 1]) * \
                (f[..., 2] if dz else 1 - f[..., 2])
            acc += w * val
        total += amp * acc
        norm += amp
    return total / norm


def shell_vdb_torch(domain=4096, leaf_fraction=0.05, thickness=0.02, seed=5, device="cuda",
                    max_shells=64):
    """Sparse VDB leaves of seeded spherical shells (radius U[0.1, 0.45] x
    domain, relative thickness `thickness`) with fractal-noise density in
    [0, 1], built in GPU memory.  Shells are added in seed order until at
    least `leaf_fraction` of the (domain/8)^3 leaf slots are active.

    Returns (origins (L,3) int32 numpy, values (L*512,) float32 CUDA tensor,
    z fastest inside each leaf, shells used, active fraction)."""
    import torch
    rng = np.random.default_rng(seed)
    n = domain // 8
    half = 0.5 * thickness * domain
    lim = half + 4 * math.sqrt(3)
    centers, radii = [], []
    active = torch.zeros((n, n, n), dtype=torch.bool, device=device)
    g = torch.arange(n, device=device, dtype=torch.float32) * 8 + 4.0
    frac = 0.0
    while frac < leaf_fraction and len(centers) < max_shells:
        c = rng.uniform(0.3, 0.7, size=3) * domain
        r = rng.uniform(0.1, 0.45) * domain
        centers.append(c)
        radii.append(r)
        for xi in range(0, n, 64):  # slabs keep the temporaries small
            dx = (g[xi:xi + 64, None, None] - c[0]) ** 2
            dist = torch.sqrt(dx + (g[None, :, None] - c[1]) ** 2 + (g[None, None, :] - c[2]) ** 2)
            active[xi:xi + 64] |= (dist - r).abs() <= lim
        frac = float(active.sum().item()) / n ** 3
    idx = torch.nonzero(active)                      # (L, 3) in (x, y, z) slot order
    origins = (idx * 8).to(torch.int32)
    L = origins.shape[0]
    values = torch.empty((L, 512), dtype=torch.float32, device=device)
    off = torch.stack(torch.meshgrid(torch.arange(8, device=device), torch.arange(8, device=device),
                                     torch.arange(8, device=device), indexing="ij"), -1).reshape(-1, 3)
    C = torch.tensor(np.array(centers), dtype=torch.float32, device=device)
    R = torch.tensor(np.array(radii), dtype=torch.float32, device=device)
    chunk = 1 << 15
    for s in range(0, L, chunk):
        e = min(L, s + chunk)
        vox = origins[s:e, None, :].to(torch.float32) + off[None].to(torch.float32) + 0.5
        dens = torch.zeros(vox.shape[:2], dtype=torch.float32, device=device)
        for k in range(C.shape[0]):
            dist = torch.linalg.norm(vox - C[k], dim=2)
            dens = torch.maximum(dens, torch.clamp(1.0 - (dist - R[k]).abs() / half, 0.0, 1.0))
        noise = _value_noise_torch(vox, seed)
        values[s:e] = torch.clamp(dens * (0.5 + noise), 0.0, 1.0)
    return origins.cpu().numpy(), values.reshape(-1), len(centers), frac
