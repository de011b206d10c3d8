"""How far results are from an FP-contracted evaluation (test infrastructure).

The device rounds every float operation in source order and equals the
oracle's parity build bit for bit (the -m gpu tests, at the benchmark sizes
too).  The reference's ISPC build lets the compiler contract a*b+c into
FMAs.  This script evaluates the benchmark workloads with the oracle's
parity build and with its contraction build (-ffp-contract=fast, FMA ISA)
and prints, per workload, the largest differences: ULPs, error relative to
max(|v|, 1), and interval / hit count mismatches.

    python tests/contraction_study.py            # all rows (a few minutes)
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import pyoracle as O  # noqa: E402
from openvkl_b200 import fields  # noqa: E402
from tests.parity import contraction_stats  # noqa: E402


def row(name, got, want, extra=""):
    s = contraction_stats(got, want)
    print(f"| {name} | {s['n']} | {s['max_ulp']} | {s['max_rel']:.2e} | {s['outside']} | {extra} |", flush=True)


def intervals_row(name, a, b, o, d, t, vr, m):
    ia, ca = a.intervals(o, d, t, value_ranges=vr, max_intervals=m)
    ib, cb = b.intervals(o, d, t, value_ranges=vr, max_intervals=m)
    same = ca == cb
    mask = (np.arange(m)[None, :] < ca[:, None]) & same[:, None]
    row(name, ia[mask], ib[mask], f"{int(np.count_nonzero(~same))} of {len(ca)} rays change count")


def main():
    threads = os.cpu_count() or 1
    print("| workload | values | max ULP | max rel. to max(\\|v\\|,1) | beyond 4 ULP and 1e-6 | counts |")
    print("|---|---|---|---|---|---|")
    # config 1: 128^3, 2^20 uniform points, trilinear sample + gradient
    v = fields.sinusoid_volume((128, 128, 128), seed=1)
    a, b = O.OracleVolume.dense_volume(v), O.OracleVolume.dense_volume(v, fma=True)
    p = fields.uniform_points(1 << 20, (0, 0, 0), (127, 127, 127), seed=2)
    row("128^3 trilinear sample", a.sample_parallel(p, threads=threads), b.sample_parallel(p, threads=threads))
    row("128^3 trilinear gradient", a.gradient_parallel(p, threads=threads), b.gradient_parallel(p, threads=threads))
    row("128^3 tricubic sample", a.sample_parallel(p, 200, threads=threads), b.sample_parallel(p, 200, threads=threads))
    row("128^3 tricubic gradient", a.gradient_parallel(p, 200, threads=threads),
        b.gradient_parallel(p, 200, threads=threads))
    # config 2: 1024^3, coherent orbit-camera rows (every 64th row) + intervals
    t0 = time.time()
    v = fields.sinusoid_volume((1024, 1024, 1024), seed=1)
    a, b = O.OracleVolume.dense_volume(v), O.OracleVolume.dense_volume(v, fma=True)
    hi = (1023, 1023, 1023)
    eye, fwd, right, up, sx, sy = fields._camera_rays(1920, 1080, (0, 0, 0), hi, 0.7)
    rng = np.random.default_rng(3)
    u = (np.arange(1920) + 0.5) / 1920 * 2 - 1
    vv = (np.arange(0, 1080, 64) + 0.5) / 1080 * 2 - 1
    uu, vvv = np.meshgrid(u, vv)
    d = fwd[None, :] + uu.reshape(-1, 1) * sx * right[None, :] + vvv.reshape(-1, 1) * sy * up[None, :]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ta, tb = fields._slab(eye, d, np.zeros(3), np.asarray(hi, np.float64))
    j = (np.arange(256)[None, :] + rng.random((d.shape[0], 256))) / 256
    tt = ta[:, None] + j * (tb - ta)[:, None]
    p = (eye[None, None, :] + tt[:, :, None] * d[:, None, :]).reshape(-1, 3).astype(np.float32)
    row("1024^3 coherent rays, trilinear sample", a.sample_parallel(p, threads=threads),
        b.sample_parallel(p, threads=threads))
    q = p[:: 8]
    row("1024^3 coherent rays, trilinear gradient", a.gradient_parallel(q, threads=threads),
        b.gradient_parallel(q, threads=threads))
    o, dd, t = fields.camera_rays(1920, 1080, (0, 0, 0), hi)
    sel = (np.arange(0, 1080, 16)[:, None] * 1920 + np.arange(1920)[None, :]).reshape(-1)
    lo, hi_ = a.value_range()
    qq = np.linspace(lo, hi_, 5, dtype=np.float32)
    vr = np.stack([qq[:-1], qq[1:]], 1)
    _, cnt = a.intervals(o[sel][:64], dd[sel][:64], t[sel][:64], value_ranges=vr, max_intervals=4096)
    intervals_row("1024^3 interval iterator, 1920x1080 rays every 16th row", a, b, o[sel], dd[sel], t[sel], vr,
                  int(cnt.max()) * 2)
    print(f"(1024^3 rows: {time.time() - t0:.0f} s)", file=sys.stderr)
    del a, b, v
    # sparse VDB shells (1024^3 domain here: the 4096^3 one needs 14 GB of
    # host memory per copy), interior points and hit iterator
    origins, values = fields.shell_leaves(domain=1024, shells=3, thickness=0.02, seed=5)
    L = len(origins)
    a = O.OracleVolume.vdb_volume(np.full(L, 3), origins, np.ones(L), values)
    b = O.OracleVolume.vdb_volume(np.full(L, 3), origins, np.ones(L), values, fma=True)
    rng = np.random.default_rng(13)
    pick = rng.integers(0, L, 1 << 20)
    p = (origins[pick] + rng.uniform(0, 8, (1 << 20, 3))).astype(np.float32)
    row(f"VDB shells ({L} leaves), trilinear sample", a.sample_parallel(p, threads=threads),
        b.sample_parallel(p, threads=threads))
    o, d, t = fields.random_rays(1 << 16, (0, 0, 0), (1024,) * 3, seed=4)
    isos = np.array([0.25, 0.5], np.float32)
    ha, ca = a.hits(o, d, t, isos, max_hits=16)
    hb, cb = b.hits(o, d, t, isos, max_hits=16)
    same = ca == cb
    mask = (np.arange(16)[None, :] < np.minimum(ca, 16)[:, None]) & same[:, None]
    row("VDB shells, hit iterator (t, sample, epsilon)", ha[mask], hb[mask],
        f"{int(np.count_nonzero(~same))} of {len(ca)} rays change hit count")


if __name__ == "__main__":
    main()
