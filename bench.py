"""Benchmark of the cuda device's hot path on B200.

Workload (default, "coherent"): structuredRegular 1024^3 float32
vertex-centered volume (seeded sum of 4 sinusoids + noise), trilinear
vklComputeSampleN over 1920x1080 orbit-camera rays x 256 jittered samples
each = 530,841,600 points per step.  Other workloads: "incoherent" (2^26
uniform random points, same volume), "cubic" (coherent points, tricubic
filter), "gradient" (coherent points, trilinear gradients).

One JSON line (rank 0):
  value       Gsamples/s over all ranks, device-timed with CUDA events on the
              launching stream over exactly --steps steps (inputs resident in
              HBM; inputs are larger than L2, so no flush is needed)
  e2e         the same metric through the C API with pinned host buffers:
              H2D of the points, kernel, D2H of the samples, every step
  roofline    dominant kernel's algorithmic bytes per launch / launch time
              against the measured HBM copy bandwidth
  cpu_baseline the oracle (C++ restatement of the reference CPU device)
              on all host cores, on a bounded sample of the same workload

--impl reference times that CPU implementation alone (rank 0) and prints its
line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DIMS = (1024, 1024, 1024)
WIDTH, HEIGHT, SPP = 1920, 1080, 256
INCOHERENT_N = 1 << 26
METRIC = "Gsamples/s and HBM GB/s (% roofline): plain FP32 vs FP16/FP8/batched/MLP at stated error"
UNIT = "Gsamples/s"
MAX_CPU_POINTS = 1 << 27  # bounded CPU sample (1.6 GB of points)
FILTER = {"coherent": 100, "incoherent": 100, "cubic": 200, "gradient": 100, "vdb": 100, "batched": 100,
          "intervals": 100, "hits": 100, "surrogate": 100,
          "render": 100, "config1": 100, "vdb_coherent": 100, "commit": 100}
BATCH_VOLUMES = 512
VDB_DOMAIN, VDB_POINTS = 4096, 1 << 26
HIT_RAYS = 1 << 24
TRAIN_STEPS = 1024


# ---------------------------------------------------------------------------
# Workload generation.
# ---------------------------------------------------------------------------
def volume_numpy(dims=None, seed=1):
    """Seeded sinusoid field, generated slab by slab in float32 (x fastest)."""
    from openvkl_b200.fields import sinusoid_volume
    return sinusoid_volume(dims or DIMS, seed)


def points_torch(workload, dims=None, device="cuda"):
    from openvkl_b200 import fields
    hi = tuple(d - 1 for d in (dims or DIMS))
    if workload == "incoherent":
        return fields.uniform_points_torch(INCOHERENT_N, (0, 0, 0), hi, seed=2, device=device)
    return fields.orbit_camera_samples_torch(WIDTH, HEIGHT, SPP, (0, 0, 0), hi, seed=3, device=device)


def points_numpy_sample(workload, n_rays_or_pts, dims=None):
    """A bounded sample of the same workload generated on the host."""
    from openvkl_b200 import fields
    hi = tuple(d - 1 for d in (dims or DIMS))
    if workload == "incoherent":
        return fields.uniform_points(n_rays_or_pts, (0, 0, 0), hi, seed=2)
    # the first rows of the image: whole rays, ray-major like the full set
    rows = max(1, n_rays_or_pts // WIDTH)
    full_h = HEIGHT
    pts = fields.orbit_camera_samples(WIDTH, full_h, SPP, (0, 0, 0), hi, seed=3) if rows >= full_h else \
        _camera_rows(rows, hi)
    return pts


def _camera_rows(rows, hi):
    """Samples of the first `rows` image rows of the orbit camera."""
    from openvkl_b200 import fields
    eye, fwd, right, up, sx, sy = fields._camera_rays(WIDTH, HEIGHT, (0, 0, 0), hi, 0.7)
    rng = np.random.default_rng(3)
    u = (np.arange(WIDTH) + 0.5) / WIDTH * 2 - 1
    v = ((np.arange(rows) + 0.5) / HEIGHT * 2 - 1)
    uu, vv = np.meshgrid(u, v)
    d = fwd[None, :] + uu.reshape(-1, 1) * sx * right[None, :] + vv.reshape(-1, 1) * sy * up[None, :]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t0, t1 = fields._slab(eye, d, np.zeros(3), np.asarray(hi, np.float64))
    j = (np.arange(SPP)[None, :] + rng.random((d.shape[0], SPP))) / SPP
    t = t0[:, None] + j * (t1 - t0)[:, None]
    return (eye[None, None, :] + t[:, :, None] * d[:, None, :]).reshape(-1, 3).astype(np.float32)


def compulsory_bytes(points, dims, filter_):
    """Unique 32-byte sectors of the volume touched by all stencils x 32."""
    import torch
    X, Y, Z = dims
    nsect = (X * Y * Z * 4 + 31) // 32
    mark = torch.zeros(nsect, dtype=torch.bool, device=points.device)
    lo, hi = (0, 2) if filter_ != 200 else (-1, 3)
    chunk = 1 << 22
    for s in range(0, points.shape[0], chunk):
        p = points[s:s + chunk]
        ic = torch.floor(p).to(torch.int64)
        for dz in range(lo, hi):
            for dy in range(lo, hi):
                for dx in range(lo, hi):
                    x, y, z = ic[:, 0] + dx, ic[:, 1] + dy, ic[:, 2] + dz
                    ok = (x >= 0) & (x < X) & (y >= 0) & (y < Y) & (z >= 0) & (z < Z)
                    e = ((z * Y + y) * X + x)[ok]
                    mark[(e * 4) // 32] = True
    return int(mark.sum().item()) * 32


# ---------------------------------------------------------------------------
# Clocks during the timed region.
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# CPU side (oracle restatement of the reference CPU device).
# ---------------------------------------------------------------------------
def cpu_baseline(vox, workload, budget_s=15.0):
    """Times the oracle on all host threads on a bounded sample sized for
    about `budget_s` seconds of work."""
    from oracle import pyoracle as O
    threads = os.cpu_count() or 1
    f = FILTER[workload]
    v = O.OracleVolume.dense_volume(vox, fast=True)
    L = O.lib(True)

    def run(pts):
        out = np.empty(len(pts), np.float32)
        t = time.perf_counter()
        if workload == "gradient":
            g = np.empty((len(pts), 3), np.float32)
            L.orc_gradient(v._h, f, 3, len(pts), pts.ctypes.data, 0, g.ctypes.data)
        else:
            L.orc_sample_parallel(v._h, f, len(pts), pts.ctypes.data, 0, out.ctypes.data, threads)
        return time.perf_counter() - t

    probe = points_numpy_sample(workload, WIDTH * 8 if workload != "incoherent" else 1 << 20)
    dt = run(probe)
    rate = len(probe) / max(dt, 1e-6)
    n = int(min(rate * budget_s, MAX_CPU_POINTS))
    n = max(n, len(probe))
    pts = points_numpy_sample(workload, n if workload == "incoherent" else max(1, n // SPP))
    reps = max(1, int(budget_s * rate / len(pts)))
    t = time.perf_counter()
    for _ in range(reps):
        run(pts)
    dt = time.perf_counter() - t
    cores = 1 if workload == "gradient" else threads
    what = "first image rows" if workload != "incoherent" else "same seed"
    return {"value": reps * len(pts) / dt / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(pts)} points of the same workload ({what}) x {reps} passes; oracle C++ "
                      f"restatement of the reference CPU device, -O3 -march=native, {cores} host "
                      f"threads, {dt:.1f} s"}


def oracle_check(vox, workload, pts, got):
    """Bitwise comparison of the timed run's results at a strided subset of
    its points with the oracle (the same volume and points, all host
    threads; NaN counts equal to NaN)."""
    from oracle import pyoracle as O
    f = FILTER[workload]
    v = O.OracleVolume.dense_volume(vox, fast=True)
    t = time.perf_counter()
    if workload == "gradient":
        want = v.gradient_parallel(pts, filter=f)
    else:
        want = v.sample_parallel(pts, filter=f)
    a = np.ascontiguousarray(got, np.float32).reshape(-1)
    b = np.ascontiguousarray(want, np.float32).reshape(-1)
    same = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    return {"points": int(len(pts)), "stride": 1021, "bit_exact": bool(same.all()),
            "mismatches": int((~same).sum()), "oracle_s": round(time.perf_counter() - t, 2)}


# ---------------------------------------------------------------------------
# Runs.
# ---------------------------------------------------------------------------
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    vox = volume_numpy()
    from oracle import pyoracle as O
    threads = os.cpu_count() or 1
    f = FILTER[args.workload]
    v = O.OracleVolume.dense_volume(vox, fast=True)
    L = O.lib(True)
    # size each step so the whole run stays within a few minutes
    probe = points_numpy_sample(args.workload, WIDTH * 4 if args.workload != "incoherent" else 1 << 20)
    out = np.empty(len(probe), np.float32)
    t = time.perf_counter()
    L.orc_sample_parallel(v._h, f, len(probe), probe.ctypes.data, 0, out.ctypes.data, threads)
    rate = len(probe) / max(time.perf_counter() - t, 1e-6)
    per_step_s = min(10.0, 120.0 / max(1, args.steps + args.warmup))
    n = max(len(probe), min(MAX_CPU_POINTS, int(rate * per_step_s)))
    pts = points_numpy_sample(args.workload, n if args.workload == "incoherent" else max(1, n // SPP))
    out = np.empty(len(pts), np.float32)
    for _ in range(args.warmup):
        L.orc_sample_parallel(v._h, f, len(pts), pts.ctypes.data, 0, out.ctypes.data, threads)
    t = time.perf_counter()
    for _ in range(args.steps):
        L.orc_sample_parallel(v._h, f, len(pts), pts.ctypes.data, 0, out.ctypes.data, threads)
    dt = (time.perf_counter() - t) / args.steps
    value = len(pts) / dt / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": config_of(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{len(pts)} points of the same workload per step; oracle C++ restatement "
                                   f"of the reference CPU device (the ISPC device cannot be built here), "
                                   f"-O3 -march=native, {threads} host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_of(args):
    n = INCOHERENT_N if args.workload == "incoherent" else WIDTH * HEIGHT * SPP
    return {"workload": f"structuredRegular 1024^3 float32 vertex-centered, "
                        f"{'tricubic' if args.workload == 'cubic' else 'trilinear'} "
                        f"{'gradient' if args.workload == 'gradient' else 'sample'}N, "
                        + ("1920x1080 orbit-camera rays x 256 jittered samples" if args.workload != "incoherent"
                           else "2^26 uniform random points"),
            "points_per_step": n, "volume_bytes": DIMS[0] * DIMS[1] * DIMS[2] * 4,
            "l2": "inputs larger than L2 (4 GiB volume, >=805 MB points), no flush",
            "parallelism": _parallelism(args)}


def _parallelism(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return "1 GPU"
    return (f"{ws} replicas, query partitioning (the points split across ranks)" if args.strong
            else f"{ws} replicas, every rank samples the full point set")


def run_cuda(args):
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    from openvkl_b200 import vkl

    dev = vkl.Device("cuda")
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    vox = volume_numpy()
    tvox = torch.from_numpy(vox).cuda()
    vol = vkl.structured_regular(dev, tvox, shared=True)
    f = FILTER[args.workload]
    smp = vkl.Sampler(vol, filter=f, gradient_filter=f)
    pts = points_torch(args.workload)
    n_total = pts.shape[0]
    if args.strong and ws > 1:
        # strong scaling: the ranks split one point set (query partitioning)
        from openvkl_b200.shard import query_slice
        a, b = query_slice(n_total, rank, ws)
        pts = pts[a:b].contiguous()
    n = pts.shape[0]
    grad = args.workload == "gradient"
    out = torch.empty((n, 3) if grad else (n,), dtype=torch.float32, device="cuda")
    call = smp.gradient if grad else smp.sample

    for _ in range(args.warmup):
        call(pts, out=out)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        time.sleep(0.3)  # let the sampler start
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            call(pts, out=out)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if ws > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
        torch.distributed.barrier()
    job_points = n_total if (args.strong and ws > 1) else n * ws
    value = job_points / (ms * 1e-3) / 1e9

    # algorithmic bytes of one launch: point in + result out + compulsory voxels
    io = n * (12 + (12 if grad else 4))
    comp = 0 if args.no_extras else compulsory_bytes(pts, DIMS, f)
    alg = io + comp
    peak, peak_kind = peaks()
    achieved = alg / (ms * 1e-3) / 1e9

    # end to end through the C API with pinned host buffers: every step copies
    # the points host->device and the samples device->host (library staging)
    e2e = None
    if not args.no_extras:
        hp = pts.cpu().pin_memory()
        ho = torch.empty(out.shape, dtype=torch.float32).pin_memory()
        call(hp, out=ho)  # first call sizes the staging buffers
        e2e_steps = max(1, min(args.steps, 5))
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        t = time.perf_counter()
        for _ in range(e2e_steps):
            call(hp, out=ho)
        e2e_s = (time.perf_counter() - t) / e2e_steps
        if ws > 1:
            tt = torch.tensor([e2e_s], device="cuda")
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            e2e_s = float(tt.item())
        e2e = {"value": job_points / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": n * 12,
               "d2h_bytes_per_step": int(ho.numel()) * 4}
        del hp, ho

    # a strided subset of the last timed step's results, checked against the
    # oracle below (every 1021st point: ~520k of the coherent set)
    chk_idx = torch.arange(0, n, 1021, device="cuda")
    chk_pts = pts[chk_idx].cpu().numpy()
    chk_out = out[chk_idx].cpu().numpy()

    patterns = None
    if rank == 0 and ws == 1 and args.workload == "coherent" and not args.no_patterns:
        # the configs' other patterns, measured after the headline in the
        # same process: the headline's buffers are released first
        del vol, smp, tvox, pts, out, call
        import gc
        gc.collect()
        torch.cuda.empty_cache()
        patterns = run_patterns(args)

    line = None
    if rank == 0:
        clocks = clk.summary()
        base = None if args.no_cpu_baseline else cpu_baseline(vox, args.workload)
        check = None if args.no_cpu_baseline else oracle_check(vox, args.workload, chk_pts, chk_out)
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            tr = json.load(open(tp)).get(args.workload)
            if tr:
                traffic = tr["bytes_per_point"] * n
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong" if (args.strong and ws > 1) else "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded sinusoid volume, generated rays)",
            "config": config_of(args),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "alg_bytes_per_launch": alg, "compulsory_voxel_bytes": comp},
            # per step: the layout detection (kDetectRuns) and the sampling
            # kernel for trilinear calls; the sampling kernel alone for tricubic
            "cpu_baseline": base, "e2e": e2e, "gpu_launches": args.steps * (1 if f == 200 else 2),
            "clocks": clocks, "check": check,
        }
        if patterns is not None:
            line["patterns"] = patterns
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_patterns(args):
    """Compact entries for the precision, batching and learned patterns,
    each measured with CUDA events over a few steps of its own workload
    (3 timed, 2 warm-up):
      compressed  2^26 points in active leaves of the 4096^3 shell VDB:
                  FP32 leaves vs FP16 / BF16 / FP8-E4M3 codes (per-leaf scale
                  and offset; 512 codes per leaf, or 8 stencil blocks of 5^3
                  codes per leaf), speed-up over FP32 and error against the
                  FP64 trilinear of the float leaves
      batched     the 512-volume batch vs per-volume launches (eager and in
                  a CUDA graph), sample + gradient of every point
      learned     the hash-grid + MLP surrogate of the shell VDB, trained on
                  2^28 points, against the plain sampler on 2^26 points"""
    import argparse
    import gc
    import torch
    sub = argparse.Namespace(**vars(args))
    sub.steps, sub.warmup, sub.collect = 3, 2, True
    out = {}
    v = run_vdb(sub)
    out["compressed"] = {"workload": v["config"]["workload"], "unit": UNIT,
                         "formats": {k: {x: f[x] for x in ("value", "speedup_vs_f32", "leaf_bytes",
                                                          "fp64_max_abs_err_rel_range", "fp64_max_rel_err",
                                                          "max_abs_err_rel_range") if x in f}
                                     for k, f in v["formats"].items()}}
    gc.collect()
    torch.cuda.empty_cache()
    b = run_batched(sub)
    out["batched"] = {"workload": b["config"]["workload"], "unit": b["unit"], "batch": b["value"],
                      "plain_eager": b["plain_eager"]["value"], "plain_graph": b["plain_graph"]["value"],
                      "speedup_vs_plain_eager": b["speedup_vs_plain_eager"],
                      "speedup_vs_plain_graph": b["speedup_vs_plain_graph"],
                      "bit_exact_vs_plain": b["bit_exact_vs_plain"]}
    gc.collect()
    torch.cuda.empty_cache()
    s = run_surrogate(sub)
    out["learned"] = {"workload": s["config"]["workload"], "unit": UNIT, "surrogate_with_fallback": s["value"],
                      "surrogate_no_fallback": s["surrogate_no_fallback"]["value"], "plain": s["plain"]["value"],
                      "train_points_per_s": s["train"]["points_per_s"],
                      "error_vs_plain": s["error_vs_plain"]}
    gc.collect()
    torch.cuda.empty_cache()
    return out


def run_vdb_coherent(args):
    """The sparse VDB (4096^3 shells) sampled along orbit-camera rays:
    1920x1080 rays x 64 jittered samples over the domain's box, trilinear
    sampleN, float leaves vs FP16 / BF16 / FP8-E4M3 codes.  Neighbouring
    samples share leaves, so leaf bytes, not access granularity, set the
    DRAM traffic."""
    run_vdb(args, coherent=True)


def run_vdb(args, coherent=False):
    """Sparse VDB (4096^3 domain, ~5 % of leaves active, shells with fractal
    noise), trilinear sampleN at 2^26 points inside active leaves: plain
    float leaves vs FP16 / BF16 / FP8-E4M3 codes with per-leaf scale+offset,
    as 512 codes per leaf or as 8 stencil blocks of 5^3 codes per leaf
    (scale and offset over the leaf's 9^3 sampling window; "_blocks").
    Errors of the compressed forms are against the float path on the same
    points, relative to the volume's value range."""
    import torch
    from openvkl_b200 import fields, vkl
    torch.cuda.set_device(0)
    dev = vkl.Device("cuda")
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    origins, values, shells, frac = fields.shell_vdb_torch(domain=VDB_DOMAIN, seed=5)
    L = origins.shape[0]
    levels = np.full(L, 3, np.uint32)
    formats = np.ones(L, np.uint32)
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    fp64 = None
    if coherent:
        pts = fields.orbit_camera_samples_torch(WIDTH, HEIGHT, 64, (0, 0, 0), (VDB_DOMAIN - 1,) * 3, seed=3)
    else:
        o_t = torch.from_numpy(origins).cuda()
        pick = torch.randint(0, L, (VDB_POINTS,), generator=g, device="cuda")
        loc = torch.rand((VDB_POINTS, 3), generator=g, device="cuda") * 8
        pts = (o_t[pick].to(torch.float32) + loc).contiguous()
        fp64 = _leaf_trilinear_fp64(values, pick, pts - o_t[pick].to(torch.float32))
        del o_t, pick, loc
    npts = pts.shape[0]
    out = torch.empty(npts, dtype=torch.float32, device="cuda")

    def volume(fmt):
        v = vkl.Volume(dev, "vdb")
        v.set_data("node.level", vkl.Data(dev, levels))
        v.set_data("node.origin", vkl.Data(dev, origins.reshape(-1), vkl_type=vkl.VKL_VEC3I))
        v.set_data("node.format", vkl.Data(dev, formats))
        v.set_data("nodesPackedDense", vkl.Data(dev, objects=[vkl.Data(dev, values, shared=True)]))
        if fmt != "f32":
            v.set_string("compression", fmt)
        t = time.perf_counter()
        v.commit()
        torch.cuda.synchronize()
        return v, time.perf_counter() - t

    results, ref = {}, None
    vrange = float(values.max().item() - values.min().item())
    for fmt in ("f32", "fp16", "bf16", "fp8", "fp16_blocks", "bf16_blocks", "fp8_blocks"):
        vol, commit_s = volume(fmt)
        smp = vkl.Sampler(vol, filter=100)
        for _ in range(args.warmup):
            smp.sample(pts, out=out)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            smp.sample(pts, out=out)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        r = {"value": npts / (ms * 1e-3) / 1e9, "ms_per_step": ms, "commit_s": commit_s,
             "leaf_bytes": L * {"f32": 2048, "fp16": 1024, "bf16": 1024, "fp8": 512, "fp16_blocks": 2048,
                                "bf16_blocks": 2048, "fp8_blocks": 1024}[fmt]}
        if ref is None:
            ref = out.clone()
        else:
            ok = ~torch.isnan(ref)
            r["max_abs_err_rel_range"] = float((out[ok] - ref[ok]).abs().max().item()) / vrange
            r["mean_abs_err_rel_range"] = float((out[ok] - ref[ok]).abs().mean().item()) / vrange
            r["speedup_vs_f32"] = results["f32"]["ms_per_step"] / ms
        if fp64 is not None:
            idx, want = fp64
            e = (out[idx].to(torch.float64) - want).abs()
            r["fp64_max_abs_err_rel_range"] = float(e.max().item()) / vrange
            r["fp64_max_rel_err"] = float((e / want.abs().clamp_min(1e-3)).max().item())
            r["fp64_points"] = int(idx.numel())
        results[fmt] = r
        del smp, vol
    line = {"metric": METRIC, "value": results["f32"]["value"], "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": results["f32"]["ms_per_step"],
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded shells + fractal noise)",
            "config": {"workload": f"vdb {VDB_DOMAIN}^3 domain, {L} leaves ({100 * frac:.2f} % active, "
                                   f"{shells} shells), nodesPackedDense, trilinear sampleN at "
                                   + (f"{WIDTH}x{HEIGHT} orbit-camera rays x 64 samples" if coherent
                                      else "2^26 points inside active leaves"),
                       "leaves": L, "points": npts},
            "formats": results}
    if getattr(args, "collect", False):
        return line
    print(json.dumps(line), flush=True)


def _leaf_trilinear_fp64(values, leaf, local):
    """FP64 trilinear of the float leaves (z fastest, 512 values per leaf) at
    the points whose 2x2x2 stencil lies inside their own leaf (local
    coordinates in [0, 7) on every axis): (indices of those points, FP64
    samples)."""
    import torch
    inside = (local < 7).all(dim=1)
    idx = torch.nonzero(inside).squeeze(1)
    lc = local[idx].to(torch.float64)
    i0 = torch.floor(lc).to(torch.int64)
    f = lc - i0
    base = leaf[idx].to(torch.int64) * 512
    acc = torch.zeros(idx.numel(), dtype=torch.float64, device=local.device)
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                v = values[base + ((i0[:, 0] + dx) << 6) + ((i0[:, 1] + dy) << 3) + (i0[:, 2] + dz)]
                w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * \
                    (f[:, 2] if dz else 1 - f[:, 2])
                acc += w * v.to(torch.float64)
    return idx, acc


def run_batched(args):
    """512 structuredRegular float32 volumes, edges log-uniform 16-256 per
    axis, seeded sinusoid fields; per volume 1k-1M uniform points (log-uniform
    count); trilinear sample + gradient of every point.  Timed three ways with
    CUDA events on the device stream: per-volume vklComputeSampleN +
    vklComputeGradientN calls (eager), the same calls captured in one CUDA
    graph, and the batch (vklCudaNewSampleBatch: persistent kernels in a
    graph, autotuned).  A unit of work is one point's sample and gradient."""
    import torch
    from openvkl_b200 import fields, vkl
    torch.cuda.set_device(0)
    dev = vkl.Device("cuda")
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    rng = np.random.default_rng(7)
    keep, jobs, total, voxels = [], [], 0, 0
    for i in range(BATCH_VOLUMES):
        dims = tuple(int(round(math.exp(rng.uniform(math.log(16), math.log(256))))) for _ in range(3))
        vox = fields.sinusoid_field_torch(dims, seed=100 + i)
        vol = vkl.structured_regular(dev, vox, shared=True)
        smp = vkl.Sampler(vol, filter=100, gradient_filter=100)
        n = int(round(math.exp(rng.uniform(math.log(1e3), math.log(1e6)))))
        pts = fields.uniform_points_torch(n, (0, 0, 0), tuple(d - 1 for d in dims), seed=200 + i)
        jobs.append((smp, pts, torch.empty(n, device="cuda"), torch.empty((n, 3), device="cuda")))
        keep.append((vox, vol))
        total += n
        voxels += dims[0] * dims[1] * dims[2]
    torch.cuda.synchronize()

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def plain():
        for smp, pts, sm, gr in jobs:
            smp.sample(pts, out=sm)
            smp.gradient(pts, out=gr)

    ms_eager = timed(plain, max(1, args.steps // 2), args.warmup)
    ref = [(sm.clone(), gr.clone()) for _, _, sm, gr in jobs]

    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        dev.set_stream(torch.cuda.current_stream().cuda_stream)
        plain()
    dev.set_stream(stream.cuda_stream)
    ms_graph = timed(graph.replay, args.steps, args.warmup)

    t = time.perf_counter()
    batch = vkl.SampleBatch(dev, jobs, autotune=True)
    tune_s = time.perf_counter() - t
    for _, _, sm, gr in jobs:
        sm.fill_(float("nan"))
        gr.fill_(float("nan"))
    ms_batch = timed(batch.run, args.steps, args.warmup)
    exact = all(torch.equal(sm.view(torch.int32), r[0].view(torch.int32)) and
                torch.equal(gr.view(torch.int32), r[1].view(torch.int32))
                for (_, _, sm, gr), r in zip(jobs, ref))
    rate = lambda ms: total / (ms * 1e-3) / 1e9
    line = {"metric": METRIC, "value": rate(ms_batch), "unit": "Gpoints/s (sample + gradient)",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_batch,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded sinusoid volumes)",
            "config": {"workload": f"batched: {BATCH_VOLUMES} structuredRegular f32 volumes "
                                   f"({voxels} voxels), {total} points, trilinear sample + gradient",
                       "points": total, "voxels": voxels},
            "plain_eager": {"value": rate(ms_eager), "ms_per_step": ms_eager},
            "plain_graph": {"value": rate(ms_graph), "ms_per_step": ms_graph},
            "speedup_vs_plain_eager": ms_eager / ms_batch, "speedup_vs_plain_graph": ms_graph / ms_batch,
            "batch_config": batch.config(), "autotune_s": tune_s, "bit_exact_vs_plain": exact}
    batch.release()
    del graph
    if getattr(args, "collect", False):
        return line
    print(json.dumps(line), flush=True)


def _threaded_oracle(fn, n, threads, chunk=4096):
    """Runs fn(start, end) over [0, n) in chunks on `threads` Python threads
    (the oracle's ctypes calls release the GIL)."""
    import concurrent.futures as cf
    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda s: fn(s, min(n, s + chunk)), range(0, n, chunk)))


def _timed_device(fn, steps, warmup, stream):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def run_intervals(args):
    """Interval iterator on the 1024^3 volume: one iterator per pixel ray of
    the 1920x1080 orbit camera, 4 value ranges (the quartile slices of the
    volume's value range), default interval resolution hint, every interval
    written out (vklIterateIntervalsN, 20 B per interval).  Unit: Mrays/s;
    intervals per second beside it.  CPU baseline: the oracle's iterator on
    all host threads over the first image rows."""
    import torch
    from openvkl_b200 import fields, vkl
    torch.cuda.set_device(0)
    dev = vkl.Device("cuda")
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    vox = volume_numpy()
    vol = vkl.structured_regular(dev, torch.from_numpy(vox).cuda(), shared=True)
    smp = vkl.Sampler(vol, filter=100)
    lo, hi = vol.value_range()
    q = np.linspace(lo, hi, 5, dtype=np.float32)
    vr = np.stack([q[:-1], q[1:]], 1)
    ctx = vkl.IntervalIteratorContext(smp, value_ranges=vr)
    o, d, t = fields.camera_rays(WIDTH, HEIGHT, (0, 0, 0), tuple(x - 1 for x in DIMS))
    n = o.shape[0]
    to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    go, gd, gt = to(o), to(d), to(t)
    _, cnt = ctx.iterate_n(go, gd, gt, max_per_ray=0)
    m = int(cnt.max().item())
    total = int(cnt.sum().item())
    out = torch.empty((n, m, 5), dtype=torch.float32, device="cuda")
    cnt = torch.empty(n, dtype=torch.int32, device="cuda")
    lib = ctx.lib
    import ctypes as C
    call = lambda: ctx._call(lib.vklIterateIntervalsN, C.byref(ctx.h), n, go.data_ptr(), gd.data_ptr(),
                             gt.data_ptr(), m, out.data_ptr(), cnt.data_ptr())
    with ClockSampler(0) as clk:
        time.sleep(0.3)
        ms = _timed_device(call, args.steps, args.warmup, stream)
    base = None
    if not args.no_cpu_baseline:
        from oracle import pyoracle as O
        ref = O.OracleVolume.dense_volume(vox, fast=True)
        threads = os.cpu_count() or 1
        rows = 64
        k = rows * WIDTH
        t0 = time.perf_counter()
        _threaded_oracle(lambda a, b: ref.intervals(o[a:b], d[a:b], t[a:b], value_ranges=vr,
                                                    max_intervals=m), k, threads)
        dt = time.perf_counter() - t0
        base = {"value": k / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
                "sample": f"first {rows} image rows ({k} rays); oracle C++ restatement of the reference "
                          f"CPU iterator, {threads} host threads, {dt:.1f} s"}
    line = {"metric": METRIC, "value": n / (ms * 1e-3) / 1e6, "unit": "Mrays/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded sinusoid volume, generated rays)",
            "config": {"workload": f"interval iterator, structuredRegular {DIMS[0]}^3 float32, {WIDTH}x{HEIGHT} "
                                   "orbit-camera rays, 4 value ranges (quartiles), default resolution hint",
                       "rays": n, "intervals_per_step": total, "max_per_ray": m},
            "intervals_per_s": total / (ms * 1e-3),
            "roofline": {"bound": "latency (per-ray serial DDA)", "alg_bytes_per_launch": n * 32 + total * 20,
                         "achieved": (n * 32 + total * 20) / (ms * 1e-3) / 1e9, "unit": "GB/s"},
            "cpu_baseline": base, "gpu_launches": args.steps, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_hits(args):
    """Hit iterator on the sparse VDB (4096^3 domain shells): 2^24 random
    rays from outside the domain towards uniform points inside it, isovalues
    {0.25, 0.5}, trilinear filter, up to 16 hits per ray written out
    (vklIterateHitsN, 12 B per hit).  Unit: Mrays/s."""
    import torch
    from openvkl_b200 import fields, vkl
    torch.cuda.set_device(0)
    dev = vkl.Device("cuda")
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    v, smp, origins, shells, frac = _shell_sampler(dev, VDB_DOMAIN)
    L = origins.shape[0]
    ctx = vkl.HitIteratorContext(smp, [0.25, 0.5])
    n = HIT_RAYS
    o, d, t = fields.random_rays(n, (0, 0, 0), (VDB_DOMAIN,) * 3, seed=4)
    to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    go, gd, gt = to(o), to(d), to(t)
    m = 16
    out = torch.empty((n, m, 3), dtype=torch.float32, device="cuda")
    cnt = torch.empty(n, dtype=torch.int32, device="cuda")
    import ctypes as C
    call = lambda: ctx._call(ctx.lib.vklIterateHitsN, C.byref(ctx.h), n, go.data_ptr(), gd.data_ptr(),
                             gt.data_ptr(), m, out.data_ptr(), cnt.data_ptr())
    with ClockSampler(0) as clk:
        time.sleep(0.3)
        ms = _timed_device(call, args.steps, args.warmup, stream)
    total = int(cnt.to(torch.int64).sum().item())
    # the compressed leaf forms on the same rays (a few steps each): their
    # decoded values differ slightly, so hit counts may differ by a few
    formats = {"f32": {"value": n / (ms * 1e-3) / 1e6, "ms_per_step": ms, "hits_per_step": total}}
    del ctx, smp, v
    for fmt in ("fp16", "fp16_blocks", "fp8_blocks"):
        vf, sf, _, _, _ = _shell_sampler(dev, VDB_DOMAIN, compression=fmt)
        cf = vkl.HitIteratorContext(sf, [0.25, 0.5])
        callf = lambda: cf._call(cf.lib.vklIterateHitsN, C.byref(cf.h), n, go.data_ptr(), gd.data_ptr(),
                                 gt.data_ptr(), m, out.data_ptr(), cnt.data_ptr())
        msf = _timed_device(callf, min(args.steps, 3), min(args.warmup, 2), stream)
        formats[fmt] = {"value": n / (msf * 1e-3) / 1e6, "ms_per_step": msf,
                        "speedup_vs_f32": ms / msf, "hits_per_step": int(cnt.to(torch.int64).sum().item())}
        del cf, sf, vf
    line = {"metric": METRIC, "value": n / (ms * 1e-3) / 1e6, "unit": "Mrays/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded shells + fractal noise, random rays)",
            "config": {"workload": f"hit iterator, vdb {VDB_DOMAIN}^3 domain, {L} leaves ({100 * frac:.2f} % "
                                   f"active, {shells} shells), {n} random rays, isovalues 0.25 / 0.5",
                       "rays": n, "hits_per_step": total, "leaves": L},
            "hits_per_s": total / (ms * 1e-3), "formats": formats,
            "cpu_baseline": None, "gpu_launches": args.steps, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def _shell_sampler(dev, domain, background=None, compression=None):
    """The sparse VDB shell volume (nodesPackedDense, float leaves) and a
    trilinear sampler over it; returns (volume, sampler, leaf origins (L,3)
    numpy, shells, active fraction).  Without `background` the volume keeps
    the reference's undefined (NaN) background; `compression` selects a
    compressed leaf form."""
    from openvkl_b200 import fields, vkl
    origins, values, shells, frac = fields.shell_vdb_torch(domain=domain, seed=5)
    L = origins.shape[0]
    v = vkl.Volume(dev, "vdb")
    v.set_data("node.level", vkl.Data(dev, np.full(L, 3, np.uint32)))
    v.set_data("node.origin", vkl.Data(dev, origins.reshape(-1), vkl_type=vkl.VKL_VEC3I))
    v.set_data("node.format", vkl.Data(dev, np.ones(L, np.uint32)))
    v.set_data("nodesPackedDense", vkl.Data(dev, objects=[vkl.Data(dev, values, shared=True)]))
    if background is not None:
        v.set_data("background", vkl.Data(dev, np.asarray([background], np.float32)))
    if compression is not None:
        v.set_string("compression", compression)
    v.commit()
    return v, vkl.Sampler(v, filter=100), origins, shells, frac


def run_surrogate(args):
    """Learned surrogate of the sparse VDB shell volume: 16-level hash grid
    (2^19 entries per level, 2 FP16 features, base resolution 16, growth
    1.5) + 32-64-64-64-1 ReLU MLP on FP16 tensor cores, trained with Adam
    (lr 1e-2) on 2^28 points (2^10 steps of 2^18) whose targets the plain
    sampler computes, half of them inside active leaves and half uniform in
    the domain; calibrated on 2^22 points at threshold 1e-2; inference on
    2^26 points of the same distribution against the plain sampler.  value =
    surrogate samples/s with the plain-sampler fallback."""
    import torch
    from openvkl_b200 import vkl
    torch.cuda.set_device(0)
    dev = vkl.Device("cuda")
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    # a fog volume: empty space has density 0 (the reference's undefined
    # background would make every sample outside the leaves NaN)
    vol, smp, origins, shells, frac = _shell_sampler(dev, VDB_DOMAIN, background=0.0)
    sur = vkl.Surrogate(smp, log2_table=19, base_resolution=16.0, growth=1.5)
    rng = np.random.default_rng(21)
    table = rng.uniform(-1e-4, 1e-4, sur.table_entries * 2).astype(np.float32)
    fan = [32, 64, 64, 64]
    weights = np.concatenate([rng.uniform(-1, 1, 64 * fan[0]) * np.sqrt(6 / fan[0]),
                              rng.uniform(-1, 1, 64 * 64) * np.sqrt(6 / 64),
                              rng.uniform(-1, 1, 64 * 64) * np.sqrt(6 / 64),
                              rng.uniform(-1, 1, 64) * np.sqrt(3 / 64)]).astype(np.float32)
    sur.set_parameters(table, weights)
    org = torch.from_numpy(origins).cuda().to(torch.float32)
    g = torch.Generator(device="cuda").manual_seed(22)

    def draw(n):
        half = n // 2
        leaf = org[torch.randint(0, org.shape[0], (half,), generator=g, device="cuda")]
        near = leaf + torch.rand((half, 3), generator=g, device="cuda") * 8
        uni = torch.rand((n - half, 3), generator=g, device="cuda") * VDB_DOMAIN
        return torch.cat([near, uni]).contiguous()

    steps, batch = TRAIN_STEPS, 1 << 18
    loss = torch.zeros(1, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    train_ms, first = 0.0, None
    for k in range(steps):
        pts = draw(batch)
        tgt = smp.sample(pts)
        e0.record(stream)
        sur.train_step(pts, tgt, 1e-2, loss)
        e1.record(stream)
        e1.synchronize()
        train_ms += e0.elapsed_time(e1)
        if k == 0:
            first = loss.item() / batch
    last = loss.item() / batch
    flagged = sur.calibrate(draw(1 << 22), 1e-2)
    n = VDB_POINTS
    pts = draw(n)
    out = torch.empty(n, device="cuda")
    with ClockSampler(0) as clk:
        time.sleep(0.3)
        ms_fb = _timed_device(lambda: sur.sample(pts, out=out, fallback=True), args.steps, args.warmup, stream)
        ms_nn = _timed_device(lambda: sur.sample(pts, out=out, fallback=False), args.steps, args.warmup, stream)
        ms_plain = _timed_device(lambda: smp.sample(pts, out=out), args.steps, args.warmup, stream)
    ref = smp.sample(pts)
    vrange = float(vol.value_range()[1] - vol.value_range()[0])

    def err(fb):
        e = (sur.sample(pts, fallback=fb) - ref).abs()
        return {"max_abs": float(e.max().item()), "mean_abs": float(e.mean().item()),
                "frac_above_1e-2": float((e > 1e-2).float().mean().item())}

    rate = lambda ms: n / (ms * 1e-3) / 1e9
    line = {"metric": METRIC, "value": rate(ms_fb), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_fb, "higher_is_better": True, "dtype": "fp16 (MLP), f32",
            "data": "synthetic (seeded shells + fractal noise)",
            "config": {"workload": f"surrogate of vdb {VDB_DOMAIN}^3 domain ({origins.shape[0]} leaves, "
                                   f"{shells} shells): hash grid 16 x 2^19 x 2 fp16, MLP 32-64-64-64-1; "
                                   f"{n} inference points, half in active leaves",
                       "train_points": steps * batch, "value_range": vrange},
            "surrogate_no_fallback": {"value": rate(ms_nn), "ms_per_step": ms_nn},
            "plain": {"value": rate(ms_plain), "ms_per_step": ms_plain},
            "train": {"points_per_s": steps * batch / (train_ms * 1e-3), "ms_total": train_ms,
                      "loss_first": first, "loss_last": last},
            "calibration": {"threshold": 1e-2, "flagged_regions": flagged, "regions": sur.num_regions},
            "error_vs_plain": {"fallback": err(True), "no_fallback": err(False)},
            "gpu_launches": 3 * args.steps, "clocks": clk.summary()}
    sur.release()
    if getattr(args, "collect", False):
        return line
    print(json.dumps(line), flush=True)


def run_render(args):
    """The reference's example renderers on the __device__ API, headless:
    1920x1080 frames of the 1024^3 volume from the orbit camera, one ray per
    pixel; ray march iterator (sampling rate 1, interval context over the
    whole value range), interval iterator debug and hit iterator renderer
    (isovalues at 40 % and 70 % of the value range).  value = ray-march
    Mpixels/s; each renderer's frame time beside it."""
    import torch
    from openvkl_b200 import render, vkl
    torch.cuda.set_device(0)
    dev = vkl.Device("cuda")
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    vox = volume_numpy()
    vol = vkl.structured_regular(dev, torch.from_numpy(vox).cuda(), shared=True)
    smp = vkl.Sampler(vol, filter=100, gradient_filter=100)
    lo, hi = (float(x) for x in vol.value_range())
    ictx = vkl.IntervalIteratorContext(smp, value_ranges=[[lo, hi]])
    hctx = vkl.HitIteratorContext(smp, [lo + 0.4 * (hi - lo), lo + 0.7 * (hi - lo)])
    cam = render.orbit_camera(vol.bounding_box(), WIDTH, HEIGHT)
    tf = render.transfer_function((lo, hi))
    out = torch.empty((HEIGHT, WIDTH, 4), dtype=torch.float32, device="cuda")
    times = {}
    with ClockSampler(0) as clk:
        time.sleep(0.3)
        for name in ("ray_march", "interval_debug", "hits"):
            fn = lambda: render.render(name, smp, cam, WIDTH, HEIGHT, tf=tf, interval_context=ictx,
                                       hit_context=hctx, out=out, stream=stream.cuda_stream)
            times[name] = _timed_device(fn, args.steps, args.warmup, stream)
    px = WIDTH * HEIGHT
    line = {"metric": METRIC, "value": px / (times["ray_march"] * 1e-3) / 1e6, "unit": "Mpixels/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": times["ray_march"],
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded sinusoid volume)",
            "config": {"workload": f"example renderers on the __device__ API, {WIDTH}x{HEIGHT}, structuredRegular "
                                   f"{DIMS[0]}^3 float32, one ray per pixel"},
            "frame_ms": times, "gpu_launches": 3 * args.steps, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_config1(args):
    """128^3 float32 vertex-centered structuredRegular (the seeded sinusoid
    field), 2^20 points uniform in the object bounds, trilinear
    vklComputeSampleN + vklComputeGradientN per step (the configuration the
    reference's CPU device runs).  value = points/s with both a sample and a
    gradient; the oracle on all host threads beside it."""
    import torch
    from openvkl_b200 import fields, vkl
    torch.cuda.set_device(0)
    dev = vkl.Device("cuda")
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    vox = volume_numpy((128, 128, 128))
    vol = vkl.structured_regular(dev, torch.from_numpy(vox).cuda())
    smp = vkl.Sampler(vol, filter=100, gradient_filter=100)
    n = 1 << 20
    pts_np = fields.uniform_points(n, (0, 0, 0), (127, 127, 127), seed=2)
    pts = torch.from_numpy(pts_np).cuda()
    s = torch.empty(n, device="cuda")
    g = torch.empty((n, 3), device="cuda")

    def step():
        smp.sample(pts, out=s)
        smp.gradient(pts, out=g)

    with ClockSampler(0) as clk:
        time.sleep(0.3)
        ms = _timed_device(step, max(args.steps, 100), args.warmup, stream)
    base = None
    if not args.no_cpu_baseline:
        from oracle import pyoracle as O
        ref = O.OracleVolume.dense_volume(vox, fast=True)
        L = O.lib(True)
        threads = os.cpu_count() or 1
        out_s = np.empty(n, np.float32)
        out_g = np.empty((n, 3), np.float32)
        t0 = time.perf_counter()
        L.orc_sample_parallel(ref._h, 100, n, pts_np.ctypes.data, 0, out_s.ctypes.data, threads)
        _threaded_oracle(lambda a, b: L.orc_gradient(ref._h, 100, 3, b - a, pts_np[a:b].ctypes.data, 0,
                                                     out_g[a:b].ctypes.data), n, threads, chunk=1 << 14)
        dt = time.perf_counter() - t0
        base = {"value": n / dt / 1e9, "unit": "Gpoints/s (sample + gradient)", "cores": threads, "kind": "port",
                "sample": f"all {n} points; oracle C++ restatement of the reference CPU device, -O3 "
                          f"-march=native, {threads} host threads, {dt:.2f} s"}
    line = {"metric": METRIC, "value": n / (ms * 1e-3) / 1e9, "unit": "Gpoints/s (sample + gradient)",
            "n_gpus": 1, "steps": max(args.steps, 100), "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded sinusoid volume, uniform points)",
            "config": {"workload": "structuredRegular 128^3 float32 vertex-centered, 2^20 uniform points, "
                                   "trilinear sampleN + gradientN (device pointers)", "points_per_step": n},
            "cpu_baseline": base, "gpu_launches": 2 * max(args.steps, 100), "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_commit(args):
    """vklCommit of the 1024^3 float32 structuredRegular volume: the bricked
    re-layout, the dense tree, the per-leaf value ranges over 10^3 voxel
    windows, their propagation up the tree and the volume range read back
    (DenseVdbVolume.cpp:21-119 with VdbVolume.cpp:338-392).  Unit:
    Gvoxels/s.  Device-resident voxels (VKL_DATA_SHARED_BUFFER) for `value`;
    `e2e` hands the voxels over from pinned host memory (vklNewData copies
    them) and reads the value range back.  Each commit is timed alone with
    events on the device stream; the release of the previous volume is
    outside the timed region.  CPU baseline: the oracle's commit of a 256^3
    volume of the same field (leaf ranges on all host threads)."""
    import torch
    from openvkl_b200 import vkl
    torch.cuda.set_device(0)
    dev = vkl.Device("cuda")
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    vox = volume_numpy()
    tvox = torch.from_numpy(vox).cuda()
    nvox = vox.size
    leaves = math.prod((d + 7) // 8 for d in DIMS)

    def timed_commits(make, steps):
        ts = []
        for _ in range(steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            v = make()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
            if v is not None:
                v.release()
            del v
        return ts

    timed_commits(lambda: vkl.structured_regular(dev, tvox, shared=True), args.warmup)
    with ClockSampler(0) as clk:
        time.sleep(0.3)
        ts = timed_commits(lambda: vkl.structured_regular(dev, tvox, shared=True), args.steps)
    ms = sum(ts) / len(ts)
    lo, hi = (float(x) for x in vkl.structured_regular(dev, tvox, shared=True).value_range())

    # a time-varying volume: the same object re-committed with a new data
    # object each step (its device buffers are reused)
    vol = vkl.structured_regular(dev, tvox, shared=True)

    def recommit():
        vol._keep.clear()
        vol.set_data("data", vkl.Data(dev, tvox, shared=True))
        vol.commit()
    timed_commits(recommit, args.warmup)
    rts = timed_commits(recommit, args.steps)
    del vol

    e2e = None
    if not args.no_extras:
        host = torch.from_numpy(vox).pin_memory()

        def from_host():
            v = vkl.structured_regular(dev, host)
            v.value_range()
            return v
        from_host().release()
        t = timed_commits(from_host, min(args.steps, 5))
        e2e = {"value": nvox / (sum(t) / len(t) * 1e-3) / 1e9, "unit": "Gvoxels/s",
               "h2d_bytes_per_step": nvox * 4, "d2h_bytes_per_step": 8}
        del host

    # bricked copy (4 B read + 4 B written per voxel), leaf ranges (4 B read
    # per voxel, 8 B written per leaf)
    alg = nvox * 12 + leaves * 8
    peak, peak_kind = peaks()
    base = None
    if not args.no_cpu_baseline:
        from oracle import pyoracle as O
        svox = volume_numpy((256, 256, 256))
        t0 = time.perf_counter()
        reps = 0
        while True:
            O.OracleVolume.dense_volume(svox, fast=True)
            reps += 1
            dt = time.perf_counter() - t0
            if dt > 10.0 or reps >= 20:
                break
        threads = os.cpu_count() or 1
        base = {"value": reps * svox.size / dt / 1e9, "unit": "Gvoxels/s", "cores": threads, "kind": "port",
                "sample": f"{reps} commits of a 256^3 volume of the same field; oracle C++ restatement of the "
                          f"reference's dense commit: leaf value ranges on {threads} host threads (as the "
                          f"reference's parallel_for), tree build and propagation on one, {dt:.1f} s"}
    line = {"metric": "commit Gvoxels/s (value-range builder)", "value": nvox / (ms * 1e-3) / 1e9,
            "unit": "Gvoxels/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "ms_per_step_all": ts, "recommit_ms_median": statistics.median(rts), "recommit_ms_all": rts,
            "recommit_gvoxels_s_median": nvox / (statistics.median(rts) * 1e-3) / 1e9,
            "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded sinusoid volume)",
            "config": {"workload": "vklCommit of a structuredRegular 1024^3 float32 volume (bricked re-layout, "
                                   "dense tree, leaf value ranges, propagation, volume range readback)",
                       "voxels": nvox, "leaves": leaves, "value_range": [lo, hi],
                       "l2": "4 GiB volume, larger than L2"},
            "roofline": {"bound": "hbm", "achieved": alg / (ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms * 1e-3) / 1e9 / peak, "peak_kind": peak_kind,
                         "alg_bytes_per_launch": alg, "traffic": None,
                         "note": "whole commit (several kernels, allocations and one readback)"},
            "cpu_baseline": base, "e2e": e2e,
            # per commit: kDenseLevel2/1/0, kDenseBrickRanges, kFillEmpty x3,
            # kLeafToParent, kReduceNodes x2, kVolumeRange (ncu launch list)
            "gpu_launches": 11 * args.steps, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    ap.add_argument("--workload", choices=list(FILTER), default="coherent")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--strong", action="store_true",
                    help="with --gpus N > 1: the ranks split the one point set (query partitioning) "
                         "instead of each sampling all of it")
    ap.add_argument("--no-patterns", action="store_true",
                    help="default workload: skip the compressed / batched / learned pattern entries")
    ap.add_argument("--no-extras", action="store_true",
                    help="timed loop only (no e2e / roofline bytes / CPU baseline): profiling runs")
    ap.add_argument("--small", action="store_true",
                    help="512^3 volume, 480x270 rays x 256 (vdb: 2048^3 domain, 2^24 points): "
                         "the ncu capture case")
    ap.add_argument("--volume-edge", type=int, default=0,
                    help="edge of the dense volume instead of 1024 (512 with --small), the rays "
                         "scaled to it: e.g. 128 for an L2-resident volume, the kernels' ceiling")
    args = ap.parse_args(argv)
    global DIMS, WIDTH, HEIGHT, INCOHERENT_N, VDB_DOMAIN, VDB_POINTS, HIT_RAYS, TRAIN_STEPS
    if args.small:
        DIMS, WIDTH, HEIGHT, INCOHERENT_N = (512, 512, 512), 480, 270, 1 << 24
        VDB_DOMAIN, VDB_POINTS, HIT_RAYS, TRAIN_STEPS = 2048, 1 << 24, 1 << 20, 64
    if args.volume_edge:
        DIMS = (args.volume_edge,) * 3
    if args.no_extras:
        args.no_cpu_baseline = True
        args.no_patterns = True
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "vdb":
        run_vdb(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "intervals":
        run_intervals(args)
    elif args.workload == "hits":
        run_hits(args)
    elif args.workload == "surrogate":
        run_surrogate(args)
    elif args.workload == "render":
        run_render(args)
    elif args.workload == "config1":
        run_config1(args)
    elif args.workload == "vdb_coherent":
        run_vdb_coherent(args)
    elif args.workload == "commit":
        run_commit(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()
