"""ORACLE — TEST INFRASTRUCTURE ONLY.

ctypes binding of oracle/build/liboracle.so, the C++ restatement of the
Open VKL v2.0.2 CPU device's VDB / structuredRegular path (vkl_oracle.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product (openvkl_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "build")

FILTER_NEAREST, FILTER_LINEAR, FILTER_CUBIC = 0, 100, 200
T_UCHAR, T_SHORT, T_USHORT, T_HALF, T_FLOAT, T_DOUBLE = 2500, 3000, 3500, 5800, 6000, 7000
_NP2VKL = {
    np.dtype(np.uint8): T_UCHAR,
    np.dtype(np.int16): T_SHORT,
    np.dtype(np.uint16): T_USHORT,
    np.dtype(np.float16): T_HALF,
    np.dtype(np.float32): T_FLOAT,
    np.dtype(np.float64): T_DOUBLE,
}
BACKGROUND_UNDEFINED = np.frombuffer(np.uint32(0xFFC068B5).tobytes(), np.float32)[0]


def _host_tag() -> str:
    """Short hash of this host's CPU model and ISA flags: the timing build is
    compiled with -march=native, so each host gets its own copy."""
    import hashlib
    try:
        info = open("/proc/cpuinfo").read()
        model = [l for l in info.splitlines() if l.startswith(("model name", "flags"))][:2]
    except OSError:
        model = ["unknown"]
    return hashlib.md5("\n".join(model).encode()).hexdigest()[:10]


def fast_path() -> str:
    return os.path.join(_BUILD, f"liboracle_fast_{_host_tag()}.so")


def build(fast: bool = True, fma: bool = False) -> None:
    """Compile the parity build with the committed Makefile and, if asked,
    the -march=native timing build for this host and the FP-contraction
    build."""
    subprocess.run(["make", "-s", "-C", _HERE, "build/liboracle.so"], check=True)
    if fma:
        subprocess.run(["make", "-s", "-C", _HERE, "build/liboracle_fma.so"], check=True)
    srcs = [os.path.join(_HERE, f) for f in ("vkl_oracle.cpp", "vkl_oracle.h")]
    stale = not os.path.exists(fast_path()) or \
        os.path.getmtime(fast_path()) < max(os.path.getmtime(f) for f in srcs)
    if fast and stale:
        subprocess.run(["make", "-s", "-C", _HERE, "build/liboracle_fast.so"], check=True)
        os.replace(os.path.join(_BUILD, "liboracle_fast.so"), fast_path())


_libs: dict = {}


def lib(fast: bool = False, fma: bool = False) -> C.CDLL:
    """The parity build; `fast`: the -march=native timing build; `fma`: the
    build whose float expressions are contracted into FMAs."""
    name = os.path.join(_BUILD, "liboracle_fma.so") if fma else (
        fast_path() if fast else os.path.join(_BUILD, "liboracle.so"))
    if name not in _libs:
        path = name
        build(fast=fast, fma=fma)
        L = C.CDLL(path)
        P, U32, U64, I32, F32, VP = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_float, C.c_void_p
        L.orc_dense_create.restype = P
        L.orc_dense_create.argtypes = [P, U32, P, P, P, C.c_int, P, P, P, P, P]
        L.orc_vdb_create.restype = P
        L.orc_vdb_create.argtypes = [U64, P, P, P, U32, U32, P, P, P, P, P]
        L.orc_destroy.argtypes = [P]
        L.orc_last_error.restype = C.c_char_p
        L.orc_get_info.argtypes = [P, P, P, P, P, P, P]
        L.orc_level_num_nodes.restype = U64
        L.orc_level_num_nodes.argtypes = [P, U32]
        L.orc_get_level.argtypes = [P, U32, P, P, P]
        L.orc_value_range.argtypes = [P, U32, P]
        L.orc_sample.argtypes = [P, C.c_int, U32, U64, P, U32, P]
        L.orc_gradient.argtypes = [P, C.c_int, U32, U64, P, U32, P]
        L.orc_sample_parallel.argtypes = [P, C.c_int, U64, P, U32, P, C.c_int]
        L.orc_gradient_parallel.argtypes = [P, C.c_int, U32, U64, P, U32, P, C.c_int]
        L.orc_macrocell_ranges.argtypes = [P, U32, P]
        L.orc_dense_create_temporal.restype = P
        L.orc_dense_create_temporal.argtypes = [P, U32, P, P, P, C.c_int, P, P, P, P, C.c_int, P, U32, U64, P,
                                                U64]
        L.orc_sample_times.argtypes = [P, C.c_int, U64, P, P, U32, P, C.c_int]
        L.orc_path_trace.argtypes = [P, C.c_int, U32, U32, P, P, C.c_int, P, C.c_int, C.c_int, P, P, P, P, P]
        L.orc_gradient_times.argtypes = [P, C.c_int, U64, P, P, U32, P, C.c_int]
        L.orc_iterate_macrocells.restype = C.c_int
        L.orc_iterate_macrocells.argtypes = [P, U32, U32, P, U64, P, P, P, U32, P, P]
        L.orc_sample_observed.argtypes = [P, C.c_int, U32, U64, P, U32, P, P]
        L.orc_sample_fp64.argtypes = [P, C.c_int, U64, P, U32, P]
        L.orc_iterate_intervals.argtypes = [P, U32, U32, P, F32, U64, P, P, P, U32, P, P]
        L.orc_iterate_hits.argtypes = [P, U32, C.c_int, U32, P, U64, P, P, P, U32, P, P]
        L.orc_render.argtypes = [P, C.c_int, C.c_int, C.c_int, U32, U32, U32, P, F32, U32, P, P, P, C.c_int, P,
                                 P, P, P]
        L.orc_tricubic_map.restype = C.c_int
        L.orc_tricubic_map.argtypes = [P, P, P]
        L.orc_inner_nodes.restype = U64
        L.orc_inner_nodes.argtypes = [P, U32, U32, U64, P]
        L.orc_round_format.argtypes = [C.c_int, U64, P, P]
        L.orc_quantize_leaves.argtypes = [C.c_int, U64, P, P, P]
        L.orc_quantize_groups.argtypes = [C.c_int, U64, U32, P, P, P]
        L.orc_vdb_leaf_windows.argtypes = [P, U32, P]
        L.orc_vdb_set_windows.argtypes = [P, U32, U64, P]
        _libs[name] = L
    return _libs[name]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OracleVolume:
    """A committed oracle volume (dense structuredRegular or sparse VDB)."""

    def __init__(self, handle, keep, fast=False, fma=False):
        self._h = handle
        self._keep = keep  # numpy buffers the oracle points into
        self._lib = lib(fast, fma)
        info = self.info()
        self.dense = keep.get("dense", False)
        self.o2i, self.i2o = info["o2i"], info["i2o"]

    def __del__(self):
        try:
            if self._h:
                self._lib.orc_destroy(self._h)
        except Exception:
            pass

    # ---- construction -------------------------------------------------
    @staticmethod
    def dense_volume(data, cell_centered=False, grid_origin=None, grid_spacing=None,
                     index_to_object=None, index_origin=None, background=None, fast=False, fma=False):
        """`data`: one array (or a list of arrays, one per attribute) shaped
        (Z, Y, X) so that x is fastest in memory."""
        arrays = data if isinstance(data, (list, tuple)) else [data]
        arrays = [np.ascontiguousarray(a) for a in arrays]
        dims = np.array(arrays[0].shape[::-1], np.int32)
        ptrs = (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
        types = np.array([_NP2VKL[a.dtype] for a in arrays], np.uint32)
        strides = np.array([a.dtype.itemsize for a in arrays], np.uint64)
        go = None if grid_origin is None else np.asarray(grid_origin, np.float32)
        gs = None if grid_spacing is None else np.asarray(grid_spacing, np.float32)
        i2o = None if index_to_object is None else np.asarray(index_to_object, np.float32)
        io = None if index_origin is None else np.asarray(index_origin, np.int32)
        bg = None if background is None else np.asarray(background, np.float32).reshape(-1)
        L = lib(fast, fma)
        h = L.orc_dense_create(_p(dims), len(arrays), ptrs, _p(types), _p(strides),
                               int(bool(cell_centered)), _p(go), _p(gs), _p(i2o), _p(io), _p(bg))
        if not h:
            raise RuntimeError(L.orc_last_error().decode())
        return OracleVolume(h, {"arrays": arrays, "dense": True}, fast, fma)

    @staticmethod
    def dense_temporal(data, dims, num_timesteps=0, indices=None, times=None, cell_centered=False,
                       grid_origin=None, grid_spacing=None, index_to_object=None, background=None, fast=False,
                       fma=False):
        """A structuredRegular volume with temporally varying data: `data` is
        one flat array per attribute (x-fastest voxels, each voxel's time
        samples consecutive), `dims` = (X, Y, Z); structured with
        num_timesteps > 0, unstructured with per-voxel `indices` (uint32 /
        uint64, X*Y*Z + 1 entries) into data and `times`."""
        arrays = data if isinstance(data, (list, tuple)) else [data]
        arrays = [np.ascontiguousarray(a).reshape(-1) for a in arrays]
        d = np.array(dims, np.int32)
        ptrs = (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
        types = np.array([_NP2VKL[a.dtype] for a in arrays], np.uint32)
        items = np.array([a.size for a in arrays], np.uint64)
        idx = None if indices is None else np.ascontiguousarray(indices)
        itype = 0 if idx is None else (5550 if idx.dtype == np.uint64 else 4500)
        tm = None if times is None else np.ascontiguousarray(times, np.float32)
        go = None if grid_origin is None else np.asarray(grid_origin, np.float32)
        gs = None if grid_spacing is None else np.asarray(grid_spacing, np.float32)
        i2o = None if index_to_object is None else np.asarray(index_to_object, np.float32)
        bg = None if background is None else np.asarray(background, np.float32).reshape(-1)
        L = lib(fast, fma)
        h = L.orc_dense_create_temporal(_p(d), len(arrays), ptrs, _p(types), _p(items), int(bool(cell_centered)),
                                        _p(go), _p(gs), _p(i2o), _p(bg), int(num_timesteps), _p(idx), itype,
                                        0 if idx is None else idx.size, _p(tm), 0 if tm is None else tm.size)
        if not h:
            raise RuntimeError(L.orc_last_error().decode())
        return OracleVolume(h, {"arrays": arrays, "idx": idx, "times": tm, "dense": True}, fast, fma)

    @staticmethod
    def vdb_volume(levels, origins, formats, packed_dense, packed_tile=None,
                   index_to_object=None, index_clipping_bounds=None, background=None, fast=False,
                   fma=False):
        levels = np.ascontiguousarray(levels, np.uint32)
        origins = np.ascontiguousarray(origins, np.int32).reshape(-1, 3)
        formats = np.ascontiguousarray(formats, np.uint32)
        pd = packed_dense if isinstance(packed_dense, (list, tuple)) else [packed_dense]
        pd = [np.ascontiguousarray(a) for a in pd]
        if packed_tile is None:
            pt = [np.zeros(0, pd[0].dtype) for _ in pd]
        else:
            pt = packed_tile if isinstance(packed_tile, (list, tuple)) else [packed_tile]
            pt = [np.ascontiguousarray(a) for a in pt]
        dtype = _NP2VKL[pd[0].dtype]
        pdp = (C.c_void_p * len(pd))(*[a.ctypes.data for a in pd])
        ptp = (C.c_void_p * len(pt))(*[a.ctypes.data for a in pt])
        i2o = None if index_to_object is None else np.asarray(index_to_object, np.float32)
        clip = None if index_clipping_bounds is None else np.asarray(index_clipping_bounds, np.int32)
        bg = None if background is None else np.asarray(background, np.float32).reshape(-1)
        L = lib(fast, fma)
        h = L.orc_vdb_create(len(levels), _p(levels), _p(origins), _p(formats), len(pd), dtype,
                             pdp, ptp, _p(i2o), _p(clip), _p(bg))
        if not h:
            raise RuntimeError(L.orc_last_error().decode())
        return OracleVolume(h, {"pd": pd, "pt": pt, "dense": False, "formats": formats}, fast, fma)

    def leaf_windows(self, attr=0):
        """(dense leaf slots, 9, 9, 9) float32: each dense leaf's voxels plus the
        next voxel on the +x/+y/+z side, by full-depth lookups (x outermost)."""
        n = int(np.count_nonzero(np.asarray(self._keep["formats"]) == 1))  # VKL_FORMAT_DENSE_ZYX
        w = np.empty((n, 9, 9, 9), np.float32)
        self._lib.orc_vdb_leaf_windows(self._h, attr, _p(w))
        return w

    def set_windows(self, decoded, attr=0):
        """Install decoded stencil-block windows: trilinear stencils whose base
        voxel lies in a dense leaf then read their corners from its window."""
        w = np.ascontiguousarray(decoded, np.float32).reshape(-1, 729)
        self._keep.setdefault("windows", {})[attr] = w
        self._lib.orc_vdb_set_windows(self._h, attr, w.shape[0], _p(w))

    # ---- introspection ------------------------------------------------
    def info(self):
        o2i = np.zeros(12, np.float32)
        i2o = np.zeros(12, np.float32)
        root = np.zeros(3, np.int32)
        active = np.zeros(3, np.uint32)
        dom = np.zeros(6, np.float32)
        bounds = np.zeros(6, np.float32)
        self._lib.orc_get_info(self._h, _p(o2i), _p(i2o), _p(root), _p(active), _p(dom), _p(bounds))
        return dict(o2i=o2i, i2o=i2o, root=root, active=active, domain=dom, bounds=bounds)

    def num_nodes(self, level):
        return int(self._lib.orc_level_num_nodes(self._h, level))

    def level(self, level, num_attributes=1):
        n = self.num_nodes(level)
        nv = n * (1 << (3 * [6, 5, 4, 3][level]))
        vox = np.zeros(nv, np.uint64)
        rng = np.zeros((nv * num_attributes, 2), np.float32)
        org = np.zeros((n, 3), np.uint32)
        self._lib.orc_get_level(self._h, level, _p(vox), _p(rng), _p(org))
        return vox, rng, org

    def value_range(self, attr=0):
        r = np.zeros(2, np.float32)
        self._lib.orc_value_range(self._h, attr, _p(r))
        return r

    # ---- sampling -----------------------------------------------------
    def sample(self, points, filter=FILTER_LINEAR, attr=0, max_sampling_depth=3):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.zeros(len(pts), np.float32)
        self._lib.orc_sample(self._h, filter, max_sampling_depth, len(pts), _p(pts), attr, _p(out))
        return out

    def sample_observed(self, points, num_leaves, filter=FILTER_LINEAR, attr=0, max_sampling_depth=3):
        """(samples, LeafNodeAccess buffer: uint32 per leaf, 1 where a walk reached it)."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.empty(len(pts), np.float32)
        acc = np.zeros(num_leaves, np.uint32)
        self._lib.orc_sample_observed(self._h, filter, max_sampling_depth, len(pts), _p(pts), attr, _p(out),
                                      _p(acc))
        return out, acc

    def sample_parallel(self, points, filter=FILTER_LINEAR, attr=0, threads=0):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.zeros(len(pts), np.float32)
        self._lib.orc_sample_parallel(self._h, filter, len(pts), _p(pts), attr, _p(out), threads)
        return out

    def gradient(self, points, filter=FILTER_LINEAR, attr=0, max_sampling_depth=3):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.zeros((len(pts), 3), np.float32)
        self._lib.orc_gradient(self._h, filter, max_sampling_depth, len(pts), _p(pts), attr, _p(out))
        return out

    def gradient_parallel(self, points, filter=FILTER_LINEAR, attr=0, max_sampling_depth=3, threads=0):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.zeros((len(pts), 3), np.float32)
        self._lib.orc_gradient_parallel(self._h, filter, max_sampling_depth, len(pts), _p(pts), attr, _p(out),
                                        threads)
        return out

    def sample_times(self, points, times, filter=FILTER_LINEAR, attr=0, threads=0):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        t = None if times is None else np.ascontiguousarray(times, np.float32).reshape(-1)
        out = np.zeros(len(pts), np.float32)
        self._lib.orc_sample_times(self._h, filter, len(pts), _p(pts), _p(t), attr, _p(out), threads)
        return out

    def gradient_times(self, points, times, filter=FILTER_LINEAR, attr=0, threads=0):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        t = None if times is None else np.ascontiguousarray(times, np.float32).reshape(-1)
        out = np.zeros((len(pts), 3), np.float32)
        self._lib.orc_gradient_times(self._h, filter, len(pts), _p(pts), _p(t), attr, _p(out), threads)
        return out

    def sample_fp64(self, points, filter=FILTER_LINEAR, attr=0):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.zeros(len(pts), np.float64)
        self._lib.orc_sample_fp64(self._h, filter, len(pts), _p(pts), attr, _p(out))
        return out

    # ---- iteration ----------------------------------------------------
    def intervals(self, origins, directions, t_ranges, value_ranges=None, hint=0.5, attr=0,
                  max_intervals=64):
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(t_ranges, np.float32).reshape(-1, 2)
        vr = None if value_ranges is None else np.ascontiguousarray(value_ranges, np.float32).reshape(-1, 2)
        nvr = 0 if vr is None else len(vr)
        out = np.zeros((len(o), max_intervals, 5), np.float32)
        cnt = np.zeros(len(o), np.uint32)
        self._lib.orc_iterate_intervals(self._h, attr, nvr, _p(vr), hint, len(o), _p(o), _p(d),
                                        _p(t), max_intervals, _p(out), _p(cnt))
        return out, cnt

    def macrocell_ranges(self, attr=0):
        """(nz, ny, nx, 2) value ranges of the 16^3-voxel macrocells."""
        d = self._keep["arrays"][0].shape  # (Z, Y, X)
        n = [((x - 1) >> 4) + 1 for x in d]
        out = np.zeros((n[0], n[1], n[2], 2), np.float32)
        self._lib.orc_macrocell_ranges(self._h, attr, _p(out))
        return out

    def macrocell_intervals(self, origins, directions, t_ranges, value_ranges=None, attr=0, max_intervals=64):
        """Intervals of the legacy 16^3 macrocell iterator: ((n, max, 5), counts)."""
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(t_ranges, np.float32).reshape(-1, 2)
        vr = None if value_ranges is None else np.ascontiguousarray(value_ranges, np.float32).reshape(-1, 2)
        nvr = 0 if vr is None else len(vr)
        out = np.zeros((len(o), max_intervals, 5), np.float32)
        cnt = np.zeros(len(o), np.uint32)
        if self._lib.orc_iterate_macrocells(self._h, attr, nvr, _p(vr), len(o), _p(o), _p(d), _p(t),
                                            max_intervals, _p(out), _p(cnt)):
            raise RuntimeError(self._lib.orc_last_error().decode())
        return out, cnt

    def hits(self, origins, directions, t_ranges, values, filter=FILTER_LINEAR, attr=0, max_hits=16):
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(t_ranges, np.float32).reshape(-1, 2)
        v = np.ascontiguousarray(values, np.float32).reshape(-1)
        out = np.zeros((len(o), max_hits, 3), np.float32)
        cnt = np.zeros(len(o), np.uint32)
        self._lib.orc_iterate_hits(self._h, attr, filter, len(v), _p(v), len(o), _p(o), _p(d),
                                   _p(t), max_hits, _p(out), _p(cnt))
        return out, cnt

    def render(self, renderer, camera, tf_colors, tf_range, width, height, bounds, filter=FILTER_LINEAR,
               gradient_filter=None, max_sampling_depth=3, attr=0, value_ranges=None, hint=0.5, iso_values=(),
               sampling_rate=1.0, interval_color_scale=4.0, interval_opacity=0.25, first_interval_only=False,
               show_interval_borders=False):
        """The example renderers restated (orc_render): (height, width, 4) RGBA float32."""
        vr = None if value_ranges is None else np.ascontiguousarray(value_ranges, np.float32).reshape(-1, 2)
        iso = np.ascontiguousarray(iso_values, np.float32).reshape(-1)
        cam = np.ascontiguousarray(camera, np.float32).reshape(14)
        tfc = np.ascontiguousarray(tf_colors, np.float32).reshape(-1, 4)
        tfr = np.ascontiguousarray(tf_range, np.float32).reshape(2)
        ip = np.array([width, height, int(first_interval_only), int(show_interval_borders)], np.int32)
        fp = np.array(list(bounds) + [sampling_rate, interval_color_scale, interval_opacity], np.float32)
        out = np.zeros((height, width, 4), np.float32)
        self._lib.orc_render(self._h, renderer, filter, filter if gradient_filter is None else gradient_filter,
                             max_sampling_depth, attr, 0 if vr is None else len(vr), _p(vr), hint, len(iso),
                             _p(iso), _p(cam), _p(tfc), len(tfc), _p(tfr), _p(ip), _p(fp), _p(out))
        return out

    def path_trace(self, camera, tf_colors, tf_range, width, height, bounds, frames=(0,), filter=FILTER_LINEAR,
                   max_sampling_depth=3, attr=0, time=0.0, shutter=0.0, motion_blur=False, sigma_t_scale=1.0,
                   sigma_s_scale=1.0, max_num_scatters=1, ambient_light_intensity=1.0, show_bbox=False):
        """The density path tracer restated (orc_path_trace): the frames'
        contributions accumulated as the renderer does; returns (rgba
        (H, W, 4), weights (H, W))."""
        cam = np.ascontiguousarray(camera, np.float32).reshape(14)
        tfc = np.ascontiguousarray(tf_colors, np.float32).reshape(-1, 4)
        tfr = np.ascontiguousarray(tf_range, np.float32).reshape(2)
        b = np.ascontiguousarray(bounds, np.float32).reshape(6)
        rgba = np.zeros((height, width, 4), np.float32)
        w = np.zeros((height, width), np.float32)
        for f in frames:
            pt = np.array([shutter, sigma_t_scale, sigma_s_scale, ambient_light_intensity, time], np.float32)
            ipt = np.array([int(motion_blur), max_num_scatters, int(show_bbox), f], np.int32)
            self._lib.orc_path_trace(self._h, filter, max_sampling_depth, attr, _p(cam), _p(tfc), len(tfc), _p(tfr),
                                     width, height, _p(b), _p(pt), _p(ipt), _p(rgba), _p(w))
        return rgba, w

    def inner_nodes(self, max_depth=1, attr=0):
        n = int(self._lib.orc_inner_nodes(self._h, max_depth, attr, 0, None))
        out = np.zeros((n, 8), np.float32)
        self._lib.orc_inner_nodes(self._h, max_depth, attr, n, _p(out))
        return out


def tricubic_map():
    """(start[65], cols[nnz], weights[nnz]) of the oracle's coefficient map."""
    L = lib()
    nnz = L.orc_tricubic_map(None, None, None)
    start = np.zeros(65, np.int32)
    cols = np.zeros(nnz, np.int32)
    w = np.zeros(nnz, np.float32)
    L.orc_tricubic_map(_p(start), _p(cols), _p(w))
    return start, cols, w


COMPRESSION_FORMATS = {"fp16": 1, "bf16": 2, "fp8": 3}


def round_format(fmt, values):
    """Each float rounded to nearest-even in fp16 / bf16 / fp8 (E4M3, saturating)."""
    x = np.ascontiguousarray(values, np.float32)
    out = np.empty_like(x)
    lib().orc_round_format(COMPRESSION_FORMATS[fmt], x.size, _p(x), _p(out))
    return out


def quantize_leaves(fmt, leaves):
    """Packed leaves (n*512 floats) -> (decoded floats, (n,2) scale/offset) as
    the cuda device's compressed storage reproduces them."""
    x = np.ascontiguousarray(leaves, np.float32).reshape(-1)
    n = x.size // 512
    dec = np.empty_like(x)
    so = np.empty((n, 2), np.float32)
    lib().orc_quantize_leaves(COMPRESSION_FORMATS[fmt], n, _p(x), _p(dec), _p(so))
    return dec, so


def quantize_groups(fmt, values, group):
    """Groups of `group` floats -> (decoded floats, (n,2) scale/offset) by the
    compressed-leaf rule (one scale and offset per group)."""
    x = np.ascontiguousarray(values, np.float32).reshape(-1)
    n = x.size // group
    dec = np.empty_like(x)
    so = np.empty((n, 2), np.float32)
    lib().orc_quantize_groups(COMPRESSION_FORMATS[fmt], n, group, _p(x), _p(dec), _p(so))
    return dec, so


def vdb_blocked_volume(fmt, levels, origins, formats, packed_dense, packed_tile=None, **kw):
    """The oracle of the cuda device's stencil-block leaves (compression
    "<fmt>_blocks"): each dense leaf's 9^3 sampling window of the float volume
    quantized with one scale and offset, the leaves' own voxels decoded from
    it, and trilinear stencils based in a dense leaf read from its window.
    Returns (volume, per-attribute (n, 2) scale/offset arrays)."""
    flt = OracleVolume.vdb_volume(levels, origins, formats, packed_dense, packed_tile, **kw)
    pd = packed_dense if isinstance(packed_dense, (list, tuple)) else [packed_dense]
    wins, sos, inner = [], [], []
    for a in range(len(pd)):
        w = flt.leaf_windows(a)
        dec, so = quantize_groups(fmt, w, 729)
        dec = dec.reshape(-1, 9, 9, 9)
        wins.append(dec)
        sos.append(so)
        inner.append(np.ascontiguousarray(dec[:, :8, :8, :8]).reshape(-1))
    vol = OracleVolume.vdb_volume(levels, origins, formats, inner if len(inner) > 1 else inner[0],
                                  packed_tile, **kw)
    for a, w in enumerate(wins):
        vol.set_windows(w, a)
    return vol, sos
