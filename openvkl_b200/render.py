"""Headless example renderers (libopenvkl_renderers.so): the reference's ray
march iterator, interval iterator debug and hit iterator renderers as CUDA
kernels that call the cuda device's __device__ API, writing an RGBA float
framebuffer in device memory instead of a window.

    from openvkl_b200 import render, vkl
    cam = render.orbit_camera(volume.bounding_box(), 640, 480)
    rgba = render.render("ray_march", sampler, cam, width=640, height=480,
                         interval_context=ctx)      # torch (H, W, 4) on cuda
    render.write_pfm("frame.pfm", rgba)

The oracle restates the same renderers (oracle/pyoracle.py
OracleVolume.render); the GPU tests compare the two images bit for bit.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import vkl

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libopenvkl_renderers.so")
RENDERERS = {"ray_march": 0, "interval_debug": 1, "hits": 2}
MAX_TF = 256
# TransferFunction.h default: blue (transparent) -> green -> red (opaque)
DEFAULT_TF = np.array([[0, 0, 1, 0], [0, 1, 0, 0.5], [1, 0, 0, 1]], np.float32)


class Camera(C.Structure):
    _fields_ = [("sensorWidth", C.c_float), ("focalLength", C.c_float), ("ctwR", C.c_float * 9),
                ("ctwT", C.c_float * 3)]

    def as_array(self):
        return np.array([self.sensorWidth, self.focalLength] + list(self.ctwR) + list(self.ctwT), np.float32)


class TransferFunction(C.Structure):
    _fields_ = [("valueRange", C.c_float * 2), ("numValues", C.c_int), ("colorsAndOpacities", C.c_float * (4 * MAX_TF))]


class PathTracerParams(C.Structure):
    _fields_ = [("shutter", C.c_float), ("motionBlur", C.c_int), ("sigmaTScale", C.c_float),
                ("sigmaSScale", C.c_float), ("maxNumScatters", C.c_int), ("ambientLightIntensity", C.c_float),
                ("showBbox", C.c_int), ("frame", C.c_uint)]


class Params(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("attributeIndex", C.c_uint), ("time", C.c_float),
                ("featureFlags", C.c_uint64), ("bounds", C.c_float * 6), ("samplingRate", C.c_float), ("intervalColorScale", C.c_float),
                ("intervalOpacity", C.c_float), ("firstIntervalOnly", C.c_int), ("showIntervalBorders", C.c_int)]


_lib = None


def load_library(path: str = LIB_PATH):
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(f"renderer library not built: {path} (run python -m openvkl_b200.build)")
        L = C.CDLL(path)
        L.vklExampleRender.restype = C.c_int
        L.vklExampleRender.argtypes = [C.c_int, vkl.VKLObject, vkl.VKLObject, vkl.VKLObject, C.POINTER(Camera),
                                       C.POINTER(TransferFunction), C.POINTER(Params), C.c_void_p, C.c_void_p]
        L.vklExamplePathTrace.restype = C.c_int
        L.vklExamplePathTrace.argtypes = [vkl.VKLObject, C.POINTER(Camera), C.POINTER(TransferFunction),
                                          C.POINTER(Params), C.POINTER(PathTracerParams), C.c_void_p, C.c_void_p,
                                          C.c_void_p]
        L.vklExampleSamplePoints.restype = C.c_int
        L.vklExampleSamplePoints.argtypes = [vkl.VKLObject, C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint,
                                             C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def orbit_camera(bounds, width, height, azimuth=0.7, elevation=0.35, distance=1.6, fov_deg=45.0):
    """A camera on an orbit around the box centre looking at it (the role of
    the examples' ArcballCamera): sensor width 1 unit, focal length from the
    horizontal field of view."""
    b = np.asarray(bounds, np.float64)
    ctr = 0.5 * (b[:3] + b[3:])
    r = distance * float(np.max(b[3:] - b[:3]))
    eye = ctr + r * np.array([math.cos(azimuth) * math.cos(elevation), math.sin(elevation),
                              math.sin(azimuth) * math.cos(elevation)])
    fwd = (ctr - eye) / np.linalg.norm(ctr - eye)
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    # camera looks down -z: columns of the camera-to-world rotation are
    # (right, up, -forward); Camera.ih stores its rows
    R = np.stack([right, up, -fwd], 1)
    cam = Camera()
    cam.sensorWidth = 1.0
    cam.focalLength = 0.5 / math.tan(math.radians(fov_deg) / 2)
    cam.ctwR[:] = [float(x) for x in R.reshape(-1)]
    cam.ctwT[:] = [float(x) for x in eye]
    return cam


def transfer_function(value_range, colors=DEFAULT_TF):
    c = np.ascontiguousarray(colors, np.float32).reshape(-1, 4)
    if len(c) > MAX_TF:
        raise ValueError(f"at most {MAX_TF} transfer function entries")
    tf = TransferFunction()
    tf.valueRange[:] = [float(value_range[0]), float(value_range[1])]
    tf.numValues = len(c)
    tf.colorsAndOpacities[:4 * len(c)] = [float(x) for x in c.reshape(-1)]
    return tf


def params(width, height, bounds, attr=0, sampling_rate=1.0, interval_color_scale=4.0, interval_opacity=0.25,
           first_interval_only=False, show_interval_borders=False):
    p = Params()
    p.width, p.height, p.attributeIndex, p.time = width, height, attr, 0.0
    p.bounds[:] = [float(x) for x in bounds]
    p.samplingRate, p.intervalColorScale, p.intervalOpacity = sampling_rate, interval_color_scale, interval_opacity
    p.firstIntervalOnly, p.showIntervalBorders = int(first_interval_only), int(show_interval_borders)
    return p


def render(renderer, sampler, camera, width, height, tf=None, interval_context=None, hit_context=None,
           out=None, stream=None, **kw):
    """One frame as a (height, width, 4) float32 CUDA tensor (row 0 at the top)."""
    import torch
    L = load_library()
    bounds = sampler.volume.bounding_box() if hasattr(sampler, "volume") else kw.pop("bounds")
    if tf is None:
        lo, hi = sampler.volume.value_range()
        tf = transfer_function((lo, hi))
    prm = params(width, height, bounds, **kw)
    prm.featureFlags = sampler.feature_flags()
    if out is None:
        out = torch.empty((height, width, 4), dtype=torch.float32, device="cuda")
    null = vkl.VKLObject(None, None)
    st = torch.cuda.current_stream().cuda_stream if stream is None else stream
    rc = L.vklExampleRender(RENDERERS[renderer], sampler.h,
                            interval_context.h if interval_context is not None else null,
                            hit_context.h if hit_context is not None else null, C.byref(camera), C.byref(tf),
                            C.byref(prm), out.data_ptr(), st)
    if rc != 0:
        raise RuntimeError(f"vklExampleRender failed: CUDA error {rc}")
    return out


def path_trace(sampler, camera, width, height, frames=(0,), tf=None, rgba=None, weights=None, stream=None,
               time=0.0, shutter=0.0, motion_blur=False, sigma_t_scale=1.0, sigma_s_scale=1.0, max_num_scatters=1,
               ambient_light_intensity=1.0, show_bbox=False, attr=0):
    """The density path tracer: each frame adds one path per pixel into
    rgba ((H, W, 4) CUDA tensor) and 1 into weights ((H, W)); the image is
    rgba / weights.  Returns (rgba, weights)."""
    import torch
    L = load_library()
    if tf is None:
        lo, hi = sampler.volume.value_range()
        tf = transfer_function((lo, hi))
    prm = params(width, height, sampler.volume.bounding_box(), attr=attr)
    prm.time = float(time)
    prm.featureFlags = sampler.feature_flags()
    if rgba is None:
        rgba = torch.zeros((height, width, 4), dtype=torch.float32, device="cuda")
    if weights is None:
        weights = torch.zeros((height, width), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream if stream is None else stream
    for f in frames:
        pt = PathTracerParams(float(shutter), int(motion_blur), float(sigma_t_scale), float(sigma_s_scale),
                              int(max_num_scatters), float(ambient_light_intensity), int(show_bbox), int(f))
        rc = L.vklExamplePathTrace(sampler.h, C.byref(camera), C.byref(tf), C.byref(prm), C.byref(pt),
                                   rgba.data_ptr(), weights.data_ptr(), st)
        if rc != 0:
            raise RuntimeError(f"vklExamplePathTrace failed: CUDA error {rc}")
    return rgba, weights


def sample_points(sampler, points, attr=0):
    """Samples and gradients of device points through the __device__ API."""
    import torch
    L = load_library()
    n = points.shape[0]
    s = torch.empty(n, dtype=torch.float32, device="cuda")
    g = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    rc = L.vklExampleSamplePoints(sampler.h, sampler.feature_flags(), n, points.data_ptr(), attr, s.data_ptr(), g.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    if rc != 0:
        raise RuntimeError(f"vklExampleSamplePoints failed: CUDA error {rc}")
    return s, g


def write_pfm(path, rgba):
    """Colour PFM (little endian, bottom row first) of an (H, W, 4) image."""
    img = rgba.cpu().numpy() if hasattr(rgba, "cpu") else np.asarray(rgba)
    h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(f"PF\n{w} {h}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(img[::-1, :, :3], np.float32).tobytes())


def write_ppm(path, rgba):
    """8-bit PPM (clamped, gamma 1) of an (H, W, 4) image."""
    img = rgba.cpu().numpy() if hasattr(rgba, "cpu") else np.asarray(rgba)
    h, w = img.shape[:2]
    rgb = (np.clip(img[:, :, :3], 0, 1) * 255 + 0.5).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(f"P6\n{w} {h}\n255\n".encode())
        f.write(rgb.tobytes())
