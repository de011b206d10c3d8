"""Python binding of the cuda device's C API (libopenvkl_device_cuda.so).

A thin ctypes layer over include/openvkl_cuda.h that mirrors the Open VKL
object API (devices, data, volumes, samplers, iterator contexts, observers)
with the reference's names, argument meaning and error behaviour: failures
set the device's last error and raise `VKLError` here.  Arrays may be numpy
arrays (host memory; the library stages them through the GPU) or CUDA
tensors / raw device pointers (used in place).

The library is required: importing a sampler path without the built .so
raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libopenvkl_device_cuda.so")

VKL_DEVICE, VKL_VOID_PTR, VKL_BOOL = 100, 200, 250
VKL_OBJECT, VKL_DATA = 0x8000000, 0x8000000 + 100
VKL_STRING = 1500
VKL_UCHAR, VKL_SHORT, VKL_USHORT = 2500, 3000, 3500
VKL_INT, VKL_VEC3I = 4000, 4002
VKL_UINT = 4500
VKL_ULONG = 5550
VKL_HALF, VKL_FLOAT, VKL_VEC3F, VKL_DOUBLE = 5800, 6000, 6002, 7000
VKL_BOX1F, VKL_BOX3I = 10000, 8002
VKL_AFFINE3F = 12003
VKL_DATA_DEFAULT, VKL_DATA_SHARED_BUFFER = 0, 1
VKL_FILTER_NEAREST, VKL_FILTER_LINEAR, VKL_FILTER_CUBIC = 0, 100, 200
VKL_FORMAT_TILE, VKL_FORMAT_DENSE_ZYX = 0, 1

_NP2VKL = {
    np.dtype(np.uint8): VKL_UCHAR,
    np.dtype(np.int16): VKL_SHORT,
    np.dtype(np.uint16): VKL_USHORT,
    np.dtype(np.float16): VKL_HALF,
    np.dtype(np.float32): VKL_FLOAT,
    np.dtype(np.float64): VKL_DOUBLE,
    np.dtype(np.int32): VKL_INT,
    np.dtype(np.uint32): VKL_UINT,
    np.dtype(np.uint64): VKL_ULONG,
}
_VKL_ITEM = {VKL_UCHAR: 1, VKL_SHORT: 2, VKL_USHORT: 2, VKL_HALF: 2, VKL_FLOAT: 4,
             VKL_DOUBLE: 8, VKL_INT: 4, VKL_UINT: 4, VKL_ULONG: 8, VKL_VEC3I: 12, VKL_VEC3F: 12, VKL_BOX1F: 8}

# Exported symbols declared in include/openvkl_cuda.h.
EXPORTS = [
    "vklInit", "vklNewDevice", "vklDeviceSetLogCallback", "vklDeviceSetErrorCallback",
    "vklDeviceSetInt", "vklDeviceSetString", "vklDeviceSetVoidPtr", "vklCommitDevice",
    "vklDeviceGetLastErrorCode", "vklDeviceGetLastErrorMsg", "vklGetNativeSIMDWidth",
    "vklCommit", "vklRelease", "vklReleaseDevice", "vklNewData", "vklNewVolume",
    "vklGetBoundingBox", "vklGetNumAttributes", "vklGetValueRange", "vklSetBool", "vklSetFloat",
    "vklSetVec3f", "vklSetInt", "vklSetVec3i", "vklSetData", "vklSetString", "vklSetVoidPtr",
    "vklSetParam", "vklNewSampler", "vklGetFeatureFlags", "vklComputeSample",
    "vklComputeSample4", "vklComputeSample8", "vklComputeSample16", "vklComputeSampleN",
    "vklComputeSampleM", "vklComputeSampleMN", "vklComputeGradient", "vklComputeGradientN",
    "vklComputeSampleM4", "vklComputeSampleM8", "vklComputeSampleM16",
    "vklComputeGradient4", "vklComputeGradient8", "vklComputeGradient16",
    "vklNewIntervalIteratorContext", "vklNewHitIteratorContext", "vklGetIntervalIteratorSize",
    "vklInitIntervalIterator", "vklIterateInterval", "vklGetHitIteratorSize",
    "vklInitHitIterator", "vklIterateHit", "vklIterateIntervalsN", "vklIterateHitsN",
    "vklNewVolumeObserver", "vklNewSamplerObserver", "vklMapObserver", "vklUnmapObserver",
    "vklGetObserverElementType", "vklGetObserverElementSize", "vklGetObserverNumElements",
    "vklCudaGetTreeLevel", "vklCudaDenseValueRangeNoAlloc",
    "vklCudaNewSampleBatch", "vklCudaRunSampleBatch", "vklCudaGetSampleBatchConfig",
    "vklCudaReleaseSampleBatch",
    "vklCudaNewSurrogate", "vklCudaSurrogateSetParameters", "vklCudaSurrogateGetParameters",
    "vklCudaSurrogateGradient", "vklCudaSurrogateTrainStep", "vklCudaSurrogateCalibrate",
    "vklCudaSurrogateSample", "vklCudaGetSurrogateInfo", "vklCudaReleaseSurrogate",
]


class VKLError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"VKL error {code}: {msg}")
        self.code = code
        self.msg = msg


class VKLObject(C.Structure):
    _fields_ = [("host", C.c_void_p), ("device", C.c_void_p)]


class vec3f(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class range1f(C.Structure):
    _fields_ = [("lower", C.c_float), ("upper", C.c_float)]


class box3f(C.Structure):
    _fields_ = [("lower", vec3f), ("upper", vec3f)]


class VKLInterval(C.Structure):
    _fields_ = [("tRange", range1f), ("valueRange", range1f), ("nominalDeltaT", C.c_float)]


class VKLHit(C.Structure):
    _fields_ = [("t", C.c_float), ("sample", C.c_float), ("epsilon", C.c_float)]


class VKLCudaSampleJob(C.Structure):
    _fields_ = [("sampler", VKLObject), ("points", C.c_void_p), ("numPoints", C.c_uint),
                ("attributeIndex", C.c_uint), ("samples", C.c_void_p), ("gradients", C.c_void_p)]


class vvec3f4(C.Structure):
    _fields_ = [("x", C.c_float * 4), ("y", C.c_float * 4), ("z", C.c_float * 4)]


class vvec3f8(C.Structure):
    _fields_ = [("x", C.c_float * 8), ("y", C.c_float * 8), ("z", C.c_float * 8)]


class vvec3f16(C.Structure):
    _fields_ = [("x", C.c_float * 16), ("y", C.c_float * 16), ("z", C.c_float * 16)]


_ERROR_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_char_p)
_LOG_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_char_p)
_lib = None


def load_library(path: str = LIB_PATH, load_only: bool = False) -> C.CDLL:
    """Loads the cuda device library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"cuda device library not built: {path} (run python -m openvkl_b200.build)")
    L = C.CDLL(path)
    P, VP, U, I, F, SZ = C.c_void_p, C.c_void_p, C.c_uint, C.c_int, C.c_float, C.c_size_t
    O = VKLObject
    sig = {
        "vklInit": (None, []),
        "vklNewDevice": (P, [C.c_char_p]),
        "vklDeviceSetErrorCallback": (None, [P, _ERROR_CB, VP]),
        "vklDeviceSetLogCallback": (None, [P, _LOG_CB, VP]),
        "vklDeviceSetInt": (None, [P, C.c_char_p, I]),
        "vklDeviceSetString": (None, [P, C.c_char_p, C.c_char_p]),
        "vklDeviceSetVoidPtr": (None, [P, C.c_char_p, VP]),
        "vklCommitDevice": (None, [P]),
        "vklDeviceGetLastErrorCode": (I, [P]),
        "vklDeviceGetLastErrorMsg": (C.c_char_p, [P]),
        "vklGetNativeSIMDWidth": (I, [P]),
        "vklCommit": (None, [O]),
        "vklRelease": (None, [O]),
        "vklReleaseDevice": (None, [P]),
        "vklNewData": (O, [P, SZ, I, VP, I, SZ]),
        "vklNewVolume": (O, [P, C.c_char_p]),
        "vklGetBoundingBox": (box3f, [O]),
        "vklGetNumAttributes": (U, [O]),
        "vklGetValueRange": (range1f, [O, U]),
        "vklSetBool": (None, [O, C.c_char_p, I]),
        "vklSetFloat": (None, [O, C.c_char_p, F]),
        "vklSetVec3f": (None, [O, C.c_char_p, F, F, F]),
        "vklSetInt": (None, [O, C.c_char_p, I]),
        "vklSetVec3i": (None, [O, C.c_char_p, I, I, I]),
        "vklSetData": (None, [O, C.c_char_p, O]),
        "vklSetString": (None, [O, C.c_char_p, C.c_char_p]),
        "vklSetVoidPtr": (None, [O, C.c_char_p, VP]),
        "vklSetParam": (None, [O, C.c_char_p, I, VP]),
        "vklNewSampler": (O, [O]),
        "vklGetFeatureFlags": (C.c_uint64, [O]),
        "vklComputeSample": (F, [C.POINTER(O), C.POINTER(vec3f), U, F]),
        "vklComputeSample4": (None, [VP, C.POINTER(O), C.POINTER(vvec3f4), VP, U, VP]),
        "vklComputeSample8": (None, [VP, C.POINTER(O), C.POINTER(vvec3f8), VP, U, VP]),
        "vklComputeSample16": (None, [VP, C.POINTER(O), C.POINTER(vvec3f16), VP, U, VP]),
        "vklComputeSampleN": (None, [C.POINTER(O), U, VP, VP, U, VP]),
        "vklComputeSampleM": (None, [C.POINTER(O), C.POINTER(vec3f), VP, U, VP, F]),
        "vklComputeSampleMN": (None, [C.POINTER(O), U, VP, VP, U, VP, VP]),
        "vklComputeGradient": (vec3f, [C.POINTER(O), C.POINTER(vec3f), U, F]),
        "vklComputeGradientN": (None, [C.POINTER(O), U, VP, VP, U, VP]),
        "vklComputeSampleM4": (None, [VP, C.POINTER(O), C.POINTER(vvec3f4), VP, U, VP, VP]),
        "vklComputeSampleM8": (None, [VP, C.POINTER(O), C.POINTER(vvec3f8), VP, U, VP, VP]),
        "vklComputeSampleM16": (None, [VP, C.POINTER(O), C.POINTER(vvec3f16), VP, U, VP, VP]),
        "vklComputeGradient4": (None, [VP, C.POINTER(O), C.POINTER(vvec3f4), C.POINTER(vvec3f4), U, VP]),
        "vklComputeGradient8": (None, [VP, C.POINTER(O), C.POINTER(vvec3f8), C.POINTER(vvec3f8), U, VP]),
        "vklComputeGradient16": (None, [VP, C.POINTER(O), C.POINTER(vvec3f16), C.POINTER(vvec3f16), U, VP]),
        "vklNewIntervalIteratorContext": (O, [O]),
        "vklNewHitIteratorContext": (O, [O]),
        "vklGetIntervalIteratorSize": (SZ, [C.POINTER(O)]),
        "vklInitIntervalIterator": (VP, [C.POINTER(O), C.POINTER(vec3f), C.POINTER(vec3f),
                                         C.POINTER(range1f), F, VP]),
        "vklIterateInterval": (I, [VP, C.POINTER(VKLInterval)]),
        "vklGetHitIteratorSize": (SZ, [C.POINTER(O)]),
        "vklInitHitIterator": (VP, [C.POINTER(O), C.POINTER(vec3f), C.POINTER(vec3f),
                                    C.POINTER(range1f), F, VP]),
        "vklIterateHit": (I, [VP, C.POINTER(VKLHit)]),
        "vklIterateIntervalsN": (None, [C.POINTER(O), U, VP, VP, VP, U, VP, VP]),
        "vklIterateHitsN": (None, [C.POINTER(O), U, VP, VP, VP, U, VP, VP]),
        "vklNewVolumeObserver": (O, [O, C.c_char_p]),
        "vklNewSamplerObserver": (O, [O, C.c_char_p]),
        "vklMapObserver": (VP, [O]),
        "vklUnmapObserver": (None, [O]),
        "vklGetObserverElementType": (I, [O]),
        "vklGetObserverElementSize": (SZ, [O]),
        "vklGetObserverNumElements": (SZ, [O]),
        "vklCudaGetTreeLevel": (C.c_uint64, [O, U, VP, VP, VP]),
        "vklCudaDenseValueRangeNoAlloc": (I, [VP, VP, I, I, I, I, C.c_float, VP]),
        "vklCudaNewSampleBatch": (VP, [VP, U, C.POINTER(VKLCudaSampleJob), I]),
        "vklCudaRunSampleBatch": (I, [VP]),
        "vklCudaGetSampleBatchConfig": (I, [VP, C.POINTER(I), C.POINTER(I), C.POINTER(I), C.POINTER(I)]),
        "vklCudaReleaseSampleBatch": (None, [VP]),
        "vklCudaNewSurrogate": (VP, [O, U, F, F]),
        "vklCudaSurrogateSetParameters": (I, [VP, VP, VP]),
        "vklCudaSurrogateGetParameters": (I, [VP, VP, VP]),
        "vklCudaSurrogateGradient": (I, [VP, U, VP, VP, VP, VP, VP]),
        "vklCudaSurrogateTrainStep": (I, [VP, U, VP, VP, F, VP]),
        "vklCudaSurrogateCalibrate": (I, [VP, U, VP, F, C.POINTER(U)]),
        "vklCudaSurrogateSample": (I, [VP, U, VP, VP, I]),
        "vklCudaGetSurrogateInfo": (None, [VP, C.POINTER(C.c_uint64), C.POINTER(U), C.POINTER(C.c_uint64), VP]),
        "vklCudaReleaseSurrogate": (None, [VP]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


# ---------------------------------------------------------------------------
# Array helpers: numpy (host) or torch CUDA tensors (device) -> pointer.
# ---------------------------------------------------------------------------
def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if _is_torch(a):
        assert a.is_contiguous()
        return a.data_ptr()
    return a.ctypes.data


def _times(times):
    """Pointer to a per-point time array (None -> NULL); numpy arrays are
    made contiguous float32 and must stay alive for the call."""
    if times is None:
        return None
    if _is_torch(times):
        return C.c_void_p(times.data_ptr())
    global _times_keep
    _times_keep = np.ascontiguousarray(times, np.float32)
    return C.c_void_p(_times_keep.ctypes.data)


_times_keep = None


def _alloc_like(ref, shape, dtype=np.float32):
    if _is_torch(ref):
        import torch
        tdt = {np.float32: torch.float32, np.uint32: torch.int32}[dtype]
        return torch.empty(shape, dtype=tdt, device=ref.device)
    return np.empty(shape, dtype)


class Device:
    def __init__(self, name: str = "cuda"):
        self.lib = load_library()
        self.lib.vklInit()
        self.handle = self.lib.vklNewDevice(name.encode())
        if not self.handle:
            raise RuntimeError(f"vklNewDevice('{name}') failed (no CUDA device?)")
        self.pending = None
        # errors arrive through the device's error callback, as in the
        # reference API; _Obj._call turns them into exceptions
        self._cb = _ERROR_CB(self._on_error)
        self.lib.vklDeviceSetErrorCallback(self.handle, self._cb, None)
        self.lib.vklCommitDevice(self.handle)

    def _on_error(self, user, code, msg):
        self.pending = (code, msg.decode() if msg else "")

    def raise_pending(self):
        if self.pending is not None:
            code, msg = self.pending
            self.pending = None
            raise VKLError(code, msg)

    def last_error(self):
        return (self.lib.vklDeviceGetLastErrorCode(self.handle),
                self.lib.vklDeviceGetLastErrorMsg(self.handle).decode())

    def set_int(self, name: str, value: int):
        self.lib.vklDeviceSetInt(self.handle, name.encode(), int(value))

    def capture_log(self, messages: list):
        """Routes the device's log messages into `messages` (a list of str);
        vklDeviceSetLogCallback."""
        self._log_cb = _LOG_CB(lambda user, msg: messages.append(msg.decode() if msg else ""))
        self.lib.vklDeviceSetLogCallback(self.handle, self._log_cb, None)

    def set_stream(self, stream_ptr: int):
        self.lib.vklDeviceSetVoidPtr(self.handle, b"cudaStream", C.c_void_p(stream_ptr))

    def release(self):
        if self.handle:
            self.lib.vklReleaseDevice(self.handle)
            self.handle = None


class _Obj:
    def __init__(self, device: Device, handle: VKLObject):
        self.device = device
        self.lib = device.lib
        self.h = handle
        self._keep = []

    def _check_handle(self, what):
        if not self.h.host:
            self.device.raise_pending()
            code, msg = self.device.last_error()
            raise VKLError(code, f"{what}: {msg}")

    def release(self):
        if self.h is not None and self.h.host:
            self.lib.vklRelease(self.h)
            self.h = VKLObject()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def _call(self, fn, *args):
        self.device.pending = None
        r = fn(*args)
        self.device.raise_pending()
        return r

    def set_int(self, name, v):
        self.lib.vklSetInt(self.h, name.encode(), int(v))
        return self

    def set_float(self, name, v):
        self.lib.vklSetFloat(self.h, name.encode(), float(v))
        return self

    def set_bool(self, name, v):
        self.lib.vklSetBool(self.h, name.encode(), int(bool(v)))
        return self

    def set_vec3f(self, name, v):
        self.lib.vklSetVec3f(self.h, name.encode(), *[float(x) for x in v])
        return self

    def set_vec3i(self, name, v):
        self.lib.vklSetVec3i(self.h, name.encode(), *[int(x) for x in v])
        return self

    def set_string(self, name, v):
        self.lib.vklSetString(self.h, name.encode(), str(v).encode())
        return self

    def set_data(self, name, data: "Data"):
        self.lib.vklSetData(self.h, name.encode(), data.h)
        self._keep.append(data)
        return self

    def set_param(self, name, vkl_type, arr):
        a = np.ascontiguousarray(arr)
        self.lib.vklSetParam(self.h, name.encode(), vkl_type, a.ctypes.data)
        return self

    def commit(self):
        self._call(self.lib.vklCommit, self.h)
        return self


class Data(_Obj):
    """vklNewData over a numpy array, a CUDA tensor or a list of Data."""

    def __init__(self, device: Device, array=None, vkl_type: Optional[int] = None,
                 shared: bool = False, objects: Optional[Sequence["Data"]] = None,
                 num_items: Optional[int] = None, byte_stride: int = 0):
        if objects is not None:
            # None entries become null handles (e.g. the per-node temporal
            # arrays of temporally constant vdb nodes)
            arr = (VKLObject * len(objects))(*[o.h if o is not None else VKLObject() for o in objects])
            h = device.lib.vklNewData(device.handle, len(objects), VKL_DATA, C.cast(arr, C.c_void_p),
                                      VKL_DATA_DEFAULT, 0)
            super().__init__(device, h)
            self._keep = [o for o in objects if o is not None]
            self._check_handle("vklNewData")
            return
        if _is_torch(array):
            import torch
            tmap = {torch.float32: VKL_FLOAT, torch.float16: VKL_HALF, torch.uint8: VKL_UCHAR,
                    torch.int16: VKL_SHORT, torch.float64: VKL_DOUBLE, torch.int32: VKL_INT}
            t = vkl_type or tmap[array.dtype]
            n = num_items if num_items is not None else array.numel() * array.element_size() // _VKL_ITEM[t]
            src = array.data_ptr()
        else:
            array = np.ascontiguousarray(array)
            t = vkl_type or _NP2VKL[array.dtype]
            n = num_items if num_items is not None else array.nbytes // _VKL_ITEM[t]
            src = array.ctypes.data
        device.pending = None
        h = device.lib.vklNewData(device.handle, n, t, C.c_void_p(src),
                                  VKL_DATA_SHARED_BUFFER if shared else VKL_DATA_DEFAULT, byte_stride)
        super().__init__(device, h)
        self._keep = [array] if shared else []
        self.num_items, self.vkl_type = n, t
        self._check_handle("vklNewData")


class Volume(_Obj):
    def __init__(self, device: Device, type_name: str):
        super().__init__(device, device.lib.vklNewVolume(device.handle, type_name.encode()))
        self._check_handle("vklNewVolume")

    def bounding_box(self):
        b = self.lib.vklGetBoundingBox(self.h)
        return np.array([b.lower.x, b.lower.y, b.lower.z, b.upper.x, b.upper.y, b.upper.z], np.float32)

    def num_attributes(self):
        return self.lib.vklGetNumAttributes(self.h)

    def value_range(self, attr=0):
        r = self.lib.vklGetValueRange(self.h, attr)
        return np.array([r.lower, r.upper], np.float32)

    def tree_level(self, level):
        """(voxels u64, value ranges (n,2*attrs) f32, origins (nodes,3) u32)."""
        n = self._call(self.lib.vklCudaGetTreeLevel, self.h, level, None, None, None)
        if level == 3:
            return n
        nv = n * (1 << (3 * [6, 5, 4][level]))
        na = self.num_attributes()
        vox = np.zeros(nv, np.uint64)
        rng = np.zeros((nv * na, 2), np.float32)
        org = np.zeros((n, 3), np.uint32)
        self._call(self.lib.vklCudaGetTreeLevel, self.h, level, vox.ctypes.data, rng.ctypes.data,
                   org.ctypes.data)
        return vox, rng, org

    def inner_nodes(self, max_depth=1):
        obs = VKLObserverObj(self.device, self.lib.vklNewVolumeObserver(self.h, b"InnerNode"))
        obs.set_int("maxDepth", max_depth)
        return obs.read()


class VKLObserverObj(_Obj):
    def __init__(self, device, handle, what="vklNewVolumeObserver"):
        super().__init__(device, handle)
        self._check_handle(what)

    def read_uint(self):
        """The mapped buffer of a uint32 observer (LeafNodeAccess)."""
        p = self._call(self.lib.vklMapObserver, self.h)
        n = self.lib.vklGetObserverNumElements(self.h)
        if n == 0:
            return np.zeros(0, np.uint32)
        out = np.array((C.c_uint32 * n).from_address(p), np.uint32)
        self.lib.vklUnmapObserver(self.h)
        return out

    def read(self):
        p = self.lib.vklMapObserver(self.h)
        n = self.lib.vklGetObserverNumElements(self.h)
        es = self.lib.vklGetObserverElementSize(self.h)
        if n == 0:
            return np.zeros((0, es // 4), np.float32)
        buf = (C.c_float * (n * es // 4)).from_address(p)
        out = np.array(buf, np.float32).reshape(n, es // 4)
        self.lib.vklUnmapObserver(self.h)
        return out


def structured_regular(device: Device, data, grid_origin=None, grid_spacing=None, cell_centered=False,
                       index_to_object=None, index_origin=None, background=None, filter=None,
                       shared=False, dims=None, num_timesteps=None, time_indices=None, times=None):
    """A committed structuredRegular volume; `data` is one array or a list
    (one per attribute), each shaped (Z, Y, X) with x fastest.  Temporally
    varying data: `dims` = (X, Y, Z) and flat data arrays with each voxel's
    time samples consecutive, plus `num_timesteps` (structured) or
    `time_indices` (uint32 / uint64, one per voxel + 1) and `times`
    (unstructured)."""
    arrays = data if isinstance(data, (list, tuple)) else [data]
    shape = tuple(arrays[0].shape) if dims is None else tuple(dims)[::-1]
    v = Volume(device, "structuredRegular")
    v.set_vec3i("dimensions", shape[::-1])
    if num_timesteps is not None:
        v.set_int("temporallyStructuredNumTimesteps", num_timesteps)
    if time_indices is not None:
        idx = np.ascontiguousarray(time_indices)
        v.set_data("temporallyUnstructuredIndices",
                   Data(device, idx, vkl_type=VKL_ULONG if idx.dtype == np.uint64 else VKL_UINT))
    if times is not None:
        v.set_data("temporallyUnstructuredTimes", Data(device, np.ascontiguousarray(times, np.float32)))
    if grid_origin is not None:
        v.set_vec3f("gridOrigin", grid_origin)
    if grid_spacing is not None:
        v.set_vec3f("gridSpacing", grid_spacing)
    if index_to_object is not None:
        v.set_param("indexToObject", VKL_AFFINE3F, np.asarray(index_to_object, np.float32))
    if index_origin is not None:
        v.set_vec3i("indexOrigin", index_origin)
    if cell_centered:
        v.set_bool("cellCentered", True)
    if background is not None:
        v.set_data("background", Data(device, np.asarray(background, np.float32).reshape(-1)))
    if filter is not None:
        v.set_int("filter", filter)
    datas = [Data(device, a, shared=shared) for a in arrays]
    if len(datas) == 1:
        v.set_data("data", datas[0])
    else:
        v.set_data("data", Data(device, objects=datas))
    v.commit()
    return v


def dense_value_range_no_alloc(device: Device, voxels, out, background=float("nan"),
                               vkl_type: Optional[int] = None):
    """vklCudaDenseValueRangeNoAlloc: the value range a structuredRegular
    volume over `voxels` (a contiguous CUDA tensor shaped (Z, Y, X), x
    fastest) would report, written as [lower, upper] into `out` (a CUDA
    float32 tensor of 2 elements) on the device's stream, with no device
    allocation.  Raises VKLError on a rejected call."""
    import torch
    tmap = {torch.float32: VKL_FLOAT, torch.float16: VKL_HALF, torch.uint8: VKL_UCHAR,
            torch.int16: VKL_SHORT, torch.float64: VKL_DOUBLE}
    assert voxels.is_contiguous() and voxels.dim() == 3
    assert out.dtype == torch.float32 and out.is_contiguous() and out.numel() >= 2
    t = vkl_type or tmap[voxels.dtype]
    Z, Y, X = voxels.shape
    device.pending = None
    code = device.lib.vklCudaDenseValueRangeNoAlloc(device.handle, C.c_void_p(voxels.data_ptr()), t,
                                                    X, Y, Z, float(background),
                                                    C.c_void_p(out.data_ptr()))
    if code != 0:
        device.pending = None
        raise VKLError(code, device.last_error()[1])


class SampleBatch:
    """vklCudaNewSampleBatch: a fixed list of (sampler, points, outputs) jobs
    run as one CUDA graph.  jobs: iterable of (sampler, points, samples,
    gradients[, attr]) with CUDA tensors (samples / gradients may be None)."""

    def __init__(self, device: Device, jobs, autotune=False):
        self.device = device
        self.lib = device.lib
        arr = (VKLCudaSampleJob * len(jobs))()
        self._keep = []
        for i, job in enumerate(jobs):
            smp, pts, smps, grads = job[:4]
            attr = job[4] if len(job) > 4 else 0
            arr[i].sampler = smp.h
            arr[i].points = pts.data_ptr()
            arr[i].numPoints = pts.shape[0]
            arr[i].attributeIndex = attr
            arr[i].samples = None if smps is None else smps.data_ptr()
            arr[i].gradients = None if grads is None else grads.data_ptr()
            self._keep.append((smp, pts, smps, grads))
        device.pending = None
        self.h = self.lib.vklCudaNewSampleBatch(device.handle, len(jobs), arr, int(bool(autotune)))
        if not self.h:
            device.raise_pending()
            raise VKLError(*device.last_error())

    def run(self):
        code = self.lib.vklCudaRunSampleBatch(self.h)
        if code != 0:
            self.device.pending = None
            raise VKLError(code, self.device.last_error()[1])

    def config(self):
        t, s, c, f = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self.lib.vklCudaGetSampleBatchConfig(self.h, C.byref(t), C.byref(s), C.byref(c), C.byref(f))
        return {"tile_points": t.value, "sorted": bool(s.value), "ctas_per_sm": c.value,
                "fused_jobs": f.value}

    def release(self):
        if self.h:
            self.lib.vklCudaReleaseSampleBatch(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class Surrogate:
    """vklCudaNewSurrogate: hash-grid + MLP surrogate of a sampler's volume
    (cuda device extension).  Arrays are CUDA tensors unless noted."""

    LEVELS, WEIGHTS = 16, 10304

    def __init__(self, sampler: "Sampler", log2_table=19, base_resolution=16.0, growth=1.5):
        self.sampler = sampler
        self.device = sampler.device
        self.lib = sampler.lib
        self.device.pending = None
        self.h = self.lib.vklCudaNewSurrogate(sampler.h, log2_table, base_resolution, growth)
        if not self.h:
            self.device.raise_pending()
            raise VKLError(*self.device.last_error())
        entries, nw, nr = C.c_uint64(), C.c_uint(), C.c_uint64()
        res = (C.c_uint * self.LEVELS)()
        self.lib.vklCudaGetSurrogateInfo(self.h, C.byref(entries), C.byref(nw), C.byref(nr), res)
        self.table_entries, self.num_weights, self.num_regions = entries.value, nw.value, nr.value
        self.resolutions = list(res)

    def _check(self, code):
        if code != 0:
            self.device.pending = None
            raise VKLError(code, self.device.last_error()[1])

    def set_parameters(self, table=None, weights=None):
        t = None if table is None else np.ascontiguousarray(table, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        self._check(self.lib.vklCudaSurrogateSetParameters(self.h, None if t is None else t.ctypes.data,
                                                           None if w is None else w.ctypes.data))

    def parameters(self):
        t = np.empty(self.table_entries * 2, np.float32)
        w = np.empty(self.num_weights, np.float32)
        self._check(self.lib.vklCudaSurrogateGetParameters(self.h, t.ctypes.data, w.ctypes.data))
        return t, w

    def gradient(self, points, targets):
        t = np.empty(self.table_entries * 2, np.float32)
        w = np.empty(self.num_weights, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(self.lib.vklCudaSurrogateGradient(self.h, points.shape[0], _ptr(points), _ptr(targets),
                                                      loss.ctypes.data, t.ctypes.data, w.ctypes.data))
        return float(loss[0]), t, w

    def train_step(self, points, targets, lr, loss=None):
        self._check(self.lib.vklCudaSurrogateTrainStep(self.h, points.shape[0], _ptr(points), _ptr(targets),
                                                       float(lr), _ptr(loss)))

    def calibrate(self, points, threshold):
        f = C.c_uint()
        self._check(self.lib.vklCudaSurrogateCalibrate(self.h, points.shape[0], _ptr(points), float(threshold),
                                                       C.byref(f)))
        return f.value

    def sample(self, points, out=None, fallback=True):
        if out is None:
            out = _alloc_like(points, (points.shape[0],))
        self._check(self.lib.vklCudaSurrogateSample(self.h, points.shape[0], _ptr(points), _ptr(out),
                                                    int(bool(fallback))))
        return out

    def release(self):
        if self.h:
            self.lib.vklCudaReleaseSurrogate(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def vdb_volume(device: Device, levels, origins, formats, packed_dense=None, packed_tile=None,
               node_data=None, index_to_object=None, index_clipping_bounds=None, background=None,
               compression=None, leaf_map=None, shared=False):
    """A committed vdb volume from packed leaves (nodesPackedDense / Tile, one
    array or a list per attribute) or per-leaf node.data arrays.
    `compression` ("fp16" | "bf16" | "fp8") stores float leaves as codes with
    a per-leaf scale and offset (cuda device extension); "fp16_blocks" |
    "bf16_blocks" | "fp8_blocks" store each leaf as 8 stencil blocks of 5^3
    codes (the leaf's voxels plus the next voxel on the +x/+y/+z side, one
    scale and offset over that 9^3 window), so a trilinear stencil based in
    the leaf reads one block.  `shared`: the
    packed leaf arrays are VKL_DATA_SHARED_BUFFER (used in place)."""
    v = Volume(device, "vdb")
    v.set_data("node.level", Data(device, np.ascontiguousarray(levels, np.uint32)))
    v.set_data("node.origin", Data(device, np.ascontiguousarray(origins, np.int32).reshape(-1),
                                   vkl_type=VKL_VEC3I))
    v.set_data("node.format", Data(device, np.ascontiguousarray(formats, np.uint32)))
    if packed_dense is not None:
        pd = packed_dense if isinstance(packed_dense, (list, tuple)) else [packed_dense]
        v.set_data("nodesPackedDense", Data(device, objects=[Data(device, a, shared=shared) for a in pd]))
        if packed_tile is not None:
            pt = packed_tile if isinstance(packed_tile, (list, tuple)) else [packed_tile]
            v.set_data("nodesPackedTile", Data(device, objects=[Data(device, a) for a in pt]))
    if node_data is not None:
        v.set_data("node.data", Data(device, objects=[Data(device, a) for a in node_data]))
    if index_to_object is not None:
        v.set_param("indexToObject", VKL_AFFINE3F, np.asarray(index_to_object, np.float32))
    if index_clipping_bounds is not None:
        v.set_param("indexClippingBounds", VKL_BOX3I, np.asarray(index_clipping_bounds, np.int32))
    if background is not None:
        v.set_data("background", Data(device, np.asarray(background, np.float32).reshape(-1)))
    if compression is not None:
        v.set_string("compression", compression)
    if leaf_map is not None:
        v.set_bool("leafMap", leaf_map)
    v.commit()
    return v


class Sampler(_Obj):
    def __init__(self, volume: Volume, filter=None, gradient_filter=None, max_sampling_depth=None):
        super().__init__(volume.device, volume.lib.vklNewSampler(volume.h))
        self._check_handle("vklNewSampler")
        self.volume = volume
        if filter is not None:
            self.set_int("filter", filter)
        if gradient_filter is not None:
            self.set_int("gradientFilter", gradient_filter)
        if max_sampling_depth is not None:
            self.set_int("maxSamplingDepth", max_sampling_depth)
        if filter is not None or gradient_filter is not None or max_sampling_depth is not None:
            self.commit()

    def feature_flags(self):
        return self.lib.vklGetFeatureFlags(self.h)

    def leaf_access_observer(self):
        """vklNewSamplerObserver(sampler, "LeafNodeAccess"); read with .read_uint()."""
        self.device.pending = None
        h = self.lib.vklNewSamplerObserver(self.h, b"LeafNodeAccess")
        self.device.raise_pending()
        return VKLObserverObj(self.device, h, "vklNewSamplerObserver")

    def sample(self, points, attr=0, out=None, times=None):
        """vklComputeSampleN; `times`: one time per point (temporally varying
        volumes), host or device array, or None."""
        n = points.shape[0]
        if out is None:
            out = _alloc_like(points, (n,))
        self._call(self.lib.vklComputeSampleN, C.byref(self.h), n, _ptr(points), _ptr(out), attr, _times(times))
        return out

    def sample_m(self, points, attrs, out=None, times=None):
        n = points.shape[0]
        a = np.ascontiguousarray(attrs, np.uint32)
        if out is None:
            out = _alloc_like(points, (n, len(a)))
        self._call(self.lib.vklComputeSampleMN, C.byref(self.h), n, _ptr(points), _ptr(out), len(a),
                   a.ctypes.data, _times(times))
        return out

    def gradient(self, points, attr=0, out=None, times=None):
        n = points.shape[0]
        if out is None:
            out = _alloc_like(points, (n, 3))
        self._call(self.lib.vklComputeGradientN, C.byref(self.h), n, _ptr(points), _ptr(out), attr,
                   _times(times))
        return out

    def sample_one(self, p, attr=0, time=0.0):
        v = vec3f(*[float(x) for x in p])
        return self._call(self.lib.vklComputeSample, C.byref(self.h), C.byref(v), attr, float(time))

    def gradient_one(self, p, attr=0, time=0.0):
        v = vec3f(*[float(x) for x in p])
        g = self._call(self.lib.vklComputeGradient, C.byref(self.h), C.byref(v), attr, float(time))
        return np.array([g.x, g.y, g.z], np.float32)

    def sample_w(self, points, valid=None, attr=0):
        """vklComputeSample4/8/16 on up to 16 points (SoA)."""
        w = {4: (vvec3f4, self.lib.vklComputeSample4), 8: (vvec3f8, self.lib.vklComputeSample8),
             16: (vvec3f16, self.lib.vklComputeSample16)}
        W = len(points)
        T, fn = w[W]
        soa = T()
        for i, p in enumerate(points):
            soa.x[i], soa.y[i], soa.z[i] = (float(p[0]), float(p[1]), float(p[2]))
        vmask = np.ones(W, np.int32) if valid is None else np.asarray(valid, np.int32)
        out = np.full(W, np.nan, np.float32)
        self._call(fn, vmask.ctypes.data, C.byref(self.h), C.byref(soa), out.ctypes.data, attr, None)
        return out

    @staticmethod
    def _soa(points):
        T = {4: vvec3f4, 8: vvec3f8, 16: vvec3f16}[len(points)]
        soa = T()
        for i, p in enumerate(points):
            soa.x[i], soa.y[i], soa.z[i] = (float(p[0]), float(p[1]), float(p[2]))
        return soa

    def sample_m_w(self, points, attrs, valid=None):
        """vklComputeSampleM4/8/16: (M, W) samples, row m = attribute attrs[m]."""
        W = len(points)
        fn = {4: self.lib.vklComputeSampleM4, 8: self.lib.vklComputeSampleM8, 16: self.lib.vklComputeSampleM16}[W]
        a = np.ascontiguousarray(attrs, np.uint32)
        vmask = np.ones(W, np.int32) if valid is None else np.asarray(valid, np.int32)
        out = np.full((len(a), W), np.nan, np.float32)
        self._call(fn, vmask.ctypes.data, C.byref(self.h), C.byref(self._soa(points)), out.ctypes.data, len(a),
                   a.ctypes.data, None)
        return out

    def gradient_w(self, points, valid=None, attr=0):
        """vklComputeGradient4/8/16: (W, 3) gradients (invalid lanes NaN)."""
        W = len(points)
        fn = {4: self.lib.vklComputeGradient4, 8: self.lib.vklComputeGradient8,
              16: self.lib.vklComputeGradient16}[W]
        vmask = np.ones(W, np.int32) if valid is None else np.asarray(valid, np.int32)
        g = self._soa(np.full((W, 3), np.nan))
        self._call(fn, vmask.ctypes.data, C.byref(self.h), C.byref(self._soa(points)), C.byref(g), attr, None)
        return np.stack([np.array(g.x[:], np.float32), np.array(g.y[:], np.float32),
                         np.array(g.z[:], np.float32)], 1)


class IntervalIteratorContext(_Obj):
    """vklNewIntervalIteratorContext.  `macrocells`: intervals of 16^3-voxel
    macrocells, the iterator of the reference's legacy structuredRegular
    volume (cuda device extension; vklIterateIntervalsN only)."""

    def __init__(self, sampler: Sampler, value_ranges=None, hint=None, attr=None, macrocells=False):
        super().__init__(sampler.device, sampler.lib.vklNewIntervalIteratorContext(sampler.h))
        self._check_handle("vklNewIntervalIteratorContext")
        self.sampler = sampler
        if value_ranges is not None:
            self.set_data("valueRanges", Data(sampler.device, np.asarray(value_ranges, np.float32).reshape(-1),
                                              vkl_type=VKL_BOX1F))
        if hint is not None:
            self.set_float("intervalResolutionHint", hint)
        if attr is not None:
            self.set_int("attributeIndex", attr)
        if macrocells:
            self.set_bool("macrocells", True)
        self.commit()

    def iterate_n(self, origins, directions, t_ranges, max_per_ray=64):
        n = origins.shape[0]
        out = _alloc_like(origins, (n, max_per_ray, 5))
        cnt = _alloc_like(origins, (n,), np.uint32)
        self._call(self.lib.vklIterateIntervalsN, C.byref(self.h), n, _ptr(origins), _ptr(directions),
                   _ptr(t_ranges), max_per_ray, _ptr(out), _ptr(cnt))
        return out, cnt

    def iterate_one(self, origin, direction, t_range):
        """Drives vklInitIntervalIterator / vklIterateInterval on one ray."""
        size = self.lib.vklGetIntervalIteratorSize(C.byref(self.h))
        buf = (C.c_uint8 * size)()
        o, d = vec3f(*map(float, origin)), vec3f(*map(float, direction))
        tr = range1f(*map(float, t_range))
        it = self._call(self.lib.vklInitIntervalIterator, C.byref(self.h), C.byref(o), C.byref(d),
                        C.byref(tr), 0.0, C.cast(buf, C.c_void_p))
        res = []
        iv = VKLInterval()
        while self._call(self.lib.vklIterateInterval, it, C.byref(iv)):
            res.append([iv.tRange.lower, iv.tRange.upper, iv.valueRange.lower, iv.valueRange.upper,
                        iv.nominalDeltaT])
        return np.array(res, np.float32).reshape(-1, 5)


class HitIteratorContext(_Obj):
    def __init__(self, sampler: Sampler, values, attr=None):
        super().__init__(sampler.device, sampler.lib.vklNewHitIteratorContext(sampler.h))
        self._check_handle("vklNewHitIteratorContext")
        self.sampler = sampler
        self.set_data("values", Data(sampler.device, np.asarray(values, np.float32).reshape(-1)))
        if attr is not None:
            self.set_int("attributeIndex", attr)
        self.commit()

    def iterate_n(self, origins, directions, t_ranges, max_per_ray=16):
        n = origins.shape[0]
        out = _alloc_like(origins, (n, max_per_ray, 3))
        cnt = _alloc_like(origins, (n,), np.uint32)
        self._call(self.lib.vklIterateHitsN, C.byref(self.h), n, _ptr(origins), _ptr(directions),
                   _ptr(t_ranges), max_per_ray, _ptr(out), _ptr(cnt))
        return out, cnt

    def iterate_one(self, origin, direction, t_range):
        size = self.lib.vklGetHitIteratorSize(C.byref(self.h))
        buf = (C.c_uint8 * size)()
        o, d = vec3f(*map(float, origin)), vec3f(*map(float, direction))
        tr = range1f(*map(float, t_range))
        it = self._call(self.lib.vklInitHitIterator, C.byref(self.h), C.byref(o), C.byref(d),
                        C.byref(tr), 0.0, C.cast(buf, C.c_void_p))
        res = []
        h = VKLHit()
        while self._call(self.lib.vklIterateHit, it, C.byref(h)):
            res.append([h.t, h.sample, h.epsilon])
        return np.array(res, np.float32).reshape(-1, 3)
