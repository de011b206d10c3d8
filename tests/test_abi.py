"""C-ABI checks that need no GPU: the cuda device library builds, loads and
exports every entry point include/openvkl_cuda.h declares; without a GPU the
device constructor reports failure instead of falling back to the CPU."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "openvkl_cuda.h")).read()
    return sorted(set(re.findall(r"OPENVKL_CUDA_INTERFACE[^;(]*?\b(vkl\w+)\s*\(", src, re.S)))


@pytest.fixture(scope="module")
def lib_path():
    from openvkl_b200 import build
    return build.build()


def test_header_declares_reference_api():
    syms = declared_symbols()
    for name in ["vklInit", "vklNewDevice", "vklNewData", "vklNewVolume", "vklCommit",
                 "vklNewSampler", "vklComputeSample", "vklComputeSampleN", "vklComputeSampleM",
                 "vklComputeSampleMN", "vklComputeGradient", "vklComputeGradientN",
                 "vklInitIntervalIterator", "vklIterateInterval", "vklInitHitIterator",
                 "vklIterateHit", "vklNewIntervalIteratorContext", "vklNewHitIteratorContext"]:
        assert name in syms, name


def test_library_exports_every_declared_symbol(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True,
                         check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing


def test_library_loads_and_binding_covers_exports(lib_path):
    from openvkl_b200 import vkl
    L = vkl.load_library(lib_path)
    for s in declared_symbols():
        assert hasattr(L, s)
    assert sorted(vkl.EXPORTS) == declared_symbols()


def test_build_targets_sm100a_only():
    from openvkl_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "--fmad=false" in build.FLAGS


def test_no_device_without_gpu(lib_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from openvkl_b200 import vkl
    L = vkl.load_library(lib_path)
    assert not L.vklNewDevice(b"cuda")
    assert not L.vklNewDevice(b"cpu")


def test_renderer_library_exports_and_device_header_compiles(lib_path):
    """The example renderer library (a consumer of include/openvkl_cuda_device.h)
    builds for sm_100a and exports its two entry points."""
    from openvkl_b200 import build
    assert os.path.exists(build.RENDERERS_LIB)
    out = subprocess.run(["nm", "-D", "--defined-only", build.RENDERERS_LIB], capture_output=True, text=True,
                         check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    assert {"vklExampleRender", "vklExampleSamplePoints"} <= exported


def test_oracle_renderer_draws_the_volume():
    """The oracle's restated ray march renderer shades pixels that see the
    volume and leaves the others black (no GPU needed)."""
    import numpy as np
    from oracle import pyoracle as O
    from openvkl_b200 import render
    from openvkl_b200.fields import sinusoid_field
    vox = sinusoid_field((24, 20, 28), seed=3)
    ref = O.OracleVolume.dense_volume(vox)
    b = ref.info()["bounds"]
    lo, hi = float(vox.min()), float(vox.max())
    cam = render.orbit_camera(b, 40, 30, distance=3.0)
    img = ref.render(0, cam.as_array(), render.DEFAULT_TF, (lo, hi), 40, 30, b, value_ranges=[[lo, hi]])
    assert np.isfinite(img).all()
    lit = img[:, :, :3].sum(-1) > 0
    assert lit[15, 20] and not lit[0, 0]
