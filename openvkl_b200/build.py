"""Builds libopenvkl_device_cuda.so, the cuda device, with nvcc for sm_100a.

Every translation unit is compiled with --fmad=false: the device math spells
out each rounding the reference CPU device performs (no contraction of
a*b+c into an FMA that the source does not write), which is what makes the
results bit-identical to the oracle.  The shared library links the CUDA
runtime statically so it loads with nothing but the driver.

    python -m openvkl_b200.build            # incremental
    python -m openvkl_b200.build --force    # rebuild everything
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libopenvkl_device_cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-O2,-fvisibility=hidden",
         "-Xptxas", "-O3", "--expt-relaxed-constexpr"]

SOURCES = ["api.cpp", "objects.cpp", "k_sample.cu", "k_sample_nearest.cu", "k_sample_linear.cu",
           "k_sample_cubic.cu", "k_build.cu", "k_iterate.cu", "k_noalloc.cu", "k_batch.cu", "k_surrogate.cu",
           "k_bin.cu", "k_macrocell.cu", "k_temporal.cu", "k_sample_rays.cu"]


# The example renderers (a consumer of the __device__ API, built separately
# from the device library they call into).
RENDERERS = os.path.join(HERE, "renderers", "renderers.cu")
RENDERERS_LIB = os.path.join(HERE, "libopenvkl_renderers.so")


INCLUDE = os.path.join(HERE, "..", "include")


def _headers():
    """Headers the library's translation units include (the __device__ API
    header is only the renderers')."""
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + [
        os.path.join(INCLUDE, "openvkl_cuda.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, force, verbose):
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ, src + ".o")
    if not force and not _stale(obj, [path] + _headers()):
        return obj
    lang = ["-x", "cu"] if src.endswith(".cu") else []
    cmd = [NVCC] + ARCH + FLAGS + lang + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def _compile_renderers(force, verbose):
    obj = os.path.join(OBJ, "renderers.cu.o")
    if not force and not _stale(obj, [RENDERERS, os.path.join(INCLUDE, "openvkl_cuda_device.h")] + _headers()):
        return obj
    cmd = [NVCC] + ARCH + FLAGS + ["-x", "cu", "-c", RENDERERS, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for renderers.cu:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        # the renderer object (the slowest translation unit) compiles beside the library's
        rend = ex.submit(_compile_renderers, force, verbose)
        objs = list(ex.map(lambda s: _compile(s, force, verbose), SOURCES))
        robj = rend.result()
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if force or _stale(RENDERERS_LIB, [robj]):
        cmd = [NVCC] + ARCH + ["-shared", "-o", RENDERERS_LIB, robj, "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed for the renderers:\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
