"""The reference's own tutorial application (examples/vklTutorialCPU.c),
compiled unchanged against this library by tests/ref_app/Makefile (its
<openvkl/openvkl.h> includes resolve to the shim headers there, which map the
"cpu" device it asks for to the cuda device), run on the GPU.  It goes
through the 1-wide, 4-wide and stream sampling / gradient / multi-attribute
calls and a per-ray interval and hit iterator; every number it prints must
equal the oracle's answer to the same call, printed the same way (%f)."""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "ref_app", "_build", "vklTutorialCPU")


def _expected(O):
    """The numbers the tutorial prints, in order, from the oracle: the
    volume is three 128^3 ramps (attribute a = voxel coordinate a)."""
    n = 128
    r = np.arange(n, dtype=np.float32)
    ramps = [np.ascontiguousarray(np.broadcast_to(r[None, None, :], (n, n, n))),
             np.ascontiguousarray(np.broadcast_to(r[None, :, None], (n, n, n))),
             np.ascontiguousarray(np.broadcast_to(r[:, None, None], (n, n, n)))]
    ref = O.OracleVolume.dense_volume(ramps, grid_origin=(0, 0, 0), grid_spacing=(1, 1, 1))
    out = []
    out += list(ref.info()["bounds"])
    for a in range(3):
        out += list(ref.value_range(a))
    c = np.array([[1, 2, 3]], np.float32)
    out += list(c[0])
    out += [ref.sample(c, attr=0)[0], *ref.gradient(c, attr=0)[0]]
    out += [ref.sample(c, attr=a)[0] for a in range(3)]
    o, d, t = [0, 1, 1], [1, 0, 0], [0, 200]
    ranges, values = [[10, 20], [50, 75]], [32, 96]
    out += o + d + t + ranges[0] + ranges[1]
    iv, ic = ref.intervals([o], [d], [t], value_ranges=ranges, attr=0)
    for k in range(int(ic[0])):
        out += list(iv[0, k])
    out += values
    h, hc = ref.hits([o], [d], [t], values, attr=0)
    for k in range(int(hc[0])):
        out += list(h[0, k])
    for m in (4, 5):  # the 4-wide demo, then the stream demo
        p = np.array([[3 * i, 3 * i + 1, 3 * i + 2] for i in range(m)], np.float32)
        out += list(p.reshape(-1))
        s, g = ref.sample(p, attr=0), ref.gradient(p, attr=0)
        for i in range(m):
            out += [s[i], *g[i]]
        sm = np.stack([ref.sample(p, attr=a) for a in range(3)])
        out += list(sm.reshape(-1)) if m == 4 else list(sm.T.reshape(-1))
    return ["%f" % float(np.float32(v)) for v in out]


def test_reference_tutorial_on_cuda_device(oracle):
    if not os.path.exists(BIN):
        pytest.skip("the tutorial is built where the reference sources are present (build())")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert r.stdout.rstrip().endswith("complete.")
    got = re.findall(r"-?\d+\.\d{6}", r.stdout)
    want = _expected(oracle)
    assert got == want
