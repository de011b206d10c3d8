"""The density path tracer's own log and sincos (openvkl_b200/renderers/
pt_math.h: Cody-Waite reduction with series / Taylor polynomials), compiled
as C on the host the way the oracle compiles them, against double-precision
libm: log within 2 ulp over the positive floats and its special cases;
sin / cos within 2 ulp of the result or 1e-7 absolute (near their zeros) on
[0, 2 pi), the arguments the renderer passes.  The CUDA renderer runs the
same source, so its images can be compared with the oracle's bit for bit."""
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include "pt_math.h"
#include <stdio.h>
#include <stdlib.h>
int main(int argc, char **argv)
{
  FILE *f = fopen(argv[1], "rb");
  FILE *g = fopen(argv[2], "wb");
  float x;
  while (fread(&x, 4, 1, f) == 1) {
    float r[3];
    r[0] = pt_log(x);
    pt_sincos(x, &r[1], &r[2]);
    fwrite(r, 4, 3, g);
  }
  fclose(f);
  fclose(g);
  return 0;
}
"""


def _run(tmp_path, xs):
    src = tmp_path / "t.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "t"
    subprocess.run(["gcc", "-std=c99", "-O2", "-ffp-contract=off", "-I",
                    os.path.join(ROOT, "openvkl_b200", "renderers"), str(src), "-o", str(exe), "-lm"], check=True)
    xs = np.ascontiguousarray(xs, np.float32)
    (tmp_path / "in.bin").write_bytes(xs.tobytes())
    subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], check=True)
    return np.frombuffer((tmp_path / "out.bin").read_bytes(), np.float32).reshape(-1, 3)


def _ulp(got, want):
    w = want.astype(np.float32)
    return np.abs(got.astype(np.float64) - want) / np.spacing(np.abs(w)).astype(np.float64)


def test_log(tmp_path):
    rng = np.random.default_rng(1)
    xs = np.concatenate([np.exp(rng.uniform(-80, 80, 200000)), 1 - rng.random(200000),
                         np.float32([1e-45, 1e-40, 1.17549435e-38, 0.5, 1.0, 2.0, 0.70710677, 1.4142135, 3.4e38])])
    xs = xs.astype(np.float32)
    r = _run(tmp_path, xs)[:, 0]
    want = np.log(xs.astype(np.float64))
    ok = xs != 1
    assert _ulp(r[ok], want[ok]).max() <= 2.0
    assert r[xs == 1][0] == 0.0
    sp = _run(tmp_path, np.float32([0.0, -1.0, np.inf, np.nan]))[:, 0]
    assert sp[0] == -np.inf and np.isnan(sp[1]) and sp[2] == np.inf and np.isnan(sp[3])


def test_sincos(tmp_path):
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.uniform(0, 2 * np.pi, 400000), np.float32([0, np.pi / 2, np.pi, 1.5 * np.pi])])
    xs = xs.astype(np.float32)
    r = _run(tmp_path, xs)
    for col, fn in ((1, np.sin), (2, np.cos)):
        want = fn(xs.astype(np.float64))
        err = np.abs(r[:, col].astype(np.float64) - want)
        assert np.all((err <= 2 * np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)) | (err <= 1e-7))
