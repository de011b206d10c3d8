"""Extracts the reference's tricubic coefficient table into a fixture.

Reads the expanded Lekien-Marsden expressions of
openvkl/devices/cpu/volume/vdb/VdbSampler_tricubic.ih (macro
__vkl_tricubic_coefficients) from a read-only Open VKL v2.0.2 checkout and
writes, for each of the 64 coefficients, the ordered list of
(weight, constraint index) terms to tricubic_coeff_map.json.  The fixture
pins the oracle's and the CUDA device's generated map to the reference.

Run where the reference tree exists, naming its root:
    python tests/golden/make_tricubic_golden.py <reference checkout>
"""
import json
import os
import re
import sys


def main(ref_root):
    src = open(os.path.join(ref_root, "openvkl/devices/cpu/volume/vdb/VdbSampler_tricubic.ih")).read()
    start = src.index("#define __vkl_tricubic_coefficients(CTR)")
    end = src.index("#define VKL_STENCIL_TRICUBIC_RES")
    body = src[start:end].split("\n", 1)[1]
    body = body.replace("\\\n", " ")
    body = body.strip().lstrip("{").rstrip().rstrip("}")
    rows = []
    for expr in body.split(","):
        terms = re.findall(r"\((-?[0-9.]+)\)\s*\*\s*CTR\[(\d+)\]", expr)
        rows.append([[float(w), int(c)] for w, c in terms])
    assert len(rows) == 64, len(rows)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tricubic_coeff_map.json")
    with open(out, "w") as f:
        json.dump({"source": "openvkl/devices/cpu/volume/vdb/VdbSampler_tricubic.ih:34-389",
                   "rows": rows}, f)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_tricubic_golden.py <reference checkout>")
    main(sys.argv[1])
