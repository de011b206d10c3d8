"""Generates tricubic_map.cuh: the Lekien-Marsden 64x64 constraint ->
coefficient map as straight-line float code.

The map is the tensor product of the 1D cubic Hermite map
    a0 = f0, a1 = d0, a2 = -3 f0 + 3 f1 - 2 d0 - d1, a3 = 2 f0 - 2 f1 + d0 + d1
over x, y, z.  Constraint layout: blocks of 8 corners (corner index 4x+2y+z)
for f, d/dx, d/dy, d/dz, d2/dxdy, d2/dxdz, d2/dydz, d3/dxdydz; coefficient
index 16i+4j+k for x^i y^j z^k.  Each coefficient is written as a
left-to-right sum over its non-zero columns in ascending order, the same
shape as the reference's expanded expressions
(openvkl/devices/cpu/volume/vdb/VdbSampler_tricubic.ih:34-389).

Run:  python openvkl_b200/csrc/gen_tricubic_map.py
"""
import os

H = [[1, 0, 0, 0], [0, 0, 1, 0], [-3, 3, -2, -1], [2, -2, 1, 1]]
BLOCK = {(0, 0, 0): 0, (1, 0, 0): 8, (0, 1, 0): 16, (0, 0, 1): 24,
         (1, 1, 0): 32, (1, 0, 1): 40, (0, 1, 1): 48, (1, 1, 1): 56}


def tricubic_rows():
    rows = []
    for i in range(4):
        for j in range(4):
            for k in range(4):
                w = [0] * 64
                for ux in range(4):
                    for uy in range(4):
                        for uz in range(4):
                            c = H[i][ux] * H[j][uy] * H[k][uz]
                            if not c:
                                continue
                            col = BLOCK[(ux >> 1, uy >> 1, uz >> 1)] + 4 * (ux & 1) + 2 * (uy & 1) + (uz & 1)
                            w[col] += c
                rows.append([(col, w[col]) for col in range(64) if w[col]])
    return rows


def main():
    lines = [
        "// GENERATED by gen_tricubic_map.py -- do not edit.",
        "// Lekien-Marsden tricubic constraint->coefficient map (see generator).",
        "#pragma once",
        "#define VKL_TRICUBIC_MAP(CTR, COEF) \\",
    ]
    for r, row in enumerate(tricubic_rows()):
        terms = " + ".join(f"({w:.1f}f) * CTR[{c}]" for c, w in row)
        lines.append(f"  COEF[{r}] = {terms}; \\")
    lines.append("")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tricubic_map.cuh")
    with open(out, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
