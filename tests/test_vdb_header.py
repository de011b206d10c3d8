"""include/openvkl/vdb.h, the cuda device's <openvkl/vdb.h>: a C and a C++
program that include it compile, and its topology helpers give the
reference's values for the 4-level 6/5/4/3 configuration
(vdb_topology.h.in: per-level log resolution, total log resolution = the sum
over the level and the levels below, resolution = 1 << total, voxels per
node = 1 << 3 * log resolution; vklVdbLevelRes(NUM_LEVELS) = 1) and its
index maps (domain offset -> voxel of a node: (offset & (res - 1)) >>
total log res of the next level; 3D -> linear with z fastest)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <openvkl/vdb.h>
#include <stdio.h>
int main(void)
{
  unsigned l;
  printf("%u\n", vklVdbNumLevels());
  for (l = 0; l <= 4; ++l)
    printf("%u %u %u %u %u %u\n", vklVdbLevelLogRes(l), vklVdbLevelTotalLogRes(l), vklVdbLevelStorageRes(l),
           vklVdbLevelRes(l), vklVdbLevelNumVoxels(l), vklVdbLevelResShift(l));
  for (l = 0; l < 4; ++l) {
    unsigned long long x;
    for (x = 0; x < 300000; x += 4099)
      printf("%llu %llu\n", (unsigned long long)vklVdbDomainOffsetToVoxel(l, (unsigned)x),
             (unsigned long long)vklVdbDomainOffsetToLinear(l, x, x * 7 + 3, x * 13 + 5));
  }
  printf("%d %d %d\n", (int)VKL_TEMPORAL_FORMAT_CONSTANT, (int)VKL_FORMAT_DENSE_ZYX, VKL_VDB_LEAF_LEVEL);
  return 0;
}
"""


def _expected():
    log = [6, 5, 4, 3]
    total = [sum(log[l:]) for l in range(4)] + [0]
    lines = ["4"]
    for l in range(5):
        lr = log[l] if l < 4 else 0
        sres = (1 << lr) if l < 4 else 0
        res = (1 << total[l]) if l < 4 else 1
        nv = (1 << 3 * lr) if l < 4 else 0
        lines.append(f"{lr} {total[l]} {sres} {res} {nv} {lr}")
    for l in range(4):
        res, nxt = 1 << total[l], total[l + 1]
        vox = lambda o: ((o & 0xFFFFFFFF) & (res - 1)) >> nxt
        for x in range(0, 300000, 4099):
            lin = (vox(x) << (2 * log[l])) + (vox(x * 7 + 3) << log[l]) + vox(x * 13 + 5)
            lines.append(f"{vox(x)} {lin}")
    lines.append("0 1 3")
    return lines


@pytest.mark.parametrize("lang", ["c", "c++"])
def test_vdb_header_compiles_and_matches_topology(tmp_path, lang):
    src = tmp_path / "t.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "t"
    cc = ["gcc", "-std=c99"] if lang == "c" else ["g++", "-std=c++11", "-x", "c++"]
    r = subprocess.run(cc + ["-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    assert out[:-1] == _expected()
