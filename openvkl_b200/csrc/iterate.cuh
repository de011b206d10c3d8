// Device-side interval and hit iteration of the cuda device.
//
// Restates, operation by operation in FP32:
//   DDA             openvkl/devices/cpu/volume/vdb/Dda.ih:17-309
//   hierarchical    HDDA.ih.in:24-101 (generated per level; unrolled here)
//   voxel queries   VdbQueryVoxelDense.ih:17-161, VdbQueryVoxel.ih.in:42-116
//   interval iter   VdbIterator.ispc:36-159
//   value ranges    common/ValueRanges.ih:22-52, math/box_utility.ih:9-77
//   hit iteration   iterator/DefaultIterator.ispc:168-258,
//                   iterator/Iterator.ih:17-197 (bisection)
#pragma once
#include "sampling.cuh"

namespace vklcuda {

constexpr float kPosInf = __builtin_huge_valf();

__device__ __forceinline__ float minx(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float maxx(float a, float b) { return a > b ? a : b; }

// rkcommon divide_safe: 1/x with |x| clamped to >= 1e-8 (sign kept).
__device__ __forceinline__ float divideSafe(float x)
{
  const float e = 1e-8f;
  return 1.f / (fabsf(x) < e ? (x >= 0.f ? e : -e) : x);
}

// Per-level DDA state, indexed [axis * 4 + level].  Every access below uses
// indices known at compile time (the level loops are unrolled, and a level
// known only at run time is dispatched through a switch to code with the
// level fixed), so the arrays stay in registers instead of local memory.
// A level's t step along an axis is res * |1/dir| and its index step
// sign(dir) * res; res is a power of two, so both are recomputed exactly from
// the per-axis 1/dir and dir instead of being stored per level.
struct Dda {
  uint32_t level;
  float t;
  f3 org, dir;
  float inv[3];  // dirRcp(dir), per axis
  int32_t idx[12];
  float tNext[12];
};

__device__ __forceinline__ int dirSign(float v) { return (int)(0.f < v) - (int)(v < 0.f); }
__device__ __forceinline__ float dirRcp(float v) { return v == 0.f ? kPosInf : divideSafe(v); }
__device__ __forceinline__ float planeT(float plane, float org, float inv)
{
  const float t = (plane - org) * inv;
  return (plane == org || isnan(t)) ? kPosInf : t;
}
__device__ __forceinline__ int32_t clampToCell(float f, int32_t res)
{
  return ifloor(maxx(f, 0.f)) & ~(res - 1);
}

__device__ inline void ddaInit(f3 org, f3 dir, float tMin, uint32_t level, Dda &d)
{
  const float oo[3] = {org.x + tMin * dir.x, org.y + tMin * dir.y, org.z + tMin * dir.z};
  const float g3[3] = {org.x, org.y, org.z};
  const float d3[3] = {dir.x, dir.y, dir.z};
  d.level = level < kNumLevels - 1 ? level : kNumLevels - 1;
  d.t     = tMin;
  d.org   = org;
  d.dir   = dir;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax)
    d.inv[ax] = dirRcp(d3[ax]);
#pragma unroll
  for (int l = 0; l < (int)kNumLevels; ++l) {
    if ((uint32_t)l <= d.level) {
      const int32_t res = (int32_t)levelRes((uint32_t)l + 1);
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const int sg      = dirSign(d3[ax]);
        const float iv    = d.inv[ax];
        const int32_t id  = clampToCell(oo[ax], res);
        const float plane = (float)(id + res * (int)(sg >= 0));
        const int k       = ax * 4 + l;
        d.idx[k]          = id;
        d.tNext[k]        = planeT(plane, g3[ax], iv);
      }
    }
  }
}

__device__ inline void ddaReinitBelow(Dda &d, uint32_t level, int32_t dx, int32_t dy, int32_t dz)
{
  const float d3[3] = {d.dir.x, d.dir.y, d.dir.z};
  const float g3[3] = {d.org.x, d.org.y, d.org.z};
  float oo[3] = {d.org.x + d.t * d.dir.x, d.org.y + d.t * d.dir.y, d.org.z + d.t * d.dir.z};
  if (dx != 0)
    oo[0] = oo[0] + (float)dirSign(d3[0]) * 1e-2f;
  else if (dy != 0)
    oo[1] = oo[1] + (float)dirSign(d3[1]) * 1e-2f;
  else
    oo[2] = oo[2] + (float)dirSign(d3[2]) * 1e-2f;
#pragma unroll
  for (int l = 1; l < (int)kNumLevels; ++l) {
    if ((uint32_t)l > level && (uint32_t)l <= d.level) {
      const int32_t res = (int32_t)levelRes((uint32_t)l + 1);
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const int k       = ax * 4 + l;
        const int sg      = dirSign(d3[ax]);
        d.idx[k]          = clampToCell(oo[ax], res);
        const float plane = (float)(d.idx[k] + res * (int)(sg >= 0));
        d.tNext[k]        = planeT(plane, g3[ax], d.inv[ax]);
      }
    }
  }
}

// One DDA step on level L: the axis whose next plane is nearest.
template <int L>
__device__ __forceinline__ void ddaStepL(Dda &d)
{
  constexpr int32_t res = (int32_t)levelRes((uint32_t)L + 1);
  const float tx = d.tNext[L], ty = d.tNext[4 + L], tz = d.tNext[8 + L];
  const float m  = minx(minx(tx, ty), tz);
  if (m == tx) {
    d.t         = tx;
    d.tNext[L]  = tx + (float)res * fabsf(d.inv[0]);
    d.idx[L]    = d.idx[L] + dirSign(d.dir.x) * res;
  } else if (m == ty) {
    d.t            = ty;
    d.tNext[4 + L] = ty + (float)res * fabsf(d.inv[1]);
    d.idx[4 + L]   = d.idx[4 + L] + dirSign(d.dir.y) * res;
  } else {
    d.t            = tz;
    d.tNext[8 + L] = tz + (float)res * fabsf(d.inv[2]);
    d.idx[8 + L]   = d.idx[8 + L] + dirSign(d.dir.z) * res;
  }
}

__device__ __forceinline__ void ddaStep(Dda &d, uint32_t l)
{
  switch (l) {
  case 0:
    ddaStepL<0>(d);
    break;
  case 1:
    ddaStepL<1>(d);
    break;
  case 2:
    ddaStepL<2>(d);
    break;
  default:
    ddaStepL<3>(d);
  }
}

// The cell (level-l voxel index per axis) the DDA is in on level l.
__device__ __forceinline__ void ddaCell(const Dda &d, uint32_t l, int32_t &x, int32_t &y, int32_t &z)
{
  switch (l) {
  case 0:
    x = d.idx[0], y = d.idx[4], z = d.idx[8];
    break;
  case 1:
    x = d.idx[1], y = d.idx[5], z = d.idx[9];
    break;
  case 2:
    x = d.idx[2], y = d.idx[6], z = d.idx[10];
    break;
  default:
    x = d.idx[3], y = d.idx[7], z = d.idx[11];
  }
}

// Runtime-level DDA: the same state and steps with the per-level arrays
// indexed by the level at run time (local memory), each step's t and index
// increments stored per level.  One copy of the step code serves every
// level, which suits the hit iterator, whose kernels are bound by
// instruction fetch and occupancy rather than by the DDA (on 2^24 random
// rays it runs 5.6 Mrays/s with this form, 4.0-4.6 with the register form);
// the interval iterator uses the register form above.  Both compute the same
// values.
struct DdaDyn {
  uint32_t level;
  float t;
  f3 org, dir;
  int32_t idx[12];
  float tNext[12];
  float tDelta[12];
  int32_t idxDelta[12];
};

__device__ inline void ddaInit(f3 org, f3 dir, float tMin, uint32_t level, DdaDyn &d)
{
  const float oo[3] = {org.x + tMin * dir.x, org.y + tMin * dir.y, org.z + tMin * dir.z};
  const float g3[3] = {org.x, org.y, org.z};
  const float d3[3] = {dir.x, dir.y, dir.z};
  d.level = level < kNumLevels - 1 ? level : kNumLevels - 1;
  d.t     = tMin;
  d.org   = org;
  d.dir   = dir;
  for (uint32_t l = 0; l <= d.level; ++l) {
    const int32_t res = (int32_t)levelRes(l + 1);
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const int sg      = dirSign(d3[ax]);
      const float iv    = dirRcp(d3[ax]);
      const int32_t id  = clampToCell(oo[ax], res);
      const float plane = (float)(id + res * (int)(sg >= 0));
      const int k       = ax * 4 + (int)l;
      d.idx[k]          = id;
      d.idxDelta[k]     = sg * res;
      d.tDelta[k]       = (float)res * fabsf(iv);
      d.tNext[k]        = planeT(plane, g3[ax], iv);
    }
  }
}

__device__ inline void ddaReinitBelow(DdaDyn &d, uint32_t level, int32_t dx, int32_t dy, int32_t dz)
{
  const float d3[3] = {d.dir.x, d.dir.y, d.dir.z};
  const float g3[3] = {d.org.x, d.org.y, d.org.z};
  float oo[3] = {d.org.x + d.t * d.dir.x, d.org.y + d.t * d.dir.y, d.org.z + d.t * d.dir.z};
  if (dx != 0)
    oo[0] = oo[0] + (float)dirSign(d3[0]) * 1e-2f;
  else if (dy != 0)
    oo[1] = oo[1] + (float)dirSign(d3[1]) * 1e-2f;
  else
    oo[2] = oo[2] + (float)dirSign(d3[2]) * 1e-2f;
  for (uint32_t l = level + 1; l <= d.level; ++l) {
    const int32_t res = (int32_t)levelRes(l + 1);
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const int k       = ax * 4 + (int)l;
      const int sg      = dirSign(d3[ax]);
      d.idx[k]          = clampToCell(oo[ax], res);
      const float plane = (float)(d.idx[k] + res * (int)(sg >= 0));
      d.tNext[k]        = planeT(plane, g3[ax], dirRcp(d3[ax]));
    }
  }
}

__device__ __forceinline__ void ddaStep(DdaDyn &d, uint32_t l)
{
  const float tx = d.tNext[l], ty = d.tNext[4 + l], tz = d.tNext[8 + l];
  const float m  = minx(minx(tx, ty), tz);
  const int k    = (m == tx) ? (int)l : (m == ty) ? 4 + (int)l : 8 + (int)l;
  d.t            = d.tNext[k];
  d.tNext[k]     = d.tNext[k] + d.tDelta[k];
  d.idx[k]       = d.idx[k] + d.idxDelta[k];
}

__device__ __forceinline__ void ddaCell(const DdaDyn &d, uint32_t l, int32_t &x, int32_t &y, int32_t &z)
{
  x = d.idx[l];
  y = d.idx[4 + l];
  z = d.idx[8 + l];
}

struct VoxelDesc {
  uint32_t level;
  bool isEmpty;
  float v0, v1;
};

__device__ __forceinline__ bool rangesOverlap(const DevValueRanges &vr, float lo, float hi)
{
  if (vr.numRanges == 0)
    return true;
  if (!(vr.minMax[1] >= lo && vr.minMax[0] <= hi))
    return false;
  for (uint32_t i = 0; i < vr.numRanges; ++i)
    if (__ldg(vr.ranges + 2 * i + 1) >= lo && __ldg(vr.ranges + 2 * i) <= hi)
      return true;
  return false;
}

// The value range of the dense tree's node voxel holding cell (x, y, z) at
// the query depth, or null outside the domain.  The reference computes the
// level-1/2 node numbers in closed form (VdbQueryVoxelDense.ih:41-113).  The
// dense tree numbers level-l nodes x-fastest over the node grid (k_build.cu
// kDenseLevel*), so the node of an in-domain cell is its node coordinates'
// linear index: the same voxel the child-pointer walk reaches, without its
// two dependent loads.
__device__ __forceinline__ const float *denseCellRange(const DevGrid &g, int32_t x, int32_t y, int32_t z,
                                                       uint32_t depth, uint32_t attr)
{
  const uint32_t ox = (uint32_t)x, oy = (uint32_t)y, oz = (uint32_t)z;
  if (!(ox < g.activeSize[0] && oy < g.activeSize[1] && oz < g.activeSize[2]))
    return nullptr;
  const uint32_t lvl = depth >= 2 ? 2u : depth;
  uint64_t ni = offsetToLinear(lvl, ox, oy, oz);
  if (lvl == 2) {
    const uint32_t n2x = (g.activeSize[0] + 127) >> 7, n2y = (g.activeSize[1] + 127) >> 7;
    ni += (((uint64_t)(oz >> 7) * n2y + (oy >> 7)) * n2x + (ox >> 7)) * levelNumVoxels(2);
  } else if (lvl == 1) {
    const uint32_t n1x = (g.activeSize[0] + 4095) >> 12, n1y = (g.activeSize[1] + 4095) >> 12;
    ni += (((uint64_t)(oz >> 12) * n1y + (oy >> 12)) * n1x + (ox >> 12)) * levelNumVoxels(1);
  }
  return g.levels[lvl].valueRange + 2 * (ni * g.numAttributes + attr);
}

__device__ inline void queryVoxelDense(const DevGrid &g, int32_t x, int32_t y, int32_t z,
                                       uint32_t depth, uint32_t attr, const DevValueRanges &vr,
                                       VoxelDesc &desc)
{
  desc.level    = depth;
  const float *r = denseCellRange(g, x, y, z, depth, attr);
  if (!r) {
    desc.isEmpty = true;
    return;
  }
  desc.v0      = __ldg(r);
  desc.v1      = __ldg(r + 1);
  desc.isEmpty = !rangesOverlap(vr, desc.v0, desc.v1);
}

__device__ inline void queryVoxelSparse(const DevGrid &g, int32_t x, int32_t y, int32_t z,
                                        uint32_t depth, uint32_t attr, const DevValueRanges &vr,
                                        VoxelDesc &desc)
{
  uint64_t node = 0;
  // int32 indices widen with sign extension before masking, as the
  // reference's uint64 parameters do.
  const uint64_t X = (uint64_t)(int64_t)x, Y = (uint64_t)(int64_t)y, Z = (uint64_t)(int64_t)z;
  for (uint32_t l = 0; l + 1 < kNumLevels; ++l) {
    const uint64_t vo   = offsetToLinear(l, X, Y, Z) + node * levelNumVoxels(l);
    const uint32_t vo32 = (uint32_t)vo;
    const uint64_t v    = __ldg(g.levels[l].voxels + vo32);
    const float *r      = g.levels[l].valueRange + 2 * ((uint64_t)vo32 * g.numAttributes + attr);
    desc.v0             = __ldg(r);
    desc.v1             = __ldg(r + 1);
    desc.level          = l;
    desc.isEmpty        = voxelIsEmpty(v) || !rangesOverlap(vr, desc.v0, desc.v1);
    if (desc.isEmpty)
      return;
    const bool atQueryDepth = (l + 1 > depth);
    const bool isLeafPtr    = voxelIsLeaf(v);
    if (isLeafPtr && !atQueryDepth)
      desc.level = l + 1;
    if (l + 2 >= kNumLevels || atQueryDepth || isLeafPtr)
      return;
    node = voxelChildIndex(v);
  }
}

// Hierarchical step: step on the lowest level the descriptor names, follow
// up the tree when a child cell leaves its parent cell.
template <int L>
__device__ inline void hddaStepL(Dda &d)
{
  if constexpr (L >= (int)kNumLevels - 1) {
    ddaStepL<(int)kNumLevels - 1>(d);
  } else {
    const int32_t x0 = d.idx[L], y0 = d.idx[4 + L], z0 = d.idx[8 + L];
    ddaStepL<L>(d);
    if ((uint32_t)L < d.level)
      ddaReinitBelow(d, (uint32_t)L, d.idx[L] - x0, d.idx[4 + L] - y0, d.idx[8 + L] - z0);
  }
  // propagate upwards: level l steps when its child (l+1) left its cell
  bool stepped = true;
#pragma unroll
  for (int l = L - 1; l >= 0; --l) {
    if (stepped) {
      const int32_t res = (int32_t)levelRes((uint32_t)l + 1);
      const bool left   = d.idx[l + 1] < d.idx[l] || d.idx[4 + l + 1] < d.idx[4 + l] ||
                        d.idx[8 + l + 1] < d.idx[8 + l] || d.idx[l + 1] >= d.idx[l] + res ||
                        d.idx[4 + l + 1] >= d.idx[4 + l] + res || d.idx[8 + l + 1] >= d.idx[8 + l] + res;
      if (left)
        ddaStep(d, (uint32_t)l);
      stepped = left;
    }
  }
}

__device__ inline void hddaStep(const VoxelDesc &desc, Dda &d)
{
  switch (desc.level) {
  case 0:
    hddaStepL<0>(d);
    break;
  case 1:
    hddaStepL<1>(d);
    break;
  case 2:
    hddaStepL<2>(d);
    break;
  default:
    hddaStepL<3>(d);
  }
}

__device__ inline void hddaStep(const VoxelDesc &desc, DdaDyn &d)
{
  const uint32_t L = desc.level;
  if (L >= kNumLevels - 1) {
    ddaStep(d, kNumLevels - 1);
  } else {
    const int32_t x0 = d.idx[L], y0 = d.idx[4 + L], z0 = d.idx[8 + L];
    ddaStep(d, L);
    if (L < d.level)
      ddaReinitBelow(d, L, d.idx[L] - x0, d.idx[4 + L] - y0, d.idx[8 + L] - z0);
  }
  bool stepped = true;
  for (int l = (int)L - 1; l >= 0 && stepped; --l) {
    const int32_t res = (int32_t)levelRes((uint32_t)l + 1);
    const bool left   = d.idx[l + 1] < d.idx[l] || d.idx[4 + l + 1] < d.idx[4 + l] ||
                      d.idx[8 + l + 1] < d.idx[8 + l] || d.idx[l + 1] >= d.idx[l] + res ||
                      d.idx[4 + l + 1] >= d.idx[4 + l] + res || d.idx[8 + l + 1] >= d.idx[8 + l] + res;
    if (left)
      ddaStep(d, (uint32_t)l);
    stepped = left;
  }
}

// Loop bounds.  The reference's loops end only when float t passes tMax;
// on a GPU a ray whose t stops advancing (t + tDelta == t at huge t, or a
// march step below t's ulp) must not spin forever, so every ray carries a
// step budget; a ray that exhausts it ends its iteration as if it had left
// the volume.  The oracle applies the same bounds, so results still match.
constexpr uint32_t kMaxDdaSteps   = 1u << 26;  // hierarchical DDA steps per ray
constexpr uint32_t kMaxMarchSteps = 1u << 24;  // bisection march steps per interval
constexpr uint32_t kMaxHitsPerRay = 1u << 24;

// D: the DDA state type, Dda (register form) or DdaDyn (runtime-level form).
template <class D>
struct IntervalItT {
  float tMax;
  float nominalDeltaT;
  uint32_t budget;
  D dda;
  // The last sparse query that ended on a leaf pointer of level 2 at full
  // depth: every elementary cell of that leaf gets the same descriptor (the
  // walk reads the same three node voxels), so the next cells reuse it.
  int32_t leafKey[3];
  bool leafKeyValid;
  VoxelDesc leafDesc;
};
using IntervalIt    = IntervalItT<Dda>;
using IntervalItDyn = IntervalItT<DdaDyn>;

// intersectBox (math/box_utility.ih:63-77)
__device__ __forceinline__ void intersectBox(f3 o, f3 d, const float *box, float lo, float hi,
                                             float &rlo, float &rhi)
{
  const float org[3] = {o.x, o.y, o.z};
  const float inv[3] = {divideSafe(d.x), divideSafe(d.y), divideSafe(d.z)};
  float mn[3], mx[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float t0 = (box[a] - org[a]) * inv[a];
    const float t1 = (box[3 + a] - org[a]) * inv[a];
    mn[a]          = minx(t0, t1);
    mx[a]          = maxx(t0, t1);
  }
  rlo = maxx(maxx(maxx(mn[0], mn[1]), mn[2]), lo);
  rhi = minx(minx(minx(mx[0], mx[1]), mx[2]), hi);
}

template <class D>
__device__ inline void intervalInit(const DevGrid &g, uint32_t depth, f3 origin, f3 direction,
                                    float tLo, float tHi, IntervalItT<D> &it)
{
  f3 org       = xfmPoint(g.objectToIndex, origin);
  org          = {org.x - (float)g.rootOrigin[0], org.y - (float)g.rootOrigin[1],
         org.z - (float)g.rootOrigin[2]};
  const f3 dir = xfmVector(g.objectToIndex, direction);
  it.nominalDeltaT = minx(minx(1.f * divideSafe(fabsf(dir.x)), 1.f * divideSafe(fabsf(dir.y))),
                          1.f * divideSafe(fabsf(dir.z)));
  float lo, hi;
  intersectBox(org, dir, g.domain, tLo, tHi, lo, hi);
  it.budget       = kMaxDdaSteps;
  it.leafKeyValid = false;
  if (hi <= lo) {
    it.tMax  = -kPosInf;
    it.dda.t = 0.f;
  } else {
    it.tMax = hi;
    ddaInit(org, dir, lo, depth, it.dda);
  }
}

template <class D>
__device__ __forceinline__ void querySparseCached(const DevGrid &g, int32_t x, int32_t y, int32_t z,
                                                  uint32_t depth, uint32_t attr, const DevValueRanges &vr,
                                                  IntervalItT<D> &it, VoxelDesc &desc)
{
  const bool full = depth >= kNumLevels - 1;
  if (full && it.leafKeyValid && (x >> 3) == it.leafKey[0] && (y >> 3) == it.leafKey[1] &&
      (z >> 3) == it.leafKey[2]) {
    desc = it.leafDesc;
    return;
  }
  queryVoxelSparse(g, x, y, z, depth, attr, vr, desc);
  if (full && desc.level == kNumLevels - 1) {
    it.leafKeyValid = true;
    it.leafKey[0]   = x >> 3;
    it.leafKey[1]   = y >> 3;
    it.leafKey[2]   = z >> 3;
    it.leafDesc     = desc;
  }
}

// The reference's loop (DefaultIterator.ispc:100-166): skip empty cells,
// then emit the first non-empty one ending where the next HDDA step lands.
// Written with one HDDA step site (the step after an empty cell and the step
// that ends an emitted interval are the same code), which keeps one copy of
// the per-level step code per caller.
template <class D>
__device__ inline bool intervalNext(const DevGrid &g, uint32_t attr, const DevValueRanges &vr,
                                    IntervalItT<D> &it, DevInterval &out)
{
  VoxelDesc desc{};
  bool emit = false;
  for (;;) {
    if (!(it.dda.t <= it.tMax))
      return false;
    const uint32_t L = it.dda.level;
    int32_t cx, cy, cz;
    ddaCell(it.dda, L, cx, cy, cz);
    if (g.dense)
      queryVoxelDense(g, cx, cy, cz, L, attr, vr, desc);
    else
      querySparseCached(g, cx, cy, cz, L, attr, vr, it, desc);
    if (!desc.isEmpty) {
      if (!(it.dda.t < it.tMax))
        return false;
      out.v0 = desc.v0;
      out.v1 = desc.v1;
      out.t0 = it.dda.t;
      emit   = true;
    }
    if (it.budget-- == 0) {
      it.tMax = -kPosInf;
      return false;
    }
    hddaStep(desc, it.dda);
    if (emit) {
      out.t1            = minx(it.dda.t, it.tMax);
      out.nominalDeltaT = it.nominalDeltaT;
      return true;
    }
  }
}

// ---------------------------------------------------------------------------
// Hit iteration.
// ---------------------------------------------------------------------------
// Out of line so the many call sites of the bisection share one copy of the
// type / filter dispatch (static: one copy per translation unit that
// includes this header).
static __device__ __noinline__ float hitSample(const DevGrid &g, int filter, uint32_t attr, uint32_t depth,
                                        f3 p, float time)
{
  return sampleObjectAny(g, filter, attr, depth, p, time);
}

// Sample hooks of the hit iterator's marching.  AnySampleHook dispatches on
// the volume's voxel type and filter out of line (one copy shared by every
// call site: the per-ray C API and the generic batched kernel); the
// specialised LinearSampleHook inlines one field type with the trilinear
// filter.  Both evaluate exactly sampleObjectAny's expression.
struct AnySampleHook {
  const DevGrid *g;
  int filter;
  uint32_t attr;
  uint32_t depth;
  float time = 0.f;  // the iterator's time (temporally varying volumes)
  __device__ __forceinline__ float operator()(f3 oc) const { return hitSample(*g, filter, attr, depth, oc, time); }
};

template <class Field>
struct LinearSampleHook {
  const DevGrid *g;
  Field F;
  __device__ __forceinline__ float operator()(f3 oc) const
  {
    return sampleLinear(F, xfmPoint(g->objectToIndex, oc));
  }
};

template <class Hook>
struct HitCtx {
  Hook sample;
  f3 o, d;
  __device__ __forceinline__ float sampleAt(float t) const
  {
    return sample({o.x + t * d.x, o.y + t * d.y, o.z + t * d.z});
  }
};

// bisect (Iterator.ih): at most 10 halvings of [t0, t] towards the iso
// crossing.
template <class Ctx>
__device__ inline float bisect(const Ctx &c, float t0, float s0, float t, float s, float iso, float tol)
{
  int iter   = 0;
  float tMid = 0.f;
  while (iter < 10) {
    tMid              = 0.5f * (t0 + t);
    const float error = 0.5f * (t - t0);
    if (error < tol)
      break;
    const float sm = c.sampleAt(tMid);
    if (isnan(sm))
      return fabsf(iso - s0) < fabsf(iso - s) ? t0 : t;
    if (sm == iso || (iso - s0) * (iso - sm) < 0.f) {
      t = tMid;
      s = sm;
    } else if (s == iso || (iso - s) * (iso - sm) < 0.f) {
      t0 = tMid;
      s0 = sm;
    } else {
      return kPosInf;
    }
    iter++;
  }
  return tMid;
}

// intersectSurfacesBisection (Iterator.ih): march [tLo, tHi) with the
// interval's nominal step, find the first iso crossing, refine it by
// bisection.  With LOOKAHEAD > 1 the t of the next LOOKAHEAD march steps
// are computed first (the same serial additions) and their samples issued
// together, so their loads overlap; the steps are then examined in order
// exactly as the one-step loop would, and samples past a hit are discarded.
//
// (cacheT, cacheS) is the last march sample of the ray, (t, sampleAt(t)): an
// interval that starts where the previous one's march ended (the usual case:
// the DDA's intervals abut and the march's last step lands on the interval
// end) reuses it instead of sampling the same t again.
template <int LOOKAHEAD, class Ctx>
__device__ inline bool intersectBisection(const Ctx &c, float tLo, float tHi, float step, uint32_t numValues,
                                          const float *values, DevHit &hit, float &cacheT, float &cacheS)
{
  float t0 = tLo;
  float s0 = t0 == cacheT ? cacheS : c.sampleAt(t0);
  for (int it = 0; (float)it < 10.f && isnan(s0) && t0 < tHi; ++it) {
    t0 += maxx(1e-5f, 1e-5f * step);
    s0 = c.sampleAt(t0);
  }
  uint32_t march = 0;
  while (t0 < tHi && march < kMaxMarchSteps) {
    float tk[LOOKAHEAD], hk[LOOKAHEAD], sk[LOOKAHEAD];
    int kn   = 0;
    float tt = t0;
#pragma unroll
    for (int k = 0; k < LOOKAHEAD; ++k)
      if (tt < tHi && march + (uint32_t)k < kMaxMarchSteps) {
        hk[k] = minx(step, tHi - tt);
        tk[k] = tt + hk[k];
        tt    = tk[k];
        kn    = k + 1;
      }
#pragma unroll
    for (int k = 0; k < LOOKAHEAD; ++k)
      if (k < kn)
        sk[k] = c.sampleAt(tk[k]);
    cacheT = tk[kn - 1];
    cacheS = sk[kn - 1];
#pragma unroll
    for (int k = 0; k < LOOKAHEAD; ++k) {
      if (k >= kn)
        break;
      const float h = hk[k];
      const float t = tk[k];
      float s       = sk[k];
      float ts      = t;
      for (int it = 0; (float)it < 10.f && isnan(s) && ts > t0; ++it) {
        ts -= maxx(1e-5f, 1e-5f * step);
        s = c.sampleAt(ts);
      }
      float tHit = kPosInf, eps = kPosInf, value = kPosInf;
      for (uint32_t i = 0; i < numValues; ++i) {
        const float vi = __ldg(values + i);
        if (fabsf(s0 - vi) < 1e-6f) {
          if (t0 < tHit && t0 <= tHi) {
            tHit  = t0;
            value = vi;
            eps   = 0.125f * step;
          }
        } else if (!isnan(s0 + s) && (vi - s0) * (vi - s) < 0.f) {
          const float tIso = bisect(c, t0, s0, ts, s, vi, minx(1e-6f, 0.01f * h));
          if (tIso < tHit && tIso <= tHi) {
            tHit  = tIso;
            value = vi;
            eps   = 0.125f * step;
          }
        }
        if (t == tHi && fabsf(s - vi) < 1e-6f) {
          if (ts < tHit && ts <= tHi) {
            tHit  = ts;
            value = vi;
            eps   = 0.125f * step;
          }
        }
      }
      if (tHit < kPosInf) {
        hit.t       = tHit;
        hit.sample  = value;
        hit.epsilon = eps * sqrtf(c.d.x * c.d.x + c.d.y * c.d.y + c.d.z * c.d.z);
        return true;
      }
      t0 = t;
      s0 = s;
    }
    march += (uint32_t)kn;
  }
  return false;
}

// Default hit iterator state (DefaultIterator.ispc:140-166).
struct HitIt {
  IntervalItDyn ii;
  f3 o, d;
  DevInterval cur;
  float lastHitOffsetT;
  float cacheT, cacheS;  // last march sample (intersectBisection)
};

__device__ inline void hitInit(const DevGrid &g, uint32_t depth, f3 o, f3 d, float tLo, float tHi,
                               HitIt &h)
{
  intervalInit(g, depth, o, d, tLo, tHi, h.ii);
  h.o              = o;
  h.d              = d;
  h.cur            = {1.f, -1.f, 0.f, 0.f, 0.f};
  h.lastHitOffsetT = -kPosInf;
  h.cacheT         = __builtin_nanf("");
  h.cacheS         = 0.f;
}

// One vklIterateHit call (DefaultIterator.ispc:168-258).
template <int LOOKAHEAD, class Hook>
__device__ inline bool hitNextWith(const DevGrid &g, const Hook &hook, uint32_t attr, const DevValueRanges &vr,
                                   uint32_t numValues, const float *values, HitIt &h, DevHit &hit)
{
  if (numValues == 0)
    return false;
  if (h.cur.t0 == kPosInf)
    return false;
  const HitCtx<Hook> c{hook, h.o, h.d};
  for (;;) {
    const bool need = h.cur.t1 <= h.cur.t0;
    bool have       = !need;
    if (need)
      have = intervalNext(g, attr, vr, h.ii, h.cur);
    if (need && have) {
      h.cur.t0 = maxx(h.cur.t0, h.lastHitOffsetT);
      if (h.cur.t1 <= h.cur.t0)
        continue;
    }
    if (!have) {
      h.cur.t0 = kPosInf;
      return false;
    }
    hit.t = kPosInf;
    if (intersectBisection<LOOKAHEAD>(c, h.cur.t0, h.cur.t1, h.cur.nominalDeltaT, numValues, values, hit,
                                      h.cacheT, h.cacheS)) {
      h.cur.t0         = hit.t + hit.epsilon;
      h.lastHitOffsetT = hit.t + hit.epsilon;
      return true;
    }
    h.cur.t0 = kPosInf;
  }
}

// ---------------------------------------------------------------------------
// Batched hit iteration as a per-lane state machine.  hitNextWith runs each
// ray's loop nest (DDA, march, NaN nudges, bisection) to completion, so the
// 32 random rays of a warp are soon in different loops and fewer than two
// lanes execute each instruction.  Here every iteration of the warp's loop
// first advances each lane through its non-sampling steps until the lane
// needs one sample (or is done), then all lanes that need one take it at a
// single call site.  Each lane performs exactly the steps, samples and
// comparisons of hitNextWith in the same order, so hits are identical.
// ---------------------------------------------------------------------------
enum HitPhase : int {
  kHpTop,          // a vklIterateHit call begins
  kHpLoop,         // hitNext's interval loop
  kHpStartSample,  // sample at the interval start arrived
  kHpStartNudge,   // NaN start sample: nudge forward
  kHpMarch,        // next march step
  kHpMarchSample,  // march sample arrived
  kHpMarchNudge,   // NaN march sample: nudge backward
  kHpNudgeSample,  // nudged march sample arrived
  kHpValue,        // test value i
  kHpBisect,       // next bisection step
  kHpBisectSample, // bisection sample arrived
  kHpValueTail,    // end-point test of value i
  kHpDone
};

// Rays: the lane's ray source.  rays.next(h, out) starts the lane's next ray
// (hitInit into h, out = its first hit slot) and returns false when the lane
// has none left; rays.finish(count) records the hit count of the ray just
// completed.  A lane that finishes a ray starts its next one within the same
// warp iteration, so a warp does not idle behind its longest ray.
template <class Hook, class Rays>
__device__ inline void hitsAllLanes(const DevGrid &g, const Hook &hook, uint32_t attr, const DevValueRanges &vr,
                                    uint32_t numValues, const float *values, uint32_t maxPerRay, Rays &rays)
{
  HitIt h;
  DevHit *out    = nullptr;
  uint32_t count = 0;
  int ph         = rays.next(h, out) ? kHpTop : kHpDone;
  float dlen     = sqrtf(h.d.x * h.d.x + h.d.y * h.d.y + h.d.z * h.d.z);
  // intersectBisection state
  float t0 = 0.f, s0 = 0.f, tHi = 0.f, step = 0.f, hs = 0.f, t = 0.f, s = 0.f, ts = 0.f;
  uint32_t march = 0;
  int nudge      = 0;
  uint32_t vi    = 0;
  float tHit = kPosInf, eps = kPosInf, value = kPosInf, iso = 0.f;
  // bisect state
  float bt0 = 0.f, bs0 = 0.f, bt = 0.f, bs = 0.f, tol = 0.f, tMid = 0.f, tIso = kPosInf;
  int iter     = 0;
  float sample = 0.f, tReq = 0.f;
  for (;;) {
    bool want = false;
    while (!want && ph != kHpDone) {
      switch (ph) {
      case kHpTop:
        if (count >= kMaxHitsPerRay || numValues == 0 || h.cur.t0 == kPosInf) {
          ph = kHpDone;
          break;
        }
        ph = kHpLoop;
        break;
      case kHpLoop: {
        const bool need = h.cur.t1 <= h.cur.t0;
        bool have       = !need;
        if (need)
          have = intervalNext(g, attr, vr, h.ii, h.cur);
        if (need && have) {
          h.cur.t0 = maxx(h.cur.t0, h.lastHitOffsetT);
          if (h.cur.t1 <= h.cur.t0)
            break;  // next interval
        }
        if (!have) {
          h.cur.t0 = kPosInf;
          ph       = kHpDone;
          break;
        }
        t0    = h.cur.t0;
        tHi   = h.cur.t1;
        step  = h.cur.nominalDeltaT;
        nudge = 0;
        march = 0;
        if (t0 == h.cacheT) {
          s0 = h.cacheS;
          ph = kHpStartNudge;
        } else {
          tReq = t0;
          want = true;
          ph   = kHpStartSample;
        }
        break;
      }
      case kHpStartSample:
        s0 = sample;
        ph = kHpStartNudge;
        break;
      case kHpStartNudge:
        if ((float)nudge < 10.f && isnan(s0) && t0 < tHi) {
          t0 += maxx(1e-5f, 1e-5f * step);
          ++nudge;
          tReq = t0;
          want = true;
          ph   = kHpStartSample;
        } else {
          ph = kHpMarch;
        }
        break;
      case kHpMarch:
        if (!(t0 < tHi && march < kMaxMarchSteps)) {
          h.cur.t0 = kPosInf;  // interval exhausted without a hit
          ph       = kHpLoop;
          break;
        }
        hs   = minx(step, tHi - t0);
        t    = t0 + hs;
        tReq = t;
        want = true;
        ph   = kHpMarchSample;
        break;
      case kHpMarchSample:
        s        = sample;
        h.cacheT = t;
        h.cacheS = s;
        ts       = t;
        nudge    = 0;
        ph       = kHpMarchNudge;
        break;
      case kHpMarchNudge:
        if ((float)nudge < 10.f && isnan(s) && ts > t0) {
          ts -= maxx(1e-5f, 1e-5f * step);
          ++nudge;
          tReq = ts;
          want = true;
          ph   = kHpNudgeSample;
        } else {
          tHit  = kPosInf;
          eps   = kPosInf;
          value = kPosInf;
          vi    = 0;
          ph    = kHpValue;
        }
        break;
      case kHpNudgeSample:
        s  = sample;
        ph = kHpMarchNudge;
        break;
      case kHpValue:
        if (vi == numValues) {
          if (tHit < kPosInf) {
            DevHit hit{tHit, value, eps * dlen};
            if (count < maxPerRay)
              out[count] = hit;
            ++count;
            h.cur.t0         = hit.t + hit.epsilon;
            h.lastHitOffsetT = hit.t + hit.epsilon;
            ph               = kHpTop;
          } else {
            t0 = t;
            s0 = s;
            ++march;
            ph = kHpMarch;
          }
          break;
        }
        iso = __ldg(values + vi);
        if (fabsf(s0 - iso) < 1e-6f) {
          if (t0 < tHit && t0 <= tHi) {
            tHit  = t0;
            value = iso;
            eps   = 0.125f * step;
          }
          ph = kHpValueTail;
        } else if (!isnan(s0 + s) && (iso - s0) * (iso - s) < 0.f) {
          bt0  = t0;
          bs0  = s0;
          bt   = ts;
          bs   = s;
          tol  = minx(1e-6f, 0.01f * hs);
          iter = 0;
          tMid = 0.f;
          ph   = kHpBisect;
        } else {
          ph = kHpValueTail;
        }
        break;
      case kHpBisect:
        if (iter < 10) {
          tMid              = 0.5f * (bt0 + bt);
          const float error = 0.5f * (bt - bt0);
          if (!(error < tol)) {
            tReq = tMid;
            want = true;
            ph   = kHpBisectSample;
            break;
          }
        }
        tIso = tMid;
        if (tIso < tHit && tIso <= tHi) {
          tHit  = tIso;
          value = iso;
          eps   = 0.125f * step;
        }
        ph = kHpValueTail;
        break;
      case kHpBisectSample: {
        const float sm = sample;
        bool finished  = false;
        if (isnan(sm)) {
          tIso     = fabsf(iso - bs0) < fabsf(iso - bs) ? bt0 : bt;
          finished = true;
        } else if (sm == iso || (iso - bs0) * (iso - sm) < 0.f) {
          bt = tMid;
          bs = sm;
        } else if (bs == iso || (iso - bs) * (iso - sm) < 0.f) {
          bt0 = tMid;
          bs0 = sm;
        } else {
          tIso     = kPosInf;
          finished = true;
        }
        if (finished) {
          if (tIso < tHit && tIso <= tHi) {
            tHit  = tIso;
            value = iso;
            eps   = 0.125f * step;
          }
          ph = kHpValueTail;
        } else {
          ++iter;
          ph = kHpBisect;
        }
        break;
      }
      case kHpValueTail:
        if (t == tHi && fabsf(s - iso) < 1e-6f) {
          if (ts < tHit && ts <= tHi) {
            tHit  = ts;
            value = iso;
            eps   = 0.125f * step;
          }
        }
        ++vi;
        ph = kHpValue;
        break;
      default:
        ph = kHpDone;
        break;
      }
      if (ph == kHpDone) {  // the ray is complete: record it, start the next
        rays.finish(count);
        if (rays.next(h, out)) {
          count = 0;
          dlen  = sqrtf(h.d.x * h.d.x + h.d.y * h.d.y + h.d.z * h.d.z);
          ph    = kHpTop;
        }
      }
    }
    if (!__any_sync(0xffffffffu, want))
      return;
    if (want)
      sample = hook({h.o.x + tReq * h.d.x, h.o.y + tReq * h.d.y, h.o.z + tReq * h.d.z});
  }
}

__device__ inline bool hitNext(const DevGrid &g, int filter, uint32_t attr, uint32_t sampleDepth,
                               const DevValueRanges &vr, uint32_t numValues, const float *values,
                               HitIt &h, DevHit &hit, float time = 0.f)
{
  return hitNextWith<1>(g, AnySampleHook{&g, filter, attr, sampleDepth, time}, attr, vr, numValues, values, h,
                        hit);
}

}  // namespace vklcuda
