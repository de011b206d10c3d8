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

struct Dda {
  uint32_t level;
  float t;
  f3 org, dir;
  int32_t idx[12];
  float tNext[12];
  float tDelta[12];
  int32_t idxDelta[12];
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

__device__ __forceinline__ void ddaStep(Dda &d, uint32_t l)
{
  const float tx = d.tNext[l], ty = d.tNext[4 + l], tz = d.tNext[8 + l];
  const float m  = minx(minx(tx, ty), tz);
  const int k    = (m == tx) ? (int)l : (m == ty) ? 4 + (int)l : 8 + (int)l;
  d.t            = d.tNext[k];
  d.tNext[k]     = d.tNext[k] + d.tDelta[k];
  d.idx[k]       = d.idx[k] + d.idxDelta[k];
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

__device__ inline void queryVoxelDense(const DevGrid &g, int32_t x, int32_t y, int32_t z,
                                       uint32_t depth, uint32_t attr, const DevValueRanges &vr,
                                       VoxelDesc &desc)
{
  desc.level = depth;
  const uint32_t ox = (uint32_t)x, oy = (uint32_t)y, oz = (uint32_t)z;
  if (!(ox < g.activeSize[0] && oy < g.activeSize[1] && oz < g.activeSize[2])) {
    desc.isEmpty = true;
    return;
  }
  // The reference computes the level-1/2 node numbers in closed form
  // (z-major over the dense node grid, VdbQueryVoxelDense.ih:41-113); walking
  // the child pointers gives the same voxel for every volume up to 4096^3
  // and never indexes past a level's arrays beyond that.
  const uint32_t lvl = depth >= 2 ? 2u : depth;
  uint64_t node = 0, ni = 0;
  for (uint32_t l = 0;; ++l) {
    ni = node * levelNumVoxels(l) + offsetToLinear(l, ox, oy, oz);
    if (l == lvl)
      break;
    node = voxelChildIndex(__ldg(g.levels[l].voxels + ni));
  }
  const float *r = g.levels[lvl].valueRange + 2 * (ni * g.numAttributes + attr);
  desc.v0        = __ldg(r);
  desc.v1        = __ldg(r + 1);
  desc.isEmpty   = !rangesOverlap(vr, desc.v0, desc.v1);
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
__device__ inline void hddaStep(const VoxelDesc &desc, Dda &d)
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
  // propagate upwards: level l steps when its child (l+1) left its cell
  bool stepped = true;
  for (int l = (int)L - 1; l >= 0 && stepped; --l) {
    const int32_t res = (int32_t)levelRes((uint32_t)l + 1);
    const bool left   = d.idx[l + 1] < d.idx[l] || d.idx[4 + l + 1] < d.idx[4 + l] ||
                      d.idx[8 + l + 1] < d.idx[8 + l] || d.idx[l + 1] >= d.idx[l] + res ||
                      d.idx[4 + l + 1] >= d.idx[4 + l] + res ||
                      d.idx[8 + l + 1] >= d.idx[8 + l] + res;
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

struct IntervalIt {
  float tMax;
  float nominalDeltaT;
  uint32_t budget;
  Dda dda;
};

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

__device__ inline void intervalInit(const DevGrid &g, uint32_t depth, f3 origin, f3 direction,
                                    float tLo, float tHi, IntervalIt &it)
{
  f3 org       = xfmPoint(g.objectToIndex, origin);
  org          = {org.x - (float)g.rootOrigin[0], org.y - (float)g.rootOrigin[1],
         org.z - (float)g.rootOrigin[2]};
  const f3 dir = xfmVector(g.objectToIndex, direction);
  it.nominalDeltaT = minx(minx(1.f * divideSafe(fabsf(dir.x)), 1.f * divideSafe(fabsf(dir.y))),
                          1.f * divideSafe(fabsf(dir.z)));
  float lo, hi;
  intersectBox(org, dir, g.domain, tLo, tHi, lo, hi);
  it.budget = kMaxDdaSteps;
  if (hi <= lo) {
    it.tMax  = -kPosInf;
    it.dda.t = 0.f;
  } else {
    it.tMax = hi;
    ddaInit(org, dir, lo, depth, it.dda);
  }
}

__device__ inline bool intervalNext(const DevGrid &g, uint32_t attr, const DevValueRanges &vr,
                                    IntervalIt &it, DevInterval &out)
{
  if (!(it.dda.t <= it.tMax))
    return false;
  VoxelDesc desc{};
  while (it.dda.t <= it.tMax) {
    const uint32_t L = it.dda.level;
    if (g.dense)
      queryVoxelDense(g, it.dda.idx[L], it.dda.idx[4 + L], it.dda.idx[8 + L], L, attr, vr, desc);
    else
      queryVoxelSparse(g, it.dda.idx[L], it.dda.idx[4 + L], it.dda.idx[8 + L], L, attr, vr, desc);
    if (!desc.isEmpty)
      break;
    if (it.budget-- == 0) {
      it.tMax = -kPosInf;
      return false;
    }
    hddaStep(desc, it.dda);
  }
  if (it.dda.t < it.tMax) {
    out.v0 = desc.v0;
    out.v1 = desc.v1;
    out.t0 = it.dda.t;
    if (it.budget-- == 0) {
      it.tMax = -kPosInf;
      return false;
    }
    hddaStep(desc, it.dda);
    out.t1            = minx(it.dda.t, it.tMax);
    out.nominalDeltaT = it.nominalDeltaT;
    return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Hit iteration.
// ---------------------------------------------------------------------------
// Out of line so the many call sites of the bisection share one copy of the
// type / filter dispatch.
__device__ __noinline__ float hitSample(const DevGrid &g, int filter, uint32_t attr, uint32_t depth,
                                        f3 p)
{
  return sampleObjectAny(g, filter, attr, depth, p);
}

struct HitCtx {
  const DevGrid *g;
  int filter;
  uint32_t attr;
  uint32_t depth;
  f3 o, d;
  __device__ __forceinline__ float sampleAt(float t) const
  {
    return hitSample(*g, filter, attr, depth, {o.x + t * d.x, o.y + t * d.y, o.z + t * d.z});
  }
};

__device__ inline float bisect(const HitCtx &c, float t0, float s0, float t, float s, float iso,
                               float tol)
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

__device__ inline bool intersectBisection(const HitCtx &c, float tLo, float tHi, float step,
                                          uint32_t numValues, const float *values, DevHit &hit)
{
  float t0 = tLo;
  float s0 = c.sampleAt(t0);
  for (int it = 0; (float)it < 10.f && isnan(s0) && t0 < tHi; ++it) {
    t0 += maxx(1e-5f, 1e-5f * step);
    s0 = c.sampleAt(t0);
  }
  for (uint32_t march = 0; t0 < tHi && march < kMaxMarchSteps; ++march) {
    const float h = minx(step, tHi - t0);
    const float t = t0 + h;
    float s       = c.sampleAt(t);
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
  return false;
}

// Default hit iterator state (DefaultIterator.ispc:140-166).
struct HitIt {
  IntervalIt ii;
  f3 o, d;
  DevInterval cur;
  float lastHitOffsetT;
};

__device__ inline void hitInit(const DevGrid &g, uint32_t depth, f3 o, f3 d, float tLo, float tHi,
                               HitIt &h)
{
  intervalInit(g, depth, o, d, tLo, tHi, h.ii);
  h.o              = o;
  h.d              = d;
  h.cur            = {1.f, -1.f, 0.f, 0.f, 0.f};
  h.lastHitOffsetT = -kPosInf;
}

// One vklIterateHit call (DefaultIterator.ispc:168-258).
__device__ inline bool hitNext(const DevGrid &g, int filter, uint32_t attr, uint32_t sampleDepth,
                               const DevValueRanges &vr, uint32_t numValues, const float *values,
                               HitIt &h, DevHit &hit)
{
  if (numValues == 0)
    return false;
  if (h.cur.t0 == kPosInf)
    return false;
  const HitCtx c{&g, filter, attr, sampleDepth, h.o, h.d};
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
    if (intersectBisection(c, h.cur.t0, h.cur.t1, h.cur.nominalDeltaT, numValues, values, hit)) {
      h.cur.t0         = hit.t + hit.epsilon;
      h.lastHitOffsetT = hit.t + hit.epsilon;
      return true;
    }
    h.cur.t0 = kPosInf;
  }
}

}  // namespace vklcuda
