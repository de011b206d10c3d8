// 16^3-voxel macrocell intervals (an extension of the cuda device; interval
// iterator context parameter "macrocells" = 1): the interval walk of the
// reference's legacy structuredRegular volume, whose GridAccelerator
// partitions the grid into macrocells of 16^3 voxel cells (built when the
// reference is configured with OPENVKL_DEVICE_CPU_STRUCTURED_REGULAR_LEGACY;
// the default structuredRegular volume walks the VDB hierarchy instead).
//
//   macrocell width          GridAccelerator.h:14-19 (CELL_WIDTH = 16)
//   macrocell value range    GridAccelerator.ispc:80-109: vertices
//                            cell * 16 + [0, 16] per axis, clamped to
//                            dims - 1, NaN skipped, a NaN range when all are
//                            NaN (a vertex's range is its value,
//                            SharedStructuredVolume.ispc:196-209)
//   cell walk                GridAccelerator_nextCell, GridAccelerator.ispc:
//                            146-240 (first cell from the entry point, then
//                            one face crossing per step)
//   interval emission        GridAcceleratorIterator.ispc:44-155
//   transforms / box         SharedStructuredVolume.ih:21-53,
//                            StructuredVolume.cpp:205-211
//
// It applies to vertex-centered volumes given by gridOrigin / gridSpacing (a
// diagonal indexToObject, index origin 0), which is what the legacy volume
// supports.  Only min / max fold the ranges, so they equal the reference's
// except for the sign of a zero bound where +0.0 and -0.0 vertices tie.
#include "iterate.cuh"
#include "kernels.h"
#include "objects.h"

namespace vklcuda {

namespace {

constexpr int kMacroBits    = 4;
constexpr int kMacroVerts   = (1 << kMacroBits) + 1;  // 17 vertices per axis
constexpr int kRangeThreads = 128;
constexpr int kWalkThreads  = 128;

// One block per macrocell: min / max over its 17^3 vertices.
template <typename T>
__global__ void __launch_bounds__(kRangeThreads)
    kMacrocellRanges(const __grid_constant__ DevGrid g, uint32_t attr, int3 nc, float2 *__restrict__ out)
{
  __shared__ float slo[kRangeThreads / 32], shi[kRangeThreads / 32];
  const uint64_t cell = blockIdx.x;
  const int cx = (int)(cell % (uint64_t)nc.x), cy = (int)((cell / (uint64_t)nc.x) % (uint64_t)nc.y),
            cz = (int)(cell / ((uint64_t)nc.x * (uint64_t)nc.y));
  const DenseField<T> F(g, attr);
  const int X = (int)g.activeSize[0], Y = (int)g.activeSize[1], Z = (int)g.activeSize[2];
  float lo = kPosInf, hi = -kPosInf;
  for (int v = threadIdx.x; v < kMacroVerts * kMacroVerts * kMacroVerts; v += kRangeThreads) {
    const int i = v % kMacroVerts, j = (v / kMacroVerts) % kMacroVerts, k = v / (kMacroVerts * kMacroVerts);
    const float s = F.at(min(X - 1, (cx << kMacroBits) + i), min(Y - 1, (cy << kMacroBits) + j),
                         min(Z - 1, (cz << kMacroBits) + k));
    if (!isnan(s)) {
      lo = minx(lo, s);
      hi = maxx(hi, s);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = minx(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = maxx(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    slo[threadIdx.x >> 5] = lo;
    shi[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kRangeThreads / 32; ++w) {
      lo = minx(lo, slo[w]);
      hi = maxx(hi, shi[w]);
    }
    // no non-NaN vertex: lo stays above hi
    const float nan = __int_as_float(0x7fffffff);
    out[cell]       = lo > hi ? make_float2(nan, nan) : make_float2(lo, hi);
  }
}

struct MacroGrid {
  int3 nc;
  float origin[3], spacing[3];
  float box[6];  // the volume's bounding box
  const float2 *ranges;
};

// isempty1f (math/box_utility.ih:6-9)
__device__ __forceinline__ bool emptyRange(float lo, float hi) { return hi <= lo; }

// transformObjectToLocal of a regular grid: 1 / spacing * (p - origin)
__device__ __forceinline__ float toLocal(const MacroGrid &m, int a, float p)
{
  return 1.f / m.spacing[a] * (p - m.origin[a]);
}

__device__ __forceinline__ void cellT(const MacroGrid &m, f3 o, f3 d, float bbLo, float bbHi, int3 c, float &lo,
                                      float &hi)
{
  // GridAccelerator_getCellBounds: the cell's corners in object space
  const int l[3] = {c.x << kMacroBits, c.y << kMacroBits, c.z << kMacroBits};
  const int u[3] = {(c.x + 1) << kMacroBits, (c.y + 1) << kMacroBits, (c.z + 1) << kMacroBits};
  float box[6];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    box[a]     = m.origin[a] + (float)l[a] * m.spacing[a];
    box[3 + a] = m.origin[a] + (float)u[a] * m.spacing[a];
  }
  intersectBox(o, d, box, bbLo, bbHi, lo, hi);
}

// GridAccelerator_nextCell: advances `cell` (x = -1 before the first call)
// and returns the cell's t range, or false past the last cell.
__device__ inline bool nextCell(const MacroGrid &m, f3 o, f3 d, float bbLo, float bbHi, int3 &cell, float &tLo,
                                float &tHi)
{
  const bool first = cell.x == -1;
  float lo = 0.f, hi = 0.f;
  if (first) {
    const float px = o.x + bbLo * d.x, py = o.y + bbLo * d.y, pz = o.z + bbLo * d.z;
    cell = make_int3(toIntX86(toLocal(m, 0, px)) >> kMacroBits, toIntX86(toLocal(m, 1, py)) >> kMacroBits,
                     toIntX86(toLocal(m, 2, pz)) >> kMacroBits);
    cellT(m, o, d, bbLo, bbHi, cell, lo, hi);
  }
  if (!first || emptyRange(lo, hi)) {
    // cell-space direction "direction * 1.f / gridSpacing * RCP_CELL_WIDTH"
    // with RCP_CELL_WIDTH the macro text "1.f / CELL_WIDTH": (d / s) / 16
    const float cd[3] = {d.x / m.spacing[0] / 16.f, d.y / m.spacing[1] / 16.f, d.z / m.spacing[2] / 16.f};
    const float co[3] = {toLocal(m, 0, o.x) / 16.f, toLocal(m, 1, o.y) / 16.f, toLocal(m, 2, o.z) / 16.f};
    const int ci[3]   = {cell.x, cell.y, cell.z};
    float tMax[3];
    int corner[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float rcd = divideSafe(cd[a]);  // rcp_safe
      corner[a]       = 1 - 2 * (int)(__float_as_uint(cd[a]) >> 31);
      const float t0  = ((float)ci[a] - co[a]) * rcd;
      const float t1  = ((float)(ci[a] + 1) - co[a]) * rcd;
      tMax[a]         = maxx(t0, t1);
    }
    const float tExit = minx(minx(tMax[0], tMax[1]), tMax[2]);
    cell = make_int3(ci[0] + (tMax[0] == tExit ? corner[0] : 0), ci[1] + (tMax[1] == tExit ? corner[1] : 0),
                     ci[2] + (tMax[2] == tExit ? corner[2] : 0));
    cellT(m, o, d, bbLo, bbHi, cell, lo, hi);
  }
  if (emptyRange(lo, hi))
    return false;
  tLo = lo;
  tHi = hi;
  return true;
}

__global__ void __launch_bounds__(kWalkThreads)
    kMacrocellIntervals(const __grid_constant__ MacroGrid m, DevValueRanges vr, uint64_t n,
                        const float *__restrict__ orgs, const float *__restrict__ dirs,
                        const float *__restrict__ tr, uint32_t maxPerRay, DevInterval *__restrict__ out,
                        uint32_t *__restrict__ counts)
{
  const uint64_t r = (uint64_t)blockIdx.x * kWalkThreads + threadIdx.x;
  if (r >= n)
    return;
  const f3 o = {__ldg(orgs + 3 * r), __ldg(orgs + 3 * r + 1), __ldg(orgs + 3 * r + 2)};
  const f3 d = {__ldg(dirs + 3 * r), __ldg(dirs + 3 * r + 1), __ldg(dirs + 3 * r + 2)};
  float bbLo, bbHi;
  intersectBox(o, d, m.box, __ldg(tr + 2 * r), __ldg(tr + 2 * r + 1), bbLo, bbHi);
  // nominalDeltaT: reduce_min(gridSpacing * rcp_safe(|direction|))
  const float ndt = minx(minx(m.spacing[0] * divideSafe(fabsf(d.x)), m.spacing[1] * divideSafe(fabsf(d.y))),
                         m.spacing[2] * divideSafe(fabsf(d.z)));
  uint32_t c = 0;
  if (!emptyRange(bbLo, bbHi)) {
    int3 cell = make_int3(-1, -1, -1);
    // a ray crosses at most nc.x + nc.y + nc.z + 3 cells
    int budget = 4 * (m.nc.x + m.nc.y + m.nc.z) + 16;
    float tLo, tHi;
    while (budget-- > 0 && nextCell(m, o, d, bbLo, bbHi, cell, tLo, tHi)) {
      // cells the walk reaches lie in the grid; the lookup clamps the index
      const int x = min(max(cell.x, 0), m.nc.x - 1), y = min(max(cell.y, 0), m.nc.y - 1),
                z = min(max(cell.z, 0), m.nc.z - 1);
      const float2 v = m.ranges[(uint64_t)x + (uint64_t)m.nc.x * ((uint64_t)y + (uint64_t)m.nc.y * (uint64_t)z)];
      if (!rangesOverlap(vr, v.x, v.y))
        continue;
      if (c < maxPerRay)
        out[r * maxPerRay + c] = DevInterval{tLo, tHi, v.x, v.y, ndt};
      ++c;
    }
  }
  counts[r] = c;
}

bool legacyGrid(const DevGrid &g)
{
  const float *M = g.indexToObject;
  return g.dense && !g.constantCellData && g.rootOrigin[0] == 0 && g.rootOrigin[1] == 0 && g.rootOrigin[2] == 0 &&
         M[1] == 0.f && M[2] == 0.f && M[3] == 0.f && M[5] == 0.f && M[6] == 0.f && M[7] == 0.f;
}

int3 macrocellCount(const DevGrid &g)
{
  return make_int3((int)((g.activeSize[0] - 1) >> kMacroBits) + 1, (int)((g.activeSize[1] - 1) >> kMacroBits) + 1,
                   (int)((g.activeSize[2] - 1) >> kMacroBits) + 1);
}

}  // namespace

void checkMacrocellVolume(const DevGrid &g)
{
  if (!legacyGrid(g))
    fail("macrocell intervals need a vertex-centered structuredRegular volume given by gridOrigin / "
         "gridSpacing (index origin 0, no rotation)",
         VKL_INVALID_OPERATION);
}

uint64_t macrocellRangeCount(const DevGrid &g)
{
  const int3 n = macrocellCount(g);
  return (uint64_t)n.x * n.y * n.z;
}

void launchMacrocellRanges(const DevGrid &g, uint32_t attr, float *ranges, cudaStream_t st)
{
  const int3 n        = macrocellCount(g);
  const uint64_t cells = (uint64_t)n.x * n.y * n.z;
  float2 *out         = (float2 *)ranges;
  switch (g.type[attr]) {
  case kUChar:
    kMacrocellRanges<uint8_t><<<(unsigned)cells, kRangeThreads, 0, st>>>(g, attr, n, out);
    break;
  case kShort:
    kMacrocellRanges<int16_t><<<(unsigned)cells, kRangeThreads, 0, st>>>(g, attr, n, out);
    break;
  case kUShort:
    kMacrocellRanges<uint16_t><<<(unsigned)cells, kRangeThreads, 0, st>>>(g, attr, n, out);
    break;
  case kHalf:
    kMacrocellRanges<__half><<<(unsigned)cells, kRangeThreads, 0, st>>>(g, attr, n, out);
    break;
  case kDouble:
    kMacrocellRanges<double><<<(unsigned)cells, kRangeThreads, 0, st>>>(g, attr, n, out);
    break;
  default:
    kMacrocellRanges<float><<<(unsigned)cells, kRangeThreads, 0, st>>>(g, attr, n, out);
  }
  cudaCheck(cudaGetLastError(), "macrocell range kernel launch");
}

void launchMacrocellIntervals(const DevGrid &g, const float *ranges, DevValueRanges vr, uint64_t n,
                              const float *origins, const float *directions, const float *tRanges,
                              uint32_t maxPerRay, DevInterval *out, uint32_t *counts, cudaStream_t st)
{
  if (!n)
    return;
  MacroGrid m{};
  m.nc = macrocellCount(g);
  const float *M = g.indexToObject;
  for (int a = 0; a < 3; ++a) {
    m.origin[a]  = M[9 + a];
    m.spacing[a] = M[4 * a];
    m.box[a]     = m.origin[a];
    // StructuredVolume.cpp:205-211: gridOrigin + (dims - 1) * gridSpacing
    m.box[3 + a] = m.origin[a] + (float)(g.activeSize[a] - 1) * m.spacing[a];
  }
  m.ranges = (const float2 *)ranges;
  kMacrocellIntervals<<<(unsigned)((n + kWalkThreads - 1) / kWalkThreads), kWalkThreads, 0, st>>>(
      m, vr, n, origins, directions, tRanges, maxPerRay, out, counts);
  cudaCheck(cudaGetLastError(), "macrocell interval kernel launch");
}

}  // namespace vklcuda
