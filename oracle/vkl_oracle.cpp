// ORACLE — TEST INFRASTRUCTURE ONLY (see vkl_oracle.h).
//
// Every function below cites the reference file and lines it restates
// (paths relative to the Open VKL v2.0.2 source tree).  Compiled with
// -ffp-contract=off so that every float expression rounds after each
// operation, in the order written; the CUDA device is compiled the same way
// (--fmad=false) so the two agree bit for bit.
#include "vkl_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>
#include <atomic>
#include <thread>

// The density path tracer's log / sincos: the one source the CUDA renderer
// compiles too (the reference's platform math differs between platforms).
#include "../openvkl_b200/renderers/pt_math.h"

namespace orc {

static thread_local std::string g_lastError;

// Splits [0, n) into chunks handed to `threads` std::threads (threads <= 0:
// all hardware threads).  Used only where iterations are independent.
template <class F>
static void parallelFor(int64_t n, int threads, int64_t chunk, const F &fn)
{
  if (threads <= 0)
    threads = (int)std::max(1u, std::thread::hardware_concurrency());
  if (threads == 1 || n <= chunk) {
    for (int64_t i = 0; i < n; ++i)
      fn(i);
    return;
  }
  std::atomic<int64_t> next(0);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&]() {
      for (;;) {
        const int64_t b = next.fetch_add(chunk);
        if (b >= n)
          break;
        const int64_t e = std::min(n, b + chunk);
        for (int64_t i = b; i < e; ++i)
          fn(i);
      }
    });
  for (auto &th : pool)
    th.join();
}

// ---------------------------------------------------------------------------
// Topology: log resolutions 6/5/4/3 (openvkl/CMakeLists.txt:37-49; macro
// generator cmake/openvkl_macros.cmake:239-310, template
// openvkl/include/openvkl/vdb_topology.h.in).  Index 4 is the "one past the
// leaf" stopper whose resolution is 1 (vdb.h vklVdbLevelRes special case).
// ---------------------------------------------------------------------------
constexpr uint32_t NUM_LEVELS        = 4;
constexpr uint32_t LOG_RES[5]        = {6, 5, 4, 3, 0};
constexpr uint32_t TOTAL_LOG_RES[5]  = {18, 12, 7, 3, 0};
inline uint32_t levelRes(uint32_t l) { return 1u << TOTAL_LOG_RES[l]; }
inline uint64_t levelNumVoxels(uint32_t l) { return 1ull << (3 * LOG_RES[l]); }

enum : uint32_t {
  T_UCHAR  = 2500,
  T_SHORT  = 3000,
  T_USHORT = 3500,
  T_HALF   = 5800,
  T_FLOAT  = 6000,
  T_DOUBLE = 7000
};
enum : uint32_t { FMT_TILE = 0, FMT_DENSE_ZYX = 1 };
enum : int { F_NEAREST = 0, F_LINEAR = 100, F_CUBIC = 200 };

// Voxel codes (VdbGrid.h:91-203).
inline bool vEmpty(uint64_t v) { return (v & 3u) == 0; }
inline bool vError(uint64_t v) { return (v & 3u) == 1; }
inline bool vChild(uint64_t v) { return (v & 3u) == 2; }
inline bool vLeaf(uint64_t v) { return (v & 3u) == 3; }
inline uint64_t mkChild(uint64_t i) { return (i << 2) | 2u; }
inline uint64_t mkLeaf(uint64_t i, uint32_t fmt, uint32_t tf)
{
  return (i << 6) + ((uint64_t)(tf & 3u) << 4) + ((uint64_t)(fmt & 3u) << 2) +
         3u;
}
inline uint64_t mkError(uint32_t level, uint32_t off)
{
  return ((uint64_t)off << 32) + ((uint64_t)level << 8) + 1u;
}
inline uint64_t childIdx(uint64_t v) { return v >> 2; }
inline uint64_t leafIdx(uint64_t v) { return v >> 6; }
inline uint32_t leafFmt(uint64_t v) { return (uint32_t)((v >> 2) & 3u); }

// __vkl_vdb_domain_offset_to_linear_*_<l> (vdb_topology.h.in:96-166): mask
// the offset to the node, shift by the child resolution, z fastest.
inline uint64_t offsetToLinear(uint32_t l, uint64_t x, uint64_t y, uint64_t z)
{
  const uint64_t mask = levelRes(l) - 1;
  const uint32_t sh   = TOTAL_LOG_RES[l + 1];
  const uint64_t vx = (x & mask) >> sh, vy = (y & mask) >> sh,
                 vz = (z & mask) >> sh;
  return (vx << (2 * LOG_RES[l])) + (vy << LOG_RES[l]) + vz;
}

struct vec3f {
  float x, y, z;
};
struct vec3i {
  int32_t x, y, z;
};
struct vec3ui {
  uint32_t x, y, z;
};
struct range1f {
  float lower = std::numeric_limits<float>::infinity();
  float upper = -std::numeric_limits<float>::infinity();
};

// ISPC min/max on float lower to minps/maxps, i.e. (a < b ? a : b) and
// (a > b ? a : b); written out so NaN handling is explicit.
inline float fmin_(float a, float b) { return a < b ? a : b; }
inline float fmax_(float a, float b) { return a > b ? a : b; }

// float -> int32 truncation as x86 cvttss2si does it (ISPC to_int): NaN and
// out-of-range values give INT32_MIN.
inline int32_t toIntX86(float x)
{
  return (x >= -2147483648.f && x < 2147483648.f) ? (int32_t)x : INT32_MIN;
}

// rkcommon lerp(factor, a, b) = (1 - factor) * a + factor * b (the form used
// by rkcommon/math; not vendored in the reference tree, so parity-unpinned).
inline float lerp(float f, float a, float b) { return (1.f - f) * a + f * b; }

// rkcommon divide_safe / rcp_safe (not vendored): 1/x with |x| clamped away
// from zero at 1e-8 keeping the sign; a correctly rounded division stands in
// for ISPC's rcp().
inline float divide_safe(float x)
{
  const float e = 1e-8f;
  return 1.f / (std::fabs(x) < e ? (x >= 0.f ? e : -e) : x);
}
inline float rcp_safe(float x) { return divide_safe(x); }

// IEEE binary16 -> binary32, exact (Data.ih:151-153 half_to_float).
inline float halfToFloat(uint16_t h)
{
  const uint32_t s = (uint32_t)(h >> 15) << 31;
  uint32_t e       = (h >> 10) & 0x1f;
  uint32_t m       = h & 0x3ff;
  uint32_t bits;
  if (e == 0) {
    if (m == 0) {
      bits = s;
    } else {
      // subnormal half: normalise
      int ee = -1;
      do {
        ee++;
        m <<= 1;
      } while ((m & 0x400) == 0);
      m &= 0x3ff;
      bits = s | ((uint32_t)(127 - 15 - ee) << 23) | (m << 13);
    }
  } else if (e == 0x1f) {
    bits = s | 0x7f800000u | (m << 13);
  } else {
    bits = s | ((e + 127 - 15) << 23) | (m << 13);
  }
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

// Typed element load (Data.ih:66-153 get_<T>).
struct Attr {
  uint32_t type;
  const uint8_t *ptr;
  uint64_t stride;
};

inline float loadAttr(const Attr &a, uint64_t i)
{
  const uint8_t *p = a.ptr + i * a.stride;
  switch (a.type) {
  case T_UCHAR:
    return (float)*p;
  case T_SHORT: {
    int16_t v;
    std::memcpy(&v, p, 2);
    return (float)v;
  }
  case T_USHORT: {
    uint16_t v;
    std::memcpy(&v, p, 2);
    return (float)v;
  }
  case T_HALF: {
    uint16_t v;
    std::memcpy(&v, p, 2);
    return halfToFloat(v);
  }
  case T_FLOAT: {
    float v;
    std::memcpy(&v, p, 4);
    return v;
  }
  case T_DOUBLE: {
    double v;
    std::memcpy(&v, p, 8);
    return (float)v;
  }
  }
  return 0.f;
}

inline uint32_t typeSize(uint32_t t)
{
  switch (t) {
  case T_UCHAR:
    return 1;
  case T_SHORT:
  case T_USHORT:
  case T_HALF:
    return 2;
  case T_FLOAT:
    return 4;
  case T_DOUBLE:
    return 8;
  }
  throw std::runtime_error("unsupported data type");
}

struct Level {
  uint64_t numNodes = 0;
  std::vector<vec3ui> origin;
  std::vector<uint64_t> voxels;
  std::vector<range1f> valueRange;
};

struct Grid {
  float o2i[12];
  float i2o[12];
  vec3i rootOrigin;
  vec3ui activeSize;
  float domain[6];
  float bounds[6];
  bool constantCellData = false;
  bool dense            = false;
  uint32_t numAttributes = 1;
  std::vector<float> background;
  // dense
  vec3i denseDims;
  // gridOrigin / gridSpacing of a vertex-centered dense volume without
  // indexToObject or indexOrigin (what the legacy macrocell iterator reads)
  bool legacyGrid = false;
  float gridOrigin[3] = {0, 0, 0}, gridSpacing[3] = {1, 1, 1};
  // temporally varying dense data (0 constant, 1 structured: numTimesteps
  // values per voxel; 2 unstructured: per-voxel [indices[v], indices[v+1])
  // into the data and times arrays)
  int temporalFormat = 0;
  int numTimesteps   = 0;
  const uint8_t *tIndices = nullptr;
  bool tIndices64         = false;
  const float *tTimes     = nullptr;
  std::vector<Attr> denseAttr;
  std::vector<std::vector<uint8_t>> denseCopies;
  // sparse packed
  uint32_t leafType = T_FLOAT;
  std::vector<std::vector<uint8_t>> packedDense, packedTile;
  // leaves
  uint64_t numLeaves = 0;
  std::vector<uint32_t> leafLevel, leafFormat;
  std::vector<vec3i> leafOrigin;
  Level levels[NUM_LEVELS - 1];
  std::vector<range1f> volumeRange;
  // stencil-block leaves (the cuda device's extension): per attribute the
  // decoded 9^3 sampling window of every dense leaf slot (empty: off)
  std::vector<std::vector<float>> blockWin;
};

// ---------------------------------------------------------------------------
// Transforms (VdbGrid.h:56-89).
// ---------------------------------------------------------------------------
inline vec3f xfmVector(const float *M, const vec3f &p)
{
  return {M[0] * p.x + M[1] * p.y + M[2] * p.z,
          M[3] * p.x + M[4] * p.y + M[5] * p.z,
          M[6] * p.x + M[7] * p.y + M[8] * p.z};
}
inline vec3f xfmNormal(const float *Mi, const vec3f &p)
{
  return {Mi[0] * p.x + Mi[3] * p.y + Mi[6] * p.z,
          Mi[1] * p.x + Mi[4] * p.y + Mi[7] * p.z,
          Mi[2] * p.x + Mi[5] * p.y + Mi[8] * p.z};
}
inline vec3f xfmPoint(const float *M, const vec3f &p)
{
  vec3f r = xfmVector(M, p);
  return {r.x + M[9], r.y + M[10], r.z + M[11]};
}

// indexToObject (column-major vx,vy,vz,p as the "indexToObject" parameter,
// VdbVolume.h:37-57) -> row-major 3x4 buffers (writeTransform, VdbVolume.h:
// 63-78).  The inverse is taken in double and rounded once (the reference
// inverts in float with rkcommon's adjoint/det, DenseVdbVolume.cpp:60-63).
static void makeTransforms(const float c[12], float *i2o, float *o2i)
{
  // row-major linear part
  const double L[3][3] = {{c[0], c[3], c[6]}, {c[1], c[4], c[7]},
                          {c[2], c[5], c[8]}};
  const double p[3]    = {c[9], c[10], c[11]};
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k)
      i2o[r * 3 + k] = (float)L[r][k];
  i2o[9]  = c[9];
  i2o[10] = c[10];
  i2o[11] = c[11];
  const double det = L[0][0] * (L[1][1] * L[2][2] - L[1][2] * L[2][1]) -
                     L[0][1] * (L[1][0] * L[2][2] - L[1][2] * L[2][0]) +
                     L[0][2] * (L[1][0] * L[2][1] - L[1][1] * L[2][0]);
  double I[3][3];
  I[0][0] = (L[1][1] * L[2][2] - L[1][2] * L[2][1]) / det;
  I[0][1] = (L[0][2] * L[2][1] - L[0][1] * L[2][2]) / det;
  I[0][2] = (L[0][1] * L[1][2] - L[0][2] * L[1][1]) / det;
  I[1][0] = (L[1][2] * L[2][0] - L[1][0] * L[2][2]) / det;
  I[1][1] = (L[0][0] * L[2][2] - L[0][2] * L[2][0]) / det;
  I[1][2] = (L[0][2] * L[1][0] - L[0][0] * L[1][2]) / det;
  I[2][0] = (L[1][0] * L[2][1] - L[1][1] * L[2][0]) / det;
  I[2][1] = (L[0][1] * L[2][0] - L[0][0] * L[2][1]) / det;
  I[2][2] = (L[0][0] * L[1][1] - L[0][1] * L[1][0]) / det;
  for (int r = 0; r < 3; ++r) {
    for (int k = 0; k < 3; ++k)
      o2i[r * 3 + k] = (float)I[r][k];
    o2i[9 + r] =
        (float)(-(I[r][0] * p[0] + I[r][1] * p[1] + I[r][2] * p[2]));
  }
}

// ---------------------------------------------------------------------------
// Voxel access.
// ---------------------------------------------------------------------------
inline bool inDomain(const vec3ui &active, const vec3ui &o)
{
  return o.x < active.x && o.y < active.y && o.z < active.z;
}
inline vec3ui toDomainOffset(const vec3i &ic, const vec3i &root)
{
  return {(uint32_t)(ic.x - root.x), (uint32_t)(ic.y - root.y),
          (uint32_t)(ic.z - root.z)};
}

// Time of the sample being computed on this thread (the `time` argument of
// the sampling calls; temporally constant data ignore it).
static thread_local float t_time = 0.f;

inline uint64_t tIndex(const Grid &g, uint64_t v)
{
  if (g.tIndices64) {
    uint64_t r;
    std::memcpy(&r, g.tIndices + 8 * v, 8);
    return r;
  }
  uint32_t r;
  std::memcpy(&r, g.tIndices + 4 * v, 4);
  return r;
}

// interpolateTemporallyStructured (temporal_data_interpolation.ih:22-55):
// N values per voxel, regularly placed in [0, 1].
inline float temporalStructured(const Attr &at, int N, uint64_t base, float time)
{
  const float tf        = time * ((float)(N - 1));
  const uint32_t ts     = (uint32_t)tf;
  const float w         = tf - (float)ts;
  const uint32_t next   = (w == 0.f) ? ts : ts + 1;
  const float v0 = loadAttr(at, base + ts), v1 = loadAttr(at, base + next);
  return (1.f - w) * v0 + w * v1;
}

// interpolateTemporallyUnstructured (temporal_data_interpolation.ih:
// 117-190): per-voxel times, clamped at both ends, binary search between.
inline float temporalUnstructured(const Grid &g, const Attr &at, uint64_t voxel, float time)
{
  const uint64_t b = tIndex(g, voxel), e = tIndex(g, voxel + 1);
  const float t0 = g.tTimes[b];
  if (time <= t0)
    return loadAttr(at, b);
  const float t1 = g.tTimes[e - 1];
  if (time >= t1)
    return loadAttr(at, e - 1);
  const uint64_t n = e - b;
  if (n == 2) {
    const float w = (time - t0) * (1.f / (t1 - t0));
    return (1.f - w) * loadAttr(at, b) + w * loadAttr(at, e - 1);
  }
  uint64_t lower = 0, upper = n;
  while (lower <= upper) {
    const uint64_t mid = (lower + upper) / 2;
    const float tm     = g.tTimes[b + mid];
    if (time >= tm && time <= g.tTimes[b + mid + 1]) {
      lower = b + mid;
      upper = lower + 1;
      break;
    } else if (time < tm) {
      upper = mid;
    } else {
      lower = mid;
    }
  }
  const float tl = g.tTimes[lower], th = g.tTimes[upper];
  const float w  = (time - tl) * (1.f / (th - tl));
  return (1.f - w) * loadAttr(at, lower) + w * loadAttr(at, upper);
}

// Dense voxel load (VdbSampler_dense.ih:282-345): x fastest, 64-bit index;
// temporally varying data interpolated at the thread's sample time (the
// structured / unstructured handlers, VdbSampler_dense.ih:347-500).
inline float denseLoad(const Grid &g, uint32_t a, const vec3ui &o)
{
  const uint64_t idx = (uint64_t)o.z * g.activeSize.y * (uint64_t)g.activeSize.x +
                       (uint64_t)o.y * (uint64_t)g.activeSize.x + (uint64_t)o.x;
  if (g.temporalFormat == 1)
    return temporalStructured(g.denseAttr[a], g.numTimesteps, (uint64_t)g.numTimesteps * idx, t_time);
  if (g.temporalFormat == 2)
    return temporalUnstructured(g, g.denseAttr[a], idx, t_time);
  return loadAttr(g.denseAttr[a], idx);
}

// VdbSampler_traverseAndSample_dense (VdbSampler_traverseAndSample.ih:
// 313-349).
inline float traverseAndSampleDense(const Grid &g, const vec3i &ic, uint32_t a)
{
  const vec3ui o = toDomainOffset(ic, g.rootOrigin);
  if (inDomain(g.activeSize, o))
    return denseLoad(g, a, o);
  return g.background[a];
}

// LeafNodeAccess observer buffer of the sampling call in progress (set by
// orc_sample_observed only): the walk marks every leaf it reaches.
thread_local uint32_t *t_leafAccess = nullptr;

// Tree walk (VdbSampler_traverse, VdbSampler_traverseAndSample.ih:85-146,
// VdbSampleInner.ih.in:33-76): returns the leaf / error / empty voxel; a
// reached leaf is observed as VdbSampleInner.ih.in:68-74 does.
inline uint64_t traverse(const Grid &g,
                         const vec3ui &domainOffset,
                         uint32_t maxSamplingDepth)
{
  const vec3ui lo = {domainOffset.x & ~7u, domainOffset.y & ~7u,
                     domainOffset.z & ~7u};
  uint64_t node = 0;
  for (uint32_t l = 0; l < NUM_LEVELS - 1; ++l) {
    const uint64_t vo =
        node * levelNumVoxels(l) + offsetToLinear(l, lo.x, lo.y, lo.z);
    const uint32_t vo32 = (uint32_t)vo;
    const uint64_t v    = g.levels[l].voxels[vo32];
    if ((vLeaf(v) || vChild(v)) && (l + 1 > maxSamplingDepth))
      return mkError(l, vo32);
    if (vChild(v) && l + 1 < NUM_LEVELS - 1) {
      node = childIdx(v);
      continue;
    }
    if (t_leafAccess && vLeaf(v))
      t_leafAccess[leafIdx(v)] = 1;
    return v;
  }
  return 0;
}

// Leaf value for a found voxel (VdbSampler_sample_inner,
// VdbSampler_traverseAndSample.ih:153-205; packed handlers
// VdbSampler_packed_denseZYX.ih:77-187, VdbSampler_packed_tile.ih).
inline float sampleVoxel(const Grid &g,
                         uint64_t voxel,
                         const vec3ui &o,
                         uint32_t a)
{
  if (vLeaf(voxel)) {
    const uint64_t li = leafIdx(voxel);
    const Attr at{g.leafType,
                  leafFmt(voxel) == FMT_TILE ? g.packedTile[a].data()
                                             : g.packedDense[a].data(),
                  typeSize(g.leafType)};
    if (leafFmt(voxel) == FMT_TILE)
      return loadAttr(at, li);
    const uint64_t vi =
        li * 512 + (((uint64_t)(o.x & 7u)) << 6) + ((uint64_t)(o.y & 7u) << 3) +
        (uint64_t)(o.z & 7u);
    return loadAttr(at, vi);
  } else if (vError(voxel)) {
    const uint32_t level = (uint32_t)((voxel >> 8) & 0xff);
    const uint32_t off   = (uint32_t)(voxel >> 32);
    const range1f &r =
        g.levels[level].valueRange[(uint64_t)off * g.numAttributes + a];
    return 0.5f * (r.lower + r.upper);
  } else if (!inDomain(g.activeSize, o)) {
    return g.background[a];
  }
  return 0.f;
}

// VdbSampler_traverseAndSample (VdbSampler_traverseAndSample.ih:216-306).
inline float traverseAndSample(const Grid &g,
                               const vec3i &ic,
                               uint32_t a,
                               uint32_t depth)
{
  const vec3ui o = toDomainOffset(ic, g.rootOrigin);
  if (!inDomain(g.activeSize, o))
    return g.background[a];
  return sampleVoxel(g, traverse(g, o, depth), o, a);
}

inline float tap(const Grid &g, const vec3i &ic, uint32_t a, uint32_t depth)
{
  return g.dense ? traverseAndSampleDense(g, ic, a)
                 : traverseAndSample(g, ic, a, depth);
}

// ---------------------------------------------------------------------------
// Filters.
// ---------------------------------------------------------------------------

// Nearest (VdbSampler_nearest.ih:15-57): +0.5 for vertex-centered data.
inline float sampleNearest(const Grid &g, const vec3f &p, uint32_t a, uint32_t d)
{
  const float off = g.constantCellData ? 0.f : 0.5f;
  const vec3i ic  = {(int32_t)std::floor(p.x + off),
                    (int32_t)std::floor(p.y + off),
                    (int32_t)std::floor(p.z + off)};
  return tap(g, ic, a, d);
}

// Trilinear corner order (VdbSampler_trilinear.ih:17-26): (x,y,z) offsets
// 000,001,010,011,100,101,110,111, i.e. s[4x+2y+z].
inline void trilinearTaps(const Grid &g,
                          const vec3i &ic,
                          uint32_t a,
                          uint32_t d,
                          float s[8])
{
  // Stencil-block leaves (the cuda device's extension, no reference
  // counterpart): a base voxel inside a dense leaf takes all 8 corners from
  // that leaf's decoded 9^3 window.
  if (!g.dense && a < g.blockWin.size() && !g.blockWin[a].empty()) {
    const vec3ui o = toDomainOffset(ic, g.rootOrigin);
    if (inDomain(g.activeSize, o)) {
      const uint64_t v = traverse(g, o, d);
      if (vLeaf(v) && leafFmt(v) != FMT_TILE) {
        const float *w = &g.blockWin[a][leafIdx(v) * 729];
        const uint32_t lx = o.x & 7u, ly = o.y & 7u, lz = o.z & 7u;
        for (int k = 0; k < 8; ++k)
          s[k] = w[(lx + (k >> 2)) * 81 + (ly + ((k >> 1) & 1)) * 9 + lz + (k & 1)];
        return;
      }
    }
  }
  for (int o = 0; o < 8; ++o)
    s[o] = tap(g, {ic.x + (o >> 2), ic.y + ((o >> 1) & 1), ic.z + (o & 1)}, a, d);
}

// VdbSampler_interpolate_denseTrilinear (VdbSampler_trilinear.ih:378-399).
inline float sampleLinear(const Grid &g, const vec3f &p, uint32_t a, uint32_t d)
{
  const vec3i ic = {(int32_t)std::floor(p.x), (int32_t)std::floor(p.y),
                    (int32_t)std::floor(p.z)};
  const vec3f delta = {p.x - (float)ic.x, p.y - (float)ic.y, p.z - (float)ic.z};
  float s[8];
  trilinearTaps(g, ic, a, d, s);
  return lerp(delta.x,
              lerp(delta.y, lerp(delta.z, s[0], s[1]), lerp(delta.z, s[2], s[3])),
              lerp(delta.y, lerp(delta.z, s[4], s[5]), lerp(delta.z, s[6], s[7])));
}

// VdbSampler_computeGradient_denseTrilinear (VdbSampler_trilinear.ih:751-780).
inline vec3f gradientLinear(const Grid &g, const vec3f &p, uint32_t a, uint32_t d)
{
  const vec3i ic = {(int32_t)std::floor(p.x), (int32_t)std::floor(p.y),
                    (int32_t)std::floor(p.z)};
  const vec3f delta = {p.x - (float)ic.x, p.y - (float)ic.y, p.z - (float)ic.z};
  float s[8];
  trilinearTaps(g, ic, a, d, s);
  vec3f r;
  r.x = lerp(delta.y,
             lerp(delta.z, s[4] - s[0], s[5] - s[1]),
             lerp(delta.z, s[6] - s[2], s[7] - s[3]));
  r.y = lerp(delta.x,
             lerp(delta.z, s[2] - s[0], s[3] - s[1]),
             lerp(delta.z, s[6] - s[4], s[7] - s[5]));
  r.z = lerp(delta.x,
             lerp(delta.y, s[1] - s[0], s[3] - s[2]),
             lerp(delta.y, s[5] - s[4], s[7] - s[6]));
  return r;
}

// Tricubic after Lekien & Marsden (VdbSampler_tricubic.ih:9-389): the 64x64
// map from constraints (f, d/dx, d/dy, d/dz, d2/dxdy, d2/dxdz, d2/dydz,
// d3/dxdydz at the 8 corners, corner index 4x+2y+z) to coefficients
// c[16i+4j+k] of x^i y^j z^k is the tensor product of the 1D cubic Hermite
// map  a0=f0, a1=d0, a2=-3f0+3f1-2d0-d1, a3=2f0-2f1+d0+d1.  Each row is
// summed over its non-zero columns in ascending order, as the reference's
// expanded expressions are (pinned by tests/golden/tricubic_coeff_map.json).
struct TricubicMap {
  std::vector<int32_t> start, col;
  std::vector<float> w;
  TricubicMap()
  {
    // H[power][basis], basis order (f0, f1, d0, d1)
    const int H[4][4] = {{1, 0, 0, 0}, {0, 0, 1, 0}, {-3, 3, -2, -1},
                         {2, -2, 1, 1}};
    // constraint block for derivative flags (dx,dy,dz)
    auto block = [](int dx, int dy, int dz) {
      const int b[2][2][2] = {{{0, 24}, {16, 48}}, {{8, 40}, {32, 56}}};
      return b[dx][dy][dz];
    };
    start.push_back(0);
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j)
        for (int k = 0; k < 4; ++k) {
          int rowW[64] = {0};
          for (int ux = 0; ux < 4; ++ux)
            for (int uy = 0; uy < 4; ++uy)
              for (int uz = 0; uz < 4; ++uz) {
                const int wgt = H[i][ux] * H[j][uy] * H[k][uz];
                if (!wgt)
                  continue;
                // basis u: 0->f corner 0, 1->f corner 1, 2->d corner 0, 3->d
                // corner 1
                const int cx = ux & 1, cy = uy & 1, cz = uz & 1;
                const int dx = ux >> 1, dy = uy >> 1, dz = uz >> 1;
                const int c  = block(dx, dy, dz) + 4 * cx + 2 * cy + cz;
                rowW[c] += wgt;
              }
          for (int c = 0; c < 64; ++c)
            if (rowW[c]) {
              col.push_back(c);
              w.push_back((float)rowW[c]);
            }
          start.push_back((int32_t)col.size());
        }
  }
};
static const TricubicMap &tricubicMap()
{
  static TricubicMap m;
  return m;
}

// 4x4x4 stencil, offsets -1..2, x outermost (VdbSampler_tricubic.ih:
// 393-409) then constraints by central differences (:411-513).
inline void tricubicCoefficients(const Grid &g,
                                 const vec3i &ic,
                                 uint32_t a,
                                 uint32_t d,
                                 float coef[64])
{
  float s[64];
  for (int o = 0; o < 64; ++o)
    s[o] = tap(g, {ic.x + (o >> 4) - 1, ic.y + ((o >> 2) & 3) - 1, ic.z + (o & 3) - 1},
               a, d);
  auto S = [&](int x, int y, int z) { return s[(x + 1) * 16 + (y + 1) * 4 + (z + 1)]; };
  float ctr[64];
  for (int c = 0; c < 8; ++c) {
    const int x = c >> 2, y = (c >> 1) & 1, z = c & 1;
    ctr[c]      = S(x, y, z);
    ctr[8 + c]  = 0.5f * (-S(x - 1, y, z) + S(x + 1, y, z));
    ctr[16 + c] = 0.5f * (-S(x, y - 1, z) + S(x, y + 1, z));
    ctr[24 + c] = 0.5f * (-S(x, y, z - 1) + S(x, y, z + 1));
    ctr[32 + c] = 0.25f * (S(x - 1, y - 1, z) - S(x - 1, y + 1, z) -
                           S(x + 1, y - 1, z) + S(x + 1, y + 1, z));
    ctr[40 + c] = 0.25f * (S(x - 1, y, z - 1) - S(x - 1, y, z + 1) -
                           S(x + 1, y, z - 1) + S(x + 1, y, z + 1));
    ctr[48 + c] = 0.25f * (S(x, y - 1, z - 1) - S(x, y - 1, z + 1) -
                           S(x, y + 1, z - 1) + S(x, y + 1, z + 1));
    ctr[56 + c] =
        0.125f * (-S(x - 1, y - 1, z - 1) + S(x - 1, y - 1, z + 1) +
                  S(x - 1, y + 1, z - 1) - S(x - 1, y + 1, z + 1) +
                  S(x + 1, y - 1, z - 1) - S(x + 1, y - 1, z + 1) -
                  S(x + 1, y + 1, z - 1) + S(x + 1, y + 1, z + 1));
  }
  const TricubicMap &m = tricubicMap();
  for (int r = 0; r < 64; ++r) {
    float acc = m.w[m.start[r]] * ctr[m.col[m.start[r]]];
    for (int e = m.start[r] + 1; e < m.start[r + 1]; ++e)
      acc = acc + m.w[e] * ctr[m.col[e]];
    coef[r] = acc;
  }
}

// Polynomial evaluation (VdbSampler_tricubic.ih:541-580, varying path).
inline float sampleCubic(const Grid &g, const vec3f &p, uint32_t a, uint32_t d)
{
  const vec3i ic = {(int32_t)std::floor(p.x), (int32_t)std::floor(p.y),
                    (int32_t)std::floor(p.z)};
  float c[64];
  tricubicCoefficients(g, ic, a, d, c);
  const vec3f dl = {p.x - (float)ic.x, p.y - (float)ic.y, p.z - (float)ic.z};
  const float x[4] = {1.f, dl.x, dl.x * dl.x, dl.x * dl.x * dl.x};
  const float y[4] = {1.f, dl.y, dl.y * dl.y, dl.y * dl.y * dl.y};
  const float z[4] = {1.f, dl.z, dl.z * dl.z, dl.z * dl.z * dl.z};
  float result = 0.f;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k)
        result += c[16 * i + 4 * j + k] * x[i] * y[j] * z[k];
  return result;
}

inline vec3f gradientCubic(const Grid &g, const vec3f &p, uint32_t a, uint32_t d)
{
  const vec3i ic = {(int32_t)std::floor(p.x), (int32_t)std::floor(p.y),
                    (int32_t)std::floor(p.z)};
  float c[64];
  tricubicCoefficients(g, ic, a, d, c);
  const vec3f dl = {p.x - (float)ic.x, p.y - (float)ic.y, p.z - (float)ic.z};
  const float x[4] = {1.f, dl.x, dl.x * dl.x, dl.x * dl.x * dl.x};
  const float y[4] = {1.f, dl.y, dl.y * dl.y, dl.y * dl.y * dl.y};
  const float z[4] = {1.f, dl.z, dl.z * dl.z, dl.z * dl.z * dl.z};
  vec3f r = {0.f, 0.f, 0.f};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        const float cc = c[16 * i + 4 * j + k];
        if (i > 0)
          r.x += cc * (float)i * x[i - 1] * y[j] * z[k];
        if (j > 0)
          r.y += cc * (float)j * x[i] * y[j - 1] * z[k];
        if (k > 0)
          r.z += cc * (float)k * x[i] * y[j] * z[k - 1];
      }
  return r;
}

inline float sampleAt(const Grid &g, int filter, const vec3f &p, uint32_t a, uint32_t d)
{
  switch (filter) {
  case F_NEAREST:
    return sampleNearest(g, p, a, d);
  case F_CUBIC:
    return sampleCubic(g, p, a, d);
  default:
    return sampleLinear(g, p, a, d);
  }
}

// VdbSampler_iterator_computeSample_varying (VdbSampler.ispc:341-374).
inline float sampleObject(const Grid &g, int filter, const vec3f &oc, uint32_t a)
{
  return sampleAt(g, filter, xfmPoint(g.o2i, oc), a, NUM_LEVELS - 1);
}

// ---------------------------------------------------------------------------
// Value ranges (VdbSampler.ispc:383-557, VdbVolume.cpp:338-392).
// ---------------------------------------------------------------------------
static range1f nodeValueRange(const Grid &g,
                              uint64_t voxel,
                              const vec3ui &dOff,
                              const uint32_t rx[2],
                              const uint32_t ry[2],
                              const uint32_t rz[2],
                              uint32_t a)
{
  const float bgOut = g.background[a];
  range1f r;
  if (g.dense) {
    if (!inDomain(g.activeSize, dOff))
      return {bgOut, bgOut};
    for (uint32_t x = rx[0]; x < rx[1]; ++x)
      for (uint32_t y = ry[0]; y < ry[1]; ++y)
        for (uint32_t z = rz[0]; z < rz[1]; ++z) {
          const vec3ui o = {dOff.x + x, dOff.y + y, dOff.z + z};
          if (!(o.x < (uint32_t)g.denseDims.x && o.y < (uint32_t)g.denseDims.y &&
                o.z < (uint32_t)g.denseDims.z))
            continue;
          const uint64_t idx = (uint64_t)o.z * g.activeSize.y * (uint64_t)g.activeSize.x +
                               (uint64_t)o.y * (uint64_t)g.activeSize.x + (uint64_t)o.x;
          if (g.temporalFormat == 1) {
            // every time step (VdbSampler_dense.ih:107-175)
            for (int t = 0; t < g.numTimesteps; ++t) {
              const float v = loadAttr(g.denseAttr[a], (uint64_t)g.numTimesteps * idx + t);
              r.lower       = fmin_(r.lower, v);
              r.upper       = fmax_(r.upper, v);
            }
          } else if (g.temporalFormat == 2) {
            // the voxel's own range, then box_extend (VdbSampler_dense.ih:
            // 177-266, temporal_data_interpolation.ih:226-260)
            range1f vr;
            for (uint64_t i = tIndex(g, idx); i < tIndex(g, idx + 1); ++i) {
              const float v = loadAttr(g.denseAttr[a], i);
              vr.lower      = fmin_(vr.lower, v);
              vr.upper      = fmax_(vr.upper, v);
            }
            r.lower = fmin_(r.lower, vr.lower);
            r.upper = fmax_(r.upper, vr.upper);
          } else {
            const float v = denseLoad(g, a, o);
            r.lower       = fmin_(r.lower, v);
            r.upper       = fmax_(r.upper, v);
          }
        }
    return r;
  }
  if (!vLeaf(voxel)) {
    if (!inDomain(g.activeSize, dOff))
      return {bgOut, bgOut};
    return {0.f, 0.f};
  }
  const uint64_t li = leafIdx(voxel);
  if (leafFmt(voxel) == FMT_TILE) {
    const Attr at{g.leafType, g.packedTile[a].data(), typeSize(g.leafType)};
    const float v = loadAttr(at, li);
    return {v, v};
  }
  const Attr at{g.leafType, g.packedDense[a].data(), typeSize(g.leafType)};
  for (uint32_t x = rx[0]; x < rx[1]; ++x)
    for (uint32_t y = ry[0]; y < ry[1]; ++y)
      for (uint32_t z = rz[0]; z < rz[1]; ++z) {
        const float v = loadAttr(at, li * 512 + (x << 6) + (y << 3) + z);
        r.lower       = fmin_(r.lower, v);
        r.upper       = fmax_(r.upper, v);
      }
  return r;
}

static range1f leafValueRange(const Grid &g, const vec3ui &center, uint32_t a)
{
  const uint32_t win[3][2] = {{7, 8}, {0, 8}, {0, 2}};
  range1f range;
  for (int ix = 0; ix < 3; ++ix)
    for (int iy = 0; iy < 3; ++iy)
      for (int iz = 0; iz < 3; ++iz) {
        const vec3i nodeOrigin = {
            g.rootOrigin.x + (int32_t)center.x + (ix - 1) * 8,
            g.rootOrigin.y + (int32_t)center.y + (iy - 1) * 8,
            g.rootOrigin.z + (int32_t)center.z + (iz - 1) * 8};
        const vec3ui dOff = toDomainOffset(nodeOrigin, g.rootOrigin);
        uint64_t voxel    = 0;
        if (!g.dense && inDomain(g.activeSize, dOff))
          voxel = traverse(g, dOff, NUM_LEVELS - 1);
        const range1f nr =
            nodeValueRange(g, voxel, dOff, win[ix], win[iy], win[iz], a);
        if (!std::isnan(nr.lower))
          range.lower = fmin_(range.lower, nr.lower);
        if (!std::isnan(nr.upper))
          range.upper = fmax_(range.upper, nr.upper);
      }
  return range;
}

// ---------------------------------------------------------------------------
// Tree build (VdbVolume.cpp:71-331, :584-1062).
// ---------------------------------------------------------------------------
static vec3ui nodeOriginOf(const vec3ui &o, uint32_t level)
{
  const uint32_t mask = ~(levelRes(level) - 1);
  return {o.x & mask, o.y & mask, o.z & mask};
}

static void buildTree(Grid &g, bool packed, const std::vector<uint64_t> &packedIndex)
{
  // binLeavesPerLevel (VdbVolume.cpp:86-106)
  std::vector<std::vector<uint64_t>> binned(NUM_LEVELS);
  for (uint64_t i = 0; i < g.numLeaves; ++i) {
    if (g.leafLevel[i] == 0)
      throw std::runtime_error("there must not be any leaf nodes on level 0");
    if (g.leafLevel[i] >= NUM_LEVELS)
      throw std::runtime_error("invalid node level for this vdb configuration");
    binned[g.leafLevel[i]].push_back(i);
  }
  // computeLeafOffsets (:114-123)
  std::vector<vec3ui> off(g.numLeaves);
  for (uint64_t i = 0; i < g.numLeaves; ++i)
    off[i] = {(uint32_t)(g.leafOrigin[i].x - g.rootOrigin.x),
              (uint32_t)(g.leafOrigin[i].y - g.rootOrigin.y),
              (uint32_t)(g.leafOrigin[i].z - g.rootOrigin.z)};
  // allocateInnerLevels (:160-225): count distinct node origins bottom-up.
  auto less = [](const vec3ui &a, const vec3ui &b) {
    return (int32_t)a.x < (int32_t)b.x ||
           (a.x == b.x && (int32_t)a.y < (int32_t)b.y) ||
           (a.x == b.x && a.y == b.y && (int32_t)a.z < (int32_t)b.z);
  };
  auto eq = [](const vec3ui &a, const vec3ui &b) {
    return a.x == b.x && a.y == b.y && a.z == b.z;
  };
  std::vector<vec3ui> old;
  for (uint32_t i = 0; i + 1 < NUM_LEVELS; ++i) {
    const uint32_t l = NUM_LEVELS - i - 1;
    std::vector<vec3ui> inner;
    for (uint64_t leaf : binned[l])
      inner.push_back(nodeOriginOf(off[leaf], l - 1));
    for (const vec3ui &o : old)
      inner.push_back(nodeOriginOf(o, l - 1));
    std::sort(inner.begin(), inner.end(), less);
    inner.erase(std::unique(inner.begin(), inner.end(), eq), inner.end());
    old = inner;
    Level &lv = g.levels[l - 1];
    lv.numNodes = 0;
    lv.origin.assign(inner.size(), {0, 0, 0});
    lv.voxels.assign(inner.size() * levelNumVoxels(l - 1), 0);
    lv.valueRange.assign(inner.size() * levelNumVoxels(l - 1) * g.numAttributes,
                         range1f());
  }
  // insertLeaves (:244-331)
  g.levels[0].numNodes = 1;
  for (uint32_t leafLevel = 0; leafLevel < NUM_LEVELS; ++leafLevel)
    for (uint64_t idx : binned[leafLevel]) {
      const vec3ui &o   = off[idx];
      uint64_t nodeIndex = 0;
      for (uint32_t l = 0; l < leafLevel; ++l) {
        const uint64_t v = nodeIndex * levelNumVoxels(l) + offsetToLinear(l, o.x, o.y, o.z);
        uint64_t &voxel  = g.levels[l].voxels[v];
        if (vLeaf(voxel)) {
          throw std::runtime_error(
              "Attempted to insert a leaf node into a leaf node");
        } else if (vEmpty(voxel)) {
          const uint32_t nl = l + 1;
          if (nl < leafLevel) {
            nodeIndex = g.levels[nl].numNodes++;
            voxel     = mkChild(nodeIndex);
            g.levels[nl].origin[nodeIndex] = nodeOriginOf(o, nl);
          } else {
            voxel = mkLeaf(packed ? packedIndex[idx] : idx, g.leafFormat[idx], 0);
          }
        } else {
          nodeIndex = childIdx(voxel);
        }
      }
    }
  // computeValueRanges (:338-392)
  std::vector<range1f> ranges(g.numLeaves * g.numAttributes);
  parallelFor((int64_t)g.numLeaves, 0, 256, [&](int64_t idx) {
    for (uint32_t a = 0; a < g.numAttributes; ++a)
      ranges[idx * g.numAttributes + a] = leafValueRange(g, off[idx], a);
  });
  for (uint64_t idx = 0; idx < g.numLeaves; ++idx) {
    uint64_t nodeIndex = 0;
    for (uint32_t l = 0; l < g.leafLevel[idx]; ++l) {
      Level &lv        = g.levels[l];
      const uint64_t v = nodeIndex * levelNumVoxels(l) +
                         offsetToLinear(l, off[idx].x, off[idx].y, off[idx].z);
      for (uint32_t a = 0; a < g.numAttributes; ++a) {
        range1f &r        = lv.valueRange[v * g.numAttributes + a];
        const range1f &lr = ranges[idx * g.numAttributes + a];
        r.lower           = std::min(r.lower, lr.lower);
        r.upper           = std::max(r.upper, lr.upper);
      }
      const uint64_t voxel = lv.voxels[v];
      if (vLeaf(voxel))
        break;
      nodeIndex = childIdx(voxel);
    }
  }
  // aggregate volume range (:1047-1057)
  g.volumeRange.assign(g.numAttributes, range1f());
  for (uint32_t a = 0; a < g.numAttributes; ++a)
    for (uint64_t i = 0; i < levelNumVoxels(0); ++i) {
      const range1f &r = g.levels[0].valueRange[i * g.numAttributes + a];
      g.volumeRange[a].lower = std::min(g.volumeRange[a].lower, r.lower);
      g.volumeRange[a].upper = std::max(g.volumeRange[a].upper, r.upper);
    }
}

static void finishBounds(Grid &g, const float lo[3], const float hi[3])
{
  // domain box (VdbVolume.cpp:808-811) and object bounds (:814-824)
  g.domain[0] = lo[0] - (float)g.rootOrigin.x;
  g.domain[1] = lo[1] - (float)g.rootOrigin.y;
  g.domain[2] = lo[2] - (float)g.rootOrigin.z;
  g.domain[3] = hi[0] - (float)g.rootOrigin.x;
  g.domain[4] = hi[1] - (float)g.rootOrigin.y;
  g.domain[5] = hi[2] - (float)g.rootOrigin.z;
  const float inf = std::numeric_limits<float>::infinity();
  float b[6]      = {inf, inf, inf, -inf, -inf, -inf};
  for (int i = 0; i < 8; ++i) {
    const vec3f v = {(i & 1) ? hi[0] : lo[0], (i & 2) ? hi[1] : lo[1],
                     (i & 4) ? hi[2] : lo[2]};
    const vec3f w = xfmPoint(g.i2o, v);
    b[0] = std::min(b[0], w.x);
    b[1] = std::min(b[1], w.y);
    b[2] = std::min(b[2], w.z);
    b[3] = std::max(b[3], w.x);
    b[4] = std::max(b[4], w.y);
    b[5] = std::max(b[5], w.z);
  }
  std::memcpy(g.bounds, b, sizeof(b));
}

// ---------------------------------------------------------------------------
// DDA (Dda.ih:17-309), hierarchical step (HDDA.ih.in:24-101), voxel queries
// (VdbQueryVoxelDense.ih:17-161, VdbQueryVoxel.ih.in:42-116).
// ---------------------------------------------------------------------------
struct Dda {
  uint32_t level;
  float t;
  vec3f org, dir;
  int32_t idx[12];
  float tNext[12], tDelta[12];
  int32_t idxDelta[12];
};
inline int ox(int l) { return l; }
inline int oy(int l) { return 4 + l; }
inline int oz(int l) { return 8 + l; }

inline int dirSign(float v) { return (int)(0 < v) - (int)(v < 0); }
inline float dirRcp(float v)
{
  return (v == 0) ? std::numeric_limits<float>::infinity() : divide_safe(v);
}
inline float planeT(float plane, float org, float inv)
{
  const float t = (plane - org) * inv;
  return (plane == org || std::isnan(t)) ? std::numeric_limits<float>::infinity() : t;
}
inline int32_t clampToCell1(float f, int32_t res)
{
  return ((int32_t)std::floor(fmax_(f, 0.f))) & ~(res - 1);
}

static void ddaInit(const vec3f &org, const vec3f &dir, float tMin, uint32_t level, Dda &d)
{
  const vec3f oo = {org.x + tMin * dir.x, org.y + tMin * dir.y, org.z + tMin * dir.z};
  const int sg[3]  = {dirSign(dir.x), dirSign(dir.y), dirSign(dir.z)};
  const float iv[3] = {dirRcp(dir.x), dirRcp(dir.y), dirRcp(dir.z)};
  d.level = std::min<uint32_t>(level, NUM_LEVELS - 1);
  d.t     = tMin;
  d.org   = org;
  d.dir   = dir;
  const float o3[3] = {oo.x, oo.y, oo.z};
  const float g3[3] = {org.x, org.y, org.z};
  for (uint32_t l = 0; l <= d.level; ++l) {
    const int32_t res = (int32_t)levelRes(l + 1);
    for (int ax = 0; ax < 3; ++ax) {
      const int32_t id  = clampToCell1(o3[ax], res);
      const float plane = (float)(id + res * (int)(sg[ax] >= 0));
      const int k       = ax * 4 + (int)l;
      d.idx[k]          = id;
      d.idxDelta[k]     = sg[ax] * res;
      d.tDelta[k]       = (float)res * std::fabs(iv[ax]);
      d.tNext[k]        = planeT(plane, g3[ax], iv[ax]);
    }
  }
}

static void ddaReinitBelow(Dda &d, uint32_t level, int32_t dx, int32_t dy, int32_t dz)
{
  const float iv[3] = {dirRcp(d.dir.x), dirRcp(d.dir.y), dirRcp(d.dir.z)};
  const int sg[3]   = {dirSign(d.dir.x), dirSign(d.dir.y), dirSign(d.dir.z)};
  float oo[3] = {d.org.x + d.t * d.dir.x, d.org.y + d.t * d.dir.y,
                 d.org.z + d.t * d.dir.z};
  if (dx != 0)
    oo[0] = oo[0] + (float)sg[0] * 1e-2f;
  else if (dy != 0)
    oo[1] = oo[1] + (float)sg[1] * 1e-2f;
  else
    oo[2] = oo[2] + (float)sg[2] * 1e-2f;
  const float g3[3] = {d.org.x, d.org.y, d.org.z};
  for (uint32_t l = level + 1; l <= d.level; ++l) {
    const int32_t res = (int32_t)levelRes(l + 1);
    for (int ax = 0; ax < 3; ++ax) {
      const int k  = ax * 4 + (int)l;
      d.idx[k]     = clampToCell1(oo[ax], res);
      const float plane = (float)(d.idx[k] + res * (int)(sg[ax] >= 0));
      d.tNext[k]   = planeT(plane, g3[ax], iv[ax]);
    }
  }
}

static void ddaStep(Dda &d, uint32_t l)
{
  const float tx = d.tNext[ox(l)], ty = d.tNext[oy(l)], tz = d.tNext[oz(l)];
  const float m  = fmin_(fmin_(tx, ty), tz);
  int k;
  if (m == tx)
    k = ox(l);
  else if (m == ty)
    k = oy(l);
  else
    k = oz(l);
  d.t        = d.tNext[k];
  d.tNext[k] = d.tNext[k] + d.tDelta[k];
  d.idx[k]   = d.idx[k] + d.idxDelta[k];
}

struct VoxelDesc {
  uint32_t level;
  bool isEmpty;
  bool isLeaf;
  uint64_t nodeIndex;
  uint64_t voxel;
  range1f valueRange;
};

struct ValueRanges {
  std::vector<range1f> ranges;
  range1f minMax;
  bool overlaps(const range1f &r) const
  {
    if (ranges.empty())
      return true;
    // overlaps1f(box1, box2) = box1.upper >= box2.lower && box1.lower <= box2.upper
    if (!(minMax.upper >= r.lower && minMax.lower <= r.upper))
      return false;
    for (const range1f &q : ranges)
      if (q.upper >= r.lower && q.lower <= r.upper)
        return true;
    return false;
  }
  void computeMinMax()
  {
    minMax.lower = std::numeric_limits<float>::infinity();
    minMax.upper = -std::numeric_limits<float>::infinity();
    for (const range1f &q : ranges) {
      minMax.lower = fmin_(minMax.lower, q.lower);
      minMax.upper = fmax_(minMax.upper, q.upper);
    }
  }
};

static void queryVoxelDense(const Grid &g, int32_t x, int32_t y, int32_t z,
                            uint32_t depth, uint32_t a, const ValueRanges &vr,
                            VoxelDesc &desc)
{
  desc.level      = depth;
  const vec3ui o = {(uint32_t)x, (uint32_t)y, (uint32_t)z};
  if (!inDomain(g.activeSize, o)) {
    desc.isEmpty = true;
    return;
  }
  const uint64_t nx1 = (g.activeSize.x + levelRes(1) - 1) >> TOTAL_LOG_RES[1];
  const uint64_t ny1 = (g.activeSize.y + levelRes(1) - 1) >> TOTAL_LOG_RES[1];
  const uint64_t l1 = (uint64_t)(o.z >> TOTAL_LOG_RES[1]) * ny1 * nx1 +
                      (uint64_t)(o.y >> TOTAL_LOG_RES[1]) * nx1 +
                      (uint64_t)(o.x >> TOTAL_LOG_RES[1]);
  uint32_t lvl;
  if (depth >= 2) {
    desc.isLeaf        = true;
    const uint64_t nx2 = (g.activeSize.x + levelRes(2) - 1) >> TOTAL_LOG_RES[2];
    const uint64_t ny2 = (g.activeSize.y + levelRes(2) - 1) >> TOTAL_LOG_RES[2];
    const uint64_t l2  = (uint64_t)(o.z >> TOTAL_LOG_RES[2]) * ny2 * nx2 +
                        (uint64_t)(o.y >> TOTAL_LOG_RES[2]) * nx2 +
                        (uint64_t)(o.x >> TOTAL_LOG_RES[2]);
    desc.nodeIndex = l1 * levelNumVoxels(1) + l2 * levelNumVoxels(2) +
                     offsetToLinear(2, o.x, o.y, o.z);
    lvl = 2;
  } else if (depth == 1) {
    desc.isLeaf    = false;
    desc.nodeIndex = l1 * levelNumVoxels(1) + offsetToLinear(1, o.x, o.y, o.z);
    lvl            = 1;
  } else {
    desc.isLeaf    = false;
    desc.nodeIndex = offsetToLinear(0, o.x, o.y, o.z);
    lvl            = 0;
  }
  desc.voxel      = g.levels[lvl].voxels[desc.nodeIndex];
  desc.valueRange = g.levels[lvl].valueRange[desc.nodeIndex * g.numAttributes + a];
  desc.isEmpty    = !vr.overlaps(desc.valueRange);
}

static void queryVoxelSparse(const Grid &g, int32_t x, int32_t y, int32_t z,
                             uint32_t depth, uint32_t a, const ValueRanges &vr,
                             VoxelDesc &desc)
{
  desc.nodeIndex = 0;
  for (uint32_t l = 0; l + 1 < NUM_LEVELS; ++l) {
    const Level &lv  = g.levels[l];
    const uint64_t vo = offsetToLinear(l, (uint64_t)(int64_t)x, (uint64_t)(int64_t)y,
                                       (uint64_t)(int64_t)z) +
                        desc.nodeIndex * levelNumVoxels(l);
    const uint32_t vo32 = (uint32_t)vo;
    desc.voxel          = lv.voxels[vo32];
    desc.valueRange     = lv.valueRange[(uint64_t)vo32 * g.numAttributes + a];
    desc.level          = l;
    desc.isEmpty        = vEmpty(desc.voxel) || !vr.overlaps(desc.valueRange);
    if (desc.isEmpty)
      return;
    const bool atQueryDepth = (l + 1 > depth);
    const bool isLeafPtr    = vLeaf(desc.voxel);
    if (isLeafPtr && !atQueryDepth) {
      desc.isLeaf = true;
      desc.level  = l + 1;
    }
    if (l + 2 >= NUM_LEVELS)
      return;
    if (atQueryDepth || isLeafPtr)
      return;
    desc.nodeIndex = childIdx(desc.voxel);
  }
}

static bool hddaStepL(uint32_t L, const VoxelDesc &desc, Dda &d)
{
  const bool lowest = (desc.level == L);
  bool stepped      = false;
  if (L + 1 < NUM_LEVELS) {
    if (lowest) {
      const int32_t x0 = d.idx[ox(L)], y0 = d.idx[oy(L)], z0 = d.idx[oz(L)];
      ddaStep(d, L);
      stepped = true;
      if (L < d.level)
        ddaReinitBelow(d, L, d.idx[ox(L)] - x0, d.idx[oy(L)] - y0, d.idx[oz(L)] - z0);
    } else {
      if (hddaStepL(L + 1, desc, d)) {
        const int32_t res = (int32_t)levelRes(L + 1);
        const bool left   = d.idx[ox(L + 1)] < d.idx[ox(L)] ||
                          d.idx[oy(L + 1)] < d.idx[oy(L)] ||
                          d.idx[oz(L + 1)] < d.idx[oz(L)] ||
                          d.idx[ox(L + 1)] >= d.idx[ox(L)] + res ||
                          d.idx[oy(L + 1)] >= d.idx[oy(L)] + res ||
                          d.idx[oz(L + 1)] >= d.idx[oz(L)] + res;
        if (left) {
          ddaStep(d, L);
          stepped = true;
        }
      }
    }
  } else {
    ddaStep(d, L);
    stepped = true;
  }
  return stepped;
}

// Per-ray loop bounds shared with the CUDA device (a ray whose float t
// stops advancing ends instead of spinning): DDA steps per ray, march steps
// per bisection interval, hits per ray.
constexpr uint32_t MAX_DDA_STEPS   = 1u << 26;
constexpr uint32_t MAX_MARCH_STEPS = 1u << 24;
constexpr uint32_t MAX_HITS        = 1u << 24;

struct IntervalIt {
  const Grid *g;
  uint32_t attr;
  float tMax;
  float nominalDeltaT;
  uint32_t budget;
  Dda dda;
};

struct Interval {
  range1f t, v;
  float nominalDeltaT;
};

// intersectBox (math/box_utility.ih:63-77).
static range1f intersectBox(const vec3f &o, const vec3f &d, const float *box,
                            const range1f &lim)
{
  const float inv[3] = {divide_safe(d.x), divide_safe(d.y), divide_safe(d.z)};
  const float org[3] = {o.x, o.y, o.z};
  float lo = lim.lower, hi = lim.upper;
  float mn[3], mx[3];
  for (int a = 0; a < 3; ++a) {
    const float t0 = (box[a] - org[a]) * inv[a];
    const float t1 = (box[3 + a] - org[a]) * inv[a];
    mn[a]          = fmin_(t0, t1);
    mx[a]          = fmax_(t0, t1);
  }
  range1f r;
  r.lower = fmax_(fmax_(fmax_(mn[0], mn[1]), mn[2]), lo);
  r.upper = fmin_(fmin_(fmin_(mx[0], mx[1]), mx[2]), hi);
  return r;
}

// VdbIterator_Initialize (VdbIterator.ispc:36-94).
static void intervalInit(IntervalIt &it, const Grid &g, uint32_t attr, uint32_t depth,
                         const vec3f &origin, const vec3f &direction,
                         const range1f &tRange)
{
  it.g    = &g;
  it.attr = attr;
  const vec3f root = {(float)g.rootOrigin.x, (float)g.rootOrigin.y, (float)g.rootOrigin.z};
  vec3f org        = xfmPoint(g.o2i, origin);
  org              = {org.x - root.x, org.y - root.y, org.z - root.z};
  const vec3f dir  = xfmVector(g.o2i, direction);
  it.nominalDeltaT = fmin_(fmin_(1.f * rcp_safe(std::fabs(dir.x)), 1.f * rcp_safe(std::fabs(dir.y))),
                           1.f * rcp_safe(std::fabs(dir.z)));
  const range1f ti = intersectBox(org, dir, g.domain, tRange);
  it.budget        = MAX_DDA_STEPS;
  if (ti.upper <= ti.lower) {
    it.tMax  = -std::numeric_limits<float>::infinity();
    it.dda.t = 0;
  } else {
    it.tMax = ti.upper;
    ddaInit(org, dir, ti.lower, depth, it.dda);
  }
}

// VdbIterator_iterateIntervalInternal (VdbIterator.ispc:96-159).
static bool intervalIterate(IntervalIt &it, const ValueRanges &vr, Interval &out)
{
  if (!(it.dda.t <= it.tMax))
    return false;
  VoxelDesc desc{};
  const Grid &g = *it.g;
  while (it.dda.t <= it.tMax) {
    const uint32_t L = it.dda.level;
    if (g.dense)
      queryVoxelDense(g, it.dda.idx[ox(L)], it.dda.idx[oy(L)], it.dda.idx[oz(L)], L,
                      it.attr, vr, desc);
    else
      queryVoxelSparse(g, it.dda.idx[ox(L)], it.dda.idx[oy(L)], it.dda.idx[oz(L)], L,
                       it.attr, vr, desc);
    if (!desc.isEmpty)
      break;
    if (it.budget-- == 0) {
      it.tMax = -std::numeric_limits<float>::infinity();
      return false;
    }
    hddaStepL(0, desc, it.dda);
  }
  if (it.dda.t < it.tMax) {
    out.v       = desc.valueRange;
    out.t.lower = it.dda.t;
    if (it.budget-- == 0) {
      it.tMax = -std::numeric_limits<float>::infinity();
      return false;
    }
    hddaStepL(0, desc, it.dda);
    out.t.upper       = fmin_(it.dda.t, it.tMax);
    out.nominalDeltaT = it.nominalDeltaT;
    return true;
  }
  return false;
}

// mapToMaxIteratorDepth for VDB / dense (IteratorContext.cpp:49-174).
static int hintToDepth(float hint)
{
  hint = std::max(std::min(1.f, hint), 0.f);
  const float th[4] = {0.f, 0.2f, 0.4f, 0.8f};
  int depth         = -1;
  for (int i = 0; i < 4; ++i) {
    if (hint >= th[i])
      depth = i;
    else
      break;
  }
  return depth;
}

// ---------------------------------------------------------------------------
// Hit iteration: bisection (Iterator.ih:17-197) driven by the default hit
// iterator (DefaultIterator.ispc:168-258).
// ---------------------------------------------------------------------------
struct HitRec {
  float t, sample, epsilon;
};

static float bisect(const Grid &g, int filter, uint32_t a, const vec3f &o, const vec3f &d,
                    float t0, float sample0, float t, float sample, float iso,
                    float tol, float &error)
{
  const int maxIter = 10;
  int iter          = 0;
  float tMid        = 0.f;
  while (iter < maxIter) {
    tMid  = 0.5f * (t0 + t);
    error = 0.5f * (t - t0);
    if (error < tol)
      break;
    const float sMid =
        sampleObject(g, filter, {o.x + tMid * d.x, o.y + tMid * d.y, o.z + tMid * d.z}, a);
    if (std::isnan(sMid)) {
      if (std::fabs(iso - sample0) < std::fabs(iso - sample))
        return t0;
      return t;
    }
    if (sMid == iso || (iso - sample0) * (iso - sMid) < 0.f) {
      t      = tMid;
      sample = sMid;
    } else if (sample == iso || (iso - sample) * (iso - sMid) < 0.f) {
      t0      = tMid;
      sample0 = sMid;
    } else {
      return std::numeric_limits<float>::infinity();
    }
    iter++;
  }
  return tMid;
}

static bool intersectBisection(const Grid &g, int filter, uint32_t a, const vec3f &o,
                               const vec3f &d, const range1f &tr, float step,
                               const std::vector<float> &values, HitRec &hit)
{
  const float inf = std::numeric_limits<float>::infinity();
  auto S = [&](float t) {
    return sampleObject(g, filter, {o.x + t * d.x, o.y + t * d.y, o.z + t * d.z}, a);
  };
  float t0      = tr.lower;
  float sample0 = S(t0);
  {
    int iters = 0;
    while ((float)iters < 10.f && std::isnan(sample0) && t0 < tr.upper) {
      t0 += fmax_(1e-5f, 1e-5f * step);
      sample0 = S(t0);
      iters++;
    }
  }
  float t;
  for (uint32_t march = 0; t0 < tr.upper && march < MAX_MARCH_STEPS; ++march) {
    const float h = fmin_(step, tr.upper - t0);
    t             = t0 + h;
    float sample  = S(t);
    float ts      = t;
    {
      int iters = 0;
      while ((float)iters < 10.f && std::isnan(sample) && ts > t0) {
        ts -= fmax_(1e-5f, 1e-5f * step);
        sample = S(ts);
        iters++;
      }
    }
    float tHit = inf, eps = inf, value = inf;
    for (size_t i = 0; i < values.size(); ++i) {
      const float vi = values[i];
      if (std::fabs(sample0 - vi) < 1e-6f) {
        if (t0 < tHit && t0 <= tr.upper) {
          tHit  = t0;
          value = vi;
          eps   = 0.125f * step;
        }
      } else if (!std::isnan(sample0 + sample) && (vi - sample0) * (vi - sample) < 0.f) {
        float err;
        const float tIso = bisect(g, filter, a, o, d, t0, sample0, ts, sample, vi,
                                  fmin_(1e-6f, 0.01f * h), err);
        if (tIso < tHit && tIso <= tr.upper) {
          tHit  = tIso;
          value = vi;
          eps   = 0.125f * step;
        }
      }
      if (t == tr.upper && std::fabs(sample - vi) < 1e-6f) {
        if (ts < tHit && ts <= tr.upper) {
          tHit  = ts;
          value = vi;
          eps   = 0.125f * step;
        }
      }
    }
    if (tHit < inf) {
      hit.t       = tHit;
      hit.sample  = value;
      hit.epsilon = eps * std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
      return true;
    }
    t0      = t;
    sample0 = sample;
  }
  return false;
}

}  // namespace orc

using namespace orc;

struct OrcVolume {
  Grid g;
};

static float bgOr(const float *bg, uint32_t a)
{
  if (bg)
    return bg[a];
  uint32_t bits = 0xFFC068B5u;
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

extern "C" {

const char *orc_last_error(void) { return g_lastError.c_str(); }

struct TemporalArgs {
  int numTimesteps;
  const void *indices;
  uint32_t indexType;
  uint64_t numIndices;
  const float *times;
  uint64_t numTimes;
  const uint64_t *numItems;  // per attribute
};

// verifyTemporalData (common/temporal_data_verification.h:10-181) for the
// structured / unstructured cases, with the reference's messages.
static void verifyTemporal(Grid &g, uint64_t numVoxels, const TemporalArgs &t, uint32_t numAttributes)
{
  uint64_t expected = numVoxels;
  if (t.numTimesteps > 0) {
    if (t.indices || t.times)
      throw std::runtime_error("Temporally structured volumes should not have temporallyUnstructuredIndices or "
                               "temporallyUnstructuredTimes provided");
    g.temporalFormat = 1;
    g.numTimesteps   = t.numTimesteps;
    expected         = numVoxels * (uint64_t)t.numTimesteps;
  } else if (t.indices) {
    if (!t.times)
      throw std::runtime_error("temporal format is VKL_TEMPORAL_FORMAT_UNSTRUCTURED but "
                               "temporallyUnstructuredTimes is not specified.");
    if (t.numIndices < numVoxels + 1)
      throw std::runtime_error("temporallyUnstructuredIndices is too small.");
    if (t.indexType != 4500 && t.indexType != 5550)
      throw std::runtime_error("temporallyUnstructuredIndices must have type VKL_UINT or VKL_ULONG");
    g.temporalFormat = 2;
    g.tIndices       = (const uint8_t *)t.indices;
    g.tIndices64     = t.indexType == 5550;
    g.tTimes         = t.times;
    uint64_t b = 0, e = 0;
    for (uint64_t i = 0; i < numVoxels; ++i) {
      b = tIndex(g, i);
      e = tIndex(g, i + 1);
      if (!(b < e))
        throw std::runtime_error("temporallyUnstructuredIndices must increase strictly monotonically.");
      if (!(e <= t.numTimes))
        throw std::runtime_error(
            "Values in temporallyUnstructuredIndices are out of bounds in temporallyUnstructredTimes.");
      for (uint64_t k = b + 1; k < e; ++k)
        if (!(t.times[k - 1] < t.times[k]))
          throw std::runtime_error(
              "temporallyUnstructuredTimes must increase strictly monotonically for every voxel.");
      if (t.times[b] < 0.f || t.times[b] > 1.f || t.times[e - 1] < 0.f || t.times[e - 1] > 1.f)
        throw std::runtime_error(
            "Values in temporallyUnstructuredTimes must be bounded by 0.0 and 1.0 for every voxel.");
    }
    expected = e;
  } else if (t.times) {
    throw std::runtime_error("Temporally constant volumes should not have temporallyUnstructuredIndices or "
                             "temporallyUnstructuredTimes provided");
  }
  for (uint32_t a = 0; a < numAttributes; ++a)
    if (t.numItems && t.numItems[a] != expected)
      throw std::runtime_error("attribute " + std::to_string(a) + " has " + std::to_string(t.numItems[a]) +
                               " elements, but expected " + std::to_string(expected));
}

static OrcVolume *denseCreate(const int32_t dims[3], uint32_t numAttributes, const void *const *data,
                              const uint32_t *types, const uint64_t *byteStrides, int cellCentered,
                              const float gridOrigin[3], const float gridSpacing[3], const float *indexToObject,
                              const int32_t indexOrigin[3], const float *background, const TemporalArgs *temporal)
{
  try {
    OrcVolume *v = new OrcVolume();
    Grid &g      = v->g;
    g.dense      = true;
    if (temporal)
      verifyTemporal(g, (uint64_t)dims[0] * (uint64_t)dims[1] * (uint64_t)dims[2], *temporal, numAttributes);
    g.constantCellData = cellCentered != 0;
    g.numAttributes    = numAttributes;
    g.denseDims        = {dims[0], dims[1], dims[2]};
    for (uint32_t a = 0; a < numAttributes; ++a) {
      typeSize(types[a]);
      g.denseAttr.push_back({types[a], (const uint8_t *)data[a],
                             (byteStrides && byteStrides[a]) ? byteStrides[a] : typeSize(types[a])});
      g.background.push_back(bgOr(background, a));
    }
    // transforms (DenseVdbVolume.cpp:42-64)
    float c[12];
    if (indexToObject) {
      std::memcpy(c, indexToObject, sizeof(c));
    } else {
      const float go[3] = {gridOrigin ? gridOrigin[0] : 0.f, gridOrigin ? gridOrigin[1] : 0.f,
                           gridOrigin ? gridOrigin[2] : 0.f};
      const float gs[3] = {gridSpacing ? gridSpacing[0] : 1.f,
                           gridSpacing ? gridSpacing[1] : 1.f,
                           gridSpacing ? gridSpacing[2] : 1.f};
      const float cc[12] = {gs[0], 0, 0, 0, gs[1], 0, 0, 0, gs[2], go[0], go[1], go[2]};
      std::memcpy(c, cc, sizeof(c));
      for (int a = 0; a < 3; ++a) {
        g.gridOrigin[a]  = go[a];
        g.gridSpacing[a] = gs[a];
      }
      g.legacyGrid = !cellCentered &&
                     (!indexOrigin || (indexOrigin[0] == 0 && indexOrigin[1] == 0 && indexOrigin[2] == 0));
    }
    makeTransforms(c, g.i2o, g.o2i);
    const vec3i io = {indexOrigin ? indexOrigin[0] : 0, indexOrigin ? indexOrigin[1] : 0,
                      indexOrigin ? indexOrigin[2] : 0};
    // leaves (DenseVdbVolume.cpp:67-119): x fastest
    const vec3i nl = {(dims[0] + 7) / 8, (dims[1] + 7) / 8, (dims[2] + 7) / 8};
    g.numLeaves    = (uint64_t)nl.x * nl.y * nl.z;
    if (g.numLeaves == 0)
      throw std::runtime_error("Vdb volumes must have at least one leaf node.");
    g.leafLevel.assign(g.numLeaves, 3);
    g.leafFormat.assign(g.numLeaves, FMT_DENSE_ZYX);
    g.leafOrigin.resize(g.numLeaves);
    uint64_t i = 0;
    for (int z = 0; z < nl.z; ++z)
      for (int y = 0; y < nl.y; ++y)
        for (int x = 0; x < nl.x; ++x)
          g.leafOrigin[i++] = {x * 8 + io.x, y * 8 + io.y, z * 8 + io.z};
    // root origin / active size / bbox (VdbVolume.cpp:749-765)
    g.rootOrigin = io;
    g.activeSize = {(uint32_t)dims[0], (uint32_t)dims[1], (uint32_t)dims[2]};
    const float lo[3] = {(float)io.x, (float)io.y, (float)io.z};
    const int e       = cellCentered ? 0 : 1;
    const float hi[3] = {(float)(io.x + dims[0] - e), (float)(io.y + dims[1] - e),
                         (float)(io.z + dims[2] - e)};
    finishBounds(g, lo, hi);
    buildTree(g, false, {});
    return v;
  } catch (const std::exception &ex) {
    g_lastError = ex.what();
    return nullptr;
  }
}

OrcVolume *orc_dense_create(const int32_t dims[3], uint32_t numAttributes,
                            const void *const *data, const uint32_t *types,
                            const uint64_t *byteStrides, int cellCentered,
                            const float gridOrigin[3], const float gridSpacing[3],
                            const float *indexToObject, const int32_t indexOrigin[3],
                            const float *background)
{
  return denseCreate(dims, numAttributes, data, types, byteStrides, cellCentered, gridOrigin, gridSpacing,
                     indexToObject, indexOrigin, background, nullptr);
}

OrcVolume *orc_dense_create_temporal(const int32_t dims[3], uint32_t numAttributes, const void *const *data,
                                     const uint32_t *types, const uint64_t *numItems, int cellCentered,
                                     const float gridOrigin[3], const float gridSpacing[3],
                                     const float *indexToObject, const float *background, int numTimesteps,
                                     const void *indices, uint32_t indexType, uint64_t numIndices,
                                     const float *times, uint64_t numTimes)
{
  const TemporalArgs t{numTimesteps, indices, indexType, numIndices, times, numTimes, numItems};
  return denseCreate(dims, numAttributes, data, types, nullptr, cellCentered, gridOrigin, gridSpacing,
                     indexToObject, nullptr, background, &t);
}

void orc_sample_times(const OrcVolume *v, int filter, uint64_t n, const float *pts, const float *times,
                      uint32_t attr, float *out, int threads)
{
  const Grid &g = v->g;
  parallelFor((int64_t)n, threads, 4096, [&](int64_t i) {
    t_time        = times ? times[i] : 0.f;
    const vec3f p = xfmPoint(g.o2i, {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]});
    out[i]        = sampleAt(g, filter, p, attr, NUM_LEVELS - 1);
  });
  t_time = 0.f;
}

void orc_gradient_times(const OrcVolume *v, int filter, uint64_t n, const float *pts, const float *times,
                        uint32_t attr, float *out, int threads)
{
  const uint64_t chunks = (n + 4095) / 4096;
  parallelFor((int64_t)chunks, threads, 1, [&](int64_t c) {
    const uint64_t b = (uint64_t)c * 4096, e = std::min<uint64_t>(n, b + 4096);
    for (uint64_t i = b; i < e; ++i) {
      t_time = times ? times[i] : 0.f;
      orc_gradient(v, filter, NUM_LEVELS - 1, 1, pts + 3 * i, attr, out + 3 * i);
    }
    t_time = 0.f;
  });
}

OrcVolume *orc_vdb_create(uint64_t numLeaves, const uint32_t *levels, const int32_t *origins,
                          const uint32_t *formats, uint32_t numAttributes, uint32_t dataType,
                          const void *const *packedDense, const void *const *packedTile,
                          const float *indexToObject, const int32_t *clip,
                          const float *background)
{
  try {
    OrcVolume *v = new OrcVolume();
    Grid &g      = v->g;
    g.dense      = false;
    g.constantCellData = true;
    g.numAttributes    = numAttributes;
    g.leafType         = dataType;
    if (numLeaves == 0)
      throw std::runtime_error("Vdb volumes must have at least one leaf node.");
    g.numLeaves = numLeaves;
    g.leafLevel.assign(levels, levels + numLeaves);
    g.leafFormat.assign(formats, formats + numLeaves);
    g.leafOrigin.resize(numLeaves);
    uint64_t nDense = 0, nTile = 0;
    std::vector<uint64_t> packedIndex(numLeaves);
    for (uint64_t i = 0; i < numLeaves; ++i) {
      g.leafOrigin[i] = {origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]};
      // verifyLevel / verifyNodeDataFormat (VdbVolume.cpp:529-551)
      if (levels[i] >= NUM_LEVELS)
        throw std::runtime_error("invalid node level " + std::to_string(levels[i]) +
                                 " for this vdb configuration");
      if (formats[i] == FMT_DENSE_ZYX) {
        if (levels[i] + 1 < NUM_LEVELS)
          throw std::runtime_error("leaf nodes are only supported on the lowest level.");
        packedIndex[i] = nDense++;
      } else if (formats[i] == FMT_TILE) {
        packedIndex[i] = nTile++;
      } else {
        throw std::runtime_error("invalid format specified");
      }
    }
    const uint32_t ts = typeSize(dataType);
    for (uint32_t a = 0; a < numAttributes; ++a) {
      g.background.push_back(bgOr(background, a));
      const uint8_t *pd = packedDense ? (const uint8_t *)packedDense[a] : nullptr;
      const uint8_t *pt = packedTile ? (const uint8_t *)packedTile[a] : nullptr;
      g.packedDense.emplace_back(pd ? pd : (const uint8_t *)"", pd ? pd + nDense * 512 * ts : (const uint8_t *)"");
      g.packedTile.emplace_back(pt ? pt : (const uint8_t *)"", pt ? pt + nTile * ts : (const uint8_t *)"");
    }
    float c[12] = {1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0};
    if (indexToObject)
      std::memcpy(c, indexToObject, sizeof(c));
    makeTransforms(c, g.i2o, g.o2i);
    // computeBbox (VdbVolume.cpp:71-81) and computeRootOrigin (:567-581)
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (uint64_t i = 0; i < numLeaves; ++i) {
      const int32_t r = (int32_t)levelRes(g.leafLevel[i]);
      const int32_t o[3] = {g.leafOrigin[i].x, g.leafOrigin[i].y, g.leafOrigin[i].z};
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], o[a]);
        hi[a] = std::max(hi[a], o[a] + r);
        lo[a] = std::min(lo[a], o[a] + r);
        hi[a] = std::max(hi[a], o[a]);
      }
    }
    for (int a = 0; a < 3; ++a)
      if ((uint32_t)(hi[a] - lo[a]) > levelRes(0))
        throw std::runtime_error("input leaves do not fit into a single root level node");
    const int32_t r1 = (int32_t)levelRes(1);
    g.rootOrigin = {r1 * (int32_t)std::floor(lo[0] / (float)r1),
                    r1 * (int32_t)std::floor(lo[1] / (float)r1),
                    r1 * (int32_t)std::floor(lo[2] / (float)r1)};
    g.activeSize = {(uint32_t)(hi[0] - g.rootOrigin.x), (uint32_t)(hi[1] - g.rootOrigin.y),
                    (uint32_t)(hi[2] - g.rootOrigin.z)};
    float flo[3] = {(float)lo[0], (float)lo[1], (float)lo[2]};
    float fhi[3] = {(float)hi[0], (float)hi[1], (float)hi[2]};
    if (clip && !(clip[3] < clip[0] || clip[4] < clip[1] || clip[5] < clip[2])) {
      for (int a = 0; a < 3; ++a) {
        flo[a] = (float)clip[a];
        fhi[a] = (float)clip[3 + a];
      }
    }
    finishBounds(g, flo, fhi);
    buildTree(g, true, packedIndex);
    return v;
  } catch (const std::exception &ex) {
    g_lastError = ex.what();
    return nullptr;
  }
}

void orc_destroy(OrcVolume *v) { delete v; }

void orc_get_info(const OrcVolume *v, float o2i[12], float i2o[12], int32_t root[3],
                  uint32_t active[3], float domain[6], float bounds[6])
{
  const Grid &g = v->g;
  if (o2i) std::memcpy(o2i, g.o2i, 48);
  if (i2o) std::memcpy(i2o, g.i2o, 48);
  if (root) { root[0] = g.rootOrigin.x; root[1] = g.rootOrigin.y; root[2] = g.rootOrigin.z; }
  if (active) { active[0] = g.activeSize.x; active[1] = g.activeSize.y; active[2] = g.activeSize.z; }
  if (domain) std::memcpy(domain, g.domain, 24);
  if (bounds) std::memcpy(bounds, g.bounds, 24);
}

uint64_t orc_level_num_nodes(const OrcVolume *v, uint32_t level)
{
  return level < NUM_LEVELS - 1 ? v->g.levels[level].numNodes : v->g.numLeaves;
}

void orc_get_level(const OrcVolume *v, uint32_t level, uint64_t *voxels, float *ranges,
                   uint32_t *origins)
{
  const Level &lv = v->g.levels[level];
  const uint64_t nv = lv.numNodes * levelNumVoxels(level);
  if (voxels) std::memcpy(voxels, lv.voxels.data(), nv * 8);
  if (ranges)
    for (uint64_t i = 0; i < nv * v->g.numAttributes; ++i) {
      ranges[2 * i]     = lv.valueRange[i].lower;
      ranges[2 * i + 1] = lv.valueRange[i].upper;
    }
  if (origins)
    for (uint64_t n = 0; n < lv.numNodes; ++n) {
      origins[3 * n]     = lv.origin[n].x;
      origins[3 * n + 1] = lv.origin[n].y;
      origins[3 * n + 2] = lv.origin[n].z;
    }
}

void orc_value_range(const OrcVolume *v, uint32_t attr, float r[2])
{
  r[0] = v->g.volumeRange[attr].lower;
  r[1] = v->g.volumeRange[attr].upper;
}

void orc_sample(const OrcVolume *v, int filter, uint32_t depth, uint64_t n, const float *pts,
                uint32_t attr, float *out)
{
  const Grid &g = v->g;
  for (uint64_t i = 0; i < n; ++i) {
    const vec3f p = xfmPoint(g.o2i, {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]});
    out[i]        = sampleAt(g, filter, p, attr, depth);
  }
}

void orc_sample_observed(const OrcVolume *v, int filter, uint32_t depth, uint64_t n, const float *pts,
                         uint32_t attr, float *out, uint32_t *leafAccess)
{
  t_leafAccess = leafAccess;
  orc_sample(v, filter, depth, n, pts, attr, out);
  t_leafAccess = nullptr;
}

void orc_sample_parallel(const OrcVolume *v, int filter, uint64_t n, const float *pts,
                         uint32_t attr, float *out, int threads)
{
  const Grid &g = v->g;
  parallelFor((int64_t)n, threads, 4096, [&](int64_t i) {
    const vec3f p = xfmPoint(g.o2i, {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]});
    out[i]        = sampleAt(g, filter, p, attr, NUM_LEVELS - 1);
  });
}

void orc_gradient(const OrcVolume *v, int filter, uint32_t depth, uint64_t n, const float *pts,
                  uint32_t attr, float *out)
{
  const Grid &g = v->g;
  for (uint64_t i = 0; i < n; ++i) {
    const vec3f p = xfmPoint(g.o2i, {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]});
    vec3f gr;
    if (filter == F_NEAREST) {
      gr = {0.f, 0.f, 0.f};
    } else {
      gr = (filter == F_CUBIC) ? gradientCubic(g, p, attr, depth)
                               : gradientLinear(g, p, attr, depth);
      gr = xfmNormal(g.o2i, gr);
    }
    out[3 * i]     = gr.x;
    out[3 * i + 1] = gr.y;
    out[3 * i + 2] = gr.z;
  }
}

void orc_gradient_parallel(const OrcVolume *v, int filter, uint32_t depth, uint64_t n,
                           const float *pts, uint32_t attr, float *out, int threads)
{
  // orc_gradient over chunks of 4096 points on `threads` host threads
  const uint64_t chunks = (n + 4095) / 4096;
  parallelFor((int64_t)chunks, threads, 1, [&](int64_t c) {
    const uint64_t b = (uint64_t)c * 4096, e = std::min<uint64_t>(n, b + 4096);
    orc_gradient(v, filter, depth, e - b, pts + 3 * b, attr, out + 3 * b);
  });
}

void orc_sample_fp64(const OrcVolume *v, int filter, uint64_t n, const float *pts,
                     uint32_t attr, double *out)
{
  // Same stencils, evaluated in double from the stored (float-converted)
  // voxel values; the index-space position is computed in double too.
  const Grid &g = v->g;
  const TricubicMap &m = tricubicMap();
  for (uint64_t i = 0; i < n; ++i) {
    const double o[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
    double p[3];
    for (int r = 0; r < 3; ++r)
      p[r] = (double)g.o2i[3 * r] * o[0] + (double)g.o2i[3 * r + 1] * o[1] +
             (double)g.o2i[3 * r + 2] * o[2] + (double)g.o2i[9 + r];
    if (filter == F_NEAREST) {
      const double off = g.constantCellData ? 0.0 : 0.5;
      out[i] = tap(g, {(int32_t)std::floor(p[0] + off), (int32_t)std::floor(p[1] + off),
                       (int32_t)std::floor(p[2] + off)}, attr, NUM_LEVELS - 1);
      continue;
    }
    const vec3i ic = {(int32_t)std::floor(p[0]), (int32_t)std::floor(p[1]),
                      (int32_t)std::floor(p[2])};
    const double dl[3] = {p[0] - ic.x, p[1] - ic.y, p[2] - ic.z};
    if (filter == F_LINEAR) {
      double acc = 0;
      for (int c = 0; c < 8; ++c) {
        const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
        const double w = (cx ? dl[0] : 1 - dl[0]) * (cy ? dl[1] : 1 - dl[1]) *
                         (cz ? dl[2] : 1 - dl[2]);
        acc += w * tap(g, {ic.x + cx, ic.y + cy, ic.z + cz}, attr, NUM_LEVELS - 1);
      }
      out[i] = acc;
      continue;
    }
    double s[64];
    for (int q = 0; q < 64; ++q)
      s[q] = tap(g, {ic.x + (q >> 4) - 1, ic.y + ((q >> 2) & 3) - 1, ic.z + (q & 3) - 1},
                 attr, NUM_LEVELS - 1);
    auto S = [&](int x, int y, int z) { return s[(x + 1) * 16 + (y + 1) * 4 + (z + 1)]; };
    double ctr[64];
    for (int c = 0; c < 8; ++c) {
      const int x = c >> 2, y = (c >> 1) & 1, z = c & 1;
      ctr[c]      = S(x, y, z);
      ctr[8 + c]  = 0.5 * (S(x + 1, y, z) - S(x - 1, y, z));
      ctr[16 + c] = 0.5 * (S(x, y + 1, z) - S(x, y - 1, z));
      ctr[24 + c] = 0.5 * (S(x, y, z + 1) - S(x, y, z - 1));
      ctr[32 + c] = 0.25 * (S(x - 1, y - 1, z) - S(x - 1, y + 1, z) - S(x + 1, y - 1, z) + S(x + 1, y + 1, z));
      ctr[40 + c] = 0.25 * (S(x - 1, y, z - 1) - S(x - 1, y, z + 1) - S(x + 1, y, z - 1) + S(x + 1, y, z + 1));
      ctr[48 + c] = 0.25 * (S(x, y - 1, z - 1) - S(x, y - 1, z + 1) - S(x, y + 1, z - 1) + S(x, y + 1, z + 1));
      ctr[56 + c] = 0.125 * (-S(x - 1, y - 1, z - 1) + S(x - 1, y - 1, z + 1) + S(x - 1, y + 1, z - 1) -
                             S(x - 1, y + 1, z + 1) + S(x + 1, y - 1, z - 1) - S(x + 1, y - 1, z + 1) -
                             S(x + 1, y + 1, z - 1) + S(x + 1, y + 1, z + 1));
    }
    double acc = 0;
    for (int r = 0; r < 64; ++r) {
      double cr = 0;
      for (int e = m.start[r]; e < m.start[r + 1]; ++e)
        cr += (double)m.w[e] * ctr[m.col[e]];
      const int pi = r >> 4, pj = (r >> 2) & 3, pk = r & 3;
      acc += cr * std::pow(dl[0], pi) * std::pow(dl[1], pj) * std::pow(dl[2], pk);
    }
    out[i] = acc;
  }
}

void orc_iterate_intervals(const OrcVolume *v, uint32_t attr, uint32_t numRanges,
                           const float *ranges, float hint, uint64_t numRays,
                           const float *origins, const float *directions,
                           const float *tRanges, uint32_t maxIntervals, float *out,
                           uint32_t *counts)
{
  const Grid &g = v->g;
  ValueRanges vr;
  for (uint32_t i = 0; i < numRanges; ++i)
    vr.ranges.push_back({ranges[2 * i], ranges[2 * i + 1]});
  vr.computeMinMax();
  const int depth = hintToDepth(hint);
  parallelFor((int64_t)numRays, 0, 64, [&](int64_t r) {
    IntervalIt it;
    intervalInit(it, g, attr, (uint32_t)depth,
                 {origins[3 * r], origins[3 * r + 1], origins[3 * r + 2]},
                 {directions[3 * r], directions[3 * r + 1], directions[3 * r + 2]},
                 {tRanges[2 * r], tRanges[2 * r + 1]});
    uint32_t c = 0;
    Interval iv;
    while (intervalIterate(it, vr, iv)) {
      if (c < maxIntervals) {
        float *o = out + ((uint64_t)r * maxIntervals + c) * 5;
        o[0] = iv.t.lower;
        o[1] = iv.t.upper;
        o[2] = iv.v.lower;
        o[3] = iv.v.upper;
        o[4] = iv.nominalDeltaT;
      }
      c++;
    }
    counts[r] = c;
  });
}

// ---------------------------------------------------------------------------
// 16^3-voxel macrocell intervals: the iterator of the reference's legacy
// structuredRegular volume (the GridAccelerator, built when
// OPENVKL_DEVICE_CPU_STRUCTURED_REGULAR_LEGACY is on).  Macrocell width
// GridAccelerator.h:14-19; macrocell value ranges GridAccelerator.ispc:80-109
// (vertices cell*16 + [0, 16] per axis, clamped to dims - 1, NaN skipped, NaN
// range if all are NaN; SharedStructuredVolume.ispc:196-209 for a vertex's
// range); cell walk GridAccelerator_nextCell, GridAccelerator.ispc:146-240;
// interval emission GridAcceleratorIterator.ispc:44-155.  Transforms
// SharedStructuredVolume.ih:21-53, bounding box StructuredVolume.cpp:205-211.
// ---------------------------------------------------------------------------
namespace {

constexpr int MACRO_BITS = 4;  // CELL_WIDTH_BITCOUNT

inline vec3i macrocellCount(const Grid &g)
{
  return {((g.denseDims.x - 1) >> MACRO_BITS) + 1, ((g.denseDims.y - 1) >> MACRO_BITS) + 1,
          ((g.denseDims.z - 1) >> MACRO_BITS) + 1};
}

range1f macrocellRange(const Grid &g, uint32_t a, int cx, int cy, int cz)
{
  range1f r;
  bool empty = true;
  const vec3i d = g.denseDims;
  for (int k = 0; k <= (1 << MACRO_BITS); ++k)
    for (int j = 0; j <= (1 << MACRO_BITS); ++j)
      for (int i = 0; i <= (1 << MACRO_BITS); ++i) {
        const int x = std::min(d.x - 1, (cx << MACRO_BITS) + i), y = std::min(d.y - 1, (cy << MACRO_BITS) + j),
                  z = std::min(d.z - 1, (cz << MACRO_BITS) + k);
        const float v = loadAttr(g.denseAttr[a], (uint64_t)x + (uint64_t)d.x * ((uint64_t)y + (uint64_t)d.y * (uint64_t)z));
        if (!std::isnan(v)) {
          r.lower = fmin_(r.lower, v);
          r.upper = fmax_(r.upper, v);
          empty   = false;
        }
      }
  if (empty)
    r.lower = r.upper = std::numeric_limits<float>::quiet_NaN();
  return r;
}

struct MacroIt {
  vec3f o, d;
  range1f bbT;
  vec3i cell;
  float nominalDeltaT;
};

inline vec3f toLocal(const Grid &g, const vec3f &p)
{
  return {1.f / g.gridSpacing[0] * (p.x - g.gridOrigin[0]), 1.f / g.gridSpacing[1] * (p.y - g.gridOrigin[1]),
          1.f / g.gridSpacing[2] * (p.z - g.gridOrigin[2])};
}

inline range1f macrocellT(const Grid &g, const MacroIt &it, const vec3i &c)
{
  // GridAccelerator_getCellBounds: lower/upper corner of the cell in object space
  float box[6];
  const int lo[3] = {c.x << MACRO_BITS, c.y << MACRO_BITS, c.z << MACRO_BITS};
  const int hi[3] = {(c.x + 1) << MACRO_BITS, (c.y + 1) << MACRO_BITS, (c.z + 1) << MACRO_BITS};
  for (int a = 0; a < 3; ++a) {
    box[a]     = g.gridOrigin[a] + (float)lo[a] * g.gridSpacing[a];
    box[3 + a] = g.gridOrigin[a] + (float)hi[a] * g.gridSpacing[a];
  }
  return intersectBox(it.o, it.d, box, it.bbT);
}

// isempty1f (math/box_utility.ih:6-9)
inline bool isEmpty1f(const range1f &r) { return r.upper <= r.lower; }

bool macroNextCell(const Grid &g, MacroIt &it, range1f &cellT)
{
  const bool first = it.cell.x == -1;
  range1f iv;
  if (first) {
    const vec3f p  = {it.o.x + it.bbT.lower * it.d.x, it.o.y + it.bbT.lower * it.d.y, it.o.z + it.bbT.lower * it.d.z};
    const vec3f lc = toLocal(g, p);
    it.cell        = {toIntX86(lc.x) >> MACRO_BITS, toIntX86(lc.y) >> MACRO_BITS, toIntX86(lc.z) >> MACRO_BITS};
    iv             = macrocellT(g, it, it.cell);
  }
  if (!first || isEmpty1f(iv)) {
    // direction * 1.f / gridSpacing * RCP_CELL_WIDTH, RCP_CELL_WIDTH being the
    // macro text "1.f / CELL_WIDTH": ((d * 1) / s * 1) / 16
    const float cd[3]  = {it.d.x / g.gridSpacing[0] / 16.f, it.d.y / g.gridSpacing[1] / 16.f,
                          it.d.z / g.gridSpacing[2] / 16.f};
    const float rcd[3] = {rcp_safe(cd[0]), rcp_safe(cd[1]), rcp_safe(cd[2])};
    const vec3f lo     = toLocal(g, it.o);
    const float co[3]  = {lo.x / 16.f, lo.y / 16.f, lo.z / 16.f};
    int corner[3];
    float tMax[3];
    const int ci[3] = {it.cell.x, it.cell.y, it.cell.z};
    for (int a = 0; a < 3; ++a) {
      uint32_t bits;
      std::memcpy(&bits, &cd[a], 4);
      corner[a]      = 1 - 2 * (int)(bits >> 31);
      const float t0 = ((float)ci[a] - co[a]) * rcd[a];
      const float t1 = ((float)(ci[a] + 1) - co[a]) * rcd[a];
      tMax[a]        = fmax_(t0, t1);
    }
    const float tExit = fmin_(fmin_(tMax[0], tMax[1]), tMax[2]);
    it.cell = {ci[0] + (tMax[0] == tExit ? corner[0] : 0), ci[1] + (tMax[1] == tExit ? corner[1] : 0),
               ci[2] + (tMax[2] == tExit ? corner[2] : 0)};
    iv      = macrocellT(g, it, it.cell);
  }
  if (isEmpty1f(iv)) {
    cellT = range1f();
    return false;
  }
  cellT = iv;
  return true;
}

}  // namespace

void orc_macrocell_ranges(const OrcVolume *v, uint32_t attr, float *out)
{
  const Grid &g = v->g;
  const vec3i n = macrocellCount(g);
  parallelFor((int64_t)n.x * n.y * n.z, 0, 64, [&](int64_t c) {
    const int cx = (int)(c % n.x), cy = (int)((c / n.x) % n.y), cz = (int)(c / ((int64_t)n.x * n.y));
    const range1f r = macrocellRange(g, attr, cx, cy, cz);
    out[2 * c]      = r.lower;
    out[2 * c + 1]  = r.upper;
  });
}

int orc_iterate_macrocells(const OrcVolume *v, uint32_t attr, uint32_t numRanges, const float *ranges,
                           uint64_t numRays, const float *origins, const float *directions,
                           const float *tRanges, uint32_t maxIntervals, float *out, uint32_t *counts)
{
  const Grid &g = v->g;
  if (!g.dense || !g.legacyGrid) {
    g_lastError = "macrocell intervals need a vertex-centered structuredRegular volume given by "
                  "gridOrigin / gridSpacing";
    return 1;
  }
  ValueRanges vr;
  for (uint32_t i = 0; i < numRanges; ++i)
    vr.ranges.push_back({ranges[2 * i], ranges[2 * i + 1]});
  vr.computeMinMax();
  const vec3i n = macrocellCount(g);
  std::vector<range1f> cr((size_t)n.x * n.y * n.z);
  parallelFor((int64_t)cr.size(), 0, 64, [&](int64_t c) {
    cr[c] = macrocellRange(g, attr, (int)(c % n.x), (int)((c / n.x) % n.y), (int)(c / ((int64_t)n.x * n.y)));
  });
  float box[6];
  for (int a = 0; a < 3; ++a) {
    const int d = a == 0 ? g.denseDims.x : a == 1 ? g.denseDims.y : g.denseDims.z;
    box[a]      = g.gridOrigin[a];
    box[3 + a]  = g.gridOrigin[a] + (float)(d - 1) * g.gridSpacing[a];
  }
  parallelFor((int64_t)numRays, 0, 64, [&](int64_t r) {
    MacroIt it;
    it.o   = {origins[3 * r], origins[3 * r + 1], origins[3 * r + 2]};
    it.d   = {directions[3 * r], directions[3 * r + 1], directions[3 * r + 2]};
    it.bbT = intersectBox(it.o, it.d, box, {tRanges[2 * r], tRanges[2 * r + 1]});
    it.cell = {-1, -1, -1};
    it.nominalDeltaT = fmin_(fmin_(g.gridSpacing[0] * rcp_safe(std::fabs(it.d.x)),
                                   g.gridSpacing[1] * rcp_safe(std::fabs(it.d.y))),
                             g.gridSpacing[2] * rcp_safe(std::fabs(it.d.z)));
    uint32_t c = 0;
    if (!isEmpty1f(it.bbT)) {
      range1f t;
      int budget = 4 * (n.x + n.y + n.z) + 16;
      while (budget-- > 0 && macroNextCell(g, it, t)) {
        // the cell's stored range (cells the walk reaches lie in the grid; the
        // index is clamped for the lookup)
        const int x = std::min(std::max(it.cell.x, 0), n.x - 1), y = std::min(std::max(it.cell.y, 0), n.y - 1),
                  z = std::min(std::max(it.cell.z, 0), n.z - 1);
        const range1f vrng = cr[(size_t)x + (size_t)n.x * ((size_t)y + (size_t)n.y * z)];
        if (!vr.overlaps(vrng))
          continue;
        if (c < maxIntervals) {
          float *o = out + ((uint64_t)r * maxIntervals + c) * 5;
          o[0] = t.lower;
          o[1] = t.upper;
          o[2] = vrng.lower;
          o[3] = vrng.upper;
          o[4] = it.nominalDeltaT;
        }
        c++;
      }
    }
    counts[r] = c;
  });
  return 0;
}

namespace {

// Default hit iterator state and one vklIterateHit call
// (DefaultIterator.ispc:140-258).
struct HitIter {
  IntervalIt it;
  Interval cur;
  float lastHitOffsetT;
  vec3f o, d;
};

ValueRanges hitRanges(const float *values, uint32_t numValues)
{
  // HitIteratorContext::commit (IteratorContext.cpp:266-336): degenerate
  // ranges at the iso values
  ValueRanges vr;
  for (uint32_t i = 0; i < numValues; ++i)
    vr.ranges.push_back({values[i], values[i]});
  vr.computeMinMax();
  return vr;
}

int hitDepth(const Grid &g) { return g.dense ? hintToDepth(0.5f) : hintToDepth(1.f); }

void hitInit(HitIter &h, const Grid &g, uint32_t attr, const vec3f &o, const vec3f &d, const range1f &tr)
{
  intervalInit(h.it, g, attr, (uint32_t)hitDepth(g), o, d, tr);
  h.cur.t             = {1.f, -1.f};
  h.cur.v             = {0.f, 0.f};
  h.cur.nominalDeltaT = 0.f;
  h.lastHitOffsetT    = -std::numeric_limits<float>::infinity();
  h.o                 = o;
  h.d                 = d;
}

bool hitNext(HitIter &h, const Grid &g, int filter, uint32_t attr, const ValueRanges &vr,
             const std::vector<float> &vals, HitRec &out)
{
  const float inf = std::numeric_limits<float>::infinity();
  if (vals.empty() || h.cur.t.lower == inf)
    return false;
  for (;;) {
    const bool need = h.cur.t.upper <= h.cur.t.lower;
    bool have       = !need;
    if (need)
      have = intervalIterate(h.it, vr, h.cur);
    if (need && have) {
      h.cur.t.lower = fmax_(h.cur.t.lower, h.lastHitOffsetT);
      if (h.cur.t.upper <= h.cur.t.lower)
        continue;
    }
    if (!have) {
      h.cur.t.lower = inf;
      return false;
    }
    HitRec hit{inf, 0.f, 0.f};
    if (intersectBisection(g, filter, attr, h.o, h.d, h.cur.t, h.cur.nominalDeltaT, vals, hit)) {
      h.cur.t.lower    = hit.t + hit.epsilon;
      h.lastHitOffsetT = hit.t + hit.epsilon;
      out              = hit;
      return true;
    }
    h.cur.t.lower = inf;
  }
}

}  // namespace

void orc_iterate_hits(const OrcVolume *v, uint32_t attr, int filter, uint32_t numValues,
                      const float *values, uint64_t numRays, const float *origins,
                      const float *directions, const float *tRanges, uint32_t maxHits,
                      float *out, uint32_t *counts)
{
  const Grid &g = v->g;
  const ValueRanges vr = hitRanges(values, numValues);
  const std::vector<float> vals(values, values + numValues);
  parallelFor((int64_t)numRays, 0, 64, [&](int64_t r) {
    HitIter h;
    hitInit(h, g, attr, {origins[3 * r], origins[3 * r + 1], origins[3 * r + 2]},
            {directions[3 * r], directions[3 * r + 1], directions[3 * r + 2]},
            {tRanges[2 * r], tRanges[2 * r + 1]});
    uint32_t c = 0;
    HitRec hit;
    while (c < MAX_HITS && hitNext(h, g, filter, attr, vr, vals, hit)) {
      if (c < maxHits) {
        float *o = out + ((uint64_t)r * maxHits + c) * 3;
        o[0]     = hit.t;
        o[1]     = hit.sample;
        o[2]     = hit.epsilon;
      }
      c++;
    }
    counts[r] = c;
  });
}

// ---------------------------------------------------------------------------
// The reference's example renderers, one ray per pixel centre
// (examples/interactive/renderer: Camera.ih Camera_createRay;
// RendererGpuKernel.h:64-93 sampleTransferFunction and :142-155
// intersectBox; RayMarchIteratorGpuKernel.cpp:9-88;
// IntervalIteratorDebugGpuKernel.cpp:9-77; HitIteratorRendererGpuKernel.cpp:
// 9-114).  The reference's approximate reciprocals and rsqrt are exact
// divisions and square roots here; min/max of possibly-NaN slab values use
// the IEEE minNum / maxNum form (std::fmin / std::fmax).
// ---------------------------------------------------------------------------
namespace {

struct RV3 {
  float x, y, z;
};
inline RV3 operator+(RV3 a, RV3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline RV3 operator-(RV3 a, RV3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline RV3 operator*(float s, RV3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline float rdot(RV3 a, RV3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline RV3 rnormalize(RV3 a)
{
  const float l = std::sqrt(rdot(a, a));
  return {a.x / l, a.y / l, a.z / l};
}
inline float clamp01(float x) { return std::fmin(std::fmax(x, 0.f), 1.f); }

struct RenderTF {
  const float *c;
  int n;
  float lo, hi;
  void at(float value, float out[4]) const
  {
    if (std::isnan(value) || n == 0) {
      out[0] = out[1] = out[2] = out[3] = 0.f;
      return;
    }
    const int last = n - 1;
    if (value <= lo) {
      std::memcpy(out, c, 16);
      return;
    }
    if (value >= hi) {
      std::memcpy(out, c + 4 * last, 16);
      return;
    }
    value                 = (value - lo) / (hi - lo) * (float)last;
    const int index       = (int)std::floor(value);
    const float remainder = value - (float)index;
    const int next        = std::min(index + 1, last);
    const float a         = 1.f - remainder;
    for (int k = 0; k < 4; ++k)
      out[k] = a * c[4 * index + k] + remainder * c[4 * next + k];
  }
};

}  // namespace

void orc_render(const OrcVolume *v, int renderer, int filter, int gradientFilter, uint32_t maxSamplingDepth,
                uint32_t attr, uint32_t numRanges, const float *ranges, float hint, uint32_t numValues,
                const float *values, const float camera[14], const float *tfColors, int tfNum,
                const float tfRange[2], const int ip[4], const float fp[9], float *rgba)
{
  const Grid &g = v->g;
  const int W = ip[0], H = ip[1];
  const bool firstOnly = ip[2] != 0, borders = ip[3] != 0;
  const float *bounds = fp;
  const float samplingRate = fp[6], colorScale = fp[7], intervalOpacity = fp[8];
  const RenderTF tf{tfColors, tfNum, tfRange[0], tfRange[1]};
  ValueRanges ivr;
  for (uint32_t i = 0; i < numRanges; ++i)
    ivr.ranges.push_back({ranges[2 * i], ranges[2 * i + 1]});
  ivr.computeMinMax();
  const ValueRanges hvr = hitRanges(values, numValues);
  const std::vector<float> vals(values, values + numValues);
  const int depth = hintToDepth(hint);
  const float inf = std::numeric_limits<float>::infinity();
  auto sampleP = [&](RV3 c) { return sampleAt(g, filter, xfmPoint(g.o2i, {c.x, c.y, c.z}), attr, maxSamplingDepth); };
  auto gradientP = [&](RV3 c) {
    if (gradientFilter == F_NEAREST)
      return RV3{0.f, 0.f, 0.f};
    const vec3f p  = xfmPoint(g.o2i, {c.x, c.y, c.z});
    const vec3f gi = gradientFilter == F_CUBIC ? gradientCubic(g, p, attr, maxSamplingDepth)
                                               : gradientLinear(g, p, attr, maxSamplingDepth);
    const vec3f r = xfmNormal(g.o2i, gi);
    return RV3{r.x, r.y, r.z};
  };
  parallelFor((int64_t)W * H, 0, 16, [&](int64_t idx) {
    // Camera_createRay at the pixel centre
    const float px = (float)(idx % W) + 0.5f, py = (float)(idx / W) + 0.5f;
    const float irx    = 1.f / (float)W;
    const float sx     = (px - 0.5f * (float)W) * irx;
    const float sy     = -(py - 0.5f * (float)H) * irx;
    const RV3 pCamera  = {camera[0] * sx, camera[0] * sy, 0.f};
    const RV3 pAperture = {0.f, 0.f, -camera[1]};
    const RV3 dCamera  = pAperture - pCamera;
    const RV3 R0 = {camera[2], camera[3], camera[4]}, R1 = {camera[5], camera[6], camera[7]},
              R2 = {camera[8], camera[9], camera[10]};
    const RV3 org = {rdot(R0, pCamera) + camera[11], rdot(R1, pCamera) + camera[12],
                     rdot(R2, pCamera) + camera[13]};
    const RV3 dir = rnormalize({rdot(R0, dCamera), rdot(R1, dCamera), rdot(R2, dCamera)});
    // intersectBox
    const float rx = 1.f / dir.x, ry = 1.f / dir.y, rz = 1.f / dir.z;
    const float x0 = (bounds[0] - org.x) * rx, y0 = (bounds[1] - org.y) * ry, z0 = (bounds[2] - org.z) * rz;
    const float x1 = (bounds[3] - org.x) * rx, y1 = (bounds[4] - org.y) * ry, z1 = (bounds[5] - org.z) * rz;
    range1f tr;
    tr.lower = std::fmax(std::fmax(std::fmax(std::fmin(x0, x1), std::fmin(y0, y1)), std::fmin(z0, z1)), 0.f);
    tr.upper = std::fmin(std::fmin(std::fmin(std::fmax(x0, x1), std::fmax(y0, y1)), std::fmax(z0, z1)), inf);
    RV3 color   = {0.f, 0.f, 0.f};
    float alpha = 0.f;
    if (renderer == 0 || renderer == 1) {
      IntervalIt it;
      intervalInit(it, g, attr, (uint32_t)depth, {org.x, org.y, org.z}, {dir.x, dir.y, dir.z}, tr);
      Interval iv;
      int count = 0;
      while (intervalIterate(it, ivr, iv) && alpha < 0.99f) {
        if (renderer == 0) {
          const float dtn = iv.nominalDeltaT / samplingRate;
          float lo = iv.t.lower, hi = std::fmin(iv.t.lower + dtn, iv.t.upper);
          while (hi - lo > 0.f && alpha < 0.99f) {
            const float t  = 0.5f * (lo + hi);
            const float dt = hi - lo;
            float sc[4];
            tf.at(sampleP(org + t * dir), sc);
            const float op = clamp01(sc[3] * dt);
            color          = color + (1.f - alpha) * RV3{sc[0] * op, sc[1] * op, sc[2] * op};
            alpha          = alpha + (1.f - alpha) * op;
            lo             = hi;
            hi             = std::fmin(lo + dtn, iv.t.upper);
          }
        } else {
          count++;
          const float dt = iv.t.upper - iv.t.lower;
          float sc[4];
          tf.at(tfRange[0] + (float)count / colorScale * (tfRange[1] - tfRange[0]), sc);
          sc[3]    = intervalOpacity;
          float op = clamp01(sc[3] * dt);
          RV3 c    = {sc[0] * op, sc[1] * op, sc[2] * op};
          if (borders && dt < iv.nominalDeltaT) {
            c  = {1.f, 1.f, 1.f};
            op = 1.f;
          }
          color = color + (1.f - alpha) * c;
          alpha = alpha + (1.f - alpha) * op;
          if (firstOnly)
            break;
        }
      }
    } else {
      const float surfaceAlpha = 0.6f;
      const float emission[2]  = {1.f, 0.8f};
      const RV3 lightDir[2]    = {rnormalize({1.f, 1.f, 1.f}), rnormalize({1.f, 1.f, -1.f})};
      HitIter h;
      hitInit(h, g, attr, {org.x, org.y, org.z}, {dir.x, dir.y, dir.z}, tr);
      HitRec hit;
      while (hitNext(h, g, filter, attr, hvr, vals, hit) && alpha < 0.99f) {
        const RV3 c = org + hit.t * dir;
        RV3 N       = rnormalize(gradientP(c));
        if (std::isnan(N.x) || std::isnan(N.y) || std::isnan(N.z))
          N = {0.f, 0.f, 0.f};
        const RV3 wi   = rnormalize({-1.f * dir.x, -1.f * dir.y, -1.f * dir.z});
        const float ci = rdot(N, wi);
        float illum    = 0.f;
        if (std::sqrt(rdot(N, N)) > 0.f) {
          illum = 0.1f;
          for (int i = 0; i < 2; ++i) {
            const RV3 wo   = lightDir[i];
            const float co = rdot(N, wo);
            if ((co > 0.f) == (ci > 0.f)) {
              HitIter sh;
              hitInit(sh, g, attr, {c.x, c.y, c.z}, {wo.x, wo.y, wo.z}, {hit.epsilon, inf});
              HitRec shadow;
              if (!hitNext(sh, g, filter, attr, hvr, vals, shadow))
                illum += std::fabs(co) * emission[i];
            }
          }
        } else {
          illum = 1.f;
        }
        float sc[4];
        tf.at(hit.sample, sc);
        color = color + ((1.f - alpha) * illum) * RV3{sc[0], sc[1], sc[2]};
        alpha = alpha + (1.f - alpha) * surfaceAlpha;
      }
    }
    rgba[4 * idx]     = color.x;
    rgba[4 * idx + 1] = color.y;
    rgba[4 * idx + 2] = color.z;
    rgba[4 * idx + 3] = 1.f;
  });
}

// The density path tracer (examples/interactive/renderer/density_path_tracer/
// DensityPathTracerGpuKernel.cpp:9-170, RandomTEA of Random.ih): one
// progressive frame added into rgba (4 floats per pixel) and weights.  The
// camera ray passes through the pixel centre as in orc_render.  pt: shutter,
// sigmaTScale, sigmaSScale, ambientLightIntensity, time; ipt: motionBlur,
// maxNumScatters, showBbox, frame.
void orc_path_trace(const OrcVolume *v, int filter, uint32_t maxSamplingDepth, uint32_t attr,
                    const float camera[14], const float *tfColors, int tfNum, const float tfRange[2], int W, int H,
                    const float bounds[6], const float pt[5], const int ipt[4], float *rgba, float *weights)
{
  const Grid &g = v->g;
  const RenderTF tf{tfColors, tfNum, tfRange[0], tfRange[1]};
  const float shutter = pt[0], sigmaMax0 = pt[1], sigmaSScale = pt[2], ambient = pt[3], time0 = pt[4];
  const bool motionBlur = ipt[0] != 0, showBbox = ipt[2] != 0;
  const int maxNumScatters = ipt[1];
  const uint32_t frame     = (uint32_t)ipt[3];
  const float inf          = std::numeric_limits<float>::infinity();
  struct Tea {
    uint32_t v0, v1;
    void floats(float &a, float &b)
    {
      uint32_t sum = 0;
      for (int i = 0; i < 8; ++i) {
        sum += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + sum) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + sum) ^ ((v0 >> 5) + 0x7e95761eu);
      }
      a = (float)v0 * 2.3283064365386962890625e-10f;
      b = (float)v1 * 2.3283064365386962890625e-10f;
    }
  };
  auto box = [&](RV3 org, RV3 dir) {
    const float rx = 1.f / dir.x, ry = 1.f / dir.y, rz = 1.f / dir.z;
    const float x0 = (bounds[0] - org.x) * rx, y0 = (bounds[1] - org.y) * ry, z0 = (bounds[2] - org.z) * rz;
    const float x1 = (bounds[3] - org.x) * rx, y1 = (bounds[4] - org.y) * ry, z1 = (bounds[5] - org.z) * rz;
    range1f tr;
    tr.lower = std::fmax(std::fmax(std::fmax(std::fmin(x0, x1), std::fmin(y0, y1)), std::fmin(z0, z1)), 0.f);
    tr.upper = std::fmin(std::fmin(std::fmin(std::fmax(x0, x1), std::fmax(y0, y1)), std::fmax(z0, z1)), inf);
    return tr;
  };
  parallelFor((int64_t)W * H, 0, 16, [&](int64_t idx) {
    const float px = (float)(idx % W) + 0.5f, py = (float)(idx / W) + 0.5f;
    const float irx     = 1.f / (float)W;
    const float sx      = (px - 0.5f * (float)W) * irx;
    const float sy      = -(py - 0.5f * (float)H) * irx;
    const RV3 pCamera   = {camera[0] * sx, camera[0] * sy, 0.f};
    const RV3 pAperture = {0.f, 0.f, -camera[1]};
    const RV3 dCamera   = pAperture - pCamera;
    const RV3 R0 = {camera[2], camera[3], camera[4]}, R1 = {camera[5], camera[6], camera[7]},
              R2 = {camera[8], camera[9], camera[10]};
    RV3 org = {rdot(R0, pCamera) + camera[11], rdot(R1, pCamera) + camera[12], rdot(R2, pCamera) + camera[13]};
    RV3 dir = rnormalize({rdot(R0, dCamera), rdot(R1, dCamera), rdot(R2, dCamera)});
    Tea rng{frame, (uint32_t)idx};
    int maxScatterIndex      = 0;
    bool primaryRayIntersect = false;
    RV3 Le = {0.f, 0.f, 0.f}, sigmaS = {0.f, 0.f, 0.f};
    for (int scatterIndex = 0; true; scatterIndex++) {
      float sample    = 0.f;
      maxScatterIndex = std::max(scatterIndex, maxScatterIndex);
      const range1f rt = box(org, dir);
      const bool empty = rt.lower > rt.upper;
      if (scatterIndex == 0 && !empty)
        primaryRayIntersect = true;
      if (empty)
        break;
      // sampleWoodcock
      float t = rt.lower, transmittance = 0.f;
      bool event = false;
      if (sigmaMax0 <= 0.f) {
        transmittance = 1.f;
      } else {
        for (int step = 0; step < (1 << 16); ++step) {
          float r0, r1, s0, s1;
          rng.floats(r0, r1);
          rng.floats(s0, s1);
          t = t + (-pt_log(1.f - r0)) / sigmaMax0;
          if (t > rt.upper) {
            transmittance = 1.f;
            break;
          }
          const RV3 c = org + t * dir;
          float time  = time0;
          if (motionBlur)
            time = time + (s0 - 0.5f) * shutter;
          t_time      = std::fmin(std::fmax(time, 0.f), 1.f);
          sample      = sampleAt(g, filter, xfmPoint(g.o2i, {c.x, c.y, c.z}), attr, maxSamplingDepth);
          t_time      = 0.f;
          float sc[4];
          tf.at(sample, sc);
          const float sigmaTSample = sigmaMax0 * sc[3];
          if (r1 < sigmaTSample / sigmaMax0) {
            event = true;
            break;
          }
          if (step + 1 == (1 << 16))
            event = true;
        }
        if (event)
          transmittance = 0.f;
      }
      if (!event) {
        if (scatterIndex > 0) {
          const float a = transmittance * ambient;
          Le            = Le + RV3{a * sigmaS.x, a * sigmaS.y, a * sigmaS.z};
        }
        break;
      }
      if (scatterIndex >= maxNumScatters)
        break;
      float sc[4];
      tf.at(sample, sc);
      sigmaS = {sigmaSScale * sc[0] * sc[3], sigmaSScale * sc[1] * sc[3], sigmaSScale * sc[2] * sc[3]};
      org    = org + t * dir;
      float s0, s1;
      rng.floats(s0, s1);
      const float phi      = 6.28318530717958647692f * s0;
      const float cosTheta = 1.f * (1.f - 2.f * s1);
      const float sinTheta = 2.f * 1.f * std::sqrt(s1 * (1.f - s1));
      float sinPhi, cosPhi;
      pt_sincos(phi, &sinPhi, &cosPhi);
      dir = {cosPhi * sinTheta, sinPhi * sinTheta, cosTheta};
    }
    RV3 color   = Le;
    float alpha = maxScatterIndex > 0 ? 1.f : 0.f;
    if (showBbox && primaryRayIntersect) {
      const float blend = 0.2f;
      alpha             = (1.f - blend) * alpha + blend * 1.f;
      color             = (1.f - blend) * color + RV3{blend * 1.f, blend * 1.f, blend * 1.f};
    }
    rgba[4 * idx]     = rgba[4 * idx] + color.x;
    rgba[4 * idx + 1] = rgba[4 * idx + 1] + color.y;
    rgba[4 * idx + 2] = rgba[4 * idx + 2] + color.z;
    rgba[4 * idx + 3] = rgba[4 * idx + 3] + alpha;
    weights[idx]      = weights[idx] + 1.f;
  });
}

int orc_tricubic_map(int32_t *start, int32_t *cols, float *weights)
{
  const TricubicMap &m = tricubicMap();
  if (start)
    std::copy(m.start.begin(), m.start.end(), start);
  if (cols)
    std::copy(m.col.begin(), m.col.end(), cols);
  if (weights)
    std::copy(m.w.begin(), m.w.end(), weights);
  return (int)m.col.size();
}

uint64_t orc_inner_nodes(const OrcVolume *v, uint32_t maxDepth, uint32_t attr, uint64_t cap,
                         float *out)
{
  const Grid &g = v->g;
  maxDepth      = std::min<uint32_t>(maxDepth, NUM_LEVELS - 1);
  uint64_t cnt  = 0;
  for (uint32_t l = 0; l <= maxDepth && l + 1 < NUM_LEVELS; ++l) {
    const Level &lv     = g.levels[l];
    const uint32_t res  = 1u << LOG_RES[l];
    const uint32_t cell = levelRes(l + 1);
    for (uint64_t n = 0; n < lv.numNodes; ++n)
      for (uint32_t vx = 0; vx < res; ++vx)
        for (uint32_t vy = 0; vy < res; ++vy)
          for (uint32_t vz = 0; vz < res; ++vz) {
            const uint64_t vi = (n << (3 * LOG_RES[l])) + ((uint64_t)vx << (2 * LOG_RES[l])) +
                                ((uint64_t)vy << LOG_RES[l]) + vz;
            const uint64_t voxel = lv.voxels[vi];
            if (!(vLeaf(voxel) || (l == maxDepth && !vEmpty(voxel))))
              continue;
            if (cnt < cap && out) {
              const float lo[3] = {(float)(g.rootOrigin.x + (int32_t)(lv.origin[n].x + cell * vx)),
                                   (float)(g.rootOrigin.y + (int32_t)(lv.origin[n].y + cell * vy)),
                                   (float)(g.rootOrigin.z + (int32_t)(lv.origin[n].z + cell * vz))};
              const float hi[3] = {lo[0] + (float)cell, lo[1] + (float)cell, lo[2] + (float)cell};
              float b[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
              for (int i = 0; i < 8; ++i) {
                const vec3f w = xfmPoint(g.i2o, {(i & 1) ? hi[0] : lo[0], (i & 2) ? hi[1] : lo[1],
                                                 (i & 4) ? hi[2] : lo[2]});
                b[0] = std::min(b[0], w.x);
                b[1] = std::min(b[1], w.y);
                b[2] = std::min(b[2], w.z);
                b[3] = std::max(b[3], w.x);
                b[4] = std::max(b[4], w.y);
                b[5] = std::max(b[5], w.z);
              }
              float *o = out + cnt * 8;
              std::memcpy(o, b, 24);
              o[6] = lv.valueRange[vi * g.numAttributes + attr].lower;
              o[7] = lv.valueRange[vi * g.numAttributes + attr].upper;
            }
            cnt++;
          }
  }
  return cnt;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Compressed leaves (extension of the cuda device, test restatement).
// Round to nearest, ties to even, to a binary format with `mant` stored
// mantissa bits and minimum normal exponent `emin` (subnormals below it):
// the value is a multiple of the format's spacing at its exponent, so
// scaling by that power of two and rounding to an integer is exact in double.
// ---------------------------------------------------------------------------
namespace {

float roundToFormat(float x, int mant, int emin, float maxFinite, bool saturate)
{
  if (std::isnan(x) || x == 0.f)
    return x;
  const float a = std::fabs(x);
  if (std::isinf(a))
    return saturate ? std::copysign(maxFinite, x) : x;
  int e = 0;
  std::frexp(a, &e);  // a = f * 2^e, f in [0.5, 1)
  int E = e - 1;
  if (E < emin)
    E = emin;
  const double q = std::ldexp(1.0, E - mant);
  double r       = std::nearbyint((double)a / q) * q;
  if (r > (double)maxFinite)
    r = saturate ? (double)maxFinite : (double)INFINITY;
  return std::copysign((float)r, x);
}

float roundFormat(int format, float x)
{
  switch (format) {
  case 1:
    return roundToFormat(x, 10, -14, 65504.f, false);
  case 2:
    return roundToFormat(x, 7, -126, 3.38953139e38f, false);
  default:
    return roundToFormat(x, 3, -6, 448.f, true);
  }
}

}  // namespace

void orc_round_format(int format, uint64_t n, const float *in, float *out)
{
  for (uint64_t i = 0; i < n; ++i)
    out[i] = roundFormat(format, in[i]);
}

void orc_quantize_leaves(int format, uint64_t numLeaves, const float *in, float *decoded,
                         float *scaleOffset)
{
  orc_quantize_groups(format, numLeaves, 512, in, decoded, scaleOffset);
}

void orc_quantize_groups(int format, uint64_t numGroups, uint32_t groupSize, const float *in,
                         float *decoded, float *scaleOffset)
{
  const float codeMax = format == 3 ? 448.f : 1.f;
  const uint64_t numLeaves = numGroups;
  for (uint64_t l = 0; l < numLeaves; ++l) {
    const float *v = in + l * groupSize;
    float lo = std::numeric_limits<float>::infinity(), hi = -lo;
    for (uint32_t i = 0; i < groupSize; ++i) {
      if (v[i] < lo)
        lo = v[i];
      if (v[i] > hi)
        hi = v[i];
    }
    lo += 0.f;
    hi += 0.f;
    float offset = 0.f, scale = 1.f;
    if (lo <= hi) {
      offset           = 0.5f * lo + 0.5f * hi;
      const float half = 0.5f * hi - 0.5f * lo;
      if (half > 0.f)
        scale = half / codeMax;
    }
    scaleOffset[2 * l]     = scale;
    scaleOffset[2 * l + 1] = offset;
    for (uint32_t i = 0; i < groupSize; ++i) {
      const float code              = roundFormat(format, (v[i] - offset) / scale);
      decoded[l * groupSize + i]    = code * scale + offset;
    }
  }
}

// Stencil-block leaves (the cuda device's extension; its kBuildLeafBlocks):
// the 9^3 sampling window of each dense leaf slot (the leaf's voxels plus
// the next voxel on the +x/+y/+z side) by full-depth lookups, x outermost,
// z fastest: windows[slot * 729 + x * 81 + y * 9 + z].
void orc_vdb_leaf_windows(const OrcVolume *v, uint32_t attr, float *windows)
{
  const Grid &g = v->g;
  uint64_t slot = 0;
  for (uint64_t i = 0; i < g.numLeaves; ++i) {
    if (g.leafFormat[i] != FMT_DENSE_ZYX)
      continue;
    const vec3i o = g.leafOrigin[i];
    float *w      = windows + slot++ * 729;
    for (int x = 0; x < 9; ++x)
      for (int y = 0; y < 9; ++y)
        for (int z = 0; z < 9; ++z)
          w[x * 81 + y * 9 + z] = traverseAndSample(g, {o.x + x, o.y + y, o.z + z}, attr, NUM_LEVELS - 1);
  }
}

void orc_vdb_set_windows(OrcVolume *v, uint32_t attr, uint64_t numSlots, const float *decodedWindows)
{
  Grid &g = v->g;
  if (g.blockWin.size() < g.numAttributes)
    g.blockWin.resize(g.numAttributes);
  g.blockWin[attr].assign(decodedWindows, decodedWindows + numSlots * 729);
}
