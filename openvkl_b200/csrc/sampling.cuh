// Device-side field access and reconstruction filters of the cuda device.
//
// Arithmetic follows the reference CPU device's float expressions operation
// by operation (the translation unit is built with --fmad=false so nothing is
// contracted into an FMA that the source does not spell out):
//   transforms      VdbGrid.h:56-89 (xfmPoint / xfmNormal)
//   nearest         VdbSampler_nearest.ih:15-57
//   trilinear       VdbSampler_trilinear.ih:378-399, gradient :751-780
//   tricubic        VdbSampler_tricubic.ih:34-580 (Lekien-Marsden map)
//   dense taps      VdbSampler_traverseAndSample.ih:313-349
//   sparse taps     VdbSampler_traverseAndSample.ih:85-306 with the
//                   generated per-level walk VdbSampleInner.ih.in:33-76
//   packed leaves   VdbSampler_packed_denseZYX.ih:77-187, _packed_tile.ih
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <stdint.h>

#include "grid.h"

namespace vklcuda {

struct f3 {
  float x, y, z;
};

// rkcommon lerp: (1 - f) * a + f * b.
__device__ __forceinline__ float lerpf(float f, float a, float b)
{
  return (1.f - f) * a + f * b;
}

// float -> int32 the way x86 cvttss2si does it (the CPU device's floor
// results go through it): NaN and out-of-range values give INT32_MIN.
__device__ __forceinline__ int32_t toIntX86(float x)
{
  return (x >= -2147483648.f && x < 2147483648.f) ? (int32_t)x : INT32_MIN;
}
// floor to int32 with the same out-of-range / NaN result (INT32_MIN); the
// round-down conversion saturates, so only |x| >= 2^31 and NaN need fixing.
__device__ __forceinline__ int32_t ifloor(float x)
{
  const int32_t i = __float2int_rd(x);
  return fabsf(x) < 2147483648.f ? i : INT32_MIN;
}

__device__ __forceinline__ f3 xfmPoint(const float *M, f3 p)
{
  return {M[0] * p.x + M[1] * p.y + M[2] * p.z + M[9],
          M[3] * p.x + M[4] * p.y + M[5] * p.z + M[10],
          M[6] * p.x + M[7] * p.y + M[8] * p.z + M[11]};
}
__device__ __forceinline__ f3 xfmVector(const float *M, f3 p)
{
  return {M[0] * p.x + M[1] * p.y + M[2] * p.z, M[3] * p.x + M[4] * p.y + M[5] * p.z,
          M[6] * p.x + M[7] * p.y + M[8] * p.z};
}
__device__ __forceinline__ f3 xfmNormal(const float *Mi, f3 p)
{
  return {Mi[0] * p.x + Mi[3] * p.y + Mi[6] * p.z, Mi[1] * p.x + Mi[4] * p.y + Mi[7] * p.z,
          Mi[2] * p.x + Mi[5] * p.y + Mi[8] * p.z};
}

// ---------------------------------------------------------------------------
// Typed loads (read-only path).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ float ldv(const T *p, uint64_t i);
template <>
__device__ __forceinline__ float ldv<float>(const float *p, uint64_t i)
{
  return __ldg(p + i);
}
template <>
__device__ __forceinline__ float ldv<uint8_t>(const uint8_t *p, uint64_t i)
{
  return (float)__ldg(p + i);
}
template <>
__device__ __forceinline__ float ldv<int16_t>(const int16_t *p, uint64_t i)
{
  return (float)__ldg(p + i);
}
template <>
__device__ __forceinline__ float ldv<uint16_t>(const uint16_t *p, uint64_t i)
{
  return (float)__ldg(p + i);
}
template <>
__device__ __forceinline__ float ldv<__half>(const __half *p, uint64_t i)
{
  return __half2float(__ldg(p + i));
}
template <>
__device__ __forceinline__ float ldv<double>(const double *p, uint64_t i)
{
  return __double2float_rn(__ldg(p + i));
}

__device__ __forceinline__ float ldAny(uint32_t type, const void *p, uint64_t i)
{
  switch (type) {
  case kUChar:
    return ldv((const uint8_t *)p, i);
  case kShort:
    return ldv((const int16_t *)p, i);
  case kUShort:
    return ldv((const uint16_t *)p, i);
  case kHalf:
    return ldv((const __half *)p, i);
  case kDouble:
    return ldv((const double *)p, i);
  default:
    return ldv((const float *)p, i);
  }
}

// ---------------------------------------------------------------------------
// Dense field: bricked voxel array (brickIndex, grid.h); out-of-domain taps
// read the background.  Which voxel a tap reads, and what it returns, is
// exactly the reference's x-fastest dense load; only the address differs.
// ---------------------------------------------------------------------------
template <typename T>
struct DenseField {
  const T *data;
  uint32_t ax, ay, az;
  int32_t rx, ry, rz;
  uint64_t yStride, zStride;  // supertile strides in elements: superX << 18, superX*superY << 18
  float bg;

  __device__ __forceinline__ DenseField(const DevGrid &g, uint32_t a)
      : data((const T *)g.data[a]),
        ax(g.activeSize[0]),
        ay(g.activeSize[1]),
        az(g.activeSize[2]),
        rx(g.rootOrigin[0]),
        ry(g.rootOrigin[1]),
        rz(g.rootOrigin[2]),
        yStride((uint64_t)g.superX << 18),
        zStride((uint64_t)g.superX * g.superY << 18),
        bg(g.background[a])
  {
  }

  // brickIndex(x, y, z) is a sum of one term per axis (its bit fields do not
  // overlap), so a stencil's addresses are sums of a few per-axis terms.
  __device__ __forceinline__ uint64_t termX(uint32_t x) const
  {
    return ((uint64_t)(x >> 6) << 18) + (((x >> 3) & 7u) << 9) + (x & 7u);
  }
  __device__ __forceinline__ uint64_t termY(uint32_t y) const
  {
    return (uint64_t)(y >> 6) * yStride + ((((y >> 3) & 7u) << 12) + ((y & 7u) << 3));
  }
  __device__ __forceinline__ uint64_t termZ(uint32_t z) const
  {
    return (uint64_t)(z >> 6) * zStride + ((((z >> 3) & 7u) << 15) + ((z & 7u) << 6));
  }

  __device__ __forceinline__ float at(int32_t x, int32_t y, int32_t z) const
  {
    const uint32_t ox = (uint32_t)(x - rx), oy = (uint32_t)(y - ry), oz = (uint32_t)(z - rz);
    if (ox < ax && oy < ay && oz < az)
      return ldv(data, termX(ox) + termY(oy) + termZ(oz));
    return bg;
  }

  // The W^3 taps s[W*W*i + W*j + k] at (x+LO+i, y+LO+j, z+LO+k); taps outside
  // the domain read the background.  Every lane issues the same W^3 loads
  // (predicated), with no branch on where its stencil falls.
  template <int W, int LO>
  __device__ __forceinline__ void stencil(int32_t x, int32_t y, int32_t z, float *s) const
  {
    const uint32_t ox = (uint32_t)(x - rx), oy = (uint32_t)(y - ry), oz = (uint32_t)(z - rz);
    uint64_t tx[W], ty[W], tz[W];
    bool vx[W], vy[W], vz[W];
#pragma unroll
    for (int i = 0; i < W; ++i) {
      const uint32_t u = ox + (uint32_t)(LO + i), v = oy + (uint32_t)(LO + i),
                     w = oz + (uint32_t)(LO + i);
      vx[i] = u < ax;
      vy[i] = v < ay;
      vz[i] = w < az;
      tx[i] = termX(u);
      ty[i] = termY(v);
      tz[i] = termZ(w);
    }
#pragma unroll
    for (int i = 0; i < W; ++i)
#pragma unroll
      for (int j = 0; j < W; ++j) {
        const uint64_t xy = tx[i] + ty[j];
        const bool ok     = vx[i] & vy[j];
#pragma unroll
        for (int k = 0; k < W; ++k)
          s[(i * W + j) * W + k] = (ok & vz[k]) ? ldv(data, xy + tz[k]) : bg;
      }
  }

  // The 8 trilinear corners s[4x+2y+z] at (x..x+1, y..y+1, z..z+1).
  __device__ __forceinline__ void corners(int32_t x, int32_t y, int32_t z, float s[8]) const
  {
    stencil<2, 0>(x, y, z, s);
  }

  // The 64 tricubic taps s[16x+4y+z] at offsets -1..2.
  __device__ __forceinline__ void stencil64(int32_t x, int32_t y, int32_t z, float s[64]) const
  {
    stencil<4, -1>(x, y, z, s);
  }
};

// ---------------------------------------------------------------------------
// Temporally varying dense data (motion blur): every tap is the voxel's
// value interpolated at the sample's time, then the spatial filter runs on
// those values as on constant data (the reference's dense structured /
// unstructured handlers, VdbSampler_dense.ih:347-500, with
// temporal_data_interpolation.ih:22-190).  The voxel arrays are x fastest
// with each voxel's time samples consecutive.  Times outside [0, 1] (which
// the reference asserts against in debug builds) are clamped into it.
// ---------------------------------------------------------------------------
template <typename T>
struct TemporalDenseField {
  const T *data;
  uint32_t ax, ay, az;
  int32_t rx, ry, rz;
  float bg;
  uint32_t format, N, idx64;
  const void *idx;
  const float *times;
  float time;

  __device__ __forceinline__ TemporalDenseField(const DevGrid &g, uint32_t a, float t)
      : data((const T *)g.data[a]),
        ax(g.activeSize[0]),
        ay(g.activeSize[1]),
        az(g.activeSize[2]),
        rx(g.rootOrigin[0]),
        ry(g.rootOrigin[1]),
        rz(g.rootOrigin[2]),
        bg(g.background[a]),
        format(g.temporal),
        N(g.numTimesteps),
        idx64(g.tIndex64),
        idx(g.tIndices),
        times(g.tTimes),
        time(fminf(fmaxf(t, 0.f), 1.f))
  {
  }

  __device__ __forceinline__ uint64_t index(uint64_t v) const
  {
    return idx64 ? __ldg((const unsigned long long *)idx + v) : (uint64_t)__ldg((const uint32_t *)idx + v);
  }

  // one voxel's value at `time`
  __device__ __forceinline__ float voxel(uint64_t v) const
  {
    if (format == 1) {
      const float tf      = time * ((float)(N - 1));
      const uint32_t ts   = (uint32_t)tf;
      const float w       = tf - (float)ts;
      const uint32_t next = (w == 0.f) ? ts : ts + 1;
      const uint64_t base = (uint64_t)N * v;
      return (1.f - w) * ldv(data, base + ts) + w * ldv(data, base + next);
    }
    const uint64_t b = index(v), e = index(v + 1);
    const float t0   = __ldg(times + b);
    if (time <= t0)
      return ldv(data, b);
    const float t1 = __ldg(times + e - 1);
    if (time >= t1)
      return ldv(data, e - 1);
    if (e - b == 2) {
      const float w = (time - t0) * (1.f / (t1 - t0));
      return (1.f - w) * ldv(data, b) + w * ldv(data, e - 1);
    }
    // binary search for the bracketing samples (at most 64 halvings: the
    // loop cannot run on when a time is out of order)
    uint64_t lower = 0, upper = e - b;
    for (int it = 0; it < 64 && lower <= upper; ++it) {
      const uint64_t mid = (lower + upper) / 2;
      const float tm     = __ldg(times + b + mid);
      if (time >= tm && time <= __ldg(times + b + mid + 1)) {
        lower = b + mid;
        upper = lower + 1;
        break;
      } else if (time < tm) {
        upper = mid;
      } else {
        lower = mid;
      }
    }
    const float tl = __ldg(times + lower), th = __ldg(times + upper);
    const float w  = (time - tl) * (1.f / (th - tl));
    return (1.f - w) * ldv(data, lower) + w * ldv(data, upper);
  }

  __device__ __forceinline__ float at(int32_t x, int32_t y, int32_t z) const
  {
    const uint32_t ox = (uint32_t)(x - rx), oy = (uint32_t)(y - ry), oz = (uint32_t)(z - rz);
    if (ox < ax && oy < ay && oz < az)
      return voxel((uint64_t)ox + (uint64_t)ax * ((uint64_t)oy + (uint64_t)ay * (uint64_t)oz));
    return bg;
  }

  __device__ __forceinline__ void corners(int32_t x, int32_t y, int32_t z, float s[8]) const
  {
#pragma unroll
    for (int c = 0; c < 8; ++c)
      s[c] = at(x + (c >> 2), y + ((c >> 1) & 1), z + (c & 1));
  }

  __device__ __forceinline__ void stencil64(int32_t x, int32_t y, int32_t z, float s[64]) const
  {
#pragma unroll 4
    for (int c = 0; c < 64; ++c)
      s[c] = at(x - 1 + (c >> 4), y - 1 + ((c >> 2) & 3), z - 1 + (c & 3));
  }
};

// ---------------------------------------------------------------------------
// Dense float attribute read through its z-plane texture atlas (DevGrid::
// atlasTex): the 8 trilinear corners are two tld4 footprint gathers, one per
// z-plane, instead of 8 loads through the L1 load/store pipe.  Point
// sampling returns the stored bits of every non-denormal float; the commit
// builds the atlas only for attributes without denormals, so the corners are
// the DenseField's.  Corners outside the domain read the background like
// DenseField::stencil: every lane issues both gathers and selects.
// tld4 returns the footprint (u0,v0)..(u1,v1), u0 = floor(u - 0.5), as
// .x (u0,v1)  .y (u1,v1)  .z (u1,v0)  .w (u0,v0).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float4 tld4Red(uint64_t tex, float u, float v)
{
  float4 r;
  asm volatile("tld4.r.2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6}];"
               : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
               : "l"(tex), "f"(u), "f"(v));
  return r;
}

struct AtlasField {
  uint64_t tex;
  uint32_t ax, ay, az;
  int32_t rx, ry, rz;
  uint32_t planeMask, planeShift;  // planes per atlas row (a power of two) - 1, log2
  float bg;

  __device__ __forceinline__ AtlasField(const DevGrid &g, uint32_t a)
      : tex(g.atlasTex[a]),
        ax(g.activeSize[0]),
        ay(g.activeSize[1]),
        az(g.activeSize[2]),
        rx(g.rootOrigin[0]),
        ry(g.rootOrigin[1]),
        rz(g.rootOrigin[2]),
        planeMask(g.atlasPlanesPerRow - 1u),
        planeShift(0u),
        bg(g.background[a])
  {
    while ((1u << planeShift) < g.atlasPlanesPerRow)
      ++planeShift;
  }

  __device__ __forceinline__ void corners(int32_t x, int32_t y, int32_t z, float s[8]) const
  {
    const uint32_t ox = (uint32_t)(x - rx), oy = (uint32_t)(y - ry), oz = (uint32_t)(z - rz);
    const bool vx0 = ox < ax, vx1 = ox + 1u < ax, vy0 = oy < ay, vy1 = oy + 1u < ay, vz0 = oz < az,
               vz1 = oz + 1u < az;
    // footprint origin inside the plane's tile: (ox, oy) when valid, else
    // (-1, -1) relative (only the +1 corner can be in the domain then).  The
    // texel coordinates are integers below 2^24 (texture rows are at most
    // 2^17 texels), so summing them as integers and converting once gives
    // the same floats as converting the parts.
    const uint32_t ux = vx0 ? ox + 1u : 0u, uy = vy0 ? oy + 1u : 0u;
    const uint32_t z0 = vz0 ? oz : 0u, z1 = vz1 ? oz + 1u : 0u;
    const float4 a = tld4Red(tex, (float)((z0 & planeMask) * ax + ux), (float)((z0 >> planeShift) * ay + uy));
    const float4 b = tld4Red(tex, (float)((z1 & planeMask) * ax + ux), (float)((z1 >> planeShift) * ay + uy));
    if (vx0 & vx1 & vy0 & vy1 & vz0 & vz1) {
      // every corner in the domain (all but the volume's outer shell)
      s[0] = a.w;
      s[1] = b.w;
      s[2] = a.x;
      s[3] = b.x;
      s[4] = a.z;
      s[5] = b.z;
      s[6] = a.y;
      s[7] = b.y;
      return;
    }
    s[0] = (vx0 & vy0 & vz0) ? a.w : bg;
    s[1] = (vx0 & vy0 & vz1) ? b.w : bg;
    s[2] = (vx0 & vy1 & vz0) ? a.x : bg;
    s[3] = (vx0 & vy1 & vz1) ? b.x : bg;
    s[4] = (vx1 & vy0 & vz0) ? a.z : bg;
    s[5] = (vx1 & vy0 & vz1) ? b.z : bg;
    s[6] = (vx1 & vy1 & vz0) ? a.y : bg;
    s[7] = (vx1 & vy1 & vz1) ? b.y : bg;
  }
};

// ---------------------------------------------------------------------------
// Leaf codecs of sparse volumes.  T = float / __half: the leaf arrays hold the
// values.  The Code* tags: compressed leaves (an extension, no reference
// counterpart) hold FP16 / BF16 / FP8-E4M3 codes, value = code * scale +
// offset with one (scale, offset) pair per packed leaf, decoded in FP32;
// tiles stay float.
// ---------------------------------------------------------------------------
struct CodeFP16 {};
struct CodeBF16 {};
struct CodeE4M3 {};
// Stencil-block leaves (kLeafBlockCodes / leafBlockCode in grid.h): the
// same codes, laid out as 8 blocks of 5^3 per leaf whose (scale, offset)
// spans the leaf's 9^3 sampling window.
template <class C>
struct Blocked {};

template <typename T>
struct LeafCodec {
  static constexpr bool kScaled  = false;
  static constexpr bool kBlocked = false;
  using Tile                     = T;
  using Code                     = T;
};
template <>
struct LeafCodec<CodeFP16> {
  static constexpr bool kScaled  = true;
  static constexpr bool kBlocked = false;
  using Tile                     = float;
  using Code                     = __half;
};
template <>
struct LeafCodec<CodeBF16> {
  static constexpr bool kScaled  = true;
  static constexpr bool kBlocked = false;
  using Tile                     = float;
  using Code                     = __nv_bfloat16;
};
template <>
struct LeafCodec<CodeE4M3> {
  static constexpr bool kScaled  = true;
  static constexpr bool kBlocked = false;
  using Tile                     = float;
  using Code                     = __nv_fp8_storage_t;
};
template <class C>
struct LeafCodec<Blocked<C>> : LeafCodec<C> {
  static constexpr bool kBlocked = true;
};

// Offset of leaf voxel (x, y, z) (low 3 bits of each used) within its
// leaf's slot of the data array: z-fastest 8^3, or the stencil-block layout.
template <typename T>
__device__ __forceinline__ uint64_t leafVoxelIndex(uint64_t li, uint32_t x, uint32_t y, uint32_t z)
{
  if constexpr (LeafCodec<T>::kBlocked)
    return li * kLeafCodes + leafBlockCode(x & 7u, y & 7u, z & 7u);
  else
    return li * 512 + ((uint64_t)(x & 7u) << 6) + ((y & 7u) << 3) + (z & 7u);
}

__device__ __forceinline__ float ldCode(const __half *p, uint64_t i)
{
  return __half2float(__ldg(p + i));
}
__device__ __forceinline__ float ldCode(const __nv_bfloat16 *p, uint64_t i)
{
  return __bfloat162float(__ldg(p + i));
}
__device__ __forceinline__ float ldCode(const __nv_fp8_storage_t *p, uint64_t i)
{
  return __half2float(__half(__nv_cvt_fp8_to_halfraw(__ldg(p + i), __NV_E4M3)));
}

// Value of voxel vi of packed leaf li (vi counts from the start of the leaf array).
template <typename T>
__device__ __forceinline__ float packedLeafValue(const DevGrid &g, uint32_t attr, uint64_t li,
                                                 uint64_t vi)
{
  if constexpr (LeafCodec<T>::kScaled) {
    const float code = ldCode((const typename LeafCodec<T>::Code *)g.data[attr], vi);
    const float2 so  = __ldg((const float2 *)g.leafScaleOffset[attr] + li);
    return code * so.x + so.y;
  } else {
    return ldv((const T *)g.data[attr], vi);
  }
}

template <typename T>
__device__ __forceinline__ float tileValue(const DevGrid &g, uint32_t attr, uint64_t li)
{
  return ldv((const typename LeafCodec<T>::Tile *)g.tile[attr], li);
}

// ---------------------------------------------------------------------------
// Sparse field: 4-level tree walk, packed leaves, tiles, error voxels.
// ---------------------------------------------------------------------------
template <typename T>
struct SparseField {
  const DevGrid &g;
  uint32_t attr;
  uint32_t maxDepth;

  __device__ __forceinline__ SparseField(const DevGrid &grid, uint32_t a, uint32_t depth)
      : g(grid), attr(a), maxDepth(depth)
  {
  }

  // The voxel holding the leaf that contains the (in-domain, root-relative)
  // offset: one load from the flat leaf map at full depth, else the walk.
  __device__ __forceinline__ uint64_t traverse(uint32_t ox, uint32_t oy, uint32_t oz) const
  {
    const uint64_t v =
        (g.leafMap && maxDepth >= kNumLevels - 1)
            ? __ldg(g.leafMap + ((uint64_t)(oz >> 3) * g.leafMapDims[1] + (oy >> 3)) * g.leafMapDims[0] + (ox >> 3))
            : walk(ox, oy, oz);
    // LeafNodeAccess observers (VdbSampleInner.ih.in:68-74): a reached leaf
    // (not an empty or depth-limited voxel) is marked in every buffer
    if (g.numLeafAccess && voxelIsLeaf(v))
      for (uint32_t i = 0; i < g.numLeafAccess; ++i)
        g.leafAccess[i][voxelLeafIndex(v)] = 1u;
    return v;
  }

  // Walk from the root to the voxel holding the leaf that contains the
  // (in-domain, root-relative) offset.
  __device__ __forceinline__ uint64_t walk(uint32_t ox, uint32_t oy, uint32_t oz) const
  {
    const uint32_t lx = ox & ~7u, ly = oy & ~7u, lz = oz & ~7u;
    uint64_t node = 0;
#pragma unroll
    for (uint32_t l = 0; l < kNumLevels - 1; ++l) {
      const uint64_t vo   = node * levelNumVoxels(l) + offsetToLinear(l, lx, ly, lz);
      const uint32_t vo32 = (uint32_t)vo;
      const uint64_t v    = __ldg(g.levels[l].voxels + vo32);
      if ((voxelIsLeaf(v) || voxelIsChild(v)) && (l + 1 > maxDepth))
        return voxelMakeError(l, vo32);
      if (voxelIsChild(v) && l + 1 < kNumLevels - 1) {
        node = voxelChildIndex(v);
        continue;
      }
      return v;
    }
    return 0;
  }

  // (scale, offset) of the packed leaf a voxel code points at; (1, 0) for
  // uncompressed leaves and everything else.
  __device__ __forceinline__ float2 leafScale(uint64_t voxel) const
  {
    if constexpr (LeafCodec<T>::kScaled) {
      if (voxelIsLeaf(voxel) && voxelLeafFormat(voxel) != kFormatTile)
        return __ldg((const float2 *)g.leafScaleOffset[attr] + voxelLeafIndex(voxel));
    }
    return make_float2(1.f, 0.f);
  }

  __device__ __forceinline__ float leafValue(uint64_t voxel, uint32_t ox, uint32_t oy,
                                             uint32_t oz) const
  {
    return leafValueWith(voxel, leafScale(voxel), ox, oy, oz);
  }

  __device__ __forceinline__ float leafValueWith(uint64_t voxel, float2 so, uint32_t ox,
                                                 uint32_t oy, uint32_t oz) const
  {
    if (voxelIsLeaf(voxel)) {
      const uint64_t li = voxelLeafIndex(voxel);
      if (voxelLeafFormat(voxel) == kFormatTile)
        return tileValue<T>(g, attr, li);
      const uint64_t vi = leafVoxelIndex<T>(li, ox, oy, oz);
      if constexpr (LeafCodec<T>::kScaled)
        return ldCode((const typename LeafCodec<T>::Code *)g.data[attr], vi) * so.x + so.y;
      else
        return ldv((const T *)g.data[attr], vi);
    } else if (voxelIsError(voxel)) {
      const uint32_t level = (uint32_t)((voxel >> 8) & 0xffu);
      const uint32_t off   = (uint32_t)(voxel >> 32);
      const float *r = g.levels[level].valueRange + 2 * ((uint64_t)off * g.numAttributes + attr);
      return 0.5f * (__ldg(r) + __ldg(r + 1));
    } else if (!(ox < g.activeSize[0] && oy < g.activeSize[1] && oz < g.activeSize[2])) {
      return g.background[attr];
    }
    return 0.f;
  }

  __device__ __forceinline__ bool inDomain(uint32_t ox, uint32_t oy, uint32_t oz) const
  {
    return ox < g.activeSize[0] && oy < g.activeSize[1] && oz < g.activeSize[2];
  }

  __device__ __forceinline__ float at(int32_t x, int32_t y, int32_t z) const
  {
    const uint32_t ox = (uint32_t)(x - g.rootOrigin[0]), oy = (uint32_t)(y - g.rootOrigin[1]),
                   oz = (uint32_t)(z - g.rootOrigin[2]);
    if (!inDomain(ox, oy, oz))
      return g.background[attr];
    return leafValue(traverse(ox, oy, oz), ox, oy, oz);
  }

  // Taps of a stencil spanning offsets [lo, lo+W) per axis reuse one walk
  // per distinct leaf: the walk result depends only on the leaf origin
  // (offset & ~7), and W <= 8 means at most two leaves per axis.
  template <int W, int LO>
  __device__ __forceinline__ void stencil(int32_t x, int32_t y, int32_t z, float *s) const
  {
    const uint32_t bx = (uint32_t)(x + LO - g.rootOrigin[0]),
                   by = (uint32_t)(y + LO - g.rootOrigin[1]),
                   bz = (uint32_t)(z + LO - g.rootOrigin[2]);
    if constexpr (W == 2) {
      // 2^3 corners: along an axis the second corner is in the next leaf
      // only when the first sits on the leaf's last voxel.  Leaf slot s
      // (bit 2 = x, 1 = y, 0 = z) is needed when its bits are a subset of
      // the crossing axes; each corner selects its slot with static selects,
      // so the codes stay in registers.
      const bool cx = (bx & 7u) == 7u, cy = (by & 7u) == 7u, cz = (bz & 7u) == 7u;
      const bool inx[2] = {bx < g.activeSize[0], bx + 1 < g.activeSize[0]};
      const bool iny[2] = {by < g.activeSize[1], by + 1 < g.activeSize[1]};
      const bool inz[2] = {bz < g.activeSize[2], bz + 1 < g.activeSize[2]};
      const uint64_t base = (inx[0] && iny[0] && inz[0]) ? traverse(bx, by, bz) : 0ull;
      if constexpr (LeafCodec<T>::kBlocked) {
        // Stencil-block leaves: when the base voxel lies in a dense leaf, all
        // 8 corners are that leaf's block codes (one leaf lookup, one block).
        if (voxelIsLeaf(base) && voxelLeafFormat(base) != kFormatTile) {
          const uint64_t li = voxelLeafIndex(base);
          const float2 so   = __ldg((const float2 *)g.leafScaleOffset[attr] + li);
          const auto *c     = (const typename LeafCodec<T>::Code *)g.data[attr] + leafVoxelIndex<T>(li, bx, by, bz);
#pragma unroll
          for (int o = 0; o < 8; ++o)
            s[o] = ldCode(c, (o >> 2) * 25 + ((o >> 1) & 1) * 5 + (o & 1)) * so.x + so.y;
          return;
        }
      }
      uint64_t code[8];
      float2 sc[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int i = q >> 2, j = (q >> 1) & 1, k = q & 1;
        const bool need = (!i || cx) && (!j || cy) && (!k || cz) && inx[i] && iny[j] && inz[k];
        code[q] = q == 0 ? base : (need ? traverse(bx + i, by + j, bz + k) : 0ull);
        sc[q]   = need ? leafScale(code[q]) : make_float2(1.f, 0.f);
      }
#pragma unroll
      for (int o = 0; o < 8; ++o) {
        const int i = o >> 2, j = (o >> 1) & 1, k = o & 1;
        const uint32_t ox = bx + i, oy = by + j, oz = bz + k;
        if (!(inx[i] && iny[j] && inz[k])) {
          s[o] = g.background[attr];
          continue;
        }
        const bool ux = i && cx, uy = j && cy, uz = k && cz;
        const uint64_t c0 = uz ? code[1] : code[0], c1 = uz ? code[3] : code[2],
                       c2 = uz ? code[5] : code[4], c3 = uz ? code[7] : code[6];
        const float2 f0 = uz ? sc[1] : sc[0], f1 = uz ? sc[3] : sc[2], f2 = uz ? sc[5] : sc[4],
                     f3 = uz ? sc[7] : sc[6];
        const uint64_t cv = ux ? (uy ? c3 : c2) : (uy ? c1 : c0);
        const float2 fv   = ux ? (uy ? f3 : f2) : (uy ? f1 : f0);
        s[o]              = leafValueWith(cv, fv, ox, oy, oz);
      }
      return;
    }
    uint64_t cache[8];
    float2 scale[8];
    uint32_t have = 0;
#pragma unroll
    for (int o = 0; o < W * W * W; ++o) {
      const int dx = o / (W * W), dy = (o / W) % W, dz = o % W;
      const uint32_t ox = bx + dx, oy = by + dy, oz = bz + dz;
      if (!inDomain(ox, oy, oz)) {
        s[o] = g.background[attr];
        continue;
      }
      const uint32_t slot = (((ox & ~7u) != (bx & ~7u)) << 2) |
                            (((oy & ~7u) != (by & ~7u)) << 1) | ((oz & ~7u) != (bz & ~7u));
      if (!(have & (1u << slot))) {
        cache[slot] = traverse(ox, oy, oz);
        scale[slot] = leafScale(cache[slot]);
        have |= 1u << slot;
      }
      s[o] = leafValueWith(cache[slot], scale[slot], ox, oy, oz);
    }
  }

  __device__ __forceinline__ void corners(int32_t x, int32_t y, int32_t z, float s[8]) const
  {
    stencil<2, 0>(x, y, z, s);
  }
  __device__ __forceinline__ void stencil64(int32_t x, int32_t y, int32_t z, float s[64]) const
  {
    stencil<4, -1>(x, y, z, s);
  }
};

// ---------------------------------------------------------------------------
// Filters.
// ---------------------------------------------------------------------------
template <class Field>
__device__ __forceinline__ float sampleNearest(const Field &F, bool cellCentered, f3 p)
{
  const float off = cellCentered ? 0.f : 0.5f;
  return F.at(ifloor(p.x + off), ifloor(p.y + off), ifloor(p.z + off));
}

template <class Field>
__device__ __forceinline__ float sampleLinear(const Field &F, f3 p)
{
  const int32_t ix = ifloor(p.x), iy = ifloor(p.y), iz = ifloor(p.z);
  const float dx = p.x - (float)ix, dy = p.y - (float)iy, dz = p.z - (float)iz;
  float s[8];
  F.corners(ix, iy, iz, s);
  return lerpf(dx, lerpf(dy, lerpf(dz, s[0], s[1]), lerpf(dz, s[2], s[3])),
               lerpf(dy, lerpf(dz, s[4], s[5]), lerpf(dz, s[6], s[7])));
}

template <class Field>
__device__ __forceinline__ f3 gradientLinear(const Field &F, f3 p)
{
  const int32_t ix = ifloor(p.x), iy = ifloor(p.y), iz = ifloor(p.z);
  const float dx = p.x - (float)ix, dy = p.y - (float)iy, dz = p.z - (float)iz;
  float s[8];
  F.corners(ix, iy, iz, s);
  f3 r;
  r.x = lerpf(dy, lerpf(dz, s[4] - s[0], s[5] - s[1]), lerpf(dz, s[6] - s[2], s[7] - s[3]));
  r.y = lerpf(dx, lerpf(dz, s[2] - s[0], s[3] - s[1]), lerpf(dz, s[6] - s[4], s[7] - s[5]));
  r.z = lerpf(dx, lerpf(dy, s[1] - s[0], s[3] - s[2]), lerpf(dy, s[5] - s[4], s[7] - s[6]));
  return r;
}

// Lekien-Marsden tricubic: constraints from central differences, then the
// 64x64 coefficient map.  The map is the tensor product of the 1D cubic
// Hermite map; its non-zero entries, summed per row in ascending column order
// exactly as the reference's expanded expressions are, live in
// tricubic_map.cuh (generated, with a test that pins it to the reference).
#include "tricubic_map.cuh"

__device__ __forceinline__ void tricubicCoefficients(const float s[64], float coef[64])
{
#define S(X, Y, Z) s[((X) + 1) * 16 + ((Y) + 1) * 4 + ((Z) + 1)]
  float ctr[64];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int x = c >> 2, y = (c >> 1) & 1, z = c & 1;
    ctr[c]      = S(x, y, z);
    ctr[8 + c]  = 0.5f * (-S(x - 1, y, z) + S(x + 1, y, z));
    ctr[16 + c] = 0.5f * (-S(x, y - 1, z) + S(x, y + 1, z));
    ctr[24 + c] = 0.5f * (-S(x, y, z - 1) + S(x, y, z + 1));
    ctr[32 + c] = 0.25f * (S(x - 1, y - 1, z) - S(x - 1, y + 1, z) - S(x + 1, y - 1, z) +
                           S(x + 1, y + 1, z));
    ctr[40 + c] = 0.25f * (S(x - 1, y, z - 1) - S(x - 1, y, z + 1) - S(x + 1, y, z - 1) +
                           S(x + 1, y, z + 1));
    ctr[48 + c] = 0.25f * (S(x, y - 1, z - 1) - S(x, y - 1, z + 1) - S(x, y + 1, z - 1) +
                           S(x, y + 1, z + 1));
    ctr[56 + c] = 0.125f * (-S(x - 1, y - 1, z - 1) + S(x - 1, y - 1, z + 1) +
                            S(x - 1, y + 1, z - 1) - S(x - 1, y + 1, z + 1) +
                            S(x + 1, y - 1, z - 1) - S(x + 1, y - 1, z + 1) -
                            S(x + 1, y + 1, z - 1) + S(x + 1, y + 1, z + 1));
  }
#undef S
  VKL_TRICUBIC_MAP(ctr, coef)
}

template <class Field>
__device__ __forceinline__ float sampleCubic(const Field &F, f3 p)
{
  const int32_t ix = ifloor(p.x), iy = ifloor(p.y), iz = ifloor(p.z);
  float s[64], c[64];
  F.stencil64(ix, iy, iz, s);
  tricubicCoefficients(s, c);
  const float dx = p.x - (float)ix, dy = p.y - (float)iy, dz = p.z - (float)iz;
  const float X[4] = {1.f, dx, dx * dx, dx * dx * dx};
  const float Y[4] = {1.f, dy, dy * dy, dy * dy * dy};
  const float Z[4] = {1.f, dz, dz * dz, dz * dz * dz};
  float r = 0.f;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k)
        r += c[16 * i + 4 * j + k] * X[i] * Y[j] * Z[k];
  return r;
}

template <class Field>
__device__ __forceinline__ f3 gradientCubic(const Field &F, f3 p)
{
  const int32_t ix = ifloor(p.x), iy = ifloor(p.y), iz = ifloor(p.z);
  float s[64], c[64];
  F.stencil64(ix, iy, iz, s);
  tricubicCoefficients(s, c);
  const float dx = p.x - (float)ix, dy = p.y - (float)iy, dz = p.z - (float)iz;
  const float X[4] = {1.f, dx, dx * dx, dx * dx * dx};
  const float Y[4] = {1.f, dy, dy * dy, dy * dy * dy};
  const float Z[4] = {1.f, dz, dz * dz, dz * dz * dz};
  f3 r = {0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float cc = c[16 * i + 4 * j + k];
        if (i > 0)
          r.x += cc * (float)i * X[i - 1] * Y[j] * Z[k];
        if (j > 0)
          r.y += cc * (float)j * X[i] * Y[j - 1] * Z[k];
        if (k > 0)
          r.z += cc * (float)k * X[i] * Y[j] * Z[k - 1];
      }
  return r;
}

template <class Field>
__device__ __forceinline__ float sampleFiltered(const Field &F, int filter, bool cellCentered, f3 p)
{
  if (filter == kFilterNearest)
    return sampleNearest(F, cellCentered, p);
  if (filter == kFilterCubic)
    return sampleCubic(F, p);
  return sampleLinear(F, p);
}

// Sample at an object-space point with runtime type dispatch (used by the
// hit iterator's marching, VdbSampler_iterator_computeSample_varying,
// VdbSampler.ispc:341-374).
// Temporally varying dense data: F is TemporalDenseField<T> at `time`.
template <class Fn>
__device__ __forceinline__ auto withTemporalField(const DevGrid &g, uint32_t attr, float time, Fn &&fn)
{
  switch (g.type[attr]) {
  case kUChar:
    return fn(TemporalDenseField<uint8_t>(g, attr, time));
  case kShort:
    return fn(TemporalDenseField<int16_t>(g, attr, time));
  case kUShort:
    return fn(TemporalDenseField<uint16_t>(g, attr, time));
  case kHalf:
    return fn(TemporalDenseField<__half>(g, attr, time));
  case kDouble:
    return fn(TemporalDenseField<double>(g, attr, time));
  default:
    return fn(TemporalDenseField<float>(g, attr, time));
  }
}

__device__ __forceinline__ float sampleIndexAny(const DevGrid &g, int filter, uint32_t attr,
                                                uint32_t depth, f3 p, float time = 0.f)
{
  const bool cc = g.constantCellData != 0;
  const uint32_t t = g.type[attr];
  if (g.temporal)
    return withTemporalField(g, attr, time, [&](const auto &F) { return sampleFiltered(F, filter, cc, p); });
  if (g.dense) {
    switch (t) {
    case kUChar:
      return sampleFiltered(DenseField<uint8_t>(g, attr), filter, cc, p);
    case kShort:
      return sampleFiltered(DenseField<int16_t>(g, attr), filter, cc, p);
    case kUShort:
      return sampleFiltered(DenseField<uint16_t>(g, attr), filter, cc, p);
    case kHalf:
      return sampleFiltered(DenseField<__half>(g, attr), filter, cc, p);
    case kDouble:
      return sampleFiltered(DenseField<double>(g, attr), filter, cc, p);
    default:
      return sampleFiltered(DenseField<float>(g, attr), filter, cc, p);
    }
  }
  switch (g.compress) {
  case kCompressFP16:
    return sampleFiltered(SparseField<CodeFP16>(g, attr, depth), filter, cc, p);
  case kCompressBF16:
    return sampleFiltered(SparseField<CodeBF16>(g, attr, depth), filter, cc, p);
  case kCompressFP8:
    return sampleFiltered(SparseField<CodeE4M3>(g, attr, depth), filter, cc, p);
  case kCompressFP16Blocks:
    return sampleFiltered(SparseField<Blocked<CodeFP16>>(g, attr, depth), filter, cc, p);
  case kCompressBF16Blocks:
    return sampleFiltered(SparseField<Blocked<CodeBF16>>(g, attr, depth), filter, cc, p);
  case kCompressFP8Blocks:
    return sampleFiltered(SparseField<Blocked<CodeE4M3>>(g, attr, depth), filter, cc, p);
  default:
    break;
  }
  if (t == kHalf)
    return sampleFiltered(SparseField<__half>(g, attr, depth), filter, cc, p);
  return sampleFiltered(SparseField<float>(g, attr, depth), filter, cc, p);
}

// Object-space gradient with runtime type dispatch: the index-space
// gradient of the filter (zero for nearest) through xfmNormal, as the
// gradient kernels compute it (VdbSampler.ispc:276-301).
template <class Field>
__device__ __forceinline__ f3 gradientFiltered(const DevGrid &g, const Field &F, int filter, f3 p)
{
  if (filter == kFilterNearest)
    return {0.f, 0.f, 0.f};
  const f3 gi = filter == kFilterCubic ? gradientCubic(F, p) : gradientLinear(F, p);
  return xfmNormal(g.objectToIndex, gi);
}

__device__ __forceinline__ f3 gradientObjectAny(const DevGrid &g, int filter, uint32_t attr, uint32_t depth, f3 oc,
                                                float time = 0.f)
{
  const f3 p       = xfmPoint(g.objectToIndex, oc);
  const uint32_t t = g.type[attr];
  if (g.temporal)
    return withTemporalField(g, attr, time, [&](const auto &F) { return gradientFiltered(g, F, filter, p); });
  if (g.dense) {
    switch (t) {
    case kUChar:
      return gradientFiltered(g, DenseField<uint8_t>(g, attr), filter, p);
    case kShort:
      return gradientFiltered(g, DenseField<int16_t>(g, attr), filter, p);
    case kUShort:
      return gradientFiltered(g, DenseField<uint16_t>(g, attr), filter, p);
    case kHalf:
      return gradientFiltered(g, DenseField<__half>(g, attr), filter, p);
    case kDouble:
      return gradientFiltered(g, DenseField<double>(g, attr), filter, p);
    default:
      return gradientFiltered(g, DenseField<float>(g, attr), filter, p);
    }
  }
  switch (g.compress) {
  case kCompressFP16:
    return gradientFiltered(g, SparseField<CodeFP16>(g, attr, depth), filter, p);
  case kCompressBF16:
    return gradientFiltered(g, SparseField<CodeBF16>(g, attr, depth), filter, p);
  case kCompressFP8:
    return gradientFiltered(g, SparseField<CodeE4M3>(g, attr, depth), filter, p);
  case kCompressFP16Blocks:
    return gradientFiltered(g, SparseField<Blocked<CodeFP16>>(g, attr, depth), filter, p);
  case kCompressBF16Blocks:
    return gradientFiltered(g, SparseField<Blocked<CodeBF16>>(g, attr, depth), filter, p);
  case kCompressFP8Blocks:
    return gradientFiltered(g, SparseField<Blocked<CodeE4M3>>(g, attr, depth), filter, p);
  default:
    break;
  }
  if (t == kHalf)
    return gradientFiltered(g, SparseField<__half>(g, attr, depth), filter, p);
  return gradientFiltered(g, SparseField<float>(g, attr, depth), filter, p);
}

__device__ __forceinline__ float sampleObjectAny(const DevGrid &g, int filter, uint32_t attr,
                                                 uint32_t depth, f3 oc, float time = 0.f)
{
  return sampleIndexAny(g, filter, attr, depth, xfmPoint(g.objectToIndex, oc), time);
}

}  // namespace vklcuda
