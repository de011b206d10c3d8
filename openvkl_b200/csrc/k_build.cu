// Commit-time kernels of the cuda device: dense tree construction and the
// value-range builder (per-leaf filter-support ranges, then propagation up
// the tree), the reference's VdbVolume::commit hot loops
// (openvkl/devices/cpu/volume/vdb/VdbVolume.cpp:338-392,
// VdbSampler.ispc:383-557) as GPU kernels.
#include "kernels.h"
#include "objects.h"
#include "sampling.cuh"

namespace vklcuda {

namespace {

constexpr float kInf = __builtin_huge_valf();

__device__ __forceinline__ float fminx(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmaxx(float a, float b) { return a > b ? a : b; }

// ---------------------------------------------------------------------------
// Dense tree.  Leaves are inserted in x-fastest order, so level-l nodes are
// numbered in (z, y, x)-lexicographic order of their origins, which is what
// the reference's first-come insertion (VdbVolume.cpp:244-331) produces.
// ---------------------------------------------------------------------------
__global__ void kDenseLevel2(uint64_t *vox2, uint32_t *org2, uint3 nl, uint3 n2)
{
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t total = (uint64_t)n2.x * n2.y * n2.z * 4096;
  if (i >= total)
    return;
  const uint64_t k2 = i >> 12;
  const uint32_t v  = (uint32_t)(i & 4095);
  const uint32_t vx = v >> 8, vy = (v >> 4) & 15, vz = v & 15;
  const uint32_t x2 = (uint32_t)(k2 % n2.x), y2 = (uint32_t)((k2 / n2.x) % n2.y),
                 z2 = (uint32_t)(k2 / ((uint64_t)n2.x * n2.y));
  const uint32_t lx = x2 * 16 + vx, ly = y2 * 16 + vy, lz = z2 * 16 + vz;
  uint64_t code = 0;
  if (lx < nl.x && ly < nl.y && lz < nl.z)
    code = voxelMakeLeaf(((uint64_t)lz * nl.y + ly) * nl.x + lx, kFormatDenseZYX, 0);
  vox2[i] = code;
  if (v == 0) {
    org2[3 * k2]     = x2 * 128;
    org2[3 * k2 + 1] = y2 * 128;
    org2[3 * k2 + 2] = z2 * 128;
  }
}

__global__ void kDenseLevel1(uint64_t *vox1, uint32_t *org1, uint3 n2, uint3 n1)
{
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t total = (uint64_t)n1.x * n1.y * n1.z * 32768;
  if (i >= total)
    return;
  const uint64_t k1 = i >> 15;
  const uint32_t v  = (uint32_t)(i & 32767);
  const uint32_t vx = v >> 10, vy = (v >> 5) & 31, vz = v & 31;
  const uint32_t x1 = (uint32_t)(k1 % n1.x), y1 = (uint32_t)((k1 / n1.x) % n1.y),
                 z1 = (uint32_t)(k1 / ((uint64_t)n1.x * n1.y));
  const uint32_t x2 = x1 * 32 + vx, y2 = y1 * 32 + vy, z2 = z1 * 32 + vz;
  uint64_t code = 0;
  if (x2 < n2.x && y2 < n2.y && z2 < n2.z)
    code = voxelMakeChild(((uint64_t)z2 * n2.y + y2) * n2.x + x2);
  vox1[i] = code;
  if (v == 0) {
    org1[3 * k1]     = x1 * 4096;
    org1[3 * k1 + 1] = y1 * 4096;
    org1[3 * k1 + 2] = z1 * 4096;
  }
}

__global__ void kDenseLevel0(uint64_t *vox0, uint3 n1)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 262144)
    return;
  const uint32_t vx = i >> 12, vy = (i >> 6) & 63, vz = i & 63;
  uint64_t code = 0;
  if (vx < n1.x && vy < n1.y && vz < n1.z)
    code = voxelMakeChild(((uint64_t)vz * n1.y + vy) * n1.x + vx);
  vox0[i] = code;
}

// ---------------------------------------------------------------------------
// Dense commit: bricked copy and leaf ranges in one pass over the voxels.
//
// The reference computes, per leaf, the range of each of its 27 neighbour
// leaves' windows [7,8) | [0,8) | [0,2) per axis, in neighbour order
// (x, y, z) and, inside a window, voxel order x outer / z inner, each fold
// being extend() = (a < b ? a : b, a > b ? a : b); a neighbour whose origin
// lies outside the domain contributes (background, background); a neighbour
// range whose bound is NaN is skipped (VdbSampler.ispc:460-557,
// VdbSampler_dense.ih:35-105).  Per axis the union of the windows is the
// voxel box [o-1, o+10) clipped to the dimensions.
//
// Without NaN in the window every order of the folds gives the same value:
// the min / max over the clipped box, plus the background when some
// neighbour origin is outside the domain and the background is not NaN.
// The bits are the same too unless a bound is zero and both +0.0 and -0.0
// take part.  The kernel computes that separably (x, then y, then z) with
// per-window flags for NaN and -0.0; a leaf whose window holds a NaN (a NaN
// voxel resets a running bound, so the order matters), or whose zero bound
// may come from a -0.0, is recomputed in the reference's own fold order.
//
// One CTA owns a column of 4x4 leaves (32x32 voxels) and kDenseChunk leaf
// layers: it streams the voxel planes z = 8*k0-1 .. 8*k1+1 through shared
// memory (35x35 with the halo), writes each interior plane to the bricked
// array, reduces every plane to per-leaf-column (lo, hi, flag), then folds
// 11 planes per leaf.  Each voxel is read from HBM about once (halo reads
// hit L2 for the x / y neighbours of concurrently running CTAs).
// ---------------------------------------------------------------------------
constexpr int kDenseChunk = 8;              // leaf layers per CTA
constexpr int kPlaneW     = 35;             // 32 + halo (1 before, 2 after)
constexpr int kMaxPlanes  = 8 * kDenseChunk + 3;

template <typename T>
__device__ __forceinline__ float toFloat(T v)
{
  return (float)v;
}
template <>
__device__ __forceinline__ float toFloat<__half>(__half v)
{
  return __half2float(v);
}
template <>
__device__ __forceinline__ float toFloat<double>(double v)
{
  return __double2float_rn(v);
}

// Values for which the fold order can change the bits: NaN (bit 0) and
// -0.0 (bit 1).
constexpr uint32_t kFlagNaN = 1u, kFlagNegZero = 2u;
__device__ __forceinline__ uint32_t orderFlags(float v)
{
  return (isnan(v) ? kFlagNaN : 0u) | (__float_as_uint(v) == 0x80000000u ? kFlagNegZero : 0u);
}

struct PartialRange {
  float lo, hi;
  uint32_t flag;
};

// The reference's fold order for one leaf at voxel origin (ox, oy, oz).
template <typename T>
__device__ float2 denseLeafRangeExact(const T *__restrict__ src, uint3 dims, int32_t ox, int32_t oy,
                                      int32_t oz, float bg)
{
  float lo = kInf, hi = -kInf;
  for (int ix = 0; ix < 3; ++ix)
    for (int iy = 0; iy < 3; ++iy)
      for (int iz = 0; iz < 3; ++iz) {
        const uint32_t nx = (uint32_t)(ox + (ix - 1) * 8), ny = (uint32_t)(oy + (iy - 1) * 8),
                       nz = (uint32_t)(oz + (iz - 1) * 8);
        float nlo, nhi;
        if (!(nx < dims.x && ny < dims.y && nz < dims.z)) {
          nlo = nhi = bg;
        } else {
          nlo = kInf;
          nhi = -kInf;
          const uint32_t xa = ix == 0 ? 7 : 0, xb = ix == 2 ? 2 : 8;
          const uint32_t ya = iy == 0 ? 7 : 0, yb = iy == 2 ? 2 : 8;
          const uint32_t za = iz == 0 ? 7 : 0, zb = iz == 2 ? 2 : 8;
          for (uint32_t x = xa; x < xb; ++x)
            for (uint32_t y = ya; y < yb; ++y)
              for (uint32_t z = za; z < zb; ++z) {
                const uint32_t px = nx + x, py = ny + y, pz = nz + z;
                if (!(px < dims.x && py < dims.y && pz < dims.z))
                  continue;
                const float v = toFloat(src[((uint64_t)pz * dims.y + py) * dims.x + px]);
                nlo           = fminx(nlo, v);
                nhi           = fmaxx(nhi, v);
              }
        }
        if (!isnan(nlo))
          lo = fminx(lo, nlo);
        if (!isnan(nhi))
          hi = fmaxx(hi, nhi);
      }
  return make_float2(lo, hi);
}

// Per-plane steps shared by both kernels.  `at(r, c)` is the voxel at
// (x, y) = (X0 - 1 + c, Y0 - 1 + r) of the staged 35x35 window.
struct TileCoords {
  int32_t X0, Y0, X, Y, Z;
  int32_t k0, k1, zBeg, zEnd;
};

__device__ __forceinline__ TileCoords tileCoords(uint3 dims, uint3 nl)
{
  TileCoords t;
  t.X0 = 32 * (int32_t)blockIdx.x;
  t.Y0 = 32 * (int32_t)blockIdx.y;
  t.X = (int32_t)dims.x, t.Y = (int32_t)dims.y, t.Z = (int32_t)dims.z;
  t.k0   = kDenseChunk * (int32_t)blockIdx.z;
  t.k1   = min(t.k0 + kDenseChunk, (int32_t)nl.z);
  t.zBeg = max(8 * t.k0 - 1, 0);
  t.zEnd = min(8 * t.k1 + 2, t.Z);
  return t;
}

// A thread's part of the bricked copy of a plane's 32x32 interior: column
// x = X0 + (tid & 31), rows y = Y0 + (tid >> 5) + 8u.  brickIndex is a sum
// of per-axis terms, so the x and y terms are computed once per thread and
// the z term once per plane.
// Texture atlas of a float attribute (DevGrid::atlasTex), written through a
// surface object in the same pass; surf = 0: none.
struct AtlasTarget {
  uint64_t surf;
  uint32_t planesPerRow;
  uint32_t *denormal;  // set to 1 when a voxel is denormal (the texture path would flush it)
};

__device__ __forceinline__ bool isDenormal(float v)
{
  const uint32_t b = __float_as_uint(v);
  return (b & 0x7f800000u) == 0 && (b & 0x007fffffu) != 0;
}

struct BrickWriter {
  uint64_t termXY[4];
  uint32_t valid;  // bit u: (x, y_u) inside the volume
  uint64_t zStride;
  uint32_t x, y0;

  __device__ __forceinline__ BrickWriter(const TileCoords &t, uint32_t superX, uint32_t superY)
  {
    x  = (uint32_t)(t.X0 + (threadIdx.x & 31));
    y0 = (uint32_t)(t.Y0 + (threadIdx.x >> 5));
    const uint64_t tx = ((uint64_t)(x >> 6) << 18) + (((x >> 3) & 7u) << 9) + (x & 7u);
    const uint64_t yStride = (uint64_t)superX << 18;
    zStride = (uint64_t)superX * superY << 18;
    valid   = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t y = (uint32_t)(t.Y0 + (threadIdx.x >> 5) + 8 * u);
      termXY[u] = tx + (uint64_t)(y >> 6) * yStride + ((((y >> 3) & 7u) << 12) + ((y & 7u) << 3));
      if ((int32_t)x < t.X && (int32_t)y < t.Y)
        valid |= 1u << u;
    }
  }
  template <typename T, class At>
  __device__ __forceinline__ void write(uint32_t z, At at, T *__restrict__ dst, const AtlasTarget &atlas,
                                        const TileCoords &t, uint32_t &denormal) const
  {
    const uint64_t tz = (uint64_t)(z >> 6) * zStride + ((((z >> 3) & 7u) << 15) + ((z & 7u) << 6));
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (valid & (1u << u)) {
        const T v = at((threadIdx.x >> 5) + 8 * u + 1, (threadIdx.x & 31) + 1);
        dst[termXY[u] + tz] = v;
        if constexpr (std::is_same<T, float>::value) {
          if (atlas.surf) {
            const uint32_t ax = (z % atlas.planesPerRow) * (uint32_t)t.X + x,
                           ay = (z / atlas.planesPerRow) * (uint32_t)t.Y + y0 + 8 * u;
            surf2Dwrite(v, (cudaSurfaceObject_t)atlas.surf, (int)(ax * sizeof(float)), (int)ay,
                        cudaBoundaryModeZero);
            denormal |= isDenormal(v) ? 1u : 0u;
          }
        }
      }
  }
};

// Bricked copy of the plane's interior and the per-row ranges of the four
// leaf x-windows (into xres).
template <typename T, class At>
__device__ __forceinline__ void planeRows(const TileCoords &t, int32_t z, At at, T *__restrict__ dst,
                                          const BrickWriter &bw, const AtlasTarget &atlas, uint32_t &denormal,
                                          PartialRange (*xres)[4])
{
  const int tid = threadIdx.x;
  if (z >= 8 * t.k0 && z < 8 * t.k1)
    bw.write((uint32_t)z, at, dst, atlas, t, denormal);
  if (tid < kPlaneW * 4) {
    const int r = tid >> 2, i = tid & 3;
    const int32_t y = t.Y0 - 1 + r;
    PartialRange pr{kInf, -kInf, 0u};
    auto fold = [&](int c) {
      const float v = toFloat(at(r, c));
      pr.flag |= orderFlags(v);
      pr.lo = fminf(pr.lo, v);
      pr.hi = fmaxf(pr.hi, v);
    };
    if ((uint32_t)y < (uint32_t)t.Y && t.X0 + 8 * i < t.X) {
      const int c0 = max(8 * i, 1 - t.X0), c1 = min(8 * i + 11, t.X - t.X0 + 1);
      for (int c = c0; c < c1; ++c)
        fold(c);
    }
    xres[r][i] = pr;
  }
}

// The plane's range per leaf column (threads 0..15).
__device__ __forceinline__ void planeColumns(const PartialRange (*xres)[4], PartialRange *out)
{
  const int tid = threadIdx.x;
  if (tid < 16) {
    const int i = tid & 3, j = tid >> 2;
    PartialRange pr{kInf, -kInf, 0u};
    for (int r = 8 * j; r < 8 * j + 11; ++r) {
      const PartialRange q = xres[r][i];
      pr.lo = fminf(pr.lo, q.lo);
      pr.hi = fmaxf(pr.hi, q.hi);
      pr.flag |= q.flag;
    }
    out[tid] = pr;
  }
}

// Folds 11 plane ranges per leaf and writes the leaf ranges (one thread per
// leaf of the CTA's column).
template <typename T>
__device__ __forceinline__ void finishLeaves(const TileCoords &t, const PartialRange (*pres)[16],
                                             const T *__restrict__ src, uint3 dims, uint3 nl, float bg,
                                             float *__restrict__ leafRanges)
{
  const int tid = threadIdx.x;
  const int layer = tid >> 4, col = tid & 15;
  const int32_t lx = 4 * (int32_t)blockIdx.x + (col & 3), ly = 4 * (int32_t)blockIdx.y + (col >> 2),
                lz = t.k0 + layer;
  if (layer >= kDenseChunk || lz >= t.k1 || lx >= (int32_t)nl.x || ly >= (int32_t)nl.y)
    return;
  PartialRange pr{kInf, -kInf, 0u};
  for (int32_t z = max(8 * lz - 1, 0); z < min(8 * lz + 10, t.Z); ++z) {
    const PartialRange q = pres[z - t.zBeg][col];
    pr.lo = fminf(pr.lo, q.lo);
    pr.hi = fmaxf(pr.hi, q.hi);
    pr.flag |= q.flag;
  }
  const int32_t ox = 8 * lx, oy = 8 * ly, oz = 8 * lz;
  const bool boundary = lx == 0 || ly == 0 || lz == 0 || ox + 8 >= t.X || oy + 8 >= t.Y || oz + 8 >= t.Z;
  float2 r = make_float2(pr.lo, pr.hi);
  if (boundary && !isnan(bg)) {
    r.x = fminf(r.x, bg);
    r.y = fmaxf(r.y, bg);
    pr.flag |= orderFlags(bg) & kFlagNegZero;
  }
  if ((pr.flag & kFlagNaN) || ((pr.flag & kFlagNegZero) && (r.x == 0.f || r.y == 0.f)))
    r = denseLeafRangeExact(src, dims, ox, oy, oz, bg);
  const uint64_t leaf = ((uint64_t)lz * nl.y + ly) * nl.x + lx;
  leafRanges[2 * leaf]     = r.x;
  leafRanges[2 * leaf + 1] = r.y;
}

// Any row pitch: the next plane is loaded into registers while the current
// one is reduced.
template <typename T>
__global__ void __launch_bounds__(256, 4) kDenseBrickRanges(const T *__restrict__ src, T *__restrict__ dst,
                                                         uint3 dims, uint3 nl, uint32_t superX, uint32_t superY,
                                                         float bg, float *__restrict__ leafRanges,
                                                         AtlasTarget atlas)
{
  __shared__ T plane[kPlaneW][kPlaneW];
  __shared__ PartialRange xres[kPlaneW][4];
  __shared__ PartialRange pres[kMaxPlanes][16];
  const int tid        = threadIdx.x;
  const TileCoords t   = tileCoords(dims, nl);
  const BrickWriter bw(t, superX, superY);
  uint32_t denormal = 0;
  // Loads: 245 threads = 7 rows x 35 columns per pass, 5 passes cover the
  // 35 rows.  A thread's column and its row validity are fixed; its voxel
  // offset within a plane is rowOff + 7 * u * X.
  constexpr int kRowsPerPass = 7, kPasses = kPlaneW / kRowsPerPass;
  const int lr = tid / kPlaneW, lc = tid - lr * kPlaneW;
  const bool loader = tid < kRowsPerPass * kPlaneW;
  const int32_t lx = t.X0 - 1 + lc;
  uint32_t rowValid = 0;
#pragma unroll
  for (int u = 0; u < kPasses; ++u)
    if (loader && (uint32_t)lx < dims.x && (uint32_t)(t.Y0 - 1 + lr + kRowsPerPass * u) < dims.y)
      rowValid |= 1u << u;
  // the first row may lie above the volume (then only the later passes load)
  const int64_t rowOff     = (int64_t)(t.Y0 - 1 + lr) * dims.x + lx;
  const int64_t planeElems = (int64_t)dims.x * dims.y, passStride = (int64_t)kRowsPerPass * dims.x;
  T next[kPasses];
  auto loadPlane = [&](int32_t z) {
    const T *p = src + ((int64_t)z * planeElems + rowOff);
#pragma unroll
    for (int u = 0; u < kPasses; ++u)
      if (rowValid & (1u << u))
        next[u] = p[u * passStride];
  };
  auto at = [&](int r, int c) { return plane[r][c]; };
  loadPlane(t.zBeg);
  for (int32_t z = t.zBeg; z < t.zEnd; ++z) {
    if (loader) {
#pragma unroll
      for (int u = 0; u < kPasses; ++u)
        plane[lr + kRowsPerPass * u][lc] = next[u];
    }
    __syncthreads();
    if (z + 1 < t.zEnd)
      loadPlane(z + 1);
    planeRows(t, z, at, dst, bw, atlas, denormal, xres);
    __syncthreads();
    planeColumns(xres, pres[z - t.zBeg]);
  }
  if (__syncthreads_or(denormal) && tid == 0)
    atomicOr(atlas.denormal, 1u);
  finishLeaves(t, pres, src, dims, nl, bg, leafRanges);
}

// ---------------------------------------------------------------------------
// Sparse leaf ranges: per leaf, walk to each of the 27 neighbour leaves and
// scan its window (VdbSampler_computeNodeValueRange, VdbSampler.ispc:
// 383-455; packed handlers VdbSampler_packed_denseZYX.ih:12-75,
// VdbSampler_packed_tile.ih).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) kSparseLeafRanges(const __grid_constant__ DevGrid g,
                                                         uint32_t attr, uint64_t numLeaves,
                                                         const uint32_t *__restrict__ offs,
                                                         float *__restrict__ leafRanges)
{
  const uint64_t leaf = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= numLeaves)
    return;
  const SparseField<T> F(g, attr, kNumLevels - 1);
  const uint32_t cx = offs[3 * leaf], cy = offs[3 * leaf + 1], cz = offs[3 * leaf + 2];
  const float bgOut = g.background[attr];
  float lo = kInf, hi = -kInf;
  for (int n = 0; n < 27; ++n) {
    const int ix = n / 9, iy = (n / 3) % 3, iz = n % 3;
    const uint32_t dx = cx + (uint32_t)((ix - 1) * 8), dy = cy + (uint32_t)((iy - 1) * 8),
                   dz = cz + (uint32_t)((iz - 1) * 8);
    float nlo, nhi;
    const bool inDom = F.inDomain(dx, dy, dz);
    const uint64_t voxel = inDom ? F.traverse(dx, dy, dz) : 0ull;
    if (!voxelIsLeaf(voxel)) {
      nlo = nhi = inDom ? 0.f : bgOut;
    } else if (voxelLeafFormat(voxel) == kFormatTile) {
      nlo = nhi = tileValue<T>(g, attr, voxelLeafIndex(voxel));
    } else {
      const uint32_t xa = ix == 0 ? 7 : 0, xb = ix == 2 ? 2 : 8;
      const uint32_t ya = iy == 0 ? 7 : 0, yb = iy == 2 ? 2 : 8;
      const uint32_t za = iz == 0 ? 7 : 0, zb = iz == 2 ? 2 : 8;
      const uint64_t li = voxelLeafIndex(voxel);
      nlo = kInf;
      nhi = -kInf;
      for (uint32_t x = xa; x < xb; ++x)
        for (uint32_t y = ya; y < yb; ++y)
          for (uint32_t z = za; z < zb; ++z) {
            const float v = packedLeafValue<T>(g, attr, li, leafVoxelIndex<T>(li, x, y, z));
            nlo           = fminx(nlo, v);
            nhi           = fmaxx(nhi, v);
          }
    }
    if (!isnan(nlo))
      lo = fminx(lo, nlo);
    if (!isnan(nhi))
      hi = fmaxx(hi, nhi);
  }
  leafRanges[2 * leaf]     = lo;
  leafRanges[2 * leaf + 1] = hi;
}

// ---------------------------------------------------------------------------
// Propagation.  Every leaf's range lands in the voxel that points at it;
// every child node's voxels reduce into the voxel that points at the node.
// This equals the reference's per-leaf `extend` up the ancestor chain
// (VdbVolume.cpp:361-391) because min/max are order-independent.
// ---------------------------------------------------------------------------
__global__ void kFillEmpty(float *r, uint64_t n)
{
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    r[2 * i]     = kInf;
    r[2 * i + 1] = -kInf;
  }
}

__global__ void kLeafToParent(const __grid_constant__ DevGrid g, uint32_t attr, uint64_t numLeaves,
                              const uint64_t *__restrict__ leafVoxel,
                              const float *__restrict__ leafRanges, uint3 nl)
{
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numLeaves)
    return;
  uint64_t lv;
  if (leafVoxel) {
    lv = leafVoxel[i];
    if (lv == ~0ull)
      return;
  } else {
    // dense: leaf (lx,ly,lz) hangs off level-2 node (l>>4) at voxel (l&15)
    const uint32_t lx = (uint32_t)(i % nl.x), ly = (uint32_t)((i / nl.x) % nl.y),
                   lz = (uint32_t)(i / ((uint64_t)nl.x * nl.y));
    const uint32_t n2x = (nl.x + 15) / 16, n2y = (nl.y + 15) / 16;
    const uint64_t k2 = ((uint64_t)(lz >> 4) * n2y + (ly >> 4)) * n2x + (lx >> 4);
    lv = (2ull << 40) | (k2 * 4096 + ((lx & 15) << 8) + ((ly & 15) << 4) + (lz & 15));
  }
  const uint32_t level = (uint32_t)(lv >> 40);
  const uint64_t v     = lv & ((1ull << 40) - 1);
  float *r = (float *)g.levels[level].valueRange + 2 * (v * g.numAttributes + attr);
  // A voxel holds exactly one leaf, so this read-modify-write has no race;
  // it extends like the reference instead of assigning.
  r[0] = fminx(r[0], leafRanges[2 * i]);
  r[1] = fmaxx(r[1], leafRanges[2 * i + 1]);
}

// One block per node on `level` (1 or 2): reduce the node's voxel ranges and
// write them into the parent voxel on level-1, found by walking down from
// the root with the node's origin.
__global__ void __launch_bounds__(256) kReduceNodes(const __grid_constant__ DevGrid g,
                                                    uint32_t attr, uint32_t level)
{
  const uint64_t node = blockIdx.x;
  const DevLevel &L   = g.levels[level];
  const uint64_t nv   = levelNumVoxels(level);
  float lo = kInf, hi = -kInf;
  for (uint64_t v = threadIdx.x; v < nv; v += blockDim.x) {
    const float *r = L.valueRange + 2 * ((node * nv + v) * g.numAttributes + attr);
    lo             = fminx(lo, r[0]);
    hi             = fmaxx(hi, r[1]);
  }
  __shared__ float slo[256], shi[256];
  slo[threadIdx.x] = lo;
  shi[threadIdx.x] = hi;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      slo[threadIdx.x] = fminx(slo[threadIdx.x], slo[threadIdx.x + s]);
      shi[threadIdx.x] = fmaxx(shi[threadIdx.x], shi[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const uint32_t ox = L.origin[3 * node], oy = L.origin[3 * node + 1], oz = L.origin[3 * node + 2];
    uint64_t pnode = 0;
    for (uint32_t l = 0; l + 1 < level; ++l) {
      const uint64_t v = g.levels[l].voxels[pnode * levelNumVoxels(l) + offsetToLinear(l, ox, oy, oz)];
      pnode            = voxelChildIndex(v);
    }
    const uint32_t pl = level - 1;
    const uint64_t pv = pnode * levelNumVoxels(pl) + offsetToLinear(pl, ox, oy, oz);
    float *r = (float *)g.levels[pl].valueRange + 2 * (pv * g.numAttributes + attr);
    r[0]     = fminx(r[0], slo[0]);
    r[1]     = fmaxx(r[1], shi[0]);
  }
}

__global__ void __launch_bounds__(1024) kVolumeRange(const __grid_constant__ DevGrid g,
                                                     uint32_t attr, float *out)
{
  float lo = kInf, hi = -kInf;
  for (uint32_t v = threadIdx.x; v < 262144; v += blockDim.x) {
    const float *r = g.levels[0].valueRange + 2 * ((uint64_t)v * g.numAttributes + attr);
    lo             = fminx(lo, r[0]);
    hi             = fmaxx(hi, r[1]);
  }
  __shared__ float slo[1024], shi[1024];
  slo[threadIdx.x] = lo;
  shi[threadIdx.x] = hi;
  __syncthreads();
  for (int s = 512; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      slo[threadIdx.x] = fminx(slo[threadIdx.x], slo[threadIdx.x + s]);
      shi[threadIdx.x] = fmaxx(shi[threadIdx.x], shi[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = slo[0];
    out[1] = shi[0];
  }
}

// ---------------------------------------------------------------------------
// Flat leaf map: for every 8^3 leaf slot of the active domain, the voxel code
// the full-depth walk reaches (VdbSampler_traverseAndSample.ih:85-306 at
// maxSamplingDepth 3).  Built once at commit so sampling replaces the
// three dependent node loads of the walk by one load.
// ---------------------------------------------------------------------------
__global__ void kBuildLeafMap(const __grid_constant__ DevGrid g, uint3 dims, uint64_t *__restrict__ map)
{
  const uint64_t i     = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t total = (uint64_t)dims.x * dims.y * dims.z;
  if (i >= total)
    return;
  const uint32_t lx = (uint32_t)(i % dims.x), ly = (uint32_t)((i / dims.x) % dims.y),
                 lz = (uint32_t)(i / ((uint64_t)dims.x * dims.y));
  const SparseField<float> F(g, 0, kNumLevels - 1);
  map[i] = F.walk(lx * 8, ly * 8, lz * 8);
}

// ---------------------------------------------------------------------------
// Leaf compression (extension): per packed leaf, offset = midpoint and
// scale = half-range / code maximum of its non-NaN values, codes = the
// round-to-nearest-even conversion of (v - offset) / scale.  One warp per
// leaf, 16 values per lane.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void encodeCode(float r, __half *p) { *p = __float2half_rn(r); }
__device__ __forceinline__ void encodeCode(float r, __nv_bfloat16 *p) { *p = __float2bfloat16_rn(r); }
__device__ __forceinline__ void encodeCode(float r, __nv_fp8_storage_t *p)
{
  *p = __nv_cvt_float_to_fp8(r, __NV_SATFINITE, __NV_E4M3);
}

template <typename C>
__global__ void __launch_bounds__(256) kCompressLeaves(const float *__restrict__ src, uint64_t numLeaves,
                                                       float codeMax, C *__restrict__ codes,
                                                       float2 *__restrict__ scaleOffset)
{
  const uint64_t leaf = (uint64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane      = threadIdx.x & 31;
  if (leaf >= numLeaves)
    return;
  const float *v = src + leaf * 512;
  float x[16];
  float lo = kInf, hi = -kInf;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    x[i] = __ldg(v + lane + 32 * i);
    if (x[i] < lo)
      lo = x[i];
    if (x[i] > hi)
      hi = x[i];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
    if (l2 < lo)
      lo = l2;
    if (h2 > hi)
      hi = h2;
  }
  lo += 0.f;  // one sign for zero
  hi += 0.f;
  float offset = 0.f, scale = 1.f;
  if (lo <= hi) {
    offset           = 0.5f * lo + 0.5f * hi;
    const float half = 0.5f * hi - 0.5f * lo;
    if (half > 0.f)
      scale = half / codeMax;
  }
  if (lane == 0)
    scaleOffset[leaf] = make_float2(scale, offset);
  C *c = codes + leaf * 512;
#pragma unroll
  for (int i = 0; i < 16; ++i)
    encodeCode((x[i] - offset) / scale, c + lane + 32 * i);
}

// ---------------------------------------------------------------------------
// Stencil-block leaves (extension): per dense leaf slot, the 9^3 sampling
// window (the leaf's voxels plus the next voxel on the +x/+y/+z side, as the
// float volume's full-depth lookup gives them: neighbouring leaves, tiles,
// zero in empty space, background outside the domain) sets the leaf's scale
// and offset by kCompressLeaves' rule over the window's non-NaN values, and
// the leaf's 8 blocks of 5^3 codes are encoded from the window (block layout:
// leafBlockCode, grid.h).  One CTA of 128 threads per slot; slots whose
// offset is ~0 (tiles of node.data input) are skipped.
// ---------------------------------------------------------------------------
template <typename C>
__global__ void __launch_bounds__(128) kBuildLeafBlocks(const __grid_constant__ DevGrid g, uint32_t attr,
                                                        const uint32_t *__restrict__ offs, float codeMax,
                                                        C *__restrict__ codes, float2 *__restrict__ scaleOffset)
{
  const uint64_t slot = blockIdx.x;
  const uint32_t cx = offs[3 * slot], cy = offs[3 * slot + 1], cz = offs[3 * slot + 2];
  if (cx == ~0u)
    return;
  __shared__ float win[729];
  __shared__ float red[2][4];
  const SparseField<float> F(g, attr, kNumLevels - 1);
  const float *leaf = (const float *)g.data[attr] + slot * 512;
  float lo = kInf, hi = -kInf;
  for (int w = threadIdx.x; w < 729; w += 128) {
    const uint32_t wx = w / 81, wy = (w / 9) % 9, wz = w % 9;
    float v;
    if (wx < 8 && wy < 8 && wz < 8)
      v = __ldg(leaf + (wx << 6) + (wy << 3) + wz);
    else
      v = F.at(g.rootOrigin[0] + (int32_t)(cx + wx), g.rootOrigin[1] + (int32_t)(cy + wy),
               g.rootOrigin[2] + (int32_t)(cz + wz));
    win[w] = v;
    if (v < lo)
      lo = v;
    if (v > hi)
      hi = v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
    if (l2 < lo)
      lo = l2;
    if (h2 > hi)
      hi = h2;
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = lo;
    red[1][threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  lo = kInf;
  hi = -kInf;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (red[0][k] < lo)
      lo = red[0][k];
    if (red[1][k] > hi)
      hi = red[1][k];
  }
  lo += 0.f;  // one sign for zero
  hi += 0.f;
  float offset = 0.f, scale = 1.f;
  if (lo <= hi) {
    offset           = 0.5f * lo + 0.5f * hi;
    const float half = 0.5f * hi - 0.5f * lo;
    if (half > 0.f)
      scale = half / codeMax;
  }
  if (threadIdx.x == 0)
    scaleOffset[slot] = make_float2(scale, offset);
  C *c = codes + slot * kLeafCodes;
  for (uint32_t k = threadIdx.x; k < kLeafCodes; k += 128) {
    const uint32_t b = k / kLeafBlockCodes, l = k % kLeafBlockCodes;
    if (l < 125) {
      const uint32_t x = ((b >> 2) & 1u) * 4 + l / 25, y = ((b >> 1) & 1u) * 4 + (l / 5) % 5,
                     z = (b & 1u) * 4 + l % 5;
      encodeCode((win[x * 81 + y * 9 + z] - offset) / scale, c + k);
    } else {
      encodeCode(0.f, c + k);
    }
  }
}

inline unsigned blocksFor(uint64_t n, unsigned b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

void launchBuildDenseTree(const DevGrid &g, uint64_t *vox0, uint64_t *vox1, uint64_t *vox2,
                          uint32_t *org1, uint32_t *org2, const uint32_t nl[3],
                          const uint32_t n1[3], const uint32_t n2[3], cudaStream_t st)
{
  (void)g;
  const uint3 NL = {nl[0], nl[1], nl[2]}, N1 = {n1[0], n1[1], n1[2]}, N2 = {n2[0], n2[1], n2[2]};
  const uint64_t t2 = (uint64_t)n2[0] * n2[1] * n2[2] * 4096;
  const uint64_t t1 = (uint64_t)n1[0] * n1[1] * n1[2] * 32768;
  kDenseLevel2<<<blocksFor(t2, 256), 256, 0, st>>>(vox2, org2, NL, N2);
  kDenseLevel1<<<blocksFor(t1, 256), 256, 0, st>>>(vox1, org1, N2, N1);
  kDenseLevel0<<<blocksFor(262144, 256), 256, 0, st>>>(vox0, N1);
  cudaCheck(cudaGetLastError(), "dense tree kernels");
}

void launchDenseBrickRanges(const void *src, uint32_t type, void *dst, const uint32_t dims[3],
                            uint32_t superX, uint32_t superY, float background, float *leafRanges,
                            uint64_t atlasSurface, uint32_t atlasPlanesPerRow, uint32_t *denormalFlag,
                            cudaStream_t st)
{
  const AtlasTarget atlas{type == kFloat ? atlasSurface : 0, atlasPlanesPerRow, denormalFlag};
  const uint3 D  = {dims[0], dims[1], dims[2]};
  const uint3 NL = {(dims[0] + 7) / 8, (dims[1] + 7) / 8, (dims[2] + 7) / 8};
  const dim3 grid((NL.x + 3) / 4, (NL.y + 3) / 4, (NL.z + kDenseChunk - 1) / kDenseChunk);
#define VKL_DENSE_BRICK(T)                                                                              \
  kDenseBrickRanges<T><<<grid, 256, 0, st>>>((const T *)src, (T *)dst, D, NL, superX, superY, background, \
                                             leafRanges, atlas)
  switch (type) {
  case kUChar:
    VKL_DENSE_BRICK(uint8_t);
    break;
  case kShort:
    VKL_DENSE_BRICK(int16_t);
    break;
  case kUShort:
    VKL_DENSE_BRICK(uint16_t);
    break;
  case kHalf:
    VKL_DENSE_BRICK(__half);
    break;
  case kDouble:
    VKL_DENSE_BRICK(double);
    break;
  default:
    VKL_DENSE_BRICK(float);
  }
#undef VKL_DENSE_BRICK
  cudaCheck(cudaGetLastError(), "dense bricking / leaf range kernel");
}

void launchSparseLeafRanges(const DevGrid &g, uint32_t attr, uint64_t numLeaves,
                            const uint32_t *leafOffsets, float *leafRanges, cudaStream_t st)
{
  const unsigned grid = blocksFor(numLeaves, 128);
  if (g.compress == kCompressFP16)
    kSparseLeafRanges<CodeFP16><<<grid, 128, 0, st>>>(g, attr, numLeaves, leafOffsets, leafRanges);
  else if (g.compress == kCompressBF16)
    kSparseLeafRanges<CodeBF16><<<grid, 128, 0, st>>>(g, attr, numLeaves, leafOffsets, leafRanges);
  else if (g.compress == kCompressFP8)
    kSparseLeafRanges<CodeE4M3><<<grid, 128, 0, st>>>(g, attr, numLeaves, leafOffsets, leafRanges);
  else if (g.compress == kCompressFP16Blocks)
    kSparseLeafRanges<Blocked<CodeFP16>><<<grid, 128, 0, st>>>(g, attr, numLeaves, leafOffsets, leafRanges);
  else if (g.compress == kCompressBF16Blocks)
    kSparseLeafRanges<Blocked<CodeBF16>><<<grid, 128, 0, st>>>(g, attr, numLeaves, leafOffsets, leafRanges);
  else if (g.compress == kCompressFP8Blocks)
    kSparseLeafRanges<Blocked<CodeE4M3>><<<grid, 128, 0, st>>>(g, attr, numLeaves, leafOffsets, leafRanges);
  else if (g.type[attr] == kHalf)
    kSparseLeafRanges<__half><<<grid, 128, 0, st>>>(g, attr, numLeaves, leafOffsets, leafRanges);
  else
    kSparseLeafRanges<float><<<grid, 128, 0, st>>>(g, attr, numLeaves, leafOffsets, leafRanges);
  cudaCheck(cudaGetLastError(), "sparse leaf range kernel");
}

void launchPropagateRanges(const DevGrid &g, uint32_t attr, uint64_t numLeaves,
                           const uint64_t *leafVoxel, const float *leafRanges,
                           float *volumeRange, const uint32_t nl[3], cudaStream_t st)
{
  if (attr == 0) {
    for (uint32_t l = 0; l < kNumLevels - 1; ++l) {
      const uint64_t n = g.levels[l].numNodes * levelNumVoxels(l) * g.numAttributes;
      kFillEmpty<<<blocksFor(n, 256), 256, 0, st>>>((float *)g.levels[l].valueRange, n);
    }
  }
  kLeafToParent<<<blocksFor(numLeaves, 256), 256, 0, st>>>(g, attr, numLeaves, leafVoxel,
                                                           leafRanges, make_uint3(nl[0], nl[1], nl[2]));
  for (uint32_t l = kNumLevels - 2; l >= 1; --l)
    if (g.levels[l].numNodes)
      kReduceNodes<<<(unsigned)g.levels[l].numNodes, 256, 0, st>>>(g, attr, l);
  kVolumeRange<<<1, 1024, 0, st>>>(g, attr, volumeRange);
  cudaCheck(cudaGetLastError(), "range propagation kernels");
}

}  // namespace vklcuda

namespace vklcuda {

uint64_t brickedElements(const uint32_t dims[3], uint32_t &superX, uint32_t &superY)
{
  superX = (dims[0] + 63) / 64;
  superY = (dims[1] + 63) / 64;
  const uint64_t superZ = (dims[2] + 63) / 64;
  return (uint64_t)superX * superY * superZ << 18;
}

void launchBuildLeafMap(const DevGrid &g, uint64_t *map, cudaStream_t st)
{
  const uint3 d = {g.leafMapDims[0], g.leafMapDims[1], g.leafMapDims[2]};
  const uint64_t n = (uint64_t)d.x * d.y * d.z;
  if (n)
    kBuildLeafMap<<<blocksFor(n, 256), 256, 0, st>>>(g, d, map);
  cudaCheck(cudaGetLastError(), "leaf map kernel");
}

void launchCompressLeaves(uint32_t format, const float *src, uint64_t numLeaves, void *codes,
                          float *scaleOffset, cudaStream_t st)
{
  if (!numLeaves)
    return;
  const unsigned grid = blocksFor(numLeaves, 8);
  float2 *so          = (float2 *)scaleOffset;
  if (format == kCompressFP16)
    kCompressLeaves<<<grid, 256, 0, st>>>(src, numLeaves, 1.f, (__half *)codes, so);
  else if (format == kCompressBF16)
    kCompressLeaves<<<grid, 256, 0, st>>>(src, numLeaves, 1.f, (__nv_bfloat16 *)codes, so);
  else
    kCompressLeaves<<<grid, 256, 0, st>>>(src, numLeaves, 448.f, (__nv_fp8_storage_t *)codes, so);
  cudaCheck(cudaGetLastError(), "leaf compression kernel");
}

void launchBuildLeafBlocks(uint32_t format, const DevGrid &g, uint32_t attr, uint64_t numSlots,
                           const uint32_t *slotOffsets, void *codes, float *scaleOffset, cudaStream_t st)
{
  if (!numSlots)
    return;
  const unsigned grid = (unsigned)numSlots;
  float2 *so          = (float2 *)scaleOffset;
  if (format == kCompressFP16Blocks)
    kBuildLeafBlocks<<<grid, 128, 0, st>>>(g, attr, slotOffsets, 1.f, (__half *)codes, so);
  else if (format == kCompressBF16Blocks)
    kBuildLeafBlocks<<<grid, 128, 0, st>>>(g, attr, slotOffsets, 1.f, (__nv_bfloat16 *)codes, so);
  else
    kBuildLeafBlocks<<<grid, 128, 0, st>>>(g, attr, slotOffsets, 448.f, (__nv_fp8_storage_t *)codes, so);
  cudaCheck(cudaGetLastError(), "leaf block kernel");
}

}  // namespace vklcuda
