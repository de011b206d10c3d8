// Device-side data contract of the cuda device: the committed grid as the
// kernels see it, passed to every launch by value (one constant-bank copy per
// launch, no pointer chase to reach it).
//
// It holds the same information as the reference's VdbGrid / VdbLevel shared
// structs (openvkl/devices/cpu/volume/vdb/VdbGridShared.h:17-86): the 4-level
// tree with log resolutions 6/5/4/3 (openvkl/CMakeLists.txt:37-49), u64 voxel
// codes (VdbGrid.h:91-203), per-voxel value ranges, the 3x4 row-major
// object<->index transforms, and either dense x-fastest voxel arrays
// (structuredRegular) or packed leaf arrays (nodesPackedDense / Tile).
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define VKL_HD __host__ __device__ __forceinline__
#else
#define VKL_HD inline
#endif

namespace vklcuda {

constexpr uint32_t kNumLevels  = 4;
constexpr uint32_t kMaxAttributes = 16;
constexpr uint32_t kLeafRes    = 8;
constexpr uint32_t kLeafVoxels = 512;

constexpr VKL_HD uint32_t logRes(uint32_t l)
{
  return l == 0 ? 6u : l == 1 ? 5u : l == 2 ? 4u : l == 3 ? 3u : 0u;
}
constexpr VKL_HD uint32_t totalLogRes(uint32_t l)
{
  return l == 0 ? 18u : l == 1 ? 12u : l == 2 ? 7u : l == 3 ? 3u : 0u;
}
// Resolution of a level-l node in leaf voxels; level 4 (one past the leaf)
// is 1, the DDA's elementary cell.
constexpr VKL_HD uint32_t levelRes(uint32_t l) { return 1u << totalLogRes(l); }
VKL_HD uint64_t levelNumVoxels(uint32_t l) { return 1ull << (3 * logRes(l)); }

// Data type codes (VKLDataType values of the public API).
enum : uint32_t {
  kUChar  = 2500,
  kShort  = 3000,
  kUShort = 3500,
  kHalf   = 5800,
  kFloat  = 6000,
  kDouble = 7000,
};

enum : uint32_t { kFormatTile = 0, kFormatDenseZYX = 1 };
enum : int { kFilterNearest = 0, kFilterLinear = 100, kFilterCubic = 200 };

// Voxel codes: empty ..00, error ..01 (level in bits 8-15, voxel offset in
// 32-63), child (index<<2)|10, leaf (index<<6)|(tf<<4)|(fmt<<2)|11.
VKL_HD bool voxelIsEmpty(uint64_t v) { return (v & 3u) == 0; }
VKL_HD bool voxelIsError(uint64_t v) { return (v & 3u) == 1; }
VKL_HD bool voxelIsChild(uint64_t v) { return (v & 3u) == 2; }
VKL_HD bool voxelIsLeaf(uint64_t v) { return (v & 3u) == 3; }
VKL_HD uint64_t voxelMakeChild(uint64_t i) { return (i << 2) | 2u; }
VKL_HD uint64_t voxelMakeLeaf(uint64_t i, uint32_t fmt, uint32_t tf)
{
  return (i << 6) + ((uint64_t)(tf & 3u) << 4) + ((uint64_t)(fmt & 3u) << 2) + 3u;
}
VKL_HD uint64_t voxelMakeError(uint32_t level, uint32_t off)
{
  return ((uint64_t)off << 32) + ((uint64_t)level << 8) + 1u;
}
VKL_HD uint64_t voxelChildIndex(uint64_t v) { return v >> 2; }
VKL_HD uint64_t voxelLeafIndex(uint64_t v) { return v >> 6; }
VKL_HD uint32_t voxelLeafFormat(uint64_t v) { return (uint32_t)((v >> 2) & 3u); }

// Linear index of the voxel containing root-relative offset (x,y,z) inside a
// level-l node (z fastest).
VKL_HD uint64_t offsetToLinear(uint32_t l, uint64_t x, uint64_t y, uint64_t z)
{
  const uint64_t mask = levelRes(l) - 1;
  const uint32_t sh   = totalLogRes(l + 1);
  const uint32_t lr   = logRes(l);
  return (((x & mask) >> sh) << (2 * lr)) + (((y & mask) >> sh) << lr) +
         ((z & mask) >> sh);
}

// Bricked dense layout: 8^3-voxel bricks (x fastest inside a brick), 8^3
// bricks per 64^3 supertile (x fastest), supertiles x fastest.  A trilinear
// stencil then touches one or two 2 KB bricks and a warp's rays stay within
// a few MB, where the x-fastest layout puts every z step 4 MB apart (1024^2
// floats) and thrashes the TLB and L2.
VKL_HD uint64_t brickIndex(uint32_t x, uint32_t y, uint32_t z, uint32_t superX, uint32_t superY)
{
  const uint32_t st = ((z >> 6) * superY + (y >> 6)) * superX + (x >> 6);
  const uint32_t b  = (((z >> 3) & 7u) << 6) | (((y >> 3) & 7u) << 3) | ((x >> 3) & 7u);
  return ((uint64_t)st << 18) | ((uint64_t)b << 9) | ((z & 7u) << 6) | ((y & 7u) << 3) | (x & 7u);
}

struct DevLevel {
  uint64_t numNodes;
  const uint32_t *origin;  // 3 per node, root-relative
  const uint64_t *voxels;  // levelNumVoxels(l) per node
  const float *valueRange; // 2 floats per voxel per attribute
};

// Compressed leaf storage (FP16/BF16/FP8-E4M3 with per-leaf scale+offset);
// `format` 0 = none (plain float/half leaves).  The *Blocks formats store
// each leaf as 8 stencil blocks (kLeafBlock* below) instead of 512 codes.
enum : uint32_t {
  kCompressNone       = 0,
  kCompressFP16       = 1,
  kCompressBF16       = 2,
  kCompressFP8        = 3,
  kCompressFP16Blocks = 4,
  kCompressBF16Blocks = 5,
  kCompressFP8Blocks  = 6,
};

// Stencil-block leaves: leaf voxel (x, y, z) in [0, 8)^3 lies in block
// ((x >> 2) << 2 | (y >> 2) << 1 | (z >> 2)); a block holds the 5^3 voxels
// 4 * b + [0, 4] per axis (its 4^3 voxels plus the next voxel on the +x/+y/+z
// side, which may lie in a neighbouring leaf), z fastest, padded to 128
// codes.  A trilinear stencil whose base voxel lies in the leaf reads all 8
// corners from one block.
constexpr uint32_t kLeafBlockCodes = 128;
constexpr uint32_t kLeafCodes      = 8 * kLeafBlockCodes;

VKL_HD uint32_t leafBlockCode(uint32_t x, uint32_t y, uint32_t z)
{
  return ((((x >> 2) & 1u) << 2 | ((y >> 2) & 1u) << 1 | ((z >> 2) & 1u)) * kLeafBlockCodes) +
         (x & 3u) * 25u + (y & 3u) * 5u + (z & 3u);
}

constexpr uint32_t kMaxLeafObservers = 4;

struct DevGrid {
  float objectToIndex[12];
  float indexToObject[12];
  int32_t rootOrigin[3];
  uint32_t activeSize[3];
  float domain[6];  // domain-space (root-relative) bounding box
  uint32_t dense;
  uint32_t constantCellData;
  uint32_t numAttributes;
  int32_t denseDims[3];
  // Dense voxels are stored bricked (see brickIndex): the number of 64^3
  // supertiles along x and y.
  uint32_t superX, superY;
  DevLevel levels[kNumLevels - 1];
  uint64_t numLeaves;
  // Dense: attribute voxel arrays (x fastest).  Sparse: packed dense leaves
  // (512 values per leaf, z fastest) per attribute.
  const void *data[kMaxAttributes];
  // Sparse: packed tile values per attribute.
  const void *tile[kMaxAttributes];
  uint32_t type[kMaxAttributes];
  float background[kMaxAttributes];
  // Compressed leaves (sparse only): per-leaf (scale, offset) pairs for each
  // attribute; value = code * scale + offset.
  uint32_t compress;
  const float *leafScaleOffset[kMaxAttributes];
  // Sparse: flat leaf map over the active domain at leaf resolution, x
  // fastest: entry = the voxel code the full-depth tree walk reaches for
  // that 8^3 leaf slot (leaf, tile or empty).  Null when it would exceed its
  // memory budget; the walk is used then, and for maxSamplingDepth < 3.
  const uint64_t *leafMap;
  uint32_t leafMapDims[3];
  // LeafNodeAccess observers of the sampler a launch runs for (sparse only):
  // every traversal that reaches a leaf sets leafAccess[i][leaf] = 1, like
  // VdbLeafAccessObserver_observe (unsynchronised stores of the same value).
  uint32_t numLeafAccess;
  uint32_t *leafAccess[kMaxLeafObservers];
  // Dense float attributes: texture object (0 = none) over a 2D atlas of the
  // attribute's z-planes, plane z at texel (X * (z % atlasPlanesPerRow),
  // Y * (z / atlasPlanesPerRow)).  The trilinear tile kernels fetch their
  // 2x2x2 corners from it with two tld4 footprint gathers; z-neighbours sit
  // side by side in the atlas, a few KB apart.
  uint64_t atlasTex[kMaxAttributes];
  uint32_t atlasPlanesPerRow;  // a power of two
  // Temporally varying (motion-blur) dense data, kept as given (x fastest,
  // each voxel's time samples consecutive, not bricked): 0 = constant,
  // 1 = structured (numTimesteps values per voxel, regularly placed in
  // [0, 1]), 2 = unstructured (voxel v's samples are data[idx[v] ..
  // idx[v+1]) at times[idx[v] .. idx[v+1]), idx 32- or 64-bit).
  uint32_t temporal;
  uint32_t numTimesteps;
  uint32_t tIndex64;
  const void *tIndices;
  const float *tTimes;
};

struct DevSampler {
  int filter;
  int gradientFilter;
  uint32_t maxSamplingDepth;
};

// Interval / hit query description shared by the iterator kernels.
struct DevValueRanges {
  uint32_t numRanges;
  float minMax[2];
  const float *ranges;  // 2 floats per range (device)
};

// What a handle's `device` pointer addresses (device memory, written at the
// object's commit, stable for the object's lifetime): the state the
// __device__ API (include/openvkl_cuda_device.h) reads.
struct DevSamplerState {
  DevGrid g;
  DevSampler s;
};
struct DevIntervalContextState {
  const DevSamplerState *sampler;
  DevValueRanges vr;
  uint32_t attr;
  uint32_t depth;
};
struct DevHitContextState {
  const DevSamplerState *sampler;
  DevValueRanges vr;
  const float *values;
  uint32_t numValues;
  uint32_t attr;
  uint32_t depth;
};

struct DevInterval {
  float t0, t1, v0, v1, nominalDeltaT;
};

struct DevHit {
  float t, sample, epsilon;
};

}  // namespace vklcuda
