/* <openvkl/vdb.h> of the cuda device: the VDB tree topology an application
 * uses to build "vdb" volumes (node levels, resolutions, voxel counts and
 * the index maps from a domain offset to a node's voxel).
 *
 * It declares the names of the reference's header (openvkl/include/openvkl/
 * vdb.h:44-230, with the constants its build generates from
 * vdb_topology.h.in for the default 4-level configuration, log resolutions
 * 6 / 5 / 4 / 3) and VKLTemporalFormat (VKLTemporalFormat.h), so code that
 * includes <openvkl/vdb.h> compiles unchanged against the cuda device.  The
 * cuda device implements exactly this configuration (grid.h, kNumLevels). */
#pragma once

#include <stdint.h>

#include "../openvkl_cuda.h"

#ifndef VKL_VDB_NUM_LEVELS
#define VKL_VDB_NUM_LEVELS 4
#endif

/* per level: log2 of the node's voxels per axis, voxels per axis, voxels
 * per node, log2 and size of the domain a node covers (leaf voxels) */
#define VKL_VDB_LOG_RES_0 6
#define VKL_VDB_LOG_RES_1 5
#define VKL_VDB_LOG_RES_2 4
#define VKL_VDB_LOG_RES_3 3
#define VKL_VDB_LOG_RES_4 0
#define VKL_VDB_STORAGE_RES_0 64
#define VKL_VDB_STORAGE_RES_1 32
#define VKL_VDB_STORAGE_RES_2 16
#define VKL_VDB_STORAGE_RES_3 8
#define VKL_VDB_STORAGE_RES_4 1
#define VKL_VDB_NUM_VOXELS_0 262144
#define VKL_VDB_NUM_VOXELS_1 32768
#define VKL_VDB_NUM_VOXELS_2 4096
#define VKL_VDB_NUM_VOXELS_3 512
#define VKL_VDB_NUM_VOXELS_4 1
#define VKL_VDB_TOTAL_LOG_RES_0 18
#define VKL_VDB_TOTAL_LOG_RES_1 12
#define VKL_VDB_TOTAL_LOG_RES_2 7
#define VKL_VDB_TOTAL_LOG_RES_3 3
#define VKL_VDB_TOTAL_LOG_RES_4 0
#define VKL_VDB_RES_0 262144
#define VKL_VDB_RES_1 4096
#define VKL_VDB_RES_2 128
#define VKL_VDB_RES_3 8
#define VKL_VDB_RES_4 1

#define VKL_VDB_LEAF_LEVEL 3
#define VKL_VDB_LOG_RES_LEAF VKL_VDB_LOG_RES_3
#define VKL_VDB_STORAGE_RES_LEAF VKL_VDB_STORAGE_RES_3
#define VKL_VDB_NUM_VOXELS_LEAF VKL_VDB_NUM_VOXELS_3
#define VKL_VDB_TOTAL_LOG_RES_LEAF VKL_VDB_TOTAL_LOG_RES_3
#define VKL_VDB_RES_LEAF VKL_VDB_RES_3

#ifdef __cplusplus
#define VKL_VDB_INLINE inline
enum VKLTemporalFormat : uint32_t
#else
#define VKL_VDB_INLINE static inline
enum VKLTemporalFormat
#endif
{
  VKL_TEMPORAL_FORMAT_CONSTANT = 0,
  VKL_TEMPORAL_FORMAT_STRUCTURED,
  VKL_TEMPORAL_FORMAT_UNSTRUCTURED,
  VKL_TEMPORAL_FORMAT_INVALID = 100
};
#ifndef __cplusplus
typedef enum VKLTemporalFormat VKLTemporalFormat;
#endif

VKL_VDB_INLINE uint32_t vklVdbNumLevels(void) { return VKL_VDB_NUM_LEVELS; }

VKL_VDB_INLINE uint32_t vklVdbLevelLogRes(uint32_t level)
{
  static const uint32_t v[4] = {VKL_VDB_LOG_RES_0, VKL_VDB_LOG_RES_1, VKL_VDB_LOG_RES_2, VKL_VDB_LOG_RES_3};
  return level < 4 ? v[level] : 0;
}
VKL_VDB_INLINE uint32_t vklVdbLevelResShift(uint32_t level) { return vklVdbLevelLogRes(level); }
VKL_VDB_INLINE uint32_t vklVdbLevelTotalLogRes(uint32_t level)
{
  static const uint32_t v[4] = {VKL_VDB_TOTAL_LOG_RES_0, VKL_VDB_TOTAL_LOG_RES_1, VKL_VDB_TOTAL_LOG_RES_2,
                                VKL_VDB_TOTAL_LOG_RES_3};
  return level < 4 ? v[level] : 0;
}
VKL_VDB_INLINE uint32_t vklVdbLevelStorageRes(uint32_t level)
{
  return level < 4 ? 1u << vklVdbLevelLogRes(level) : 0;
}
/* the domain a node of `level` covers, per axis; level == VKL_VDB_NUM_LEVELS
 * (one leaf voxel) gives 1, the cell resolution below the leaves */
VKL_VDB_INLINE uint32_t vklVdbLevelRes(uint32_t level)
{
  if (level == VKL_VDB_NUM_LEVELS)
    return 1;
  return level < 4 ? 1u << vklVdbLevelTotalLogRes(level) : 0;
}
VKL_VDB_INLINE uint32_t vklVdbLevelNumVoxels(uint32_t level)
{
  return level < 4 ? 1u << (3 * vklVdbLevelLogRes(level)) : 0;
}

/* a 1D domain offset (leaf voxels, relative to the root node) -> the index
 * of the voxel of a level-`level` node that contains it */
VKL_VDB_INLINE uint64_t vklVdbDomainOffsetToVoxel(uint32_t level, uint32_t offset)
{
  if (level >= 4)
    return 0;
  return (uint64_t)(offset & (vklVdbLevelRes(level) - 1)) >> vklVdbLevelTotalLogRes(level + 1);
}
/* a node's 3D voxel index -> its linear index; x is the slowest axis (z
 * fastest), as VDB nodes store their voxels */
VKL_VDB_INLINE uint64_t vklVdb3DToLinear(uint32_t level, uint64_t offsetX, uint64_t offsetY, uint64_t offsetZ)
{
  if (level >= 4)
    return 0;
  const uint32_t l = vklVdbLevelLogRes(level);
  return (offsetX << (2 * l)) + (offsetY << l) + offsetZ;
}
VKL_VDB_INLINE uint64_t vklVdbDomainOffsetToLinear(uint32_t level, uint64_t offsetX, uint64_t offsetY,
                                                   uint64_t offsetZ)
{
  return vklVdb3DToLinear(level, vklVdbDomainOffsetToVoxel(level, (uint32_t)offsetX),
                          vklVdbDomainOffsetToVoxel(level, (uint32_t)offsetY),
                          vklVdbDomainOffsetToVoxel(level, (uint32_t)offsetZ));
}
