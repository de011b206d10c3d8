// Host-callable launchers of the cuda device's kernels.  All pointers are
// device pointers; every launcher enqueues on `stream` and returns without
// synchronizing.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "grid.h"

namespace vklcuda {

// Sampling / gradients over N object-space points (AoS float3).  `attrs`
// lists M attribute indices (M <= kMaxAttributes, host array); output is
// out[i*M + m] for samples and out[3*i ...] for gradients (M == 1).
void launchSample(const DevGrid &g, int filter, uint32_t maxDepth, uint64_t n,
                  const float *points, uint32_t M, const uint32_t *attrs, float *out,
                  cudaStream_t stream);
void launchGradient(const DevGrid &g, int filter, uint32_t maxDepth, uint64_t n,
                    const float *points, uint32_t attr, float *out, cudaStream_t stream);

// Flat leaf map of a sparse grid (g.leafMapDims set, g.leafMap unused):
// map[slot] = full-depth walk result per 8^3 leaf slot, x fastest.
void launchBuildLeafMap(const DevGrid &g, uint64_t *map, cudaStream_t stream);
// Compressed leaves: `numLeaves` packed float leaves (512 values each) ->
// codes (2 or 1 bytes per value by `format`, kCompress*) and one
// (scale, offset) float pair per leaf.
void launchCompressLeaves(uint32_t format, const float *src, uint64_t numLeaves, void *codes,
                          float *scaleOffset, cudaStream_t stream);
// Stencil-block leaves (format kCompress*Blocks): from the float volume g
// (leaf map built), per dense slot (root-relative leaf offsets, 3 per slot,
// ~0 for slots to skip) kLeafCodes codes and one (scale, offset) pair.
void launchBuildLeafBlocks(uint32_t format, const DevGrid &g, uint32_t attr, uint64_t numSlots,
                           const uint32_t *slotOffsets, void *codes, float *scaleOffset, cudaStream_t stream);
// Element count of the bricked copy of a dense x-fastest voxel array
// (brickIndex, grid.h) and its supertile counts.
uint64_t brickedElements(const uint32_t dims[3], uint32_t &superX, uint32_t &superY);

// Commit-time tree construction for dense volumes: fills the voxel codes and
// node origins of levels 0..2 (closed form of the reference's insertion
// order for x-fastest leaves).
void launchBuildDenseTree(const DevGrid &g, uint64_t *vox0, uint64_t *vox1, uint64_t *vox2,
                          uint32_t *org1, uint32_t *org2, const uint32_t nl[3],
                          const uint32_t n1[3], const uint32_t n2[3], cudaStream_t stream);

// Dense commit of one attribute: writes the bricked copy of the x-fastest
// voxel array `src` (element type `type`, kUChar..kDouble) to `dst`, and the
// per-leaf value ranges (2 floats per leaf, leaves x-fastest) over each
// leaf's 3x3x3-leaf filter neighbourhood window.  For a float attribute with
// `atlasSurface` != 0 it also writes the z-plane texture atlas (DevGrid::
// atlasTex) through that surface and sets *denormalFlag (a device word the
// caller zeroes) to 1 if any voxel is denormal.
void launchDenseBrickRanges(const void *src, uint32_t type, void *dst, const uint32_t dims[3],
                            uint32_t superX, uint32_t superY, float background, float *leafRanges,
                            uint64_t atlasSurface, uint32_t atlasPlanesPerRow, uint32_t *denormalFlag,
                            cudaStream_t stream);
// Same for sparse volumes, leaves given by root-relative offsets (3 u32).
void launchSparseLeafRanges(const DevGrid &g, uint32_t attr, uint64_t numLeaves,
                            const uint32_t *leafOffsets, float *leafRanges,
                            cudaStream_t stream);
// Writes leaf ranges into the parent voxels (leafVoxel[i] = level*2^40 +
// voxel index on that level, ~0 to skip; NULL for dense volumes, whose
// parents follow from the leaf counts nl), then reduces level 2 -> 1 -> 0
// child nodes into their parent voxels, and the level-0 node into
// volumeRange.  Attribute 0's call first resets all ranges to empty.
void launchPropagateRanges(const DevGrid &g, uint32_t attr, uint64_t numLeaves,
                           const uint64_t *leafVoxel, const float *leafRanges,
                           float *volumeRange, const uint32_t nl[3], cudaStream_t stream);

// Batched interval iteration: one thread per ray.
void launchIntervals(const DevGrid &g, uint32_t attr, uint32_t depth, DevValueRanges vr,
                     uint64_t n, const float *origins, const float *directions,
                     const float *tRanges, uint32_t maxPerRay, DevInterval *out,
                     uint32_t *counts, cudaStream_t stream);
// Temporally varying dense volumes (k_temporal.cu): samples / gradients at
// per-point times (times NULL: time 0; M > 1: samples of M attributes) and
// the commit's leaf value ranges over all time samples.
void launchSampleTemporal(const DevGrid &g, int filter, uint64_t n, const float *points, const float *times,
                          uint32_t M, const uint32_t *attrs, float *out, bool grad, cudaStream_t stream);
void launchTemporalLeafRanges(const DevGrid &g, uint32_t attr, const uint32_t nl[3], float *leafRanges,
                              cudaStream_t stream);
// 16^3-voxel macrocell intervals (k_macrocell.cu): the volume check (throws
// for volumes the legacy iterator does not cover), the number of
// macrocells, their value ranges (2 floats each) and the batched walk.
void checkMacrocellVolume(const DevGrid &g);
uint64_t macrocellRangeCount(const DevGrid &g);
void launchMacrocellRanges(const DevGrid &g, uint32_t attr, float *ranges, cudaStream_t stream);
void launchMacrocellIntervals(const DevGrid &g, const float *ranges, DevValueRanges vr, uint64_t n,
                              const float *origins, const float *directions, const float *tRanges,
                              uint32_t maxPerRay, DevInterval *out, uint32_t *counts, cudaStream_t stream);
// Batched hit iteration: one thread per ray.
void launchHits(const DevGrid &g, uint32_t attr, int filter, uint32_t depth, DevValueRanges vr,
                uint32_t numValues, const float *values, uint64_t n, const float *origins,
                const float *directions, const float *tRanges, uint32_t maxPerRay,
                DevHit *out, uint32_t *counts, cudaStream_t stream);

// Per-ray stateful iterators of the C API: the state lives in the caller's
// buffer; each call advances it on the GPU by one interval / hit.
struct IntervalIterState;
struct HitIterState;
size_t intervalIterStateSize();
size_t hitIterStateSize();
void launchIntervalIterInit(const DevGrid &g, uint32_t attr, uint32_t depth, const float *ray,
                            void *state, cudaStream_t stream);
void launchIntervalIterNext(const DevGrid &g, DevValueRanges vr, void *state,
                            DevInterval *out, int *result, cudaStream_t stream);
void launchHitIterInit(const DevGrid &g, uint32_t attr, uint32_t depth, const float *ray,
                       void *state, cudaStream_t stream);
void launchHitIterNext(const DevGrid &g, int filter, DevValueRanges vr, uint32_t numValues,
                       const float *values, void *state, DevHit *out, int *result,
                       cudaStream_t stream);

}  // namespace vklcuda
