// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// C++ restatement of the Open VKL v2.0.2 CPU device's VDB / structuredRegular
// hot path (commit-time tree build and value ranges, nearest / trilinear /
// tricubic sampling and gradients, DDA interval iterator, default hit
// iterator).  It is the checker for the CUDA device in openvkl_b200/: only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it,
// never the product path.
//
// Parity status: the reference CPU device (ISPC 1.30 + rkcommon 1.15.2) cannot
// be built in this environment, so this restatement is pinned against the
// reference's own test assertions and tolerances (tests/test_oracle_*.py) and
// against the reference's tricubic coefficient table (tests/golden/).  The
// exact float forms of rkcommon's lerp / rcp_safe / divide_safe and ISPC's FMA
// contraction are not visible in the reference tree; the forms chosen here are
// documented at each helper.
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcVolume OrcVolume;

// Dense structuredRegular volume (DenseVdbVolume.cpp:21-199).
//   dims: voxel counts; data: one pointer per attribute, each x-fastest with
//   byte stride `byteStrides[a]`; types: VKLDataType codes (UCHAR 2500, SHORT
//   3000, USHORT 3500, HALF 5800, FLOAT 6000, DOUBLE 7000).
//   indexToObject: 12 floats, column-major [vx vy vz p] like the reference's
//   "indexToObject" parameter, or NULL to use gridOrigin / gridSpacing.
//   background: one float per attribute (NaN bits 0xFFC068B5 = undefined).
OrcVolume *orc_dense_create(const int32_t dims[3],
                            uint32_t numAttributes,
                            const void *const *data,
                            const uint32_t *types,
                            const uint64_t *byteStrides,
                            int cellCentered,
                            const float gridOrigin[3],
                            const float gridSpacing[3],
                            const float *indexToObject,
                            const int32_t indexOrigin[3],
                            const float *background);

// Sparse VDB volume with packed leaf storage (VdbVolume.cpp:584-1062).
//   levels/origins(3 x i32)/formats per leaf; packedDense[a] holds
//   numDenseLeaves*512 values (z fastest inside a leaf), packedTile[a] holds
//   numTileLeaves values, both of type `dataType` (HALF or FLOAT).
//   indexClippingBounds: 6 ints (lower, upper) or NULL.
OrcVolume *orc_vdb_create(uint64_t numLeaves,
                          const uint32_t *levels,
                          const int32_t *origins,
                          const uint32_t *formats,
                          uint32_t numAttributes,
                          uint32_t dataType,
                          const void *const *packedDense,
                          const void *const *packedTile,
                          const float *indexToObject,
                          const int32_t *indexClippingBounds,
                          const float *background);

void orc_destroy(OrcVolume *v);
const char *orc_last_error(void);

// Introspection (bit-exact tree comparison).
void orc_get_info(const OrcVolume *v,
                  float objectToIndex[12],
                  float indexToObject[12],
                  int32_t rootOrigin[3],
                  uint32_t activeSize[3],
                  float domainBBox[6],
                  float bounds[6]);
uint64_t orc_level_num_nodes(const OrcVolume *v, uint32_t level);
// Copies voxels (u64), value ranges (2 floats per voxel per attribute) and node
// origins (3 u32 per node) of `level` into caller buffers (any may be NULL).
void orc_get_level(const OrcVolume *v,
                   uint32_t level,
                   uint64_t *voxels,
                   float *ranges,
                   uint32_t *origins);
void orc_value_range(const OrcVolume *v, uint32_t attr, float range[2]);

// Sampling (VdbSampler.ispc:97-129, :303-335).  filter: 0 nearest, 100
// linear, 200 cubic.  maxSamplingDepth as the sampler parameter.
void orc_sample(const OrcVolume *v,
                int filter,
                uint32_t maxSamplingDepth,
                uint64_t n,
                const float *points,
                uint32_t attr,
                float *out);
void orc_gradient(const OrcVolume *v,
                  int filter,
                  uint32_t maxSamplingDepth,
                  uint64_t n,
                  const float *points,
                  uint32_t attr,
                  float *out);
// orc_sample with a LeafNodeAccess observer buffer (one uint32 per leaf):
// every leaf a tap's tree walk reaches is set to 1 (VdbLeafAccessObserver.ih).
void orc_sample_observed(const OrcVolume *v, int filter, uint32_t maxSamplingDepth, uint64_t n,
                         const float *points, uint32_t attr, float *out, uint32_t *leafAccess);
// Same as orc_sample but split over `threads` host threads (CPU baseline,
// and the large parity cases).
void orc_sample_parallel(const OrcVolume *v,
                         int filter,
                         uint64_t n,
                         const float *points,
                         uint32_t attr,
                         float *out,
                         int threads);
// 16^3-voxel macrocell intervals of the reference's legacy structuredRegular
// volume (GridAccelerator): per-macrocell value ranges (2 floats per cell,
// x fastest) and the batched interval walk (out: maxIntervals x 5 floats per
// ray, counts: all intervals of the ray).  Returns nonzero (orc_last_error)
// for volumes the legacy iterator does not cover.
void orc_macrocell_ranges(const OrcVolume *v, uint32_t attr, float *out);
int orc_iterate_macrocells(const OrcVolume *v, uint32_t attr, uint32_t numRanges, const float *ranges,
                           uint64_t numRays, const float *origins, const float *directions,
                           const float *tRanges, uint32_t maxIntervals, float *out, uint32_t *counts);
// A structuredRegular volume with temporally varying data (motion blur):
// numTimesteps > 0 for structured data (numTimesteps values per voxel), or
// per-voxel indices (VKL_UINT 4500 / VKL_ULONG 5550, numVoxels + 1 entries)
// into the data and `times` arrays for unstructured data.  numItems: the
// element count of each attribute array (validated as the reference does).
OrcVolume *orc_dense_create_temporal(const int32_t dims[3], uint32_t numAttributes, const void *const *data,
                                     const uint32_t *types, const uint64_t *numItems, int cellCentered,
                                     const float gridOrigin[3], const float gridSpacing[3],
                                     const float *indexToObject, const float *background, int numTimesteps,
                                     const void *indices, uint32_t indexType, uint64_t numIndices,
                                     const float *times, uint64_t numTimes);
// Samples / gradients at per-point times (NULL: time 0) on `threads` host
// threads.
void orc_sample_times(const OrcVolume *v, int filter, uint64_t n, const float *points, const float *times,
                      uint32_t attr, float *out, int threads);
void orc_gradient_times(const OrcVolume *v, int filter, uint64_t n, const float *points, const float *times,
                        uint32_t attr, float *out, int threads);
// The density path tracer, one progressive frame added into rgba / weights
// (pt: shutter, sigmaTScale, sigmaSScale, ambientLightIntensity, time; ipt:
// motionBlur, maxNumScatters, showBbox, frame).
void orc_path_trace(const OrcVolume *v, int filter, uint32_t maxSamplingDepth, uint32_t attr,
                    const float camera[14], const float *tfColors, int tfNum, const float tfRange[2], int W, int H,
                    const float bounds[6], const float pt[5], const int ipt[4], float *rgba, float *weights);
// orc_gradient split over `threads` host threads.
void orc_gradient_parallel(const OrcVolume *v, int filter, uint32_t maxSamplingDepth, uint64_t n,
                           const float *points, uint32_t attr, float *out, int threads);

// FP64 evaluation of the same filter on the stored voxel values (error
// reporting only).
void orc_sample_fp64(const OrcVolume *v,
                     int filter,
                     uint64_t n,
                     const float *points,
                     uint32_t attr,
                     double *out);

// Interval iteration (VdbIterator.ispc:36-159).  For each ray writes up to
// maxIntervals intervals (5 floats: t0 t1 v0 v1 nominalDeltaT) at
// out + ray*maxIntervals*5 and the number produced in counts[ray] (which may
// exceed maxIntervals; extra intervals are counted but not stored).
void orc_iterate_intervals(const OrcVolume *v,
                           uint32_t attr,
                           uint32_t numRanges,
                           const float *ranges,
                           float intervalResolutionHint,
                           uint64_t numRays,
                           const float *origins,
                           const float *directions,
                           const float *tRanges,
                           uint32_t maxIntervals,
                           float *out,
                           uint32_t *counts);

// Hit iteration (DefaultIterator.ispc:168-258, Iterator.ih:17-197).  Hits are
// 3 floats (t, sample, epsilon).  filter is the sampler filter used to march.
void orc_iterate_hits(const OrcVolume *v,
                      uint32_t attr,
                      int filter,
                      uint32_t numValues,
                      const float *values,
                      uint64_t numRays,
                      const float *origins,
                      const float *directions,
                      const float *tRanges,
                      uint32_t maxHits,
                      float *out,
                      uint32_t *counts);

// The reference's example renderers restated (one ray per pixel centre):
// renderer 0 ray march iterator, 1 interval iterator debug, 2 hit iterator
// renderer.  camera = {sensorWidth, focalLength, camera-to-world rotation
// rows (9), translation (3)}; tfColors = tfNum RGBA quadruples over
// tfRange; ip = {width, height, firstIntervalOnly, showIntervalBorders};
// fp = {bounds (6), samplingRate, intervalColorScale, intervalOpacity}.
// Interval context: numRanges ranges and the resolution hint; hit context:
// numValues iso values.  Writes width*height RGBA floats, row 0 at the top.
void orc_render(const OrcVolume *v, int renderer, int filter, int gradientFilter, uint32_t maxSamplingDepth,
                uint32_t attr, uint32_t numRanges, const float *ranges, float hint, uint32_t numValues,
                const float *values, const float camera[14], const float *tfColors, int tfNum,
                const float tfRange[2], const int ip[4], const float fp[9], float *rgba);

// Tricubic coefficient map as generated here: for row r (coefficient
// 16i+4j+k) entries [start[r], start[r+1]) of (col, weight).
int orc_tricubic_map(int32_t *start, int32_t *cols, float *weights);

// InnerNode observer (VdbInnerNodeObserver.cpp:20-185): nodes at maxDepth
// as 6 float bbox + 2 float range.  Returns the number of nodes; writes at
// most cap of them.
uint64_t orc_inner_nodes(const OrcVolume *v,
                         uint32_t maxDepth,
                         uint32_t attr,
                         uint64_t cap,
                         float *out);

// Compressed leaves (the cuda device's extension; no reference
// counterpart).  format: 1 = FP16, 2 = BF16, 3 = FP8-E4M3 (saturating).
// orc_round_format: each input rounded to nearest-even in the format,
// returned as float.  orc_quantize_leaves: per leaf of 512 values,
// offset = 0.5*lo + 0.5*hi and scale = (0.5*hi - 0.5*lo) / codeMax over the
// non-NaN values (scale 1 for a constant leaf); decoded = round((v - offset)
// / scale) * scale + offset in float; scaleOffset gets 2 floats per leaf.
void orc_round_format(int format, uint64_t n, const float *in, float *out);
void orc_quantize_leaves(int format,
                         uint64_t numLeaves,
                         const float *in,
                         float *decoded,
                         float *scaleOffset);
// orc_quantize_groups: the same rule over groups of groupSize values.
void orc_quantize_groups(int format, uint64_t numGroups, uint32_t groupSize, const float *in,
                         float *decoded, float *scaleOffset);
// Stencil-block leaves (the cuda device's extension): orc_vdb_leaf_windows
// writes each dense leaf slot's 9^3 sampling window (full-depth lookups, x
// outermost, z fastest); orc_vdb_set_windows installs decoded windows of an
// attribute, whose trilinear stencils then take their 8 corners from the
// window of the dense leaf holding the base voxel.
void orc_vdb_leaf_windows(const OrcVolume *v, uint32_t attr, float *windows);
void orc_vdb_set_windows(OrcVolume *v, uint32_t attr, uint64_t numSlots, const float *decodedWindows);

#ifdef __cplusplus
}
#endif
