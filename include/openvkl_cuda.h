// Open VKL C API as exported by the B200 `cuda` device
// (libopenvkl_device_cuda.so).
//
// Every declaration below re-states the signature of the reference interface
// it replaces (Open VKL v2.0.2; file:line relative to its source tree) so an
// application's existing sampling / traversal calls link against this library
// unchanged.  Handles are the reference's {host, device} pair
// (openvkl/include/openvkl/types.h:56-69).  Entry points marked EXTENSION have
// no counterpart in the reference; they are the batched GPU forms of the
// per-ray iterator calls and the precision / batching / learned patterns.
//
// Pointer arguments of the N / MN / batched calls may be host or device
// memory; device memory is used in place, host memory is staged through the
// device and the call synchronizes before returning.  All work runs on the
// device's CUDA stream (vklDeviceSetVoidPtr(device, "cudaStream", stream)).
#pragma once

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>  // as the reference's sampler.h / volume.h / observer.h

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define OPENVKL_CUDA_INTERFACE __declspec(dllexport)
#else
#define OPENVKL_CUDA_INTERFACE __attribute__((visibility("default")))
#endif

// ---------------------------------------------------------------------------
// Types (openvkl/include/openvkl/types.h, VKLDataType.h, VKLFilter.h,
// VKLFormat.h, VKLError.h, VKLLogLevel.h, data.h).
// ---------------------------------------------------------------------------
typedef struct { float x, y, z; } vkl_vec3f;
typedef struct { int x, y, z; } vkl_vec3i;
typedef struct { float lower, upper; } vkl_range1f;
typedef struct { vkl_vec3f lower, upper; } vkl_box3f;
typedef struct { float x[4], y[4], z[4]; } vkl_vvec3f4;
typedef struct { float x[8], y[8], z[8]; } vkl_vvec3f8;
typedef struct { float x[16], y[16], z[16]; } vkl_vvec3f16;
typedef struct { float lower[4], upper[4]; } vkl_vrange1f4;
typedef struct { float lower[8], upper[8]; } vkl_vrange1f8;
typedef struct { float lower[16], upper[16]; } vkl_vrange1f16;

typedef struct
{
  void *host;
  void *device;
} VKLObject;

typedef struct VKLDeviceInternal *VKLDevice;
typedef VKLObject VKLData;
typedef VKLObject VKLVolume;
typedef VKLObject VKLSampler;
typedef VKLObject VKLIntervalIteratorContext;
typedef VKLObject VKLHitIteratorContext;
typedef VKLObject VKLObserver;
typedef uint64_t VKLFeatureFlags;

typedef enum
{
  VKL_DEVICE = 100, VKL_VOID_PTR = 200, VKL_BOOL = 250,
  VKL_OBJECT = 0x8000000, VKL_DATA = 0x8000000 + 100, VKL_VOLUME,
  VKL_STRING = 1500,
  VKL_CHAR = 2000, VKL_UCHAR = 2500, VKL_SHORT = 3000, VKL_USHORT = 3500,
  VKL_INT = 4000, VKL_VEC2I, VKL_VEC3I, VKL_VEC4I,
  VKL_UINT = 4500, VKL_VEC2UI, VKL_VEC3UI, VKL_VEC4UI,
  VKL_LONG = 5000, VKL_ULONG = 5550,
  VKL_HALF = 5800,
  VKL_FLOAT = 6000, VKL_VEC2F, VKL_VEC3F, VKL_VEC4F,
  VKL_DOUBLE = 7000,
  VKL_BOX1I = 8000, VKL_BOX2I, VKL_BOX3I, VKL_BOX4I,
  VKL_BOX1F = 10000, VKL_BOX2F, VKL_BOX3F, VKL_BOX4F,
  VKL_LINEAR2F = 12000, VKL_LINEAR3F, VKL_AFFINE2F, VKL_AFFINE3F,
  VKL_UNKNOWN = 9999999
} VKLDataType;

typedef enum { VKL_DATA_DEFAULT = 0, VKL_DATA_SHARED_BUFFER = 1 } VKLDataCreationFlags;
typedef enum { VKL_FILTER_NEAREST = 0, VKL_FILTER_LINEAR = 100, VKL_FILTER_CUBIC = 200 } VKLFilter;
typedef enum { VKL_FORMAT_TILE = 0, VKL_FORMAT_DENSE_ZYX = 1, VKL_FORMAT_INVALID = 100 } VKLFormat;
typedef enum
{
  VKL_NO_ERROR = 0, VKL_UNKNOWN_ERROR = 1, VKL_INVALID_ARGUMENT = 2,
  VKL_INVALID_OPERATION = 3, VKL_OUT_OF_MEMORY = 4, VKL_UNSUPPORTED_CPU = 5
} VKLError;
typedef enum
{
  VKL_LOG_DEBUG = 1, VKL_LOG_INFO = 2, VKL_LOG_WARNING = 3, VKL_LOG_ERROR = 4,
  VKL_LOG_NONE = 5
} VKLLogLevel;

// VKLInterval / VKLHit (openvkl/devices/cpu/include/openvkl/device/openvkl.h:
// 174-180, :315-320).
typedef struct
{
  vkl_range1f tRange;
  vkl_range1f valueRange;
  float nominalDeltaT;
} VKLInterval;

typedef struct
{
  float t;
  float sample;
  float epsilon;
} VKLHit;

typedef struct IntervalIterator *VKLIntervalIterator;
typedef struct HitIterator *VKLHitIterator;

typedef void (*VKLLogCallback)(void *userData, const char *message);
typedef void (*VKLErrorCallback)(void *userData, VKLError error, const char *message);

// ---------------------------------------------------------------------------
// Device (openvkl/include/openvkl/device.h:15-75; init
// devices/cpu/include/openvkl/device/openvkl.h:23).
// ---------------------------------------------------------------------------
OPENVKL_CUDA_INTERFACE void vklInit(void);
OPENVKL_CUDA_INTERFACE VKLDevice vklNewDevice(const char *deviceName);
OPENVKL_CUDA_INTERFACE void vklDeviceSetLogCallback(VKLDevice, VKLLogCallback, void *userData);
OPENVKL_CUDA_INTERFACE void vklDeviceSetErrorCallback(VKLDevice, VKLErrorCallback, void *userData);
OPENVKL_CUDA_INTERFACE void vklDeviceSetInt(VKLDevice, const char *name, int x);
OPENVKL_CUDA_INTERFACE void vklDeviceSetString(VKLDevice, const char *name, const char *s);
OPENVKL_CUDA_INTERFACE void vklDeviceSetVoidPtr(VKLDevice, const char *name, void *v);
OPENVKL_CUDA_INTERFACE void vklCommitDevice(VKLDevice);
OPENVKL_CUDA_INTERFACE VKLError vklDeviceGetLastErrorCode(VKLDevice);
OPENVKL_CUDA_INTERFACE const char *vklDeviceGetLastErrorMsg(VKLDevice);
OPENVKL_CUDA_INTERFACE int vklGetNativeSIMDWidth(VKLDevice);
OPENVKL_CUDA_INTERFACE void vklCommit(VKLObject object);
OPENVKL_CUDA_INTERFACE void vklRelease(VKLObject object);
OPENVKL_CUDA_INTERFACE void vklReleaseDevice(VKLDevice);

// ---------------------------------------------------------------------------
// Data (openvkl/include/openvkl/data.h:38-44).
// ---------------------------------------------------------------------------
OPENVKL_CUDA_INTERFACE VKLData vklNewData(VKLDevice device,
                                          size_t numItems,
                                          VKLDataType dataType,
                                          const void *source,
                                          VKLDataCreationFlags dataCreationFlags,
                                          size_t byteStride);

// ---------------------------------------------------------------------------
// Volumes and parameters (openvkl/include/openvkl/volume.h:53-63,
// parameters.h:12-32).
// ---------------------------------------------------------------------------
OPENVKL_CUDA_INTERFACE VKLVolume vklNewVolume(VKLDevice device, const char *type);
OPENVKL_CUDA_INTERFACE vkl_box3f vklGetBoundingBox(VKLVolume volume);
OPENVKL_CUDA_INTERFACE unsigned int vklGetNumAttributes(VKLVolume volume);
OPENVKL_CUDA_INTERFACE vkl_range1f vklGetValueRange(VKLVolume volume, unsigned int attributeIndex);

OPENVKL_CUDA_INTERFACE void vklSetBool(VKLObject object, const char *name, int b);
OPENVKL_CUDA_INTERFACE void vklSetFloat(VKLObject object, const char *name, float x);
OPENVKL_CUDA_INTERFACE void vklSetVec3f(VKLObject object, const char *name, float x, float y, float z);
OPENVKL_CUDA_INTERFACE void vklSetInt(VKLObject object, const char *name, int x);
OPENVKL_CUDA_INTERFACE void vklSetVec3i(VKLObject object, const char *name, int x, int y, int z);
OPENVKL_CUDA_INTERFACE void vklSetData(VKLObject object, const char *name, VKLData data);
OPENVKL_CUDA_INTERFACE void vklSetString(VKLObject object, const char *name, const char *s);
OPENVKL_CUDA_INTERFACE void vklSetVoidPtr(VKLObject object, const char *name, void *v);
OPENVKL_CUDA_INTERFACE void vklSetParam(VKLObject object, const char *name, VKLDataType dataType,
                                        const void *mem);

// ---------------------------------------------------------------------------
// Samplers (openvkl/include/openvkl/sampler.h:30-41).
// ---------------------------------------------------------------------------
OPENVKL_CUDA_INTERFACE VKLSampler vklNewSampler(VKLVolume volume);
OPENVKL_CUDA_INTERFACE VKLFeatureFlags vklGetFeatureFlags(VKLSampler sampler);

// ---------------------------------------------------------------------------
// Sampling and gradients
// (openvkl/devices/cpu/include/openvkl/device/openvkl.h:32-160).
// ---------------------------------------------------------------------------
OPENVKL_CUDA_INTERFACE float vklComputeSample(const VKLSampler *sampler,
                                              const vkl_vec3f *objectCoordinates,
                                              unsigned int attributeIndex,
                                              float time);
OPENVKL_CUDA_INTERFACE void vklComputeSample4(const int *valid, const VKLSampler *sampler,
                                              const vkl_vvec3f4 *objectCoordinates,
                                              float *samples, unsigned int attributeIndex,
                                              const float *times);
OPENVKL_CUDA_INTERFACE void vklComputeSample8(const int *valid, const VKLSampler *sampler,
                                              const vkl_vvec3f8 *objectCoordinates,
                                              float *samples, unsigned int attributeIndex,
                                              const float *times);
OPENVKL_CUDA_INTERFACE void vklComputeSample16(const int *valid, const VKLSampler *sampler,
                                               const vkl_vvec3f16 *objectCoordinates,
                                               float *samples, unsigned int attributeIndex,
                                               const float *times);
// Multi-attribute samples of 4 / 8 / 16 SoA points; samples[m * W + i] is
// attribute attributeIndices[m] at lane i (openvkl/devices/cpu/include/
// openvkl/device/openvkl.h:79-104).
OPENVKL_CUDA_INTERFACE void vklComputeSampleM4(const int *valid, const VKLSampler *sampler,
                                               const vkl_vvec3f4 *objectCoordinates, float *samples,
                                               unsigned int M, const unsigned int *attributeIndices,
                                               const float *times);
OPENVKL_CUDA_INTERFACE void vklComputeSampleM8(const int *valid, const VKLSampler *sampler,
                                               const vkl_vvec3f8 *objectCoordinates, float *samples,
                                               unsigned int M, const unsigned int *attributeIndices,
                                               const float *times);
OPENVKL_CUDA_INTERFACE void vklComputeSampleM16(const int *valid, const VKLSampler *sampler,
                                                const vkl_vvec3f16 *objectCoordinates, float *samples,
                                                unsigned int M, const unsigned int *attributeIndices,
                                                const float *times);
// Gradients of 4 / 8 / 16 SoA points (openvkl/devices/cpu/include/openvkl/
// device/openvkl.h:121-143).
OPENVKL_CUDA_INTERFACE void vklComputeGradient4(const int *valid, const VKLSampler *sampler,
                                                const vkl_vvec3f4 *objectCoordinates, vkl_vvec3f4 *gradients,
                                                unsigned int attributeIndex, const float *times);
OPENVKL_CUDA_INTERFACE void vklComputeGradient8(const int *valid, const VKLSampler *sampler,
                                                const vkl_vvec3f8 *objectCoordinates, vkl_vvec3f8 *gradients,
                                                unsigned int attributeIndex, const float *times);
OPENVKL_CUDA_INTERFACE void vklComputeGradient16(const int *valid, const VKLSampler *sampler,
                                                 const vkl_vvec3f16 *objectCoordinates, vkl_vvec3f16 *gradients,
                                                 unsigned int attributeIndex, const float *times);
OPENVKL_CUDA_INTERFACE void vklComputeSampleN(const VKLSampler *sampler,
                                              unsigned int N,
                                              const vkl_vec3f *objectCoordinates,
                                              float *samples,
                                              unsigned int attributeIndex,
                                              const float *times);
OPENVKL_CUDA_INTERFACE void vklComputeSampleM(const VKLSampler *sampler,
                                              const vkl_vec3f *objectCoordinates,
                                              float *samples,
                                              unsigned int M,
                                              const unsigned int *attributeIndices,
                                              float time);
OPENVKL_CUDA_INTERFACE void vklComputeSampleMN(const VKLSampler *sampler,
                                               unsigned int N,
                                               const vkl_vec3f *objectCoordinates,
                                               float *samples,
                                               unsigned int M,
                                               const unsigned int *attributeIndices,
                                               const float *times);
OPENVKL_CUDA_INTERFACE vkl_vec3f vklComputeGradient(const VKLSampler *sampler,
                                                    const vkl_vec3f *objectCoordinates,
                                                    unsigned int attributeIndex,
                                                    float time);
OPENVKL_CUDA_INTERFACE void vklComputeGradientN(const VKLSampler *sampler,
                                                unsigned int N,
                                                const vkl_vec3f *objectCoordinates,
                                                vkl_vec3f *gradients,
                                                unsigned int attributeIndex,
                                                const float *times);

// ---------------------------------------------------------------------------
// Iterator contexts (openvkl/include/openvkl/iterator.h:30-37) and the
// per-ray iterator calls (devices/cpu/include/openvkl/device/openvkl.h:
// 208-279, :348-416).
// ---------------------------------------------------------------------------
OPENVKL_CUDA_INTERFACE VKLIntervalIteratorContext vklNewIntervalIteratorContext(VKLSampler sampler);
OPENVKL_CUDA_INTERFACE VKLHitIteratorContext vklNewHitIteratorContext(VKLSampler sampler);
OPENVKL_CUDA_INTERFACE size_t vklGetIntervalIteratorSize(const VKLIntervalIteratorContext *context);
OPENVKL_CUDA_INTERFACE VKLIntervalIterator vklInitIntervalIterator(
    const VKLIntervalIteratorContext *context, const vkl_vec3f *origin,
    const vkl_vec3f *direction, const vkl_range1f *tRange, float time, void *buffer);
OPENVKL_CUDA_INTERFACE int vklIterateInterval(VKLIntervalIterator iterator, VKLInterval *interval);
OPENVKL_CUDA_INTERFACE size_t vklGetHitIteratorSize(const VKLHitIteratorContext *context);
OPENVKL_CUDA_INTERFACE VKLHitIterator vklInitHitIterator(const VKLHitIteratorContext *context,
                                                         const vkl_vec3f *origin,
                                                         const vkl_vec3f *direction,
                                                         const vkl_range1f *tRange,
                                                         float time, void *buffer);
OPENVKL_CUDA_INTERFACE int vklIterateHit(VKLHitIterator iterator, VKLHit *hit);

// EXTENSION: batched iteration, one GPU thread per ray.  Ray i writes up to
// `maxPerRay` records at out[i*maxPerRay ...] and its full count to
// counts[i] (a count above maxPerRay means the ray had more records than
// were stored).  Records and counts equal what repeated vklIterateInterval /
// vklIterateHit calls on the same ray return.
OPENVKL_CUDA_INTERFACE void vklIterateIntervalsN(const VKLIntervalIteratorContext *context,
                                                 unsigned int N,
                                                 const vkl_vec3f *origins,
                                                 const vkl_vec3f *directions,
                                                 const vkl_range1f *tRanges,
                                                 unsigned int maxPerRay,
                                                 VKLInterval *intervals,
                                                 unsigned int *counts);
OPENVKL_CUDA_INTERFACE void vklIterateHitsN(const VKLHitIteratorContext *context,
                                            unsigned int N,
                                            const vkl_vec3f *origins,
                                            const vkl_vec3f *directions,
                                            const vkl_range1f *tRanges,
                                            unsigned int maxPerRay,
                                            VKLHit *hits,
                                            unsigned int *counts);

// ---------------------------------------------------------------------------
// Observers (openvkl/include/openvkl/observer.h:36-75).
// ---------------------------------------------------------------------------
OPENVKL_CUDA_INTERFACE VKLObserver vklNewVolumeObserver(VKLVolume volume, const char *type);
OPENVKL_CUDA_INTERFACE VKLObserver vklNewSamplerObserver(VKLSampler sampler, const char *type);
OPENVKL_CUDA_INTERFACE const void *vklMapObserver(VKLObserver observer);
OPENVKL_CUDA_INTERFACE void vklUnmapObserver(VKLObserver observer);
OPENVKL_CUDA_INTERFACE VKLDataType vklGetObserverElementType(VKLObserver observer);
OPENVKL_CUDA_INTERFACE size_t vklGetObserverElementSize(VKLObserver observer);
OPENVKL_CUDA_INTERFACE size_t vklGetObserverNumElements(VKLObserver observer);

// EXTENSION: copies level `level` (0..2) of a committed volume's tree into
// host memory: the u64 voxel codes of all nodes (levelNumVoxels per node),
// their value ranges (2 floats per voxel per attribute) and the node origins
// (3 u32 per node, relative to the root origin).  Any output may be NULL.
// Returns the number of nodes on the level (level 3: the number of leaves).
// Exposes the VdbGrid levels of the reference
// (openvkl/devices/cpu/volume/vdb/VdbGridShared.h:17-33) for inspection.
OPENVKL_CUDA_INTERFACE uint64_t vklCudaGetTreeLevel(VKLVolume volume, unsigned int level,
                                                    uint64_t *voxels, float *valueRanges,
                                                    uint32_t *origins);

// EXTENSION (no counterpart in the reference): batched multi-volume
// sampling.  One job = a committed sampler, `numPoints` object-space points
// and outputs for samples (`numPoints` floats) and / or gradients
// (`numPoints` vec3f), all in device memory (an output may be NULL).  The
// batch records every job into one CUDA graph: dense volumes and plain
// sparse volumes with the trilinear filter run in persistent kernels that
// compute each point's sample and gradient from one gather; other jobs run
// as the vklComputeSampleN / vklComputeGradientN launches.  Results equal
// those calls bit for bit.  `autotune` != 0 times candidate tile sizes,
// brick sorting and CTAs per SM on the batch and keeps the fastest
// (remembered for later batches of the same shape).  Running enqueues the
// graph on the device's stream; the job list is fixed at creation (the
// points and outputs are re-read at every run).
typedef struct {
  VKLSampler sampler;
  const vkl_vec3f *points;
  unsigned int numPoints;
  unsigned int attributeIndex;
  float *samples;
  vkl_vec3f *gradients;
} VKLCudaSampleJob;

typedef struct VKLCudaSampleBatch_ *VKLCudaSampleBatch;

OPENVKL_CUDA_INTERFACE VKLCudaSampleBatch vklCudaNewSampleBatch(VKLDevice device,
                                                                unsigned int numJobs,
                                                                const VKLCudaSampleJob *jobs,
                                                                int autotune);
OPENVKL_CUDA_INTERFACE VKLError vklCudaRunSampleBatch(VKLCudaSampleBatch batch);
// The configuration the batch runs its largest fused class with, and how
// many jobs are fused (the rest run as plain launches).
OPENVKL_CUDA_INTERFACE VKLError vklCudaGetSampleBatchConfig(VKLCudaSampleBatch batch,
                                                           int *tilePoints, int *sorted,
                                                           int *ctasPerSM, int *fusedJobs);
OPENVKL_CUDA_INTERFACE void vklCudaReleaseSampleBatch(VKLCudaSampleBatch batch);

// EXTENSION (no counterpart in the reference): learned surrogate of a
// volume.  A 16-level hash-grid encoding (2^log2TableSize entries of 2 FP16
// features per level, resolution floor(baseResolution * growth^level) over
// the volume's object bounding box) feeds a 32-64-64-64-1 ReLU MLP (FP16
// weights, tensor cores).  The sampler must be trilinear over float voxels;
// its plain samples are the training targets, the fallback and the measure of
// the surrogate's error.  Parameters (host or device memory): the table as
// levels x entries x 2 floats, the weights as W1 (64x32), W2 (64x64),
// W3 (64x64), W4 (64), row-major, concatenated (10304 floats).  Points,
// targets, samples and the train-step loss are device memory.
typedef struct VKLCudaSurrogate_ *VKLCudaSurrogate;

OPENVKL_CUDA_INTERFACE VKLCudaSurrogate vklCudaNewSurrogate(VKLSampler sampler,
                                                            unsigned int log2TableSize,
                                                            float baseResolution, float growth);
OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateSetParameters(VKLCudaSurrogate surrogate,
                                                             const float *table,
                                                             const float *weights);
OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateGetParameters(VKLCudaSurrogate surrogate,
                                                             float *table, float *weights);
// Gradients of sum((y - target)^2) over the n points (no update); outputs in
// host or device memory, any may be NULL.
OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateGradient(VKLCudaSurrogate surrogate,
                                                        unsigned int n,
                                                        const vkl_vec3f *points,
                                                        const float *targets, float *loss,
                                                        float *tableGradient,
                                                        float *weightGradient);
// One Adam step (beta 0.9 / 0.99) on the loss sum((y - target)^2) / n;
// `loss` (device, may be NULL) receives the sum of squared errors.
OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateTrainStep(VKLCudaSurrogate surrogate,
                                                         unsigned int n, const vkl_vec3f *points,
                                                         const float *targets, float learningRate,
                                                         float *loss);
// Flags every 32^3-voxel region where |surrogate - plain sampler| exceeds
// `threshold` at one of the points, or that none of the points reached.
OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateCalibrate(VKLCudaSurrogate surrogate,
                                                         unsigned int n, const vkl_vec3f *points,
                                                         float threshold,
                                                         unsigned int *flaggedRegions);
// Surrogate samples; with `fallback` != 0 the plain sample in flagged regions
// and outside the volume's domain (every region is flagged until calibrated).
OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateSample(VKLCudaSurrogate surrogate, unsigned int n,
                                                      const vkl_vec3f *points, float *samples,
                                                      int fallback);
OPENVKL_CUDA_INTERFACE void vklCudaGetSurrogateInfo(VKLCudaSurrogate surrogate,
                                                    uint64_t *tableEntries,
                                                    unsigned int *numWeights,
                                                    uint64_t *numRegions,
                                                    unsigned int *levelResolutions);
OPENVKL_CUDA_INTERFACE void vklCudaReleaseSurrogate(VKLCudaSurrogate surrogate);

// EXTENSION (no counterpart in the reference): the value range that
// vklGetValueRange would report for a structuredRegular volume of
// dimensions (dimX, dimY, dimZ) over `voxels` (x-fastest, device memory,
// type uchar / short / ushort / half / float / double) with the given
// "background", written as {lower, upper} to `valueRange` (2 floats, device
// memory) asynchronously on the device's stream.  It allocates no memory:
// its scratch is a fixed static device array, which bounds the volume to
// 16,777,216 leaves (8^3 voxel blocks, e.g. 2048^3 voxels); larger volumes
// return VKL_INVALID_ARGUMENT before anything is launched.  The first call
// on a device is a one-time set-up (it resolves the scratch and loads the
// kernels) and belongs before any stream capture.  Calls whose work
// overlaps on one device share the scratch and race: issue them on one
// stream.  The calling thread's current CUDA device must be the VKL
// device's.  For volumes with NaN voxels the result may differ from the
// committed volume's, whose NaN handling depends on reduction order; so may
// the sign of a zero bound where +0.0 and -0.0 voxels meet (the two folds
// visit them in different orders), which compares equal by value.
// Returns VKL_NO_ERROR once launched, else the error code (also reported
// through the device's error callback).
OPENVKL_CUDA_INTERFACE VKLError vklCudaDenseValueRangeNoAlloc(VKLDevice device, const void *voxels,
                                                             VKLDataType voxelType, int dimX,
                                                             int dimY, int dimZ, float background,
                                                             float *valueRange);

#ifdef __cplusplus
}
#endif
