// __device__ API of the cuda device: sampling and iteration called from an
// application's own CUDA kernels, with the signatures of the reference's
// GPU (SYCL) device API (openvkl/devices/gpu/include/openvkl/device/
// openvkl.h:30-120).  The handles are passed by value into the kernel; their
// `device` pointers address the objects' device-resident state, which
// vklNew* / vklCommit write and which stays valid while the object lives.
// After re-committing a volume, commit its samplers and contexts again.
//
// Two differences from the SYCL header, both forced by CUDA:
// - Every function takes its VKLFeatureFlags argument explicitly. The host C
//   API declares functions of the same names without it, and CUDA cannot
//   overload on __host__ / __device__ alone.
// - The iterator buffer sizes are the compile-time constants
//   VKL_CUDA_INTERVAL_ITERATOR_SIZE / VKL_CUDA_HIT_ITERATOR_SIZE instead of
//   vklGet*IteratorSize. The reference's GPU device publishes its
//   VKL_MAX_*_ITERATOR_SIZE the same way (max_iterator_size.h).
// Feature flags (vklGetFeatureFlags: the reference's bit layout,
// VKLFeatureFlagsInternal.h) name the volume types and sample / gradient
// filters a sampling call may meet; vklComputeSample / SampleM / Gradient
// skip the excluded paths, and drop them from the inlined code when the
// argument is a compile-time constant.  VKL_FEATURE_FLAGS_DEFAULT (all bits)
// and 0 keep every path.  Results are identical either way.  The iterators
// accept the flags and do not need them.  `time` is the sample time of
// temporally varying structuredRegular volumes (feature flags
// VKL_FEATURE_FLAG_HAS_TEMPORAL_FORMAT_STRUCTURED / _UNSTRUCTURED, bits 13 and
// 14); other volumes ignore it.
//
// Results are bit-identical to the host API's when the including
// translation unit is compiled like the library: nvcc -gencode
// arch=compute_100a,code=sm_100a --fmad=false -I<repo>/include.
#pragma once
#ifdef __CUDACC__

#include "openvkl_cuda.h"
#include "../openvkl_b200/csrc/iterate.cuh"

#define VKL_CUDA_INTERVAL_ITERATOR_SIZE 512
#define VKL_CUDA_HIT_ITERATOR_SIZE 768

namespace vklcuda {
namespace device_api {

// The iterators' state lives in the caller's buffer (local memory of the
// calling thread), so both use the DDA form indexed by the level at run time:
// one copy of its step code per call site instead of one per tree level.
struct IntervalIteratorState {
  IntervalItDyn it;
  const DevIntervalContextState *ctx;
};
struct HitIteratorState {
  HitIt h;
  const DevHitContextState *ctx;
  float time;
};
static_assert(sizeof(IntervalIteratorState) <= VKL_CUDA_INTERVAL_ITERATOR_SIZE, "interval iterator size");
static_assert(sizeof(HitIteratorState) <= VKL_CUDA_HIT_ITERATOR_SIZE, "hit iterator size");

__device__ __forceinline__ f3 toF3(const vkl_vec3f *v) { return {v->x, v->y, v->z}; }

constexpr VKLFeatureFlags kStructuredRegular = 1ull << 0, kVdb = 1ull << 5;
constexpr VKLFeatureFlags kSampleNearest = 1ull << 6, kSampleLinear = 1ull << 7, kSampleCubic = 1ull << 8;
constexpr VKLFeatureFlags kGradientNearest = 1ull << 9, kGradientLinear = 1ull << 10, kGradientCubic = 1ull << 11;
constexpr VKLFeatureFlags kTemporalVarying = (1ull << 13) | (1ull << 14);

// Runs f(field) with the sampler's field type, over the volume kinds the
// flags allow (the type dispatch of sampleIndexAny).
template <class F>
__device__ __forceinline__ auto withField(const DevGrid &g, uint32_t attr, uint32_t depth, VKLFeatureFlags ff, F &&f,
                                          float time = 0.f)
{
  const bool denseOk = ff & kStructuredRegular, vdbOk = ff & kVdb;
  const uint32_t t   = g.type[attr];
  if ((ff & kTemporalVarying) && g.temporal)
    return withTemporalField(g, attr, time, f);
  if (denseOk && (g.dense || !vdbOk)) {
    switch (t) {
    case kUChar:
      return f(DenseField<uint8_t>(g, attr));
    case kShort:
      return f(DenseField<int16_t>(g, attr));
    case kUShort:
      return f(DenseField<uint16_t>(g, attr));
    case kHalf:
      return f(DenseField<__half>(g, attr));
    case kDouble:
      return f(DenseField<double>(g, attr));
    default:
      return f(DenseField<float>(g, attr));
    }
  }
  switch (g.compress) {
  case kCompressFP16:
    return f(SparseField<CodeFP16>(g, attr, depth));
  case kCompressBF16:
    return f(SparseField<CodeBF16>(g, attr, depth));
  case kCompressFP8:
    return f(SparseField<CodeE4M3>(g, attr, depth));
  case kCompressFP16Blocks:
    return f(SparseField<Blocked<CodeFP16>>(g, attr, depth));
  case kCompressBF16Blocks:
    return f(SparseField<Blocked<CodeBF16>>(g, attr, depth));
  case kCompressFP8Blocks:
    return f(SparseField<Blocked<CodeE4M3>>(g, attr, depth));
  default:
    break;
  }
  if (t == kHalf)
    return f(SparseField<__half>(g, attr, depth));
  return f(SparseField<float>(g, attr, depth));
}

// A dense float attribute with a texture atlas samples its trilinear corners
// from it (AtlasField): the same bits as the bricked loads.
__device__ __forceinline__ bool atlasLinear(const DevGrid &g, int filter, uint32_t attr, VKLFeatureFlags ff,
                                            VKLFeatureFlags filterBit)
{
  return (ff & kStructuredRegular) && (ff & filterBit) && filter == kFilterLinear && g.dense &&
         g.atlasTex[attr] != 0;
}

__device__ __forceinline__ float sample(const DevGrid &g, int filter, uint32_t depth, uint32_t attr, f3 oc,
                                        VKLFeatureFlags ff, float time = 0.f)
{
  if (ff == 0)
    ff = ~0ull;
  const f3 p    = xfmPoint(g.objectToIndex, oc);
  if (atlasLinear(g, filter, attr, ff, kSampleLinear))
    return sampleLinear(AtlasField(g, attr), p);
  const bool cc = g.constantCellData != 0;
  return withField(
      g, attr, depth, ff,
      [&](const auto &F) -> float {
        if ((ff & kSampleNearest) && filter == kFilterNearest)
          return sampleNearest(F, cc, p);
        if ((ff & kSampleCubic) && filter == kFilterCubic)
          return sampleCubic(F, p);
        return sampleLinear(F, p);
      },
      time);
}

__device__ __forceinline__ f3 gradient(const DevSamplerState *st, uint32_t attr, f3 oc, VKLFeatureFlags ff,
                                       float time = 0.f)
{
  if (ff == 0)
    ff = ~0ull;
  const DevGrid &g = st->g;
  const int filter = st->s.gradientFilter;
  if ((ff & kGradientNearest) && filter == kFilterNearest)
    return {0.f, 0.f, 0.f};
  const f3 p = xfmPoint(g.objectToIndex, oc);
  if (atlasLinear(g, filter, attr, ff, kGradientLinear))
    return xfmNormal(g.objectToIndex, gradientLinear(AtlasField(g, attr), p));
  return withField(
      g, attr, st->s.maxSamplingDepth, ff,
      [&](const auto &F) -> f3 {
        const f3 gi =
            ((ff & kGradientCubic) && filter == kFilterCubic) ? gradientCubic(F, p) : gradientLinear(F, p);
        return xfmNormal(g.objectToIndex, gi);
      },
      time);
}

}  // namespace device_api
}  // namespace vklcuda

// Sample of one attribute at an object-space point (vklComputeSample).
__device__ inline float vklComputeSample(const VKLSampler *sampler, const vkl_vec3f *objectCoordinates,
                                         unsigned int attributeIndex, float time,
                                         const VKLFeatureFlags featureFlags)
{
  const auto *st = (const vklcuda::DevSamplerState *)sampler->device;
  return vklcuda::device_api::sample(st->g, st->s.filter, st->s.maxSamplingDepth, attributeIndex,
                                     vklcuda::device_api::toF3(objectCoordinates), featureFlags, time);
}

// Samples of M attributes (vklComputeSampleM).
__device__ inline void vklComputeSampleM(const VKLSampler *sampler, const vkl_vec3f *objectCoordinates,
                                         float *samples, unsigned int M, const unsigned int *attributeIndices,
                                         float time, const VKLFeatureFlags featureFlags)
{
  for (unsigned int m = 0; m < M; ++m)
    samples[m] = vklComputeSample(sampler, objectCoordinates, attributeIndices[m], time, featureFlags);
}

// Object-space gradient with the sampler's gradient filter (vklComputeGradient).
__device__ inline vkl_vec3f vklComputeGradient(const VKLSampler *sampler, const vkl_vec3f *objectCoordinates,
                                               unsigned int attributeIndex, float time,
                                               const VKLFeatureFlags featureFlags)
{
  const vklcuda::f3 r = vklcuda::device_api::gradient((const vklcuda::DevSamplerState *)sampler->device,
                                                      attributeIndex, vklcuda::device_api::toF3(objectCoordinates),
                                                      featureFlags, time);
  return vkl_vec3f{r.x, r.y, r.z};
}

// Interval iterator in a caller buffer of VKL_CUDA_INTERVAL_ITERATOR_SIZE
// bytes (8-byte aligned), e.g. a local array.
__device__ inline VKLIntervalIterator vklInitIntervalIterator(const VKLIntervalIteratorContext *context,
                                                              const vkl_vec3f *origin,
                                                              const vkl_vec3f *direction,
                                                              const vkl_range1f *tRange, float time,
                                                              void *buffer, const VKLFeatureFlags featureFlags)
{
  (void)time;
  (void)featureFlags;
  auto *s = (vklcuda::device_api::IntervalIteratorState *)buffer;
  s->ctx  = (const vklcuda::DevIntervalContextState *)context->device;
  vklcuda::intervalInit(s->ctx->sampler->g, s->ctx->depth, vklcuda::device_api::toF3(origin),
                        vklcuda::device_api::toF3(direction), tRange->lower, tRange->upper, s->it);
  return (VKLIntervalIterator)buffer;
}

__device__ inline int vklIterateInterval(VKLIntervalIterator iterator, VKLInterval *interval,
                                         const VKLFeatureFlags featureFlags)
{
  (void)featureFlags;
  auto *s = (vklcuda::device_api::IntervalIteratorState *)iterator;
  vklcuda::DevInterval iv;
  if (!vklcuda::intervalNext(s->ctx->sampler->g, s->ctx->attr, s->ctx->vr, s->it, iv))
    return 0;
  interval->tRange.lower     = iv.t0;
  interval->tRange.upper     = iv.t1;
  interval->valueRange.lower = iv.v0;
  interval->valueRange.upper = iv.v1;
  interval->nominalDeltaT    = iv.nominalDeltaT;
  return 1;
}

// Hit iterator in a caller buffer of VKL_CUDA_HIT_ITERATOR_SIZE bytes.
__device__ inline VKLHitIterator vklInitHitIterator(const VKLHitIteratorContext *context, const vkl_vec3f *origin,
                                                    const vkl_vec3f *direction, const vkl_range1f *tRange,
                                                    float time, void *buffer, const VKLFeatureFlags featureFlags)
{
  (void)featureFlags;
  auto *s = (vklcuda::device_api::HitIteratorState *)buffer;
  s->ctx  = (const vklcuda::DevHitContextState *)context->device;
  s->time = time;
  vklcuda::hitInit(s->ctx->sampler->g, s->ctx->depth, vklcuda::device_api::toF3(origin),
                   vklcuda::device_api::toF3(direction), tRange->lower, tRange->upper, s->h);
  return (VKLHitIterator)buffer;
}

__device__ inline int vklIterateHit(VKLHitIterator iterator, VKLHit *hit, const VKLFeatureFlags featureFlags)
{
  auto *s                   = (vklcuda::device_api::HitIteratorState *)iterator;
  const auto *c             = s->ctx;
  const vklcuda::DevGrid &g = c->sampler->g;
  vklcuda::DevHit h;
  (void)featureFlags;
  // the march samples through the generic sampler, out of line (one copy
  // for every sampling site of the march and bisection)
  if (!vklcuda::hitNext(g, c->sampler->s.filter, c->attr, vklcuda::kNumLevels - 1, c->vr, c->numValues,
                        c->values, s->h, h, s->time))
    return 0;
  hit->t       = h.t;
  hit->sample  = h.sample;
  hit->epsilon = h.epsilon;
  return 1;
}

#endif  // __CUDACC__
