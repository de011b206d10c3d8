// Iterator kernels of the cuda device.  Batched forms run one thread per
// ray through the whole DDA / hit loop; the per-call forms back the C API's
// stateful vklIterateInterval / vklIterateHit by advancing a state struct
// that lives in the caller's buffer by one step.
#include <algorithm>

#include "iterate.cuh"
#include "kernels.h"
#include "objects.h"

namespace vklcuda {

namespace {

constexpr int kBlock = 128;
// Resident blocks per SM asked of the compiler for the interval kernel,
// whose DDA state lives in registers (measured on the 1920x1080-ray
// workload): 4 x 128 threads (128 registers) ran fastest; 6 x 128 fits it in
// 80 registers but ran 10 % slower.
constexpr int kIntervalMinBlocks = 4;
// The specialised (persistent) hit kernels run fastest at 6 x 128 threads per
// SM (80 registers): 7.39 vs 6.86 Mrays/s at 5 (96 registers) on 2^24 random
// rays through the 4096^3 shell VDB.
constexpr int kHitMinBlocks = 6;

__device__ __forceinline__ f3 ld3(const float *p, uint64_t i)
{
  return {__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2)};
}

__global__ void __launch_bounds__(kBlock, kIntervalMinBlocks) kIntervals(const __grid_constant__ DevGrid g,
                                                     uint32_t attr, uint32_t depth,
                                                     DevValueRanges vr, uint64_t n,
                                                     const float *__restrict__ orgs,
                                                     const float *__restrict__ dirs,
                                                     const float *__restrict__ tr,
                                                     uint32_t maxPerRay,
                                                     DevInterval *__restrict__ out,
                                                     uint32_t *__restrict__ counts)
{
  const uint64_t r = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
  if (r >= n)
    return;
  IntervalIt it;
  intervalInit(g, depth, ld3(orgs, r), ld3(dirs, r), __ldg(tr + 2 * r), __ldg(tr + 2 * r + 1), it);
  uint32_t c = 0;
  DevInterval iv;
  while (intervalNext(g, attr, vr, it, iv)) {
    if (c < maxPerRay)
      out[r * maxPerRay + c] = iv;
    ++c;
  }
  counts[r] = c;
}

// Dense volumes: a cell's query never changes the DDA's path (the node
// level is always the query depth), so the steps can run ahead of the value
// range loads.  Each round records up to kIntervalLookahead steps (cell
// range address, t before and after the step, the budget), then loads their
// ranges together and applies intervalNext's tests to them in order: a
// non-empty cell whose t is not below tMax ends the ray, a spent budget ends
// it without emitting, a non-empty cell emits [t before, min(t after,
// tMax)].  Steps recorded past the end of a ray are dropped.  The intervals
// are those of intervalNext, in the same order.
constexpr int kIntervalLookahead = 8;

__global__ void __launch_bounds__(kBlock, kIntervalMinBlocks)
    kIntervalsDense(const __grid_constant__ DevGrid g, uint32_t attr, uint32_t depth, DevValueRanges vr, uint64_t n,
                    const float *__restrict__ orgs, const float *__restrict__ dirs, const float *__restrict__ tr,
                    uint32_t maxPerRay, DevInterval *__restrict__ out, uint32_t *__restrict__ counts)
{
  constexpr int K  = kIntervalLookahead;
  const uint64_t r = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
  if (r >= n)
    return;
  IntervalIt it;
  intervalInit(g, depth, ld3(orgs, r), ld3(dirs, r), __ldg(tr + 2 * r), __ldg(tr + 2 * r + 1), it);
  const float tMax = it.tMax;  // changes only when the ray ends
  uint32_t c = 0;
  bool live  = true;
  while (live) {
    const float *addr[K];
    float tb[K], ta[K];
    int nb = 0, budgetEnd = -1;
    bool topEnd = false;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (nb == j && budgetEnd < 0 && !topEnd) {
        if (!(it.dda.t <= tMax)) {
          topEnd = true;
        } else {
          const uint32_t L = it.dda.level;
          int32_t cx, cy, cz;
          ddaCell(it.dda, L, cx, cy, cz);
          addr[j] = denseCellRange(g, cx, cy, cz, L, attr);
          tb[j]   = it.dda.t;
          nb      = j + 1;
          if (it.budget-- == 0) {
            budgetEnd = j;
          } else {
            VoxelDesc d{};
            d.level = L;
            hddaStep(d, it.dda);
            ta[j] = it.dda.t;
          }
        }
      }
    }
    float v0[K], v1[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      v0[j] = v1[j] = 0.f;
      if (j < nb && addr[j]) {
        v0[j] = __ldg(addr[j]);
        v1[j] = __ldg(addr[j] + 1);
      }
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (live && j < nb) {
        const bool empty = !addr[j] || !rangesOverlap(vr, v0[j], v1[j]);
        if ((!empty && !(tb[j] < tMax)) || j == budgetEnd) {
          live = false;
        } else if (!empty) {
          if (c < maxPerRay)
            out[r * maxPerRay + c] = DevInterval{tb[j], minx(ta[j], tMax), v0[j], v1[j], it.nominalDeltaT};
          ++c;
        }
      }
    }
    if (topEnd)
      live = false;
  }
  counts[r] = c;
}

// The ray source of the persistent hit kernels: rays first, first + stride,
// ... below n, each with its slots out[r * maxPerRay ..] and count counts[r].
struct StridedRays {
  const DevGrid *g;
  uint32_t depth;
  uint64_t r, stride, n;
  const float *orgs, *dirs, *tr;
  DevHit *outBase;
  uint32_t maxPerRay;
  uint32_t *counts;
  bool started = false;

  __device__ __forceinline__ bool next(HitIt &h, DevHit *&out)
  {
    if (started)
      r += stride;
    started = true;
    if (r >= n)
      return false;
    hitInit(*g, depth, ld3(orgs, r), ld3(dirs, r), __ldg(tr + 2 * r), __ldg(tr + 2 * r + 1), h);
    out = outBase + r * maxPerRay;
    return true;
  }
  __device__ __forceinline__ void finish(uint32_t count) { counts[r] = count; }
};

// Field specialisations of the batched hit kernel: the generic one samples
// through the out-of-line type / filter dispatch; the float trilinear ones
// inline their field (far fewer registers, so more rays in flight per SM)
// and look LOOKAHEAD march steps ahead.  All give the same hits.
enum HitKind {
  kHitAny               = 0,
  kHitDenseFloatLinear  = 1,
  kHitSparseFloatLinear = 2,
  kHitSparseFP16Blocks  = 3,
  kHitSparseBF16Blocks  = 4,
  kHitSparseFP8Blocks   = 5,
  kHitSparseFP16        = 6,
  kHitSparseBF16        = 7,
  kHitSparseFP8         = 8,
};
constexpr int kHitLookahead = 1;

// Leaf codec of a sparse persistent hit kernel kind.
template <int KIND>
struct HitSparseCodec {
  using T = float;
};
template <>
struct HitSparseCodec<kHitSparseFP16Blocks> {
  using T = Blocked<CodeFP16>;
};
template <>
struct HitSparseCodec<kHitSparseBF16Blocks> {
  using T = Blocked<CodeBF16>;
};
template <>
struct HitSparseCodec<kHitSparseFP8Blocks> {
  using T = Blocked<CodeE4M3>;
};
template <>
struct HitSparseCodec<kHitSparseFP16> {
  using T = CodeFP16;
};
template <>
struct HitSparseCodec<kHitSparseBF16> {
  using T = CodeBF16;
};
template <>
struct HitSparseCodec<kHitSparseFP8> {
  using T = CodeE4M3;
};

template <int KIND, int LOOKAHEAD>
__global__ void __launch_bounds__(kBlock, KIND == kHitAny ? 1 : kHitMinBlocks) kHits(const __grid_constant__ DevGrid g, uint32_t attr,
                                                int filter, uint32_t depth, DevValueRanges vr,
                                                uint32_t numValues,
                                                const float *__restrict__ values, uint64_t n,
                                                const float *__restrict__ orgs,
                                                const float *__restrict__ dirs,
                                                const float *__restrict__ tr,
                                                uint32_t maxPerRay, DevHit *__restrict__ out,
                                                uint32_t *__restrict__ counts)
{
  const uint64_t r = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
  if constexpr (KIND == kHitAny) {
    if (r >= n)
      return;
    HitIt h;
    hitInit(g, depth, ld3(orgs, r), ld3(dirs, r), __ldg(tr + 2 * r), __ldg(tr + 2 * r + 1), h);
    uint32_t c = 0;
    DevHit hit;
    const AnySampleHook hook{&g, filter, attr, kNumLevels - 1};
    while (c < kMaxHitsPerRay && hitNextWith<LOOKAHEAD>(g, hook, attr, vr, numValues, values, h, hit)) {
      if (c < maxPerRay)
        out[r * maxPerRay + c] = hit;
      ++c;
    }
    counts[r] = c;
  } else {
    // Persistent: lane r takes rays r, r + stride, ... (stride = the grid's
    // threads) and starts the next as soon as one is done.  Every lane of
    // the warp stays in the state machine's warp-wide loop until all its
    // lanes are out of rays.
    StridedRays rays{&g, depth, r, (uint64_t)gridDim.x * kBlock, n, orgs, dirs, tr, out, maxPerRay, counts};
    if constexpr (KIND == kHitDenseFloatLinear)
      hitsAllLanes(g, LinearSampleHook<DenseField<float>>{&g, DenseField<float>(g, attr)}, attr, vr, numValues,
                   values, maxPerRay, rays);
    else {
      using SF = SparseField<typename HitSparseCodec<KIND>::T>;
      hitsAllLanes(g, LinearSampleHook<SF>{&g, SF(g, attr, kNumLevels - 1)}, attr, vr, numValues, values,
                   maxPerRay, rays);
    }
  }
}

struct IntervalIterStateImpl {
  uint32_t attr;
  IntervalIt it;
};
struct HitIterStateImpl {
  uint32_t attr;
  float time;
  HitIt h;
};

__global__ void kIntervalIterInit(const __grid_constant__ DevGrid g, uint32_t attr, uint32_t depth,
                                  const float *ray, IntervalIterStateImpl *s)
{
  s->attr = attr;
  intervalInit(g, depth, {ray[0], ray[1], ray[2]}, {ray[3], ray[4], ray[5]}, ray[6], ray[7], s->it);
}

__global__ void kIntervalIterNext(const __grid_constant__ DevGrid g, DevValueRanges vr,
                                  IntervalIterStateImpl *s, DevInterval *out, int *result)
{
  DevInterval iv;
  const bool ok = intervalNext(g, s->attr, vr, s->it, iv);
  if (ok)
    *out = iv;
  *result = ok ? 1 : 0;
}

__global__ void kHitIterInit(const __grid_constant__ DevGrid g, uint32_t attr, uint32_t depth,
                             const float *ray, HitIterStateImpl *s)
{
  s->attr = attr;
  s->time = ray[8];
  hitInit(g, depth, {ray[0], ray[1], ray[2]}, {ray[3], ray[4], ray[5]}, ray[6], ray[7], s->h);
}

__global__ void kHitIterNext(const __grid_constant__ DevGrid g, int filter, DevValueRanges vr,
                             uint32_t numValues, const float *values, HitIterStateImpl *s,
                             DevHit *out, int *result)
{
  DevHit hit;
  const bool ok = hitNext(g, filter, s->attr, kNumLevels - 1, vr, numValues, values, s->h, hit, s->time);
  if (ok)
    *out = hit;
  *result = ok ? 1 : 0;
}

inline unsigned blocksFor(uint64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

}  // namespace

void launchIntervals(const DevGrid &g, uint32_t attr, uint32_t depth, DevValueRanges vr,
                     uint64_t n, const float *origins, const float *directions,
                     const float *tRanges, uint32_t maxPerRay, DevInterval *out,
                     uint32_t *counts, cudaStream_t st)
{
  if (!n)
    return;
  if (g.dense)
    kIntervalsDense<<<blocksFor(n), kBlock, 0, st>>>(g, attr, depth, vr, n, origins, directions, tRanges,
                                                      maxPerRay, out, counts);
  else
    kIntervals<<<blocksFor(n), kBlock, 0, st>>>(g, attr, depth, vr, n, origins, directions, tRanges, maxPerRay,
                                                 out, counts);
  cudaCheck(cudaGetLastError(), "interval kernel launch");
}

void launchHits(const DevGrid &g, uint32_t attr, int filter, uint32_t depth, DevValueRanges vr,
                uint32_t numValues, const float *values, uint64_t n, const float *origins,
                const float *directions, const float *tRanges, uint32_t maxPerRay, DevHit *out,
                uint32_t *counts, cudaStream_t st)
{
  if (!n)
    return;
  const bool lin = filter == kFilterLinear && g.type[attr] == kFloat && !g.temporal;
  auto k         = kHits<kHitAny, 1>;
  unsigned grid  = blocksFor(n);
  if (lin) {
    if (g.dense)
      k = kHits<kHitDenseFloatLinear, kHitLookahead>;
    else if (g.compress == kCompressFP16Blocks)
      k = kHits<kHitSparseFP16Blocks, kHitLookahead>;
    else if (g.compress == kCompressBF16Blocks)
      k = kHits<kHitSparseBF16Blocks, kHitLookahead>;
    else if (g.compress == kCompressFP8Blocks)
      k = kHits<kHitSparseFP8Blocks, kHitLookahead>;
    else if (g.compress == kCompressFP16)
      k = kHits<kHitSparseFP16, kHitLookahead>;
    else if (g.compress == kCompressBF16)
      k = kHits<kHitSparseBF16, kHitLookahead>;
    else if (g.compress == kCompressFP8)
      k = kHits<kHitSparseFP8, kHitLookahead>;
    else
      k = kHits<kHitSparseFloatLinear, kHitLookahead>;
    // persistent: as many CTAs as are resident at once
    int dev = 0, sms = 0, perSM = 0;
    cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
    cudaCheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
    cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k, kBlock, 0), "occupancy");
    grid = (unsigned)std::min<uint64_t>(grid, (uint64_t)sms * (uint64_t)std::max(perSM, 1));
  }
  k<<<grid, kBlock, 0, st>>>(g, attr, filter, depth, vr, numValues, values, n, origins, directions, tRanges,
                             maxPerRay, out, counts);
  cudaCheck(cudaGetLastError(), "hit kernel launch");
}

size_t intervalIterStateSize() { return sizeof(IntervalIterStateImpl); }
size_t hitIterStateSize() { return sizeof(HitIterStateImpl); }

void launchIntervalIterInit(const DevGrid &g, uint32_t attr, uint32_t depth, const float *ray,
                            void *state, cudaStream_t st)
{
  kIntervalIterInit<<<1, 1, 0, st>>>(g, attr, depth, ray, (IntervalIterStateImpl *)state);
  cudaCheck(cudaGetLastError(), "interval iterator init");
}

void launchIntervalIterNext(const DevGrid &g, DevValueRanges vr, void *state, DevInterval *out,
                            int *result, cudaStream_t st)
{
  kIntervalIterNext<<<1, 1, 0, st>>>(g, vr, (IntervalIterStateImpl *)state, out, result);
  cudaCheck(cudaGetLastError(), "interval iterator step");
}

void launchHitIterInit(const DevGrid &g, uint32_t attr, uint32_t depth, const float *ray,
                       void *state, cudaStream_t st)
{
  kHitIterInit<<<1, 1, 0, st>>>(g, attr, depth, ray, (HitIterStateImpl *)state);
  cudaCheck(cudaGetLastError(), "hit iterator init");
}

void launchHitIterNext(const DevGrid &g, int filter, DevValueRanges vr, uint32_t numValues,
                       const float *values, void *state, DevHit *out, int *result,
                       cudaStream_t st)
{
  kHitIterNext<<<1, 1, 0, st>>>(g, filter, vr, numValues, values, (HitIterStateImpl *)state, out,
                                result);
  cudaCheck(cudaGetLastError(), "hit iterator step");
}

}  // namespace vklcuda
