// Ray-run tiles: sampling of point arrays laid out as runs of S consecutive
// samples per ray, the order a renderer passes the samples of many rays to
// vklComputeSampleN / vklComputeGradientN.
//
// Within such an array the samples with the same index on neighbouring rays
// lie close together, consecutive samples of one ray do not.  A CTA takes 8
// consecutive runs (8 * S points) and lane l of a warp computes run l % 8 at
// sample l / 8 (+ 4 per warp and per step), so a warp's 32 points are 4
// consecutive sample indices of 8 neighbouring rays and its texture gathers
// share cache lines.  This is the locality the spatially sorted tile kernel
// (kSampleTile) buys with a counting sort through shared memory; here the
// order is read off the layout, and shared memory only stages the runs:
//  - the 8 runs are copied into padded shared-memory rows by 8 bulk copies
//    (cp.async.bulk, completion on an mbarrier, bounded wait);
//  - the row pitch (3 S + 4 words) puts every lane's loads in distinct
//    banks;
//  - the results go straight to global memory.
// Each point is computed by the same code as in the other kernels, so the
// results do not depend on the order.  A detector (kDetectRuns) picks S from
// the points themselves: it counts, on a sample of warps, the distinct
// 16x16x2-voxel blocks the 32 points of a warp touch under each candidate S;
// the run kernel is used with the S whose warps touch fewest blocks, when
// that is at most 12 (points with no locality touch about 32).
#include <atomic>

#include "kernels.h"
#include "objects.h"
#include "sample_kernels.cuh"

namespace vklcuda {

namespace {

constexpr int kRunThreads = 256;
constexpr int kRuns       = 8;  // runs per tile
constexpr int kRunGroup   = 4;  // samples computed before their stores

__device__ __forceinline__ uint32_t smemAddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Waits for phase 0 of the mbarrier, at most 2^22 polls; false if it gave up.
__device__ __forceinline__ bool waitPhase0(uint64_t *bar)
{
  for (uint32_t it = 0; it < (1u << 22); ++it) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smemAddr(bar))
        : "memory");
    if (ok)
      return true;
  }
  return false;
}

template <int S>
struct RunSmem {
  static constexpr int kPtPitch = 3 * S + 4;  // words
  static constexpr size_t bytes = 16 + 4 * (size_t)kRuns * kPtPitch;
};

// At least 5 CTAs per SM (51 registers) for the texture-atlas field, whose
// gathers are latency bound, 4 otherwise.
template <class Field>
constexpr int runMinBlocks()
{
  return std::is_same<Field, AtlasField>::value ? 5 : 4;
}

template <class Field, int FILTER, bool GRAD, int S>
__global__ void __launch_bounds__(kRunThreads, runMinBlocks<Field>())
    kSampleRuns(const __grid_constant__ DevGrid g, uint32_t maxDepth, uint64_t n, const float *__restrict__ pts,
                uint32_t attr, float *__restrict__ out, uint32_t *__restrict__ error)
{
  using L            = RunSmem<S>;
  constexpr int TILE = kRuns * S;
  constexpr int PPT  = TILE / kRunThreads;
  extern __shared__ __align__(128) unsigned char smemRaw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smemRaw);
  float *rows   = reinterpret_cast<float *>(smemRaw + 16);
  const uint64_t base = (uint64_t)blockIdx.x * TILE;
  // whole tiles of 16-byte aligned point arrays go through the bulk copies
  const bool bulk = base + TILE <= n && (reinterpret_cast<uintptr_t>(pts) & 15) == 0;
  if (bulk && threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(TILE * 12)
                 : "memory");
#pragma unroll 1
    for (int r = 0; r < kRuns; ++r)
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smemAddr(rows + r * L::kPtPitch)),
          "l"(pts + 3 * (base + (uint64_t)r * S)), "r"(S * 12), "r"(smemAddr(bar))
          : "memory");
  }
  if (!bulk) {
    for (int k = threadIdx.x; k < TILE * 3; k += kRunThreads) {
      const int r = k / (3 * S), w = k - r * 3 * S;
      const uint64_t e = 3 * base + (uint64_t)k;
      rows[r * L::kPtPitch + w] = e < 3 * n ? __ldg(pts + e) : 0.f;
    }
  }
  __syncthreads();
  if (!__syncthreads_and(bulk ? waitPhase0(bar) : true)) {
    if (threadIdx.x == 0)
      atomicExch(error, 1u);
    return;
  }
  const bool cc = g.constantCellData != 0;
  const Field F = makeField<Field>(g, attr, maxDepth);
  // Results go straight to global memory: a warp's stores are 8 runs x 4
  // consecutive samples, 8 segments of 16 B (48 B for gradients).  Staging
  // them in shared memory between the samples (the rows share one array)
  // kept the compiler from overlapping consecutive samples' gathers: 7.85 vs
  // 3.57 ms on the 1024^3 coherent workload.  kRunGroup samples are computed
  // before their stores, so their gathers are in flight together; points
  // past the end of the array (zero rows of a partial tile) are computed
  // and not stored.
  constexpr int G = kRunGroup < PPT ? kRunGroup : PPT;
#pragma unroll
  for (int j0 = 0; j0 < PPT; j0 += G) {
    float res[G][GRAD ? 3 : 1];
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int k    = threadIdx.x + (j0 + u) * kRunThreads;
      const int r    = k & (kRuns - 1), s = k >> 3;
      const float *q = rows + r * L::kPtPitch + 3 * s;
      const f3 p     = xfmPoint(g.objectToIndex, f3{q[0], q[1], q[2]});
      if constexpr (GRAD) {
        f3 gr = {0.f, 0.f, 0.f};
        if constexpr (FILTER == kFilterCubic)
          gr = xfmNormal(g.objectToIndex, gradientCubic(F, p));
        else if constexpr (FILTER == kFilterLinear)
          gr = xfmNormal(g.objectToIndex, gradientLinear(F, p));
        res[u][0] = gr.x;
        res[u][GRAD ? 1 : 0] = gr.y;
        res[u][GRAD ? 2 : 0] = gr.z;
      } else {
        res[u][0] = filterAt<Field, FILTER>(F, cc, p);
      }
    }
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int k      = threadIdx.x + (j0 + u) * kRunThreads;
      const int r      = k & (kRuns - 1), s = k >> 3;
      const uint64_t i = base + (uint64_t)r * S + s;
      if (i < n) {
        if constexpr (GRAD) {
          __stcs(out + 3 * i, res[u][0]);
          __stcs(out + 3 * i + 1, res[u][GRAD ? 1 : 0]);
          __stcs(out + 3 * i + 2, res[u][GRAD ? 2 : 0]);
        } else {
          __stcs(out + i, res[u][0]);
        }
      }
    }
  }
}

// Candidates: 0 = the plain order, then S = 64, 128, 256, 512.
constexpr int kCandidates        = 5;
constexpr int kCandidateS[kCandidates] = {0, 64, 128, 256, 512};
constexpr int kDetectBlocks      = 64;

// Each block looks at one spot of the array; each warp counts the distinct
// 16x16x2 blocks of its 32 points under every candidate order.  out[c] sums
// the distinct counts, out[kCandidates + c] the warps counted.
__global__ void __launch_bounds__(256) kDetectRuns(const __grid_constant__ DevGrid g, uint64_t n,
                                                   const float *__restrict__ pts, uint32_t *__restrict__ out)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t span = (uint64_t)kRuns * 512;
  if (n < span)
    return;
  const uint64_t spot = (n - span) / kDetectBlocks * blockIdx.x;
#pragma unroll 1
  for (int c = 0; c < kCandidates; ++c) {
    const int S     = c == 0 ? 0 : (32 << c);  // kCandidateS[c]
    const uint64_t i = S == 0 ? spot + 32 * warp + lane : spot + (uint64_t)(lane & 7) * S + 4 * warp + (lane >> 3);
    const f3 p       = xfmPoint(g.objectToIndex, f3{__ldg(pts + 3 * i), __ldg(pts + 3 * i + 1), __ldg(pts + 3 * i + 2)});
    const uint32_t key  = tileKey<true>(p);
    const uint32_t same = __match_any_sync(0xffffffffu, key);
    const bool leader   = lane == __ffs(same) - 1;
    const uint32_t distinct = __popc(__ballot_sync(0xffffffffu, leader));
    if (lane == 0) {
      atomicAdd(out + c, distinct);
      atomicAdd(out + kCandidates + c, 1u);
    }
  }
}

template <class Field, int FILTER, bool GRAD, int S>
void launchRuns(const DevGrid &g, uint32_t maxDepth, uint64_t n, const float *pts, uint32_t attr, float *out,
                uint32_t *error, cudaStream_t st)
{
  constexpr size_t smem = RunSmem<S>::bytes;
  // the dynamic shared-memory limit is raised once per instantiation and
  // device (bit = device ordinal)
  static std::atomic<uint64_t> configured{0};
  int dev = 0;
  cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
  const uint64_t bit = 1ull << (dev & 63);
  if (!(configured.load() & bit)) {
    cudaCheck(cudaFuncSetAttribute(kSampleRuns<Field, FILTER, GRAD, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem),
              "ray-run kernel shared memory");
    configured.fetch_or(bit);
  }
  const uint64_t tile = (uint64_t)kRuns * S;
  kSampleRuns<Field, FILTER, GRAD, S>
      <<<(unsigned)((n + tile - 1) / tile), kRunThreads, smem, st>>>(g, maxDepth, n, pts, attr, out, error);
}

template <class Field, int FILTER, bool GRAD>
void launchRunsS(const DevGrid &g, uint32_t maxDepth, uint64_t n, const float *pts, uint32_t attr, float *out,
                 int S, uint32_t *error, cudaStream_t st)
{
  switch (S) {
  case 64:
    return launchRuns<Field, FILTER, GRAD, 64>(g, maxDepth, n, pts, attr, out, error, st);
  case 128:
    return launchRuns<Field, FILTER, GRAD, 128>(g, maxDepth, n, pts, attr, out, error, st);
  case 256:
    return launchRuns<Field, FILTER, GRAD, 256>(g, maxDepth, n, pts, attr, out, error, st);
  default:
    return launchRuns<Field, FILTER, GRAD, 512>(g, maxDepth, n, pts, attr, out, error, st);
  }
}

}  // namespace

bool rayRunsApply(const DevGrid &g, int filter, uint32_t attr)
{
  return g.dense && !g.temporal && filter == kFilterLinear && g.type[attr] == kFloat;
}

int detectRayRuns(const DevGrid &g, uint64_t n, const float *pts, RunScratch &scratch, cudaStream_t st)
{
  if (n < (uint64_t)kRuns * 512 * 4)
    return 0;
  if (!scratch.counts.ptr) {
    scratch.counts.alloc(4 * 2 * kCandidates + 4);
    cudaCheck(cudaMemsetAsync(scratch.counts.ptr, 0, 4 * 2 * kCandidates + 4, st), "ray-run scratch");
  }
  uint32_t *c = scratch.counts.as<uint32_t>();
  cudaCheck(cudaMemsetAsync(c, 0, 4 * 2 * kCandidates, st), "ray-run detection");
  kDetectRuns<<<kDetectBlocks, 256, 0, st>>>(g, n, pts, c);
  cudaCheck(cudaGetLastError(), "ray-run detection launch");
  uint32_t h[2 * kCandidates + 1];
  cudaCheck(cudaMemcpyAsync(h, c, sizeof(h), cudaMemcpyDeviceToHost, st), "ray-run detection readback");
  cudaCheck(cudaStreamSynchronize(st), "ray-run detection");
  if (h[2 * kCandidates]) {
    // a ray-run launch since the last detection gave up waiting for its
    // point copy (its CTAs returned without writing their results)
    cudaCheck(cudaMemsetAsync(c + 2 * kCandidates, 0, 4, st), "ray-run error reset");
    fail("a ray-run sampling launch timed out waiting for its point copy; its results are invalid",
         VKL_UNKNOWN_ERROR);
  }
  if (!h[kCandidates])
    return 0;
  int best        = 0;
  double bestMean = 1e9;
  for (int k = 1; k < kCandidates; ++k) {
    const double m = h[kCandidates + k] ? (double)h[k] / h[kCandidates + k] : 1e9;
    if (m < bestMean) {
      bestMean = m;
      best     = k;
    }
  }
  // warps whose 32 points touch at most 12 blocks (of 32 for points with no
  // locality, e.g. uniform random points): the run kernel has the locality
  // the sorted kernel would build, without the sort.  The plain order is
  // counted for the record (candidate 0) but not used: the sorted kernel is
  // the alternative.
  if (best && bestMean <= 12.0)
    return kCandidateS[best];
  return 0;
}

void launchSampleRays(const DevGrid &g, uint32_t maxDepth, uint64_t n, const float *pts, uint32_t attr, float *out,
                      bool grad, int S, RunScratch &scratch, cudaStream_t st)
{
  if (!n)
    return;
  if (!scratch.counts.ptr) {
    scratch.counts.alloc(4 * 2 * kCandidates + 4);
    cudaCheck(cudaMemsetAsync(scratch.counts.ptr, 0, 4 * 2 * kCandidates + 4, st), "ray-run scratch");
  }
  uint32_t *error = scratch.counts.as<uint32_t>() + 2 * kCandidates;
  if (g.atlasTex[attr]) {
    if (grad)
      launchRunsS<AtlasField, kFilterLinear, true>(g, maxDepth, n, pts, attr, out, S, error, st);
    else
      launchRunsS<AtlasField, kFilterLinear, false>(g, maxDepth, n, pts, attr, out, S, error, st);
  } else {
    if (grad)
      launchRunsS<DenseField<float>, kFilterLinear, true>(g, maxDepth, n, pts, attr, out, S, error, st);
    else
      launchRunsS<DenseField<float>, kFilterLinear, false>(g, maxDepth, n, pts, attr, out, S, error, st);
  }
  cudaCheck(cudaGetLastError(), "ray-run kernel launch");
}

}  // namespace vklcuda
