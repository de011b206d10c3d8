// Binned sampling of incoherent point sets on dense float volumes.
//
// A tile of 2048 uniformly random points over a volume far larger than L2
// shares no bricks, so every tap is an independent DRAM (and TLB) access and
// the sorted tile kernel runs at a few percent of HBM bandwidth.  For such
// inputs the points are first counting-sorted, device-wide, by the coarse
// cell of index space they fall in (a "bin": 64^3 voxels, or larger for big
// volumes so that there are at most kMaxBins bins); the tile kernel then
// runs over the points in bin order, where a bin's voxels stay in L2 while
// its points are sampled, and writes each result back to the point's
// original slot.  Each point is filtered by exactly the expressions of the
// unbinned path, so results are bit-identical; only the order of work
// changes.
//
// Whether a call is binned is decided per call by kBinDetect: a few spread
// out tiles of the input count their distinct brick keys; coherent inputs
// (samples along rays) hit few bricks per tile and run unbinned.
#include <algorithm>

#include "kernels.h"
#include "objects.h"
#include "sample_kernels.cuh"

namespace vklcuda {

namespace {

constexpr int kBinThreads      = 256;
constexpr int kBinPerThread    = 16;
constexpr int kBinCtaPoints    = kBinThreads * kBinPerThread;  // 4096 points per counting / scattering CTA
constexpr uint32_t kMaxBins    = 4096;                         // + 1 for points outside the domain
constexpr int kDetectTiles     = 64;
constexpr int kDetectTile      = 2048;
constexpr uint64_t kBinChunk   = uint64_t(1) << 27;  // points per binning pass (2 GiB of entries)
constexpr uint64_t kBinMinPts  = uint64_t(1) << 24;  // smaller calls are never binned
constexpr uint64_t kBinMinVoxelBytes = uint64_t(256) << 20;  // nor volumes that L2 mostly holds

struct BinGrid {
  uint32_t shift;       // bin edge = 2^shift voxels
  uint32_t nx, ny;      // bins per axis (x, y)
  uint32_t inside;      // bins covering the domain; bin `inside` holds the rest
};

__device__ __forceinline__ uint32_t binOf(const DevGrid &g, const BinGrid &B, f3 p)
{
  // only the grouping depends on this, so the one-instruction floor is used
  const uint32_t ox = (uint32_t)(__float2int_rd(p.x) - g.rootOrigin[0]);
  const uint32_t oy = (uint32_t)(__float2int_rd(p.y) - g.rootOrigin[1]);
  const uint32_t oz = (uint32_t)(__float2int_rd(p.z) - g.rootOrigin[2]);
  if (ox >= g.activeSize[0] || oy >= g.activeSize[1] || oz >= g.activeSize[2])
    return B.inside;
  return ((oz >> B.shift) * B.ny + (oy >> B.shift)) * B.nx + (ox >> B.shift);
}

__device__ __forceinline__ f3 loadPt(const float *__restrict__ pts, uint64_t i)
{
  return {__ldg(pts + 3 * i), __ldg(pts + 3 * i + 1), __ldg(pts + 3 * i + 2)};
}

// counts[0] += distinct brick keys, counts[1] += points, over kDetectTiles
// tiles spread evenly over the input.
__global__ void __launch_bounds__(kTileThreads) kBinDetect(const __grid_constant__ DevGrid g, uint64_t n,
                                                           const float *__restrict__ pts,
                                                           unsigned long long *counts)
{
  __shared__ int hist[kSortBins];
  __shared__ int distinct;
  for (int k = threadIdx.x; k < kSortBins; k += kTileThreads)
    hist[k] = 0;
  if (threadIdx.x == 0)
    distinct = 0;
  __syncthreads();
  const uint64_t start = (n / kDetectTiles) * blockIdx.x;
  const int cnt        = (int)min((uint64_t)kDetectTile, n - start);
  for (int k = threadIdx.x; k < cnt; k += kTileThreads)
    atomicAdd(&hist[tileKey(xfmPoint(g.objectToIndex, loadPt(pts, start + k)))], 1);
  __syncthreads();
  int mine = 0;
  for (int k = threadIdx.x; k < kSortBins; k += kTileThreads)
    mine += hist[k] != 0;
  atomicAdd(&distinct, mine);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(counts, (unsigned long long)distinct);
    atomicAdd(counts + 1, (unsigned long long)cnt);
  }
}

// Global bin histogram of points [0, n).
__global__ void __launch_bounds__(kBinThreads) kBinCount(const __grid_constant__ DevGrid g, BinGrid B, uint64_t n,
                                                         const float *__restrict__ pts, uint32_t *gHist)
{
  __shared__ uint32_t hist[kMaxBins + 1];
  for (uint32_t b = threadIdx.x; b <= B.inside; b += kBinThreads)
    hist[b] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kBinCtaPoints;
  const uint64_t end  = min(base + kBinCtaPoints, n);
  for (uint64_t k = base + threadIdx.x; k < end; k += kBinThreads)
    atomicAdd(&hist[binOf(g, B, xfmPoint(g.objectToIndex, loadPt(pts, k)))], 1u);
  __syncthreads();
  for (uint32_t b = threadIdx.x; b <= B.inside; b += kBinThreads)
    if (hist[b])
      atomicAdd(gHist + b, hist[b]);
}

// Exclusive scan of the bin histogram into the bins' write cursors (one CTA).
__global__ void __launch_bounds__(1024) kBinScan(const uint32_t *gHist, uint32_t numBins, uint32_t *gCursor)
{
  constexpr int kPer = (kMaxBins + 1 + 1023) / 1024;
  __shared__ uint32_t warpSum[32];
  uint32_t v[kPer], sum = 0;
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const uint32_t b = threadIdx.x * kPer + i;
    v[i]             = b < numBins ? gHist[b] : 0u;
    sum += v[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o)
      incl += t;
  }
  if (lane == 31)
    warpSum[warp] = incl;
  __syncthreads();
  uint32_t before = incl - sum;
  for (int w = 0; w < warp; ++w)
    before += warpSum[w];
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const uint32_t b = threadIdx.x * kPer + i;
    if (b < numBins)
      gCursor[b] = before;
    before += v[i];
  }
}

// Scatter: entry = (index-space point, position in the chunk) at its bin's
// next free slots.  Each CTA ranks its points per bin in shared memory
// (ranks kept in registers), reserves one contiguous range per bin with one
// global atomic, and writes each entry at range start + rank.
__global__ void __launch_bounds__(kBinThreads) kBinScatter(const __grid_constant__ DevGrid g, BinGrid B,
                                                           uint64_t n, const float *__restrict__ pts,
                                                           uint32_t *gCursor, float4 *__restrict__ binned)
{
  __shared__ uint32_t hist[kMaxBins + 1];
  for (uint32_t b = threadIdx.x; b <= B.inside; b += kBinThreads)
    hist[b] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kBinCtaPoints;
  uint32_t slot[kBinPerThread];  // bin | rank within this CTA's share of the bin << 13
#pragma unroll
  for (int j = 0; j < kBinPerThread; ++j) {
    const uint64_t k = base + threadIdx.x + (uint64_t)j * kBinThreads;
    if (k < n) {
      const uint32_t b = binOf(g, B, xfmPoint(g.objectToIndex, loadPt(pts, k)));
      slot[j]          = b | (atomicAdd(&hist[b], 1u) << 13);
    }
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b <= B.inside; b += kBinThreads)
    if (hist[b])
      hist[b] = atomicAdd(gCursor + b, hist[b]);
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kBinPerThread; ++j) {
    const uint64_t k = base + threadIdx.x + (uint64_t)j * kBinThreads;
    if (k < n) {
      const f3 p       = xfmPoint(g.objectToIndex, loadPt(pts, k));
      const uint32_t b = slot[j] & 0x1fffu;
      binned[hist[b] + (slot[j] >> 13)] = make_float4(p.x, p.y, p.z, __uint_as_float((uint32_t)k));
    }
  }
}

// The sorted tile kernel over binned entries: the entries are already in
// index space; each result goes to the entry's slot in the chunk's output.
template <int FILTER, bool GRAD, int TILE>
__global__ void __launch_bounds__(kTileThreads) kSampleBinned(const __grid_constant__ DevGrid g, uint32_t attr,
                                                              uint64_t n, const float4 *__restrict__ binned,
                                                              float *__restrict__ out)
{
  constexpr int PPT = TILE / kTileThreads;
  __shared__ __align__(16) float4 spt[TILE];
  __shared__ __align__(16) int hist[kSortBins];
  const uint64_t base = (uint64_t)blockIdx.x * TILE;
  const int cnt       = (int)min((uint64_t)TILE, n - base);
  for (int k = threadIdx.x; k < kSortBins; k += kTileThreads)
    hist[k] = 0;
  __syncthreads();
  float4 e[PPT];
  uint32_t slot[PPT];
#pragma unroll
  for (int j = 0; j < PPT; ++j) {
    const int k = threadIdx.x + j * kTileThreads;
    if (k < cnt) {
      e[j]             = __ldcs(binned + base + k);
      const uint32_t b = tileKey(f3{e[j].x, e[j].y, e[j].z});
      slot[j]          = b | ((uint32_t)atomicAdd(&hist[b], 1) << 10);
    }
  }
  __syncthreads();
  tileScan(hist);
  __syncthreads();
#pragma unroll
  for (int j = 0; j < PPT; ++j) {
    const int k = threadIdx.x + j * kTileThreads;
    if (k < cnt)
      spt[hist[slot[j] & (kSortBins - 1)] + (int)(slot[j] >> 10)] = e[j];
  }
  __syncthreads();
  const bool cc = g.constantCellData != 0;
  const DenseField<float> F(g, attr);
  auto compute = [&](int j) {
    const int k = threadIdx.x + j * kTileThreads;
    if (k < cnt) {
      const float4 v   = spt[k];
      const f3 q       = {v.x, v.y, v.z};
      const uint64_t o = __float_as_uint(v.w);
      if (GRAD) {
        f3 r = {0.f, 0.f, 0.f};
        if (FILTER != kFilterNearest) {
          const f3 gi = FILTER == kFilterCubic ? gradientCubic(F, q) : gradientLinear(F, q);
          r           = xfmNormal(g.objectToIndex, gi);
        }
        __stcs(out + 3 * o, r.x);
        __stcs(out + 3 * o + 1, r.y);
        __stcs(out + 3 * o + 2, r.z);
      } else {
        __stcs(out + o, filterAt<DenseField<float>, FILTER>(F, cc, q));
      }
    }
  };
  if constexpr (FILTER == kFilterCubic) {
#pragma unroll 1
    for (int j = 0; j < PPT; ++j)
      compute(j);
  } else {
#pragma unroll
    for (int j = 0; j < PPT; ++j)
      compute(j);
  }
}

template <int FILTER, bool GRAD>
void launchBinnedTiles(const DevGrid &g, uint32_t attr, uint64_t n, const float4 *binned, float *out,
                       cudaStream_t st)
{
  constexpr int TILE = (GRAD || FILTER == kFilterCubic) ? 1024 : 2048;
  kSampleBinned<FILTER, GRAD, TILE>
      <<<(unsigned)((n + TILE - 1) / TILE), kTileThreads, 0, st>>>(g, attr, n, binned, out);
}

BinGrid binGridOf(const DevGrid &g)
{
  BinGrid B{};
  for (B.shift = 6;; ++B.shift) {
    const uint64_t nx = (g.activeSize[0] + (1u << B.shift) - 1) >> B.shift;
    const uint64_t ny = (g.activeSize[1] + (1u << B.shift) - 1) >> B.shift;
    const uint64_t nz = (g.activeSize[2] + (1u << B.shift) - 1) >> B.shift;
    if (nx * ny * nz <= kMaxBins) {
      B.nx     = (uint32_t)nx;
      B.ny     = (uint32_t)ny;
      B.inside = (uint32_t)(nx * ny * nz);
      return B;
    }
  }
}

}  // namespace

bool binnedSamplingApplies(const DevGrid &g, int filter, uint64_t n, uint32_t attr)
{
  if (!g.dense || g.temporal || g.type[attr] != kFloat || n < kBinMinPts)
    return false;
  // trilinear taps from a texture atlas need no binning: the texture path
  // takes incoherent points faster unsorted (16.6 vs 13-14 Gsamples/s on
  // 2^26 random points of a 1024^3 volume)
  if (filter == kFilterLinear && g.atlasTex[attr])
    return false;
  const uint64_t voxels = (uint64_t)g.activeSize[0] * g.activeSize[1] * g.activeSize[2];
  return voxels * 4 >= kBinMinVoxelBytes;
}

bool launchSampleBinned(const DevGrid &g, int filter, uint64_t n, const float *pts, uint32_t attr,
                        float *out, bool grad, BinScratch &scratch, cudaStream_t st)
{
  // decide: mean distinct brick keys per detection tile
  scratch.counts.reserve(2 * sizeof(unsigned long long));
  cudaCheck(cudaMemsetAsync(scratch.counts.ptr, 0, 2 * sizeof(unsigned long long), st), "memset");
  kBinDetect<<<kDetectTiles, kTileThreads, 0, st>>>(g, n, pts, scratch.counts.as<unsigned long long>());
  cudaCheck(cudaGetLastError(), "bin detect launch");
  unsigned long long c[2] = {0, 0};
  cudaCheck(cudaMemcpyAsync(c, scratch.counts.ptr, sizeof(c), cudaMemcpyDeviceToHost, st), "bin detect");
  cudaCheck(cudaStreamSynchronize(st), "bin detect");
  if (c[1] == 0 || c[0] * 4 < c[1])  // fewer than one distinct brick per 4 points: coherent
    return false;

  const BinGrid B        = binGridOf(g);
  const uint32_t numBins = B.inside + 1;
  const uint64_t C       = std::min(n, kBinChunk);
  scratch.entries.reserve(C * sizeof(float4));
  scratch.bins.reserve(2 * (kMaxBins + 1) * sizeof(uint32_t));
  uint32_t *hist = scratch.bins.as<uint32_t>(), *cursor = hist + (kMaxBins + 1);
  for (uint64_t off = 0; off < n; off += C) {
    const uint64_t m    = std::min(C, n - off);
    const float *p      = pts + 3 * off;
    const unsigned ctas = (unsigned)((m + kBinCtaPoints - 1) / kBinCtaPoints);
    cudaCheck(cudaMemsetAsync(hist, 0, numBins * sizeof(uint32_t), st), "memset");
    kBinCount<<<ctas, kBinThreads, 0, st>>>(g, B, m, p, hist);
    kBinScan<<<1, 1024, 0, st>>>(hist, numBins, cursor);
    kBinScatter<<<ctas, kBinThreads, 0, st>>>(g, B, m, p, cursor, scratch.entries.as<float4>());
    cudaCheck(cudaGetLastError(), "bin launch");
    const float4 *e = scratch.entries.as<float4>();
    float *o        = out + (grad ? 3 : 1) * off;
    if (filter == kFilterNearest)
      grad ? launchBinnedTiles<kFilterNearest, true>(g, attr, m, e, o, st)
           : launchBinnedTiles<kFilterNearest, false>(g, attr, m, e, o, st);
    else if (filter == kFilterCubic)
      grad ? launchBinnedTiles<kFilterCubic, true>(g, attr, m, e, o, st)
           : launchBinnedTiles<kFilterCubic, false>(g, attr, m, e, o, st);
    else
      grad ? launchBinnedTiles<kFilterLinear, true>(g, attr, m, e, o, st)
           : launchBinnedTiles<kFilterLinear, false>(g, attr, m, e, o, st);
    cudaCheck(cudaGetLastError(), "binned sample launch");
  }
  return true;
}

}  // namespace vklcuda
