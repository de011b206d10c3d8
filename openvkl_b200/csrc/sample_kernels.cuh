// Sampling and gradient kernel templates of the cuda device: one thread per
// query point, field access and filter fixed at compile time per
// (dense | sparse) x voxel type x filter so the inner loop is straight-line
// loads and FP32 arithmetic (the reference's per-filter dispatch,
// VdbSampler.ispc:97-129 / :303-335, restated as template instantiation).
// Each filter is instantiated in its own translation unit (k_sample_*.cu).
#pragma once
#include <type_traits>

#include "kernels.h"
#include "objects.h"
#include "sampling.cuh"

namespace vklcuda {

constexpr int kBlock = 256;

__device__ __forceinline__ f3 loadPoint(const float *__restrict__ pts, uint64_t i)
{
  return {__ldg(pts + 3 * i), __ldg(pts + 3 * i + 1), __ldg(pts + 3 * i + 2)};
}

template <class Field, int FILTER>
__device__ __forceinline__ float filterAt(const Field &F, bool cc, f3 p)
{
  if constexpr (FILTER == kFilterNearest)
    return sampleNearest(F, cc, p);
  else if constexpr (FILTER == kFilterCubic)
    return sampleCubic(F, p);
  else
    return sampleLinear(F, p);
}

// ---------------------------------------------------------------------------
// Spatially sorted tiles.  A CTA takes TILE consecutive query points, moves
// them to index space, counting-sorts them in shared memory by a hash of
// their 8^3 brick, computes them in that order and writes the results back
// in the caller's order.  Consecutive points of a coherent batch (samples
// along a ray) are several voxels apart, so without the sort every lane of a
// warp gathers from a different cache line; after it, a warp's lanes share a
// few bricks.  Results are unchanged: each point is computed by the same
// code, only by a different thread.
// ---------------------------------------------------------------------------
constexpr int kTileThreads = 256;
constexpr int kSortBins    = 1024;

template <typename T>
__device__ __forceinline__ DenseField<T> makeFieldAs(const DevGrid &g, uint32_t a, uint32_t,
                                                     DenseField<T> *)
{
  return DenseField<T>(g, a);
}
template <typename T>
__device__ __forceinline__ SparseField<T> makeFieldAs(const DevGrid &g, uint32_t a, uint32_t depth,
                                                      SparseField<T> *)
{
  return SparseField<T>(g, a, depth);
}
__device__ __forceinline__ AtlasField makeFieldAs(const DevGrid &g, uint32_t a, uint32_t, AtlasField *)
{
  return AtlasField(g, a);
}
template <class Field>
__device__ __forceinline__ Field makeField(const DevGrid &g, uint32_t attr, uint32_t maxDepth)
{
  return makeFieldAs(g, attr, maxDepth, (Field *)nullptr);
}

// Sort key: hash of the point's 8^3 brick (bricked loads), or of its
// 16x16x2 block for the texture atlas, whose planes are stored side by
// side: grouping two planes and a wider x/y block gave 91.2 vs 87.6
// Gsamples/s on the coherent 1024^3 workload.  Only the grouping depends on
// it, so the single-instruction round-down conversion is used.
template <bool ATLAS = false>
__device__ __forceinline__ uint32_t tileKey(f3 p)
{
  constexpr uint32_t sxy = ATLAS ? 4 : 3, sz = ATLAS ? 1 : 3;
  const uint32_t bx = (uint32_t)__float2int_rd(p.x) >> sxy, by = (uint32_t)__float2int_rd(p.y) >> sxy,
                 bz = (uint32_t)__float2int_rd(p.z) >> sz;
  return ((bx * 73856093u) ^ (by * 19349663u) ^ (bz * 83492791u)) & (kSortBins - 1);
}

// Exclusive scan of a tile's kSortBins-bin histogram in place (all
// kTileThreads threads; 4 bins per thread, warp scans, then the warp totals).
__device__ __forceinline__ void tileScan(int *hist)
{
  static_assert(kSortBins == 4 * kTileThreads && kSortBins == 1024, "scan layout");
  __shared__ int warpSum[kTileThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int4 h   = reinterpret_cast<const int4 *>(hist)[threadIdx.x];
  const int tot  = h.x + h.y + h.z + h.w;
  int incl       = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o)
      incl += t;
  }
  if (lane == 31)
    warpSum[warp] = incl;
  __syncthreads();
  int before = incl - tot;
  for (int w = 0; w < warp; ++w)
    before += warpSum[w];
  reinterpret_cast<int4 *>(hist)[threadIdx.x] =
      make_int4(before, before + h.x, before + h.x + h.y, before + h.x + h.y + h.z);
}

// The tricubic instances are held to two CTAs per SM (128 registers, a few
// spilled): the extra resident warps hide more of the 64-tap stencil's load
// latency than the spills cost (8.8 vs 8.2 Gsamples/s on the coherent
// 1024^3 workload).  The texture-atlas instances are held to four (64
// registers): they are bound by gather latency, and the fourth CTA gives
// 90.7 vs 84 Gsamples/s on the coherent workload (16.6 vs 17.5 on random
// points).  The sparse (VDB) instances are held to three (85 registers, no
// spills; 2 CTAs at 86-118 registers otherwise): on orbit-camera rays over
// the 4096^3 shells the compressed leaf forms gain 24-35 % (stencil blocks
// 13.7 -> 17.0 Gsamples/s), float leaves stay at 19.9-20.0, random
// interior points move by -3 % (float, stencil blocks) to +6 % (per-leaf
// codes).
// ATLAS: a dense float attribute's corners come from its texture atlas
// (AtlasField, trilinear only).
template <typename T, bool DENSE, int FILTER, bool GRAD, int TILE, bool ATLAS = false>
__global__ void __launch_bounds__(kTileThreads, FILTER == kFilterCubic ? 2 : (ATLAS ? 4 : (DENSE ? 1 : 3)))
    kSampleTile(const __grid_constant__ DevGrid g, uint32_t maxDepth, uint64_t n, const float *__restrict__ pts,
                uint32_t attr, float *__restrict__ out)
{
  constexpr int PPT  = TILE / kTileThreads;
  constexpr int OUTF = GRAD ? 3 : 1;
  // Before the sort these words hold the tile's points as the caller laid
  // them out (x, y, z per point); after it, spt[k] = the k-th point in
  // brick order (index space) with its position in the tile as w.
  __shared__ __align__(16) float4 spt[TILE];
  float *const sxyz = reinterpret_cast<float *>(spt);
  __shared__ float res[TILE * OUTF];
  __shared__ __align__(16) int hist[kSortBins];
  const uint64_t base = (uint64_t)blockIdx.x * TILE;
  const int cnt       = (int)min((uint64_t)TILE, n - base);
  for (int k = threadIdx.x; k < kSortBins; k += kTileThreads)
    hist[k] = 0;
  {
    // the tile's 12-byte points are one contiguous run: load it with 16-byte
    // loads when it is 16-byte aligned (whole tiles always are if pts is)
    const float *src = pts + 3 * base;
    const int nf     = 3 * cnt;
    int k0           = 0;
    if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
      const int n4 = nf >> 2;
      for (int k = threadIdx.x; k < n4; k += kTileThreads)
        reinterpret_cast<float4 *>(sxyz)[k] = __ldcs(reinterpret_cast<const float4 *>(src) + k);
      k0 = n4 << 2;
    }
    for (int k = k0 + threadIdx.x; k < nf; k += kTileThreads)
      sxyz[k] = __ldcs(src + k);
  }
  f3 p[PPT];
  uint32_t slot[PPT];  // bin (low 10 bits) | rank within the bin (high bits)
  __syncthreads();
#pragma unroll
  for (int j = 0; j < PPT; ++j) {
    const int k = threadIdx.x + j * kTileThreads;
    if (k < cnt) {
      p[j]             = xfmPoint(g.objectToIndex, f3{sxyz[3 * k], sxyz[3 * k + 1], sxyz[3 * k + 2]});
      const uint32_t b = tileKey<ATLAS>(p[j]);
      slot[j]          = b | ((uint32_t)atomicAdd(&hist[b], 1) << 10);
    }
  }
  // after this barrier no thread reads the raw points again, so the scatter
  // may overwrite them
  __syncthreads();
  tileScan(hist);
  __syncthreads();
#pragma unroll
  for (int j = 0; j < PPT; ++j) {
    const int k = threadIdx.x + j * kTileThreads;
    if (k < cnt) {
      const int pos = hist[slot[j] & (kSortBins - 1)] + (int)(slot[j] >> 10);
      spt[pos]      = make_float4(p[j].x, p[j].y, p[j].z, __int_as_float(k));
    }
  }
  __syncthreads();
  const bool cc = g.constantCellData != 0;
  // field parameters read from the launch's constant bank once per thread
  using Field = typename std::conditional<
      ATLAS, AtlasField, typename std::conditional<DENSE, DenseField<T>, SparseField<T>>::type>::type;
  const Field F = makeField<Field>(g, attr, maxDepth);
  auto compute = [&](int j) {
    const int k = threadIdx.x + j * kTileThreads;
    if (k < cnt) {
      const float4 e = spt[k];
      const f3 q     = {e.x, e.y, e.z};
      const int o    = __float_as_int(e.w);
      if (GRAD) {
        f3 r = {0.f, 0.f, 0.f};
        if constexpr (FILTER == kFilterCubic)
          r = xfmNormal(g.objectToIndex, gradientCubic(F, q));
        else if constexpr (FILTER == kFilterLinear)
          r = xfmNormal(g.objectToIndex, gradientLinear(F, q));
        res[3 * o]     = r.x;
        res[3 * o + 1] = r.y;
        res[3 * o + 2] = r.z;
      } else {
        res[o] = filterAt<Field, FILTER>(F, cc, q);
      }
    }
  };
  // Unrolled, the loads of all PPT points of a thread are in flight at once;
  // the 64-tap tricubic stays rolled to bound its register use.
  if constexpr (FILTER == kFilterCubic) {
#pragma unroll 1
    for (int j = 0; j < PPT; ++j)
      compute(j);
  } else {
#pragma unroll
    for (int j = 0; j < PPT; ++j)
      compute(j);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < cnt * OUTF; k += kTileThreads)
    __stcs(out + base * OUTF + k, res[k]);
}

template <typename T, bool DENSE, int FILTER>
void launchTyped(const DevGrid &g, uint32_t maxDepth, uint64_t n, const float *pts, uint32_t attr,
                 float *out, bool grad, cudaStream_t st)
{
  // 2048-point tiles for samples (44 KB shared), 1024 for gradients and the
  // register-heavy tricubic.
  if constexpr (DENSE && FILTER == kFilterLinear && std::is_same<T, float>::value) {
    if (g.atlasTex[attr]) {
      if (grad) {
        constexpr int TILE = 1024;
        kSampleTile<T, true, FILTER, true, TILE, true>
            <<<(unsigned)((n + TILE - 1) / TILE), kTileThreads, 0, st>>>(g, maxDepth, n, pts, attr, out);
      } else {
        constexpr int TILE = 2048;
        kSampleTile<T, true, FILTER, false, TILE, true>
            <<<(unsigned)((n + TILE - 1) / TILE), kTileThreads, 0, st>>>(g, maxDepth, n, pts, attr, out);
      }
      return;
    }
  }
  if (grad) {
    constexpr int TILE = 1024;
    kSampleTile<T, DENSE, FILTER, true, TILE>
        <<<(unsigned)((n + TILE - 1) / TILE), kTileThreads, 0, st>>>(g, maxDepth, n, pts, attr, out);
  } else if (FILTER == kFilterCubic) {
    constexpr int TILE = 1024;
    kSampleTile<T, DENSE, FILTER, false, TILE>
        <<<(unsigned)((n + TILE - 1) / TILE), kTileThreads, 0, st>>>(g, maxDepth, n, pts, attr, out);
  } else {
    constexpr int TILE = 2048;
    kSampleTile<T, DENSE, FILTER, false, TILE>
        <<<(unsigned)((n + TILE - 1) / TILE), kTileThreads, 0, st>>>(g, maxDepth, n, pts, attr, out);
  }
}

// Type dispatch for one filter (defined per filter in k_sample_<filter>.cu).
template <int FILTER>
void dispatchFilter(const DevGrid &g, uint32_t maxDepth, uint64_t n, const float *pts,
                    uint32_t attr, float *out, bool grad, cudaStream_t st)
{
  const uint32_t t = g.type[attr];
  if (g.dense) {
    switch (t) {
    case kUChar:
      return launchTyped<uint8_t, true, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
    case kShort:
      return launchTyped<int16_t, true, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
    case kUShort:
      return launchTyped<uint16_t, true, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
    case kHalf:
      return launchTyped<__half, true, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
    case kDouble:
      return launchTyped<double, true, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
    default:
      return launchTyped<float, true, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
    }
  }
  switch (g.compress) {
  case kCompressFP16:
    return launchTyped<CodeFP16, false, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
  case kCompressBF16:
    return launchTyped<CodeBF16, false, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
  case kCompressFP8:
    return launchTyped<CodeE4M3, false, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
  case kCompressFP16Blocks:
    return launchTyped<Blocked<CodeFP16>, false, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
  case kCompressBF16Blocks:
    return launchTyped<Blocked<CodeBF16>, false, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
  case kCompressFP8Blocks:
    return launchTyped<Blocked<CodeE4M3>, false, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
  default:
    break;
  }
  if (t == kHalf)
    return launchTyped<__half, false, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
  return launchTyped<float, false, FILTER>(g, maxDepth, n, pts, attr, out, grad, st);
}

extern template void dispatchFilter<kFilterNearest>(const DevGrid &, uint32_t, uint64_t,
                                                    const float *, uint32_t, float *, bool,
                                                    cudaStream_t);
extern template void dispatchFilter<kFilterLinear>(const DevGrid &, uint32_t, uint64_t,
                                                   const float *, uint32_t, float *, bool,
                                                   cudaStream_t);
extern template void dispatchFilter<kFilterCubic>(const DevGrid &, uint32_t, uint64_t,
                                                  const float *, uint32_t, float *, bool,
                                                  cudaStream_t);

}  // namespace vklcuda
