// Sampling and gradient kernel templates of the cuda device: one thread per
// query point, field access and filter fixed at compile time per
// (dense | sparse) x voxel type x filter so the inner loop is straight-line
// loads and FP32 arithmetic (the reference's per-filter dispatch,
// VdbSampler.ispc:97-129 / :303-335, restated as template instantiation).
// Each filter is instantiated in its own translation unit (k_sample_*.cu).
#pragma once
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
  if (FILTER == kFilterNearest)
    return sampleNearest(F, cc, p);
  if (FILTER == kFilterCubic)
    return sampleCubic(F, p);
  return sampleLinear(F, p);
}

template <typename T, bool DENSE, int FILTER>
__global__ void __launch_bounds__(kBlock) kSample(const __grid_constant__ DevGrid g,
                                                  uint32_t maxDepth, uint64_t n,
                                                  const float *__restrict__ pts, uint32_t attr,
                                                  float *__restrict__ out)
{
  const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
  if (i >= n)
    return;
  const f3 p = xfmPoint(g.objectToIndex, loadPoint(pts, i));
  float v;
  if (DENSE)
    v = filterAt<DenseField<T>, FILTER>(DenseField<T>(g, attr), g.constantCellData != 0, p);
  else
    v = filterAt<SparseField<T>, FILTER>(SparseField<T>(g, attr, maxDepth),
                                         g.constantCellData != 0, p);
  out[i] = v;
}

template <typename T, bool DENSE, int FILTER>
__global__ void __launch_bounds__(kBlock) kGradient(const __grid_constant__ DevGrid g,
                                                    uint32_t maxDepth, uint64_t n,
                                                    const float *__restrict__ pts,
                                                    uint32_t attr, float *__restrict__ out)
{
  const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
  if (i >= n)
    return;
  f3 r = {0.f, 0.f, 0.f};
  if (FILTER != kFilterNearest) {
    const f3 p = xfmPoint(g.objectToIndex, loadPoint(pts, i));
    f3 gi;
    if (DENSE) {
      DenseField<T> F(g, attr);
      gi = FILTER == kFilterCubic ? gradientCubic(F, p) : gradientLinear(F, p);
    } else {
      SparseField<T> F(g, attr, maxDepth);
      gi = FILTER == kFilterCubic ? gradientCubic(F, p) : gradientLinear(F, p);
    }
    r = xfmNormal(g.objectToIndex, gi);
  }
  out[3 * i]     = r.x;
  out[3 * i + 1] = r.y;
  out[3 * i + 2] = r.z;
}


template <typename T, bool DENSE, int FILTER>
void launchTyped(const DevGrid &g, uint32_t maxDepth, uint64_t n, const float *pts, uint32_t attr,
                 float *out, bool grad, cudaStream_t st)
{
  const dim3 grid((unsigned)((n + kBlock - 1) / kBlock));
  if (grad)
    kGradient<T, DENSE, FILTER><<<grid, kBlock, 0, st>>>(g, maxDepth, n, pts, attr, out);
  else
    kSample<T, DENSE, FILTER><<<grid, kBlock, 0, st>>>(g, maxDepth, n, pts, attr, out);
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
