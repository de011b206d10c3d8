// Sampling entry points of the cuda device: filter dispatch to the
// per-filter instantiations and the multi-attribute kernel
// (vklComputeSampleMN, VdbSampler.ispc:131-252).
#include "sample_kernels.cuh"

namespace vklcuda {

namespace {

struct AttrList {
  uint32_t a[kMaxAttributes];
};

__global__ void __launch_bounds__(kBlock) kSampleM(const __grid_constant__ DevGrid g, int filter,
                                                   uint32_t maxDepth, uint64_t n,
                                                   const float *__restrict__ pts, uint32_t M,
                                                   AttrList attrs, float *__restrict__ out)
{
  const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
  if (i >= n)
    return;
  const f3 p = xfmPoint(g.objectToIndex, loadPoint(pts, i));
  for (uint32_t m = 0; m < M; ++m)
    out[i * M + m] = sampleIndexAny(g, filter, attrs.a[m], maxDepth, p);
}

void dispatch(const DevGrid &g, int filter, uint32_t maxDepth, uint64_t n, const float *pts,
              uint32_t attr, float *out, bool grad, cudaStream_t st)
{
  if (n == 0)
    return;
  if (filter == kFilterNearest)
    dispatchFilter<kFilterNearest>(g, maxDepth, n, pts, attr, out, grad, st);
  else if (filter == kFilterCubic)
    dispatchFilter<kFilterCubic>(g, maxDepth, n, pts, attr, out, grad, st);
  else
    dispatchFilter<kFilterLinear>(g, maxDepth, n, pts, attr, out, grad, st);
}

}  // namespace
void launchSample(const DevGrid &g, int filter, uint32_t maxDepth, uint64_t n,
                  const float *points, uint32_t M, const uint32_t *attrs, float *out,
                  cudaStream_t stream)
{
  if (g.temporal) {  // temporally varying data, sampled at time 0
    launchSampleTemporal(g, filter, n, points, nullptr, M, attrs, out, false, stream);
    return;
  }
  if (M == 1) {
    dispatch(g, filter, maxDepth, n, points, attrs[0], out, false, stream);
  } else if (n) {
    AttrList al{};
    for (uint32_t m = 0; m < M; ++m)
      al.a[m] = attrs[m];
    kSampleM<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, stream>>>(g, filter, maxDepth, n,
                                                                          points, M, al, out);
  }
  cudaCheck(cudaGetLastError(), "sample kernel launch");
}

void launchGradient(const DevGrid &g, int filter, uint32_t maxDepth, uint64_t n,
                    const float *points, uint32_t attr, float *out, cudaStream_t stream)
{
  if (g.temporal) {
    launchSampleTemporal(g, filter, n, points, nullptr, 1, &attr, out, true, stream);
    return;
  }
  dispatch(g, filter, maxDepth, n, points, attr, out, true, stream);
  cudaCheck(cudaGetLastError(), "gradient kernel launch");
}

}  // namespace vklcuda
