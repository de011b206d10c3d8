// Temporally varying (motion-blur) structuredRegular volumes: sampling at
// per-point times and the commit's leaf value ranges over all time samples.
//
// The reference takes a structuredRegular volume's data as
// temporallyStructuredNumTimesteps values per voxel, or as per-voxel index
// ranges (temporallyUnstructuredIndices) into the data and
// temporallyUnstructuredTimes (DenseVdbVolume.cpp:149-186, validated by
// common/temporal_data_verification.h).  A tap's value is the voxel's value
// interpolated at the sample's time (TemporalDenseField, sampling.cuh), so
// these volumes skip the bricked copy and the texture atlas and keep the
// data as given; every filter, gradient and the hit iterator run on the
// interpolated taps.  A leaf's value range covers every time sample of the
// voxels in its filter-support window (VdbSampler_dense.ih:107-266).
#include "kernels.h"
#include "objects.h"
#include "sample_kernels.cuh"

namespace vklcuda {

namespace {

constexpr int kTemporalBlock = 128;
constexpr float kInfF     = __builtin_huge_valf();

template <typename T, int FILTER, bool GRAD>
__global__ void __launch_bounds__(kTemporalBlock)
    kSampleTemporal(const __grid_constant__ DevGrid g, uint64_t n, const float *__restrict__ pts,
                    const float *__restrict__ times, uint32_t attr, float *__restrict__ out)
{
  const uint64_t i = (uint64_t)blockIdx.x * kTemporalBlock + threadIdx.x;
  if (i >= n)
    return;
  const f3 p = xfmPoint(g.objectToIndex, loadPoint(pts, i));
  const TemporalDenseField<T> F(g, attr, times ? __ldg(times + i) : 0.f);
  if constexpr (GRAD) {
    f3 r = {0.f, 0.f, 0.f};
    if constexpr (FILTER == kFilterCubic)
      r = xfmNormal(g.objectToIndex, gradientCubic(F, p));
    else if constexpr (FILTER == kFilterLinear)
      r = xfmNormal(g.objectToIndex, gradientLinear(F, p));
    out[3 * i]     = r.x;
    out[3 * i + 1] = r.y;
    out[3 * i + 2] = r.z;
  } else {
    out[i] = filterAt<TemporalDenseField<T>, FILTER>(F, g.constantCellData != 0, p);
  }
}

struct AttrList {
  uint32_t a[kMaxAttributes];
};

__global__ void __launch_bounds__(kTemporalBlock)
    kSampleTemporalM(const __grid_constant__ DevGrid g, int filter, uint64_t n, const float *__restrict__ pts,
                     const float *__restrict__ times, uint32_t M, AttrList attrs, float *__restrict__ out)
{
  const uint64_t i = (uint64_t)blockIdx.x * kTemporalBlock + threadIdx.x;
  if (i >= n)
    return;
  const f3 p     = xfmPoint(g.objectToIndex, loadPoint(pts, i));
  const float tm = times ? __ldg(times + i) : 0.f;
  for (uint32_t m = 0; m < M; ++m)
    out[i * M + m] = sampleIndexAny(g, filter, attrs.a[m], kNumLevels - 1, p, tm);
}

// One thread per leaf: the leaf's range over the 3x3x3 neighbourhood
// windows [7,8) | [0,8) | [0,2) (VdbSampler.ispc:460-557), every time sample
// of each voxel, folded in the reference's order (x outer, z inner, time
// innermost; an unstructured voxel's own range first, then box_extend);
// neighbours outside the domain contribute the background, and a window
// whose bound is NaN leaves the leaf's bound as it is.
template <typename T>
__global__ void __launch_bounds__(kTemporalBlock)
    kTemporalLeafRanges(const __grid_constant__ DevGrid g, uint32_t attr, uint3 nl, float *__restrict__ ranges)
{
  const uint64_t leaf = (uint64_t)blockIdx.x * kTemporalBlock + threadIdx.x;
  const uint64_t numLeaves = (uint64_t)nl.x * nl.y * nl.z;
  if (leaf >= numLeaves)
    return;
  const uint32_t lx = (uint32_t)(leaf % nl.x), ly = (uint32_t)((leaf / nl.x) % nl.y),
                 lz = (uint32_t)(leaf / ((uint64_t)nl.x * nl.y));
  const T *data = (const T *)g.data[attr];
  const uint32_t X = g.activeSize[0], Y = g.activeSize[1], Z = g.activeSize[2];
  const float bg = g.background[attr];
  const uint32_t win[3][2] = {{7, 8}, {0, 8}, {0, 2}};
  const TemporalDenseField<T> F(g, attr, 0.f);
  float lo = kInfF, hi = -kInfF;
  for (int ix = 0; ix < 3; ++ix)
    for (int iy = 0; iy < 3; ++iy)
      for (int iz = 0; iz < 3; ++iz) {
        // neighbour node origin in domain offsets (unsigned: -8 wraps and is
        // outside the domain)
        const uint32_t nx = lx * 8 + (uint32_t)(ix - 1) * 8u, ny = ly * 8 + (uint32_t)(iy - 1) * 8u,
                       nz = lz * 8 + (uint32_t)(iz - 1) * 8u;
        float wlo = kInfF, whi = -kInfF;
        if (!(nx < X && ny < Y && nz < Z)) {
          wlo = whi = bg;
        } else {
          for (uint32_t x = win[ix][0]; x < win[ix][1]; ++x)
            for (uint32_t y = win[iy][0]; y < win[iy][1]; ++y)
              for (uint32_t z = win[iz][0]; z < win[iz][1]; ++z) {
                const uint32_t ox = nx + x, oy = ny + y, oz = nz + z;
                if (!(ox < X && oy < Y && oz < Z))
                  continue;
                const uint64_t v = (uint64_t)ox + (uint64_t)X * ((uint64_t)oy + (uint64_t)Y * (uint64_t)oz);
                if (g.temporal == 1) {
                  for (uint32_t t = 0; t < g.numTimesteps; ++t) {
                    const float s = ldv(data, (uint64_t)g.numTimesteps * v + t);
                    wlo           = wlo < s ? wlo : s;
                    whi           = whi > s ? whi : s;
                  }
                } else {
                  float vlo = kInfF, vhi = -kInfF;
                  const uint64_t e = F.index(v + 1);
                  for (uint64_t k = F.index(v); k < e; ++k) {
                    const float s = ldv(data, k);
                    vlo           = vlo < s ? vlo : s;
                    vhi           = vhi > s ? vhi : s;
                  }
                  wlo = wlo < vlo ? wlo : vlo;
                  whi = whi > vhi ? whi : vhi;
                }
              }
        }
        if (!isnan(wlo))
          lo = lo < wlo ? lo : wlo;
        if (!isnan(whi))
          hi = hi > whi ? hi : whi;
      }
  ranges[2 * leaf]     = lo;
  ranges[2 * leaf + 1] = hi;
}

template <typename T>
void sampleTyped(const DevGrid &g, int filter, uint64_t n, const float *pts, const float *times, uint32_t attr,
                 float *out, bool grad, cudaStream_t st)
{
  const unsigned blocks = (unsigned)((n + kTemporalBlock - 1) / kTemporalBlock);
  if (filter == kFilterNearest) {
    if (grad)
      kSampleTemporal<T, kFilterNearest, true><<<blocks, kTemporalBlock, 0, st>>>(g, n, pts, times, attr, out);
    else
      kSampleTemporal<T, kFilterNearest, false><<<blocks, kTemporalBlock, 0, st>>>(g, n, pts, times, attr, out);
  } else if (filter == kFilterCubic) {
    if (grad)
      kSampleTemporal<T, kFilterCubic, true><<<blocks, kTemporalBlock, 0, st>>>(g, n, pts, times, attr, out);
    else
      kSampleTemporal<T, kFilterCubic, false><<<blocks, kTemporalBlock, 0, st>>>(g, n, pts, times, attr, out);
  } else {
    if (grad)
      kSampleTemporal<T, kFilterLinear, true><<<blocks, kTemporalBlock, 0, st>>>(g, n, pts, times, attr, out);
    else
      kSampleTemporal<T, kFilterLinear, false><<<blocks, kTemporalBlock, 0, st>>>(g, n, pts, times, attr, out);
  }
}

}  // namespace

void launchSampleTemporal(const DevGrid &g, int filter, uint64_t n, const float *points, const float *times,
                          uint32_t M, const uint32_t *attrs, float *out, bool grad, cudaStream_t st)
{
  if (!n)
    return;
  if (M > 1) {
    AttrList al{};
    for (uint32_t m = 0; m < M; ++m)
      al.a[m] = attrs[m];
    kSampleTemporalM<<<(unsigned)((n + kTemporalBlock - 1) / kTemporalBlock), kTemporalBlock, 0, st>>>(
        g, filter, n, points, times, M, al, out);
  } else {
    const uint32_t attr = attrs[0];
    switch (g.type[attr]) {
    case kUChar:
      sampleTyped<uint8_t>(g, filter, n, points, times, attr, out, grad, st);
      break;
    case kShort:
      sampleTyped<int16_t>(g, filter, n, points, times, attr, out, grad, st);
      break;
    case kUShort:
      sampleTyped<uint16_t>(g, filter, n, points, times, attr, out, grad, st);
      break;
    case kHalf:
      sampleTyped<__half>(g, filter, n, points, times, attr, out, grad, st);
      break;
    case kDouble:
      sampleTyped<double>(g, filter, n, points, times, attr, out, grad, st);
      break;
    default:
      sampleTyped<float>(g, filter, n, points, times, attr, out, grad, st);
    }
  }
  cudaCheck(cudaGetLastError(), "temporal sample kernel launch");
}

void launchTemporalLeafRanges(const DevGrid &g, uint32_t attr, const uint32_t nl[3], float *leafRanges,
                              cudaStream_t st)
{
  const uint3 n         = make_uint3(nl[0], nl[1], nl[2]);
  const uint64_t leaves = (uint64_t)nl[0] * nl[1] * nl[2];
  const unsigned blocks = (unsigned)((leaves + kTemporalBlock - 1) / kTemporalBlock);
  switch (g.type[attr]) {
  case kUChar:
    kTemporalLeafRanges<uint8_t><<<blocks, kTemporalBlock, 0, st>>>(g, attr, n, leafRanges);
    break;
  case kShort:
    kTemporalLeafRanges<int16_t><<<blocks, kTemporalBlock, 0, st>>>(g, attr, n, leafRanges);
    break;
  case kUShort:
    kTemporalLeafRanges<uint16_t><<<blocks, kTemporalBlock, 0, st>>>(g, attr, n, leafRanges);
    break;
  case kHalf:
    kTemporalLeafRanges<__half><<<blocks, kTemporalBlock, 0, st>>>(g, attr, n, leafRanges);
    break;
  case kDouble:
    kTemporalLeafRanges<double><<<blocks, kTemporalBlock, 0, st>>>(g, attr, n, leafRanges);
    break;
  default:
    kTemporalLeafRanges<float><<<blocks, kTemporalBlock, 0, st>>>(g, attr, n, leafRanges);
  }
  cudaCheck(cudaGetLastError(), "temporal leaf range kernel launch");
}

}  // namespace vklcuda
