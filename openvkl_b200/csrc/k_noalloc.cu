// vklCudaDenseValueRangeNoAlloc: the value range a structuredRegular volume
// over a caller's device voxel array would report, computed without
// allocating anything.
//
// Why this exists.  vklNewVolume + vklCommit allocate device memory (the
// bricked voxel copy, the tree, the range buffers), and cudaFree makes the
// whole device wait.  Some callers cannot take that: a renderer whose frame
// loop must not stall the device, an application whose memory pool already
// owns all free device memory, or a streaming simulation that rewrites its
// voxel buffer every step and only needs the range to place its transfer
// function before it commits anything.  This entry point gives them the
// commit path's range result (the filter-support window of every 8^3 leaf,
// plus the background where a window leaves the volume; see
// kDenseBrickRanges in k_build.cu) in one kernel launch on the device's stream,
// with its scratch in static device memory instead of an allocation.
//
// Scratch.  One file-scope __device__ array per device context, fixed size:
// one [lo, hi] partial per thread block, plus a completion counter.  A launch
// has at most kMaxBlocks blocks of kThreads threads, one thread per leaf, so
// at most kMaxLeaves leaves; larger volumes are rejected on the host before
// anything is launched.  The partials need no initial value (each block
// writes its own before the last block reads them); the counter must be zero
// when a launch starts: the set-up zeroes it once and the last block of every
// launch puts it back to zero.
//
// Set-up.  The first call on a device, with that device current, resolves
// the scratch address with cudaGetSymbolAddress, zeroes the counter, and
// forces the kernels to load; all of this may make the driver load this
// module's code and static memory, so the first call belongs before any
// stream capture or allocation-free region.  Later calls look the address up
// again (no allocation) and launch; a call whose launch fails makes the next
// call repeat the set-up, which re-arms the counter.
//
// Concurrency.  All calls on one device share the one scratch array: two calls
// whose launches overlap on the device (different streams, or threads)
// corrupt each other's partials and counter.  Callers serialize them, e.g. by
// issuing them on one stream.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "objects.h"
#include "sampling.cuh"

namespace vklcuda {

namespace {

constexpr unsigned kThreads   = 256;
constexpr unsigned kMaxBlocks = 65536;
constexpr uint64_t kMaxLeaves = (uint64_t)kMaxBlocks * kThreads;  // 16,777,216
constexpr int kMaxDevices     = 64;
constexpr float kInf          = __builtin_huge_valf();

struct RangeScratch {
  float partial[2 * kMaxBlocks];  // [lo, hi] per block of the current launch
  unsigned int blocksDone;        // must be 0 when a launch starts
};

// 512 KiB + 4 bytes per device context.
static __device__ __align__(256) RangeScratch g_rangeScratch;

__device__ __forceinline__ float fminx(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmaxx(float a, float b) { return a > b ? a : b; }

__device__ __forceinline__ void blockMinMax(float &lo, float &hi, float *slo, float *shi)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminx(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxx(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    slo[w] = lo;
    shi[w] = hi;
  }
  __syncthreads();
  if (w == 0) {
    lo = l < (int)(kThreads / 32) ? slo[l] : kInf;
    hi = l < (int)(kThreads / 32) ? shi[l] : -kInf;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fminx(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmaxx(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
  }
}

// One thread per leaf: the leaf's range over its window of the x-fastest
// voxel array (same window and background rule as the commit path's
// kDenseBrickRanges), reduced per block into the scratch partials; the block
// that finishes last reduces the partials into out[0..1] and re-arms the
// counter.
template <typename T>
__global__ void __launch_bounds__(kThreads)
    kDenseRangeNoAlloc(const T *__restrict__ data, int3 dims, uint3 nl, float bg,
                       RangeScratch *__restrict__ s, float *__restrict__ out)
{
  __shared__ float slo[kThreads / 32], shi[kThreads / 32];
  __shared__ bool last;
  const uint64_t numLeaves = (uint64_t)nl.x * nl.y * nl.z;
  const uint64_t leaf      = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  float lo = kInf, hi = -kInf;
  if (leaf < numLeaves) {
    const uint32_t lx = (uint32_t)(leaf % nl.x), ly = (uint32_t)((leaf / nl.x) % nl.y),
                   lz = (uint32_t)(leaf / ((uint64_t)nl.x * nl.y));
    const int32_t X = dims.x, Y = dims.y, Z = dims.z;
    const int32_t ox = (int32_t)lx * 8, oy = (int32_t)ly * 8, oz = (int32_t)lz * 8;
    const int32_t x0 = max(ox - 1, 0), x1 = min(ox + 10, X);
    const int32_t y0 = max(oy - 1, 0), y1 = min(oy + 10, Y);
    const int32_t z0 = max(oz - 1, 0), z1 = min(oz + 10, Z);
    for (int32_t z = z0; z < z1; ++z)
      for (int32_t y = y0; y < y1; ++y) {
        const uint64_t row = ((uint64_t)z * (uint64_t)Y + (uint64_t)y) * (uint64_t)X;
        for (int32_t x = x0; x < x1; ++x) {
          const float v = ldv(data, row + (uint64_t)x);
          lo            = fminx(lo, v);
          hi            = fmaxx(hi, v);
        }
      }
    const bool boundary = ox - 8 < 0 || oy - 8 < 0 || oz - 8 < 0 || ox + 8 >= X || oy + 8 >= Y ||
                          oz + 8 >= Z;
    if (boundary && !isnan(bg)) {
      lo = fminx(lo, bg);
      hi = fmaxx(hi, bg);
    }
  }
  blockMinMax(lo, hi, slo, shi);
  if (threadIdx.x == 0) {
    s->partial[2 * blockIdx.x]     = lo;
    s->partial[2 * blockIdx.x + 1] = hi;
    __threadfence();
    last = atomicAdd(&s->blocksDone, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last)
    return;
  __threadfence();
  lo = kInf;
  hi = -kInf;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += kThreads) {
    lo = fminx(lo, __ldcg(&s->partial[2 * b]));
    hi = fmaxx(hi, __ldcg(&s->partial[2 * b + 1]));
  }
  __syncthreads();  // slo/shi are reused
  blockMinMax(lo, hi, slo, shi);
  if (threadIdx.x == 0) {
    out[0]        = lo;
    out[1]        = hi;
    s->blocksDone = 0;
  }
}

// ---------------------------------------------------------------------------
// Per-device set-up.  The scratch address is looked up on every call (a table
// lookup once the module is loaded, no allocation) and compared with the one
// the set-up was done for: a new context (after cudaDeviceReset, say) gets a
// new address and so a new set-up.  A call whose launch reports an error
// clears the cached address too, so the next call re-arms the counter: an
// aborted launch may have left it counting.
// ---------------------------------------------------------------------------
std::mutex g_setupMutex;
RangeScratch *g_scratch[kMaxDevices] = {};

template <typename T>
void loadKernel()
{
  cudaFuncAttributes attr;
  cudaCheck(cudaFuncGetAttributes(&attr, kDenseRangeNoAlloc<T>), "vklCudaDenseValueRangeNoAlloc set-up");
}

// The calling thread's current device must be `dev`.
RangeScratch *scratchFor(int dev)
{
  if (dev < 0 || dev >= kMaxDevices)
    fail("vklCudaDenseValueRangeNoAlloc: CUDA device ordinal " + std::to_string(dev) +
             " out of range",
         VKL_INVALID_ARGUMENT);
  std::lock_guard<std::mutex> lock(g_setupMutex);
  RangeScratch *p = nullptr;
  cudaCheck(cudaGetSymbolAddress((void **)&p, g_rangeScratch),
            "vklCudaDenseValueRangeNoAlloc set-up: scratch symbol");
  if (g_scratch[dev] == p)
    return p;
  g_scratch[dev] = nullptr;
  cudaCheck(cudaMemset(&p->blocksDone, 0, sizeof(unsigned int)),
            "vklCudaDenseValueRangeNoAlloc set-up: counter");
  cudaCheck(cudaDeviceSynchronize(), "vklCudaDenseValueRangeNoAlloc set-up");
  loadKernel<uint8_t>();
  loadKernel<int16_t>();
  loadKernel<uint16_t>();
  loadKernel<__half>();
  loadKernel<float>();
  loadKernel<double>();
  g_scratch[dev] = p;
  return p;
}

// After a failed launch: the next call runs the set-up again.
void forgetScratch(int dev)
{
  std::lock_guard<std::mutex> lock(g_setupMutex);
  if (dev >= 0 && dev < kMaxDevices)
    g_scratch[dev] = nullptr;
}

template <typename T>
void launch(const void *voxels, int3 dims, uint3 nl, unsigned blocks, float bg, RangeScratch *s,
            float *out, cudaStream_t st)
{
  kDenseRangeNoAlloc<T><<<blocks, kThreads, 0, st>>>((const T *)voxels, dims, nl, bg, s, out);
}

}  // namespace

}  // namespace vklcuda

using namespace vklcuda;

extern "C" OPENVKL_CUDA_INTERFACE VKLError vklCudaDenseValueRangeNoAlloc(
    VKLDevice device, const void *voxels, VKLDataType voxelType, int dimX, int dimY, int dimZ,
    float background, float *valueRange)
{
  if (!device)
    return VKL_INVALID_ARGUMENT;
  Device *d = (Device *)device;
  try {
    if (!voxels || !valueRange)
      fail("vklCudaDenseValueRangeNoAlloc: NULL voxel or output pointer", VKL_INVALID_ARGUMENT);
    if (dimX <= 0 || dimY <= 0 || dimZ <= 0)
      fail("vklCudaDenseValueRangeNoAlloc: dimensions must be positive", VKL_INVALID_ARGUMENT);
    const uint3 nl = {((uint32_t)dimX + 7) / 8, ((uint32_t)dimY + 7) / 8, ((uint32_t)dimZ + 7) / 8};
    const uint64_t numLeaves = (uint64_t)nl.x * nl.y * nl.z;
    if (numLeaves > kMaxLeaves)
      fail("vklCudaDenseValueRangeNoAlloc: " + std::to_string(numLeaves) +
               " leaves (8^3 voxel blocks) exceed the maximum of " + std::to_string(kMaxLeaves) +
               " that its static scratch holds (e.g. 2048^3 voxels)",
           VKL_INVALID_ARGUMENT);
    switch (voxelType) {
    case VKL_UCHAR:
    case VKL_SHORT:
    case VKL_USHORT:
    case VKL_HALF:
    case VKL_FLOAT:
    case VKL_DOUBLE:
      break;
    default:
      fail("vklCudaDenseValueRangeNoAlloc: unsupported voxel type", VKL_INVALID_ARGUMENT);
    }
    int cur = 0;
    cudaCheck(cudaGetDevice(&cur), "vklCudaDenseValueRangeNoAlloc: cudaGetDevice");
    if (cur != d->cudaDevice)
      fail("vklCudaDenseValueRangeNoAlloc: the calling thread's current CUDA device (" +
               std::to_string(cur) + ") is not the VKL device's (" +
               std::to_string(d->cudaDevice) + ")",
           VKL_INVALID_OPERATION);
    RangeScratch *s = scratchFor(d->cudaDevice);
    const int3 dims       = {dimX, dimY, dimZ};
    const unsigned blocks = (unsigned)((numLeaves + kThreads - 1) / kThreads);
    cudaStream_t st       = d->stream;
    switch (voxelType) {
    case VKL_UCHAR:
      launch<uint8_t>(voxels, dims, nl, blocks, background, s, valueRange, st);
      break;
    case VKL_SHORT:
      launch<int16_t>(voxels, dims, nl, blocks, background, s, valueRange, st);
      break;
    case VKL_USHORT:
      launch<uint16_t>(voxels, dims, nl, blocks, background, s, valueRange, st);
      break;
    case VKL_HALF:
      launch<__half>(voxels, dims, nl, blocks, background, s, valueRange, st);
      break;
    case VKL_DOUBLE:
      launch<double>(voxels, dims, nl, blocks, background, s, valueRange, st);
      break;
    default:
      launch<float>(voxels, dims, nl, blocks, background, s, valueRange, st);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      forgetScratch(d->cudaDevice);
      cudaCheck(e, "vklCudaDenseValueRangeNoAlloc launch");
    }
    return VKL_NO_ERROR;
  } catch (const VklError &e) {
    d->setError(e.code, e.what());
    return e.code;
  } catch (const std::exception &e) {
    d->setError(VKL_UNKNOWN_ERROR, e.what());
    return VKL_UNKNOWN_ERROR;
  }
}
