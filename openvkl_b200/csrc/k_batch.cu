// Batched multi-volume sampling (extension; no reference counterpart).
//
// A batch is a fixed list of jobs (sampler, device points, device outputs for
// samples and / or gradients).  Running it replays one CUDA graph on the
// device's stream.  The graph holds one persistent kernel per job class
// (dense voxel type or sparse leaf type, trilinear filter for samples and
// gradients); its CTAs take point tiles from an atomic counter until every
// job's tiles are done, so hundreds of small volumes and uneven query counts
// keep all SMs busy in one launch.  Each tile computes samples and gradients
// from one gather of the 8 corners: the same expressions as sampleLinear /
// gradientLinear, so the results are bit-identical to vklComputeSampleN and
// vklComputeGradientN.  Jobs outside the fused classes (other filters,
// compressed leaves) are recorded in the same graph as ordinary launches.
//
// The tile size, whether tiles are sorted by brick, and the CTAs per SM of
// the dense float class are chosen by timing each candidate on the batch
// itself (autotune), and remembered per batch shape for later batches.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "kernels.h"
#include "objects.h"
#include "sampling.cuh"

namespace vklcuda {

namespace {

struct BatchJob {
  const DevGrid *grid;  // device copy of the job's grid
  const float *points;
  float *samples;
  float *gradients;
  uint32_t numPoints;
  uint32_t attr;
};

constexpr int kBatchThreads = 256;
constexpr int kBatchBins    = 1024;

__device__ __forceinline__ uint32_t batchKey(f3 p)
{
  const uint32_t bx = (uint32_t)__float2int_rd(p.x) >> 3, by = (uint32_t)__float2int_rd(p.y) >> 3,
                 bz = (uint32_t)__float2int_rd(p.z) >> 3;
  return ((bx * 73856093u) ^ (by * 19349663u) ^ (bz * 83492791u)) & (kBatchBins - 1);
}

// Trilinear sample and index-space gradient from one corner gather
// (the expressions of sampleLinear and gradientLinear).
template <class Field>
__device__ __forceinline__ void sampleGradLinear(const Field &F, f3 p, float &v, f3 &gi)
{
  const int32_t ix = ifloor(p.x), iy = ifloor(p.y), iz = ifloor(p.z);
  const float dx = p.x - (float)ix, dy = p.y - (float)iy, dz = p.z - (float)iz;
  float s[8];
  F.corners(ix, iy, iz, s);
  v    = lerpf(dx, lerpf(dy, lerpf(dz, s[0], s[1]), lerpf(dz, s[2], s[3])),
               lerpf(dy, lerpf(dz, s[4], s[5]), lerpf(dz, s[6], s[7])));
  gi.x = lerpf(dy, lerpf(dz, s[4] - s[0], s[5] - s[1]), lerpf(dz, s[6] - s[2], s[7] - s[3]));
  gi.y = lerpf(dx, lerpf(dz, s[2] - s[0], s[3] - s[1]), lerpf(dz, s[6] - s[4], s[7] - s[5]));
  gi.z = lerpf(dx, lerpf(dy, s[1] - s[0], s[3] - s[2]), lerpf(dy, s[5] - s[4], s[7] - s[6]));
}

// ATLAS: dense float jobs whose attribute has a texture atlas fetch their
// corners from it (AtlasField), as vklComputeSampleN does.
template <typename T, bool DENSE, int TILE, bool SORT, bool ATLAS = false>
__global__ void __launch_bounds__(kBatchThreads)
    kBatchLinear(const BatchJob *__restrict__ jobs, const uint32_t *__restrict__ tileJob,
                 const uint32_t *__restrict__ jobFirstTile, uint32_t numTiles,
                 unsigned int *__restrict__ counter)
{
  constexpr int PPT = TILE / kBatchThreads;
  __shared__ __align__(16) float sxyz[3 * TILE];
  __shared__ __align__(16) float res[4 * TILE];  // sample, then gradient xyz
  __shared__ uint16_t sidx[SORT ? TILE : 1];
  __shared__ __align__(16) int hist[SORT ? kBatchBins : 4];
  __shared__ int warpSum[kBatchThreads / 32];
  __shared__ __align__(16) uint32_t gridWords[(sizeof(DevGrid) + 3) / 4];
  __shared__ uint32_t sTile;
  const DevGrid &g = *reinterpret_cast<const DevGrid *>(gridWords);
  float *const sx = sxyz, *const sy = sxyz + TILE, *const sz = sxyz + 2 * TILE;

  for (;;) {
    if (threadIdx.x == 0)
      sTile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t tile = sTile;
    if (tile >= numTiles)
      return;
    const uint32_t j   = tileJob[tile];
    const BatchJob job = jobs[j];
    {
      const uint32_t *src = reinterpret_cast<const uint32_t *>(job.grid);
      for (int k = threadIdx.x; k < (int)((sizeof(DevGrid) + 3) / 4); k += kBatchThreads)
        gridWords[k] = __ldg(src + k);
    }
    const uint32_t base = (tile - jobFirstTile[j]) * TILE;
    const int cnt       = (int)min((uint32_t)TILE, job.numPoints - base);
    if (SORT)
      for (int k = threadIdx.x; k < kBatchBins; k += kBatchThreads)
        hist[k] = 0;
    {
      const float *src = job.points + 3 * (uint64_t)base;
      const int nf     = 3 * cnt;
      int k0           = 0;
      if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
        const int n4 = nf >> 2;
        for (int k = threadIdx.x; k < n4; k += kBatchThreads)
          reinterpret_cast<float4 *>(sxyz)[k] = __ldcs(reinterpret_cast<const float4 *>(src) + k);
        k0 = n4 << 2;
      }
      for (int k = k0 + threadIdx.x; k < nf; k += kBatchThreads)
        sxyz[k] = __ldcs(src + k);
    }
    __syncthreads();
    f3 p[PPT];
    uint32_t key[PPT];
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
      const int k = threadIdx.x + q * kBatchThreads;
      if (k < cnt) {
        p[q] = xfmPoint(g.objectToIndex, f3{sxyz[3 * k], sxyz[3 * k + 1], sxyz[3 * k + 2]});
        if (SORT) {
          key[q] = batchKey(p[q]);
          atomicAdd(&hist[key[q]], 1);
        }
      }
    }
    __syncthreads();
    if (SORT) {
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
      __syncthreads();
#pragma unroll
      for (int q = 0; q < PPT; ++q) {
        const int k = threadIdx.x + q * kBatchThreads;
        if (k < cnt) {
          const int pos = atomicAdd(&hist[key[q]], 1);
          sx[pos]       = p[q].x;
          sy[pos]       = p[q].y;
          sz[pos]       = p[q].z;
          sidx[pos]     = (uint16_t)k;
        }
      }
      __syncthreads();
    }
    using Field = typename std::conditional<
        ATLAS, AtlasField, typename std::conditional<DENSE, DenseField<T>, SparseField<T>>::type>::type;
    const Field F = [&]() {
      if constexpr (ATLAS)
        return AtlasField(g, job.attr);
      else if constexpr (DENSE)
        return DenseField<T>(g, job.attr);
      else
        return SparseField<T>(g, job.attr, kNumLevels - 1);
    }();
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
      const int k = threadIdx.x + q * kBatchThreads;
      if (k < cnt) {
        const f3 pt = SORT ? f3{sx[k], sy[k], sz[k]} : p[q];
        const int o = SORT ? (int)sidx[k] : k;
        float v;
        f3 gi;
        sampleGradLinear(F, pt, v, gi);
        const f3 gr        = xfmNormal(g.objectToIndex, gi);
        res[o]             = v;
        res[TILE + 3 * o]     = gr.x;
        res[TILE + 3 * o + 1] = gr.y;
        res[TILE + 3 * o + 2] = gr.z;
      }
    }
    __syncthreads();
    if (job.samples)
      for (int k = threadIdx.x; k < cnt; k += kBatchThreads)
        __stcs(job.samples + base + k, res[k]);
    if (job.gradients)
      for (int k = threadIdx.x; k < 3 * cnt; k += kBatchThreads)
        __stcs(job.gradients + 3 * (uint64_t)base + k, res[TILE + k]);
    __syncthreads();  // shared buffers are reused by the next tile
  }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
struct Config {
  int tile   = 1024;
  bool sort  = true;
  int ctasPerSM = 0;  // 0: the occupancy maximum
};

using Kernel = void (*)(const BatchJob *, const uint32_t *, const uint32_t *, uint32_t, unsigned int *);

// Job classes fused into persistent kernels: dense voxel types and plain
// sparse leaves, trilinear filter for both outputs.
enum ClassId : int {
  kDenseU8,
  kDenseI16,
  kDenseU16,
  kDenseF16,
  kDenseF32,
  kDenseF32Atlas,
  kDenseF64,
  kSparseF32,
  kSparseF16,
  kNumClasses
};

template <typename T, bool DENSE, bool ATLAS = false>
Kernel kernelFor(const Config &c)
{
  if (c.tile == 512)
    return c.sort ? kBatchLinear<T, DENSE, 512, true, ATLAS> : kBatchLinear<T, DENSE, 512, false, ATLAS>;
  return c.sort ? kBatchLinear<T, DENSE, 1024, true, ATLAS> : kBatchLinear<T, DENSE, 1024, false, ATLAS>;
}

Kernel classKernel(int cls, const Config &c)
{
  switch (cls) {
  case kDenseU8:
    return kernelFor<uint8_t, true>(c);
  case kDenseI16:
    return kernelFor<int16_t, true>(c);
  case kDenseU16:
    return kernelFor<uint16_t, true>(c);
  case kDenseF16:
    return kernelFor<__half, true>(c);
  case kDenseF64:
    return kernelFor<double, true>(c);
  case kSparseF32:
    return kernelFor<float, false>(c);
  case kSparseF16:
    return kernelFor<__half, false>(c);
  case kDenseF32Atlas:
    return kernelFor<float, true, true>(c);
  default:
    return kernelFor<float, true>(c);
  }
}

// The class of a job on attribute `attr` (its voxel type decides).
int classOf(const Sampler *s, bool wantGrad, uint32_t attr)
{
  const DevGrid &g = s->volume->grid;
  if (s->s.filter != kFilterLinear || (wantGrad && s->s.gradientFilter != kFilterLinear))
    return -1;
  if (g.dense) {
    if (g.type[attr] == kFloat && g.atlasTex[attr])
      return kDenseF32Atlas;
    switch (g.type[attr]) {
    case kUChar:
      return kDenseU8;
    case kShort:
      return kDenseI16;
    case kUShort:
      return kDenseU16;
    case kHalf:
      return kDenseF16;
    case kDouble:
      return kDenseF64;
    default:
      return kDenseF32;
    }
  }
  if (g.compress != kCompressNone || g.temporal || s->s.maxSamplingDepth < kNumLevels - 1)
    return -1;
  return g.type[attr] == kHalf ? kSparseF16 : kSparseF32;
}

struct ClassPlan {
  std::vector<uint32_t> jobs;     // indices into the batch's job list
  Config cfg;
  DeviceBuffer dJobs, dTileJob, dFirst;
  uint32_t numTiles = 0;
  int maxCtasPerSM  = 0;
};

std::mutex g_tuneMutex;
std::map<std::tuple<int, int, uint32_t>, Config> g_tuned;  // (device, class, tiles/64) -> config

bool isDeviceMemory(const void *p)
{
  if (!p)
    return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

struct SampleBatch {
  Device *device = nullptr;
  std::vector<VKLCudaSampleJob> jobs;
  std::vector<Ref<Sampler>> samplers;
  DeviceBuffer dGrids, dCounters;
  ClassPlan plans[kNumClasses];
  std::vector<uint32_t> plainJobs;
  int numSMs = 0;
  cudaStream_t capture = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool tuned           = false;

  ~SampleBatch()
  {
    if (exec)
      cudaGraphExecDestroy(exec);
    if (capture)
      cudaStreamDestroy(capture);
  }

  void buildPlan(int cls)
  {
    ClassPlan &P = plans[cls];
    if (P.jobs.empty())
      return;
    const uint32_t T = (uint32_t)P.cfg.tile;
    std::vector<BatchJob> dj;
    std::vector<uint32_t> tileJob, first;
    for (uint32_t k = 0; k < P.jobs.size(); ++k) {
      const uint32_t i           = P.jobs[k];
      const VKLCudaSampleJob &jb = jobs[i];
      BatchJob b;
      b.grid      = dGrids.as<DevGrid>() + i;
      b.points    = (const float *)jb.points;
      b.samples   = jb.samples;
      b.gradients = (float *)jb.gradients;
      b.numPoints = jb.numPoints;
      b.attr      = jb.attributeIndex;
      dj.push_back(b);
      first.push_back((uint32_t)tileJob.size());
      const uint32_t nt = (jb.numPoints + T - 1) / T;
      tileJob.insert(tileJob.end(), nt, k);
    }
    P.numTiles = (uint32_t)tileJob.size();
    P.dJobs.alloc(dj.size() * sizeof(BatchJob));
    P.dTileJob.alloc(std::max<size_t>(tileJob.size(), 1) * 4);
    P.dFirst.alloc(first.size() * 4);
    cudaCheck(cudaMemcpy(P.dJobs.ptr, dj.data(), dj.size() * sizeof(BatchJob), cudaMemcpyHostToDevice),
              "batch upload");
    if (!tileJob.empty())
      cudaCheck(cudaMemcpy(P.dTileJob.ptr, tileJob.data(), tileJob.size() * 4, cudaMemcpyHostToDevice),
                "batch upload");
    cudaCheck(cudaMemcpy(P.dFirst.ptr, first.data(), first.size() * 4, cudaMemcpyHostToDevice),
              "batch upload");
    const Kernel k = classKernel(cls, P.cfg);
    int occ        = 0;
    cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, kBatchThreads, 0), "occupancy");
    P.maxCtasPerSM = std::max(occ, 1);
  }

  // Records every launch of one run on `st` (a capturing stream).
  void record(cudaStream_t st)
  {
    cudaCheck(cudaMemsetAsync(dCounters.ptr, 0, kNumClasses * sizeof(unsigned int), st), "batch reset");
    for (int c = 0; c < kNumClasses; ++c) {
      ClassPlan &P = plans[c];
      if (P.jobs.empty() || P.numTiles == 0)
        continue;
      const int per  = P.cfg.ctasPerSM > 0 ? std::min(P.cfg.ctasPerSM, P.maxCtasPerSM) : P.maxCtasPerSM;
      const uint32_t grid = std::min<uint32_t>((uint32_t)(per * numSMs), P.numTiles);
      classKernel(c, P.cfg)<<<grid, kBatchThreads, 0, st>>>(
          P.dJobs.as<BatchJob>(), P.dTileJob.as<uint32_t>(), P.dFirst.as<uint32_t>(), P.numTiles,
          dCounters.as<unsigned int>() + c);
    }
    for (uint32_t i : plainJobs) {
      const VKLCudaSampleJob &jb = jobs[i];
      const Sampler *s           = samplers[i].p;
      const uint32_t attr        = jb.attributeIndex;
      if (jb.samples)
        launchSample(s->volume->grid, s->s.filter, s->s.maxSamplingDepth, jb.numPoints,
                     (const float *)jb.points, 1, &attr, jb.samples, st);
      if (jb.gradients)
        launchGradient(s->volume->grid, s->s.gradientFilter, s->s.maxSamplingDepth, jb.numPoints,
                       (const float *)jb.points, attr, (float *)jb.gradients, st);
    }
    cudaCheck(cudaGetLastError(), "batch launches");
  }

  void capture_()
  {
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    cudaCheck(cudaStreamBeginCapture(capture, cudaStreamCaptureModeThreadLocal), "graph capture");
    try {
      record(capture);
    } catch (...) {
      cudaStreamEndCapture(capture, &graph);
      if (graph)
        cudaGraphDestroy(graph);
      throw;
    }
    cudaCheck(cudaStreamEndCapture(capture, &graph), "graph capture");
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    cudaCheck(e, "graph instantiate");
  }

  void run(cudaStream_t st) { cudaCheck(cudaGraphLaunch(exec, st), "graph launch"); }

  // Times `reps` runs of the current graph on the device stream (ms per run).
  float time(int reps)
  {
    cudaStream_t st = device->stream;
    cudaEvent_t a, b;
    cudaCheck(cudaEventCreate(&a), "event");
    cudaCheck(cudaEventCreate(&b), "event");
    run(st);
    cudaEventRecord(a, st);
    for (int r = 0; r < reps; ++r)
      run(st);
    cudaEventRecord(b, st);
    float ms = 0;
    const cudaError_t e = cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaCheck(e, "autotune timing");
    return ms / reps;
  }

  // Tries tile size x sort x CTAs per SM for the largest class and keeps the
  // fastest; the other classes keep the default configuration.
  void autotune()
  {
    int best = -1;
    uint32_t most = 0;
    for (int c = 0; c < kNumClasses; ++c)
      if (plans[c].numTiles > most) {
        most = plans[c].numTiles;
        best = c;
      }
    if (best < 0)
      return;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(dev, best, most / 64);
    {
      std::lock_guard<std::mutex> lock(g_tuneMutex);
      auto it = g_tuned.find(key);
      if (it != g_tuned.end()) {
        plans[best].cfg = it->second;
        buildPlan(best);
        capture_();
        tuned = true;
        return;
      }
    }
    ClassPlan &P = plans[best];
    Config bestCfg = P.cfg;
    float bestMs   = 1e30f;
    for (int tile : {512, 1024})
      for (bool sort : {true, false})
        for (int frac : {1, 2}) {
          Config c;
          c.tile = tile;
          c.sort = sort;
          P.cfg  = c;
          buildPlan(best);
          P.cfg.ctasPerSM = std::max(1, P.maxCtasPerSM / frac);
          capture_();
          const float ms = time(3);
          if (ms < bestMs) {
            bestMs  = ms;
            bestCfg = P.cfg;
          }
        }
    P.cfg = bestCfg;
    buildPlan(best);
    capture_();
    tuned = true;
    std::lock_guard<std::mutex> lock(g_tuneMutex);
    g_tuned[key] = bestCfg;
  }
};

}  // namespace vklcuda

using namespace vklcuda;

extern "C" OPENVKL_CUDA_INTERFACE VKLCudaSampleBatch vklCudaNewSampleBatch(VKLDevice device,
                                                                          unsigned int numJobs,
                                                                          const VKLCudaSampleJob *jobs,
                                                                          int autotune)
{
  if (!device)
    return nullptr;
  Device *d = (Device *)device;
  SampleBatch *b = nullptr;
  try {
    if (numJobs == 0 || !jobs)
      fail("vklCudaNewSampleBatch: no jobs", VKL_INVALID_ARGUMENT);
    b         = new SampleBatch();
    b->device = d;
    b->jobs.assign(jobs, jobs + numJobs);
    std::vector<DevGrid> grids(numJobs);
    for (unsigned int i = 0; i < numJobs; ++i) {
      const VKLCudaSampleJob &jb = jobs[i];
      Sampler *s = dynamic_cast<Sampler *>((ManagedObject *)jb.sampler.host);
      if (!s || !s->volume || !s->volume->committed)
        fail("vklCudaNewSampleBatch: job " + std::to_string(i) + " has no committed sampler",
             VKL_INVALID_ARGUMENT);
      if (jb.attributeIndex >= s->volume->grid.numAttributes)
        fail("vklCudaNewSampleBatch: job " + std::to_string(i) + " has an invalid attribute index",
             VKL_INVALID_ARGUMENT);
      if (jb.numPoints && (!isDeviceMemory(jb.points) || (jb.samples && !isDeviceMemory(jb.samples)) ||
                           (jb.gradients && !isDeviceMemory(jb.gradients))))
        fail("vklCudaNewSampleBatch: job " + std::to_string(i) +
                 " points and outputs must be device memory",
             VKL_INVALID_ARGUMENT);
      b->samplers.emplace_back(s);
      grids[i] = s->volume->grid;
      if (jb.numPoints == 0 || (!jb.samples && !jb.gradients))
        continue;
      const int cls = classOf(s, jb.gradients != nullptr, jb.attributeIndex);
      if (cls < 0)
        b->plainJobs.push_back(i);
      else
        b->plans[cls].jobs.push_back(i);
    }
    b->dGrids.alloc(grids.size() * sizeof(DevGrid));
    cudaCheck(cudaMemcpy(b->dGrids.ptr, grids.data(), grids.size() * sizeof(DevGrid),
                         cudaMemcpyHostToDevice),
              "batch upload");
    b->dCounters.alloc(kNumClasses * sizeof(unsigned int));
    cudaCheck(cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, d->cudaDevice),
              "device attribute");
    cudaCheck(cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking), "stream");
    for (int c = 0; c < kNumClasses; ++c)
      b->buildPlan(c);
    b->capture_();
    if (autotune)
      b->autotune();
    return (VKLCudaSampleBatch)b;
  } catch (const VklError &e) {
    delete b;
    d->setError(e.code, e.what());
  } catch (const std::exception &e) {
    delete b;
    d->setError(VKL_UNKNOWN_ERROR, e.what());
  }
  return nullptr;
}

extern "C" OPENVKL_CUDA_INTERFACE VKLError vklCudaRunSampleBatch(VKLCudaSampleBatch batch)
{
  if (!batch)
    return VKL_INVALID_ARGUMENT;
  SampleBatch *b = (SampleBatch *)batch;
  try {
    b->run(b->device->stream);
    return VKL_NO_ERROR;
  } catch (const VklError &e) {
    b->device->setError(e.code, e.what());
    return e.code;
  }
}

extern "C" OPENVKL_CUDA_INTERFACE VKLError vklCudaGetSampleBatchConfig(VKLCudaSampleBatch batch,
                                                                      int *tilePoints, int *sorted,
                                                                      int *ctasPerSM, int *fusedJobs)
{
  if (!batch)
    return VKL_INVALID_ARGUMENT;
  SampleBatch *b = (SampleBatch *)batch;
  int best = 0, fused = 0;
  uint32_t most = 0;
  for (int c = 0; c < kNumClasses; ++c) {
    fused += (int)b->plans[c].jobs.size();
    if (b->plans[c].numTiles > most) {
      most = b->plans[c].numTiles;
      best = c;
    }
  }
  const ClassPlan &P = b->plans[best];
  if (tilePoints)
    *tilePoints = P.cfg.tile;
  if (sorted)
    *sorted = P.cfg.sort ? 1 : 0;
  if (ctasPerSM)
    *ctasPerSM = P.cfg.ctasPerSM > 0 ? std::min(P.cfg.ctasPerSM, P.maxCtasPerSM) : P.maxCtasPerSM;
  if (fusedJobs)
    *fusedJobs = fused;
  return VKL_NO_ERROR;
}

extern "C" OPENVKL_CUDA_INTERFACE void vklCudaReleaseSampleBatch(VKLCudaSampleBatch batch)
{
  delete (SampleBatch *)batch;
}
