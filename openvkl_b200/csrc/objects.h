// Host object model of the cuda device: devices, data arrays, volumes,
// samplers, iterator contexts and observers, with the reference's parameter
// and reference-counting semantics (openvkl/common/ManagedObject.h,
// openvkl/api/Device.h:42-185).  Errors are C++ exceptions inside the
// library and are turned into the device's last-error code / message and
// error callback at the C boundary (api.cpp), as the reference does
// (openvkl/api/API.cpp:37-89).  Commit-time validation errors carry
// VKL_UNKNOWN_ERROR (1) like the reference's runtimeError() throws.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/openvkl_cuda.h"
#include "grid.h"

namespace vklcuda {

struct VklError : std::runtime_error {
  VKLError code;
  VklError(VKLError c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(const std::string &msg, VKLError code = VKL_UNKNOWN_ERROR)
{
  throw VklError(code, msg);
}

inline void cudaCheck(cudaError_t e, const char *what)
{
  if (e != cudaSuccess)
    fail(std::string(what) + ": " + cudaGetErrorString(e),
         e == cudaErrorMemoryAllocation ? VKL_OUT_OF_MEMORY : VKL_UNKNOWN_ERROR);
}

size_t sizeOfType(VKLDataType t);

struct Device;

// ---------------------------------------------------------------------------
// Reference-counted object with a parameter table.
// ---------------------------------------------------------------------------
struct ManagedObject {
  std::atomic<int> refs{1};
  Device *device = nullptr;
  // The device this object keeps alive (taken when its handle is made,
  // dropped when it is destroyed): as in the reference, vklReleaseDevice
  // frees a device only once its objects are gone.
  Device *heldDevice = nullptr;

  struct Param {
    VKLDataType type = VKL_UNKNOWN;
    std::vector<uint8_t> bytes;
    std::string str;
    ManagedObject *obj = nullptr;
  };
  std::map<std::string, Param> params;

  virtual ~ManagedObject();
  virtual void commit() {}
  virtual const char *typeName() const = 0;

  void refInc() { refs.fetch_add(1); }
  void refDec()
  {
    if (refs.fetch_sub(1) == 1)
      delete this;
  }

  void setParam(const char *name, VKLDataType type, const void *mem);
  bool has(const std::string &name) const { return params.count(name) != 0; }
  const Param *find(const std::string &name) const
  {
    auto it = params.find(name);
    return it == params.end() ? nullptr : &it->second;
  }
  int getInt(const std::string &name, int def) const;
  float getFloat(const std::string &name, float def) const;
  bool getBool(const std::string &name, bool def) const;
  void getVec3f(const std::string &name, float out[3], const float def[3]) const;
  void getVec3i(const std::string &name, int out[3], const int def[3]) const;
  struct Data *getData(const std::string &name) const;
};

template <class T>
struct Ref {
  T *p = nullptr;
  Ref() = default;
  explicit Ref(T *x) : p(x)
  {
    if (p)
      p->refInc();
  }
  Ref(const Ref &o) : p(o.p)
  {
    if (p)
      p->refInc();
  }
  Ref &operator=(const Ref &o)
  {
    if (o.p)
      o.p->refInc();
    if (p)
      p->refDec();
    p = o.p;
    return *this;
  }
  ~Ref()
  {
    if (p)
      p->refDec();
  }
  T *operator->() const { return p; }
  T &operator*() const { return *p; }
  explicit operator bool() const { return p != nullptr; }
};

// ---------------------------------------------------------------------------
// Device memory owned by an object.
// ---------------------------------------------------------------------------
struct DeviceBuffer {
  void *ptr    = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  ~DeviceBuffer() { release(); }
  void release()
  {
    if (ptr)
      cudaFree(ptr);
    ptr   = nullptr;
    bytes = 0;
  }
  void alloc(size_t n)
  {
    release();
    if (n) {
      cudaCheck(cudaMalloc(&ptr, n), "cudaMalloc");
      bytes = n;
    }
  }
  // Grow-only (scratch use).
  void reserve(size_t n)
  {
    if (n > bytes)
      alloc(n + n / 4);
  }
  template <class T>
  T *as() const
  {
    return (T *)ptr;
  }
};

// ---------------------------------------------------------------------------
// Device.
// ---------------------------------------------------------------------------
// Device scratch of the ray-run sampling path (k_sample_rays.cu): the
// detector's counters and the kernels' error word.
struct RunScratch {
  DeviceBuffer counts;
};
// Ray-run sampling of dense float volumes with the trilinear filter:
// rayRunsApply says whether the path covers the call, detectRayRuns returns
// the run length S the points are laid out in (0: not ray runs; reads back
// a few counters, so it synchronizes the stream), launchSampleRays samples
// (grad: gradients) as launchSample / launchGradient do.
bool rayRunsApply(const DevGrid &g, int filter, uint32_t attr);
int detectRayRuns(const DevGrid &g, uint64_t n, const float *pts, RunScratch &scratch, cudaStream_t stream);
void launchSampleRays(const DevGrid &g, uint32_t maxDepth, uint64_t n, const float *pts, uint32_t attr, float *out,
                      bool grad, int S, RunScratch &scratch, cudaStream_t stream);

// Device scratch of binned sampling (launchSampleBinned): detection
// counters, the binned entries of one pass, bin histogram and cursors.
struct BinScratch {
  DeviceBuffer counts, entries, bins;
};

// Binned sampling of incoherent point sets (k_bin.cu).  `applies` is the
// cheap host test (dense float volume larger than L2, large call);
// launchSampleBinned then measures the points' coherence on the device (one
// small kernel and a 16-byte read-back, so it synchronizes `stream`) and,
// for incoherent points, bins and samples them and returns true; for
// coherent points it returns false and launches nothing else.  Points and
// output are device memory; results equal launchSample's / launchGradient's.
bool binnedSamplingApplies(const DevGrid &g, int filter, uint64_t n, uint32_t attr);
bool launchSampleBinned(const DevGrid &g, int filter, uint64_t n, const float *pts, uint32_t attr,
                        float *out, bool grad, BinScratch &scratch, cudaStream_t stream);

struct TextureAtlas;

struct Device {
  // 1 for the application's handle plus 1 per live object of the device.
  std::atomic<int> refs{1};
  void refInc() { refs.fetch_add(1); }
  void refDec();
  int cudaDevice = 0;
  cudaStream_t stream = nullptr;
  VKLError lastErrorCode = VKL_NO_ERROR;
  std::string lastErrorMsg;
  VKLErrorCallback errorCb = nullptr;
  void *errorUser = nullptr;
  VKLLogCallback logCb = nullptr;
  void *logUser = nullptr;
  int logLevel = VKL_LOG_WARNING;
  bool committed = false;
  std::map<std::string, int> intParams;
  std::map<std::string, std::string> stringParams;

  // Staging memory for host-pointer calls; guarded by `stagingMutex`.
  std::mutex stagingMutex;
  DeviceBuffer stageIn, stageOut, stageAux;

  // Chunked host-pointer calls overlap the host->device copy of chunk k+1
  // and the device->host copy of chunk k-1 with the kernel on chunk k:
  // copies run on two streams of their own, ordered against `stream` by
  // events, through kPipeSlots staging slots.  Created on first use.
  static constexpr int kPipeSlots = 3;
  cudaStream_t copyIn = nullptr, copyOut = nullptr;
  cudaEvent_t pipeStart = nullptr;
  cudaEvent_t inReady[kPipeSlots]{}, computed[kPipeSlots]{}, drained[kPipeSlots]{};
  void ensurePipeline();
  ~Device();

  // Scratch of binned sampling; `binMutex` serialises its users.  Binning
  // is on by default for the calls it applies to; device parameter
  // "binnedSampling" 0 turns it off.
  std::mutex binMutex;
  BinScratch binScratch;
  // ray-run detection and kernel scratch; `runMutex` serialises its users;
  // device parameter "rayRunSampling" 0 turns the path off
  std::mutex runMutex;
  RunScratch runScratch;
  bool rayRuns = true;
  bool binning = true;
  // Texture atlases of dense float attributes (DevGrid::atlasTex): on by
  // default; device parameter "textureSampling" 0 turns them off for volumes
  // committed afterwards.
  bool textureSampling = true;
  // Atlases of released or re-shaped volumes, kept for the next commit of
  // an atlas of the same size (a volume released and created again each
  // frame then allocates none); at most kAtlasPool are kept, and all are
  // dropped when an atlas allocation fails.
  static constexpr size_t kAtlasPool = 2;
  std::mutex atlasMutex;
  std::vector<std::unique_ptr<TextureAtlas>> atlasPool;
  std::unique_ptr<TextureAtlas> takeAtlas(uint32_t width, uint32_t height);
  void giveAtlas(std::unique_ptr<TextureAtlas> atlas);
  void dropAtlases();

  void setError(VKLError code, const std::string &msg);
  void log(int level, const std::string &msg);
};

// ---------------------------------------------------------------------------
// Data arrays (openvkl/common/Data.h): always held compact in device memory
// (strided sources are compacted on upload); a host copy is kept for the
// small metadata arrays the commit logic reads on the host.
// ---------------------------------------------------------------------------
struct Data : ManagedObject {
  VKLDataType type = VKL_UNKNOWN;
  size_t numItems  = 0;
  size_t itemSize  = 0;
  const void *dev  = nullptr;  // compact device array
  DeviceBuffer owned;
  std::vector<uint8_t> host;   // compact host copy (may be empty)
  std::vector<ManagedObject *> objects;  // object arrays (VKL_DATA etc.)

  ~Data() override;
  const char *typeName() const override { return "Data"; }
  // Compact host bytes (copied back from the device on first use).
  const uint8_t *hostBytes();
  template <class T>
  const T *hostAs()
  {
    return (const T *)hostBytes();
  }
};

// ---------------------------------------------------------------------------
// 2D float texture atlas of one dense attribute's z-planes (DevGrid::
// atlasTex): a cudaArray written through a surface object at commit and
// read through a texture object (point sampling, unnormalized coordinates,
// border addressing).
// ---------------------------------------------------------------------------
struct TextureAtlas {
  cudaArray_t array        = nullptr;
  cudaSurfaceObject_t surf = 0;
  cudaTextureObject_t tex  = 0;
  uint32_t width = 0, height = 0;
  TextureAtlas() = default;
  TextureAtlas(const TextureAtlas &) = delete;
  TextureAtlas &operator=(const TextureAtlas &) = delete;
  ~TextureAtlas() { release(); }
  void release();
  // Creates (or keeps, if the size is unchanged) a width x height atlas;
  // false if the device cannot allocate it.
  bool ensure(uint32_t w, uint32_t h);
};

// ---------------------------------------------------------------------------
// Volumes.
// ---------------------------------------------------------------------------
struct Volume : ManagedObject {
  bool isDense = false;
  bool committed = false;
  DevGrid grid{};
  std::vector<std::unique_ptr<DeviceBuffer>> buffers;
  std::vector<Ref<Data>> keep;   // data referenced by the grid
  std::vector<float> rangeLo, rangeHi;  // per attribute
  vkl_box3f bounds{};
  int filter = VKL_FILTER_LINEAR;
  int gradientFilter = VKL_FILTER_LINEAR;
  uint32_t maxSamplingDepth = kNumLevels - 1;
  uint64_t levelNodes[kNumLevels] = {0, 0, 0, 0};

  const char *typeName() const override { return isDense ? "structuredRegular" : "vdb"; }
  void commit() override;
  ~Volume() override;
  // Value ranges of the 16^3-voxel macrocells of one attribute (interval
  // contexts with "macrocells" = 1), built on first use after a commit.
  std::unique_ptr<DeviceBuffer> macroRanges[kMaxAttributes];
  const float *macrocellRanges(uint32_t attr, cudaStream_t st);
  std::unique_ptr<TextureAtlas> atlases[kMaxAttributes];
  // Device buffers of the previous commit.  A re-commit takes buffers of
  // the sizes it needs from here (a time-varying volume re-committed with
  // new data of the same shape allocates nothing); the rest are freed when
  // the commit ends.
  std::vector<std::unique_ptr<DeviceBuffer>> recycled;
  DeviceBuffer *newBuffer(size_t bytes)
  {
    for (auto it = recycled.begin(); it != recycled.end(); ++it)
      if ((*it)->bytes == bytes) {
        buffers.push_back(std::move(*it));
        recycled.erase(it);
        return buffers.back().get();
      }
    buffers.emplace_back(new DeviceBuffer());
    buffers.back()->alloc(bytes);
    return buffers.back().get();
  }

 private:
  void commitDense();
  void commitVdb();
  void finishCommit(const float indexLo[3], const float indexHi[3]);
};

struct Observer;

struct Sampler : ManagedObject {
  Ref<Volume> volume;
  DevSampler s{};
  DeviceBuffer devState;  // DevSamplerState for the device-side API
  // LeafNodeAccess observers (VdbSampler::newObserver); each removes itself
  // when released.
  std::vector<Observer *> leafObservers;
  const char *typeName() const override { return "Sampler"; }
  void commit() override;
  // The volume's grid with this sampler's observer buffers: what its
  // sampling and hit-iteration launches read.
  DevGrid launchGrid() const;
  void uploadState();
};

struct IntervalContext : ManagedObject {
  Ref<Sampler> sampler;
  uint32_t attr = 0;
  std::vector<float> ranges;  // 2 per range
  float minMax[2]   = {0, 0};
  uint32_t depth    = 2;
  bool elementary   = false;
  // extension: intervals of 16^3-voxel macrocells (the reference's legacy
  // structuredRegular iterator) instead of the hierarchy walk
  bool macrocells = false;
  DeviceBuffer devRanges;
  DeviceBuffer devState;  // DevIntervalContextState for the device-side API
  const char *typeName() const override { return "IntervalIteratorContext"; }
  void commit() override;
  DevValueRanges devValueRanges() const;
};

struct HitContext : ManagedObject {
  Ref<Sampler> sampler;
  uint32_t attr = 0;
  std::vector<float> values;
  std::vector<float> ranges;
  float minMax[2] = {0, 0};
  uint32_t depth  = 2;
  DeviceBuffer devRanges, devValues;
  DeviceBuffer devState;  // DevHitContextState for the device-side API
  const char *typeName() const override { return "HitIteratorContext"; }
  void commit() override;
  DevValueRanges devValueRanges() const;
};

struct Observer : ManagedObject {
  Ref<Volume> volume;
  Ref<Sampler> sampler;
  std::string kind;
  std::vector<float> buffer;
  size_t elementFloats = 0;
  size_t numElements   = 0;
  std::vector<uint32_t> leafAccess;  // LeafNodeAccess buffer (host copy at map)
  DeviceBuffer devCounters;          // LeafNodeAccess buffer, one uint32 per leaf
  ~Observer() override;
  const char *typeName() const override { return "Observer"; }
  void commit() override;
};

}  // namespace vklcuda
