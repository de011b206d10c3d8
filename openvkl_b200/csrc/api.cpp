// C entry points of the cuda device (include/openvkl_cuda.h).
//
// Each call unwraps the {host, device} handle, runs inside a try/catch and
// converts exceptions into the device's last error plus error callback,
// returning the reference's sentinel values (NaN sample, null handle, 0)
// (openvkl/api/API.cpp:37-89, devices/cpu/api/DeviceAPI.cpp:25-57).
#include <algorithm>
#include <cmath>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <mutex>

#include "kernels.h"
#include "objects.h"

using namespace vklcuda;

namespace {

std::mutex g_devicesMutex;
Device *g_lastDevice = nullptr;

Device *deviceOf(const VKLObject &o)
{
  return o.host ? ((ManagedObject *)o.host)->device : g_lastDevice;
}

template <class F>
auto guarded(Device *d, F &&f, decltype(f()) onError) -> decltype(f())
{
  try {
    return f();
  } catch (const VklError &e) {
    if (d)
      d->setError(e.code, e.what());
  } catch (const std::exception &e) {
    if (d)
      d->setError(VKL_UNKNOWN_ERROR, e.what());
  } catch (...) {
    if (d)
      d->setError(VKL_UNKNOWN_ERROR, "unknown error");
  }
  return onError;
}

template <class F>
void guardedVoid(Device *d, F &&f)
{
  guarded(
      d,
      [&]() {
        f();
        return 0;
      },
      0);
}

template <class T>
T *objectAs(const VKLObject &o, const char *what)
{
  T *t = dynamic_cast<T *>((ManagedObject *)o.host);
  if (!t)
    fail(std::string("invalid ") + what + " handle", VKL_INVALID_ARGUMENT);
  return t;
}

VKLObject handleOf(ManagedObject *o, void *dev = nullptr)
{
  if (o->device && !o->heldDevice) {
    o->heldDevice = o->device;
    o->heldDevice->refInc();
  }
  VKLObject h;
  h.host   = o;
  h.device = dev;
  return h;
}

bool isDevicePtr(const void *p)
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

const float kNaN = std::numeric_limits<float>::quiet_NaN();

Sampler *committedSampler(const VKLSampler *s)
{
  if (!s)
    fail("sampler is NULL", VKL_INVALID_ARGUMENT);
  Sampler *sp = objectAs<Sampler>(*s, "sampler");
  if (!sp->volume || !sp->volume->committed)
    fail("sampler or its volume is not committed", VKL_INVALID_OPERATION);
  return sp;
}

// Points per chunk of a pipelined host-pointer call (a multiple of the
// sampling kernels' 2048-point tile, so every chunk starts 16-byte aligned).
constexpr uint64_t kPipeChunk = uint64_t(1) << 23;
// Host-pointer calls below this many input bytes are staged in one piece.
constexpr size_t kPipeMinBytes = size_t(32) << 20;

// Runs `launch(n, devIn, devOut)` over N independent items (inStride /
// outStride bytes each) on the device stream, with inputs / outputs that
// may be host or device memory.  Host arrays are staged through device
// buffers and the call synchronizes before returning; large host-pointer
// calls are cut into chunks whose copies overlap the kernels of their
// neighbours (copy streams ordered against the device stream by events).
template <class Launch>
void staged(Device *d, uint64_t N, size_t inStride, const void *in, size_t outStride, void *out,
            Launch &&launch)
{
  const bool inDev = isDevicePtr(in), outDev = isDevicePtr(out);
  if (inDev && outDev) {
    launch(N, in, out);
    return;
  }
  std::lock_guard<std::mutex> lock(d->stagingMutex);
  if (N * inStride < kPipeMinBytes) {
    const void *din = in;
    void *dout      = out;
    if (!inDev) {
      d->stageIn.reserve(N * inStride);
      cudaCheck(cudaMemcpyAsync(d->stageIn.ptr, in, N * inStride, cudaMemcpyHostToDevice,
                                d->stream),
                "stage in");
      din = d->stageIn.ptr;
    }
    if (!outDev) {
      d->stageOut.reserve(N * outStride);
      dout = d->stageOut.ptr;
    }
    launch(N, din, dout);
    if (!outDev)
      cudaCheck(cudaMemcpyAsync(out, dout, N * outStride, cudaMemcpyDeviceToHost, d->stream),
                "stage out");
    cudaCheck(cudaStreamSynchronize(d->stream), "synchronize");
    return;
  }

  // Chunk k uses slot k % S: its input copy waits for the kernel of chunk
  // k - S (which read the slot), its kernel for that chunk's output copy.
  constexpr int S = Device::kPipeSlots;
  d->ensurePipeline();
  const uint64_t C = kPipeChunk;
  if (!inDev)
    d->stageIn.reserve(S * C * inStride);
  if (!outDev)
    d->stageOut.reserve(S * C * outStride);
  cudaCheck(cudaEventRecord(d->pipeStart, d->stream), "pipeline");
  cudaCheck(cudaStreamWaitEvent(d->copyIn, d->pipeStart, 0), "pipeline");
  cudaCheck(cudaStreamWaitEvent(d->copyOut, d->pipeStart, 0), "pipeline");
  const uint64_t K = (N + C - 1) / C;
  for (uint64_t k = 0; k < K; ++k) {
    const int s        = int(k % S);
    const uint64_t off = k * C, n = std::min(C, N - off);
    const void *din    = (const uint8_t *)in + off * inStride;
    void *dout         = (uint8_t *)out + off * outStride;
    if (!inDev) {
      void *slot = (uint8_t *)d->stageIn.ptr + s * C * inStride;
      if (k >= (uint64_t)S)
        cudaCheck(cudaStreamWaitEvent(d->copyIn, d->computed[s], 0), "pipeline");
      cudaCheck(cudaMemcpyAsync(slot, din, n * inStride, cudaMemcpyHostToDevice, d->copyIn),
                "stage in");
      cudaCheck(cudaEventRecord(d->inReady[s], d->copyIn), "pipeline");
      cudaCheck(cudaStreamWaitEvent(d->stream, d->inReady[s], 0), "pipeline");
      din = slot;
    }
    void *hostOut = dout;
    if (!outDev) {
      if (k >= (uint64_t)S)
        cudaCheck(cudaStreamWaitEvent(d->stream, d->drained[s], 0), "pipeline");
      dout = (uint8_t *)d->stageOut.ptr + s * C * outStride;
    }
    launch(n, din, dout);
    cudaCheck(cudaEventRecord(d->computed[s], d->stream), "pipeline");
    if (!outDev) {
      cudaCheck(cudaStreamWaitEvent(d->copyOut, d->computed[s], 0), "pipeline");
      cudaCheck(cudaMemcpyAsync(hostOut, dout, n * outStride, cudaMemcpyDeviceToHost, d->copyOut),
                "stage out");
      cudaCheck(cudaEventRecord(d->drained[s], d->copyOut), "pipeline");
    }
  }
  // the device stream resumes after the last copies (and the call returns then)
  if (!outDev)
    cudaCheck(cudaStreamWaitEvent(d->stream, d->drained[(K - 1) % S], 0), "pipeline");
  cudaCheck(cudaStreamSynchronize(d->stream), "synchronize");
}

// Incoherent large calls on dense float volumes go through binned sampling
// (k_bin.cu); returns false where the ordinary launch is to run.
bool binned(Device *d, Sampler *s, int filter, uint64_t n, const float *pts, uint32_t attr, float *out,
            bool grad)
{
  const DevGrid &g = s->volume->grid;
  if (!d->binning || !binnedSamplingApplies(g, filter, n, attr))
    return false;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaCheck(cudaStreamIsCapturing(d->stream, &cs), "capture status");
  if (cs != cudaStreamCaptureStatusNone)  // the coherence test reads back a count
    return false;
  std::lock_guard<std::mutex> lock(d->binMutex);
  return launchSampleBinned(g, filter, n, pts, attr, out, grad, d->binScratch, d->stream);
}

// Temporally varying volumes: points, times and results staged through the
// device buffers in one piece (no copy pipeline), one kernel launch.
void sampleTemporal(Device *d, Sampler *s, uint64_t N, const void *pts, const float *times, void *out,
                    uint32_t M, const uint32_t *attrs, bool grad)
{
  const DevGrid &g        = s->launchGrid();
  const int filter        = grad ? s->s.gradientFilter : s->s.filter;
  const size_t outStride  = grad ? 12 : 4 * (size_t)M;
  const bool ptsDev = isDevicePtr(pts), outDev = isDevicePtr(out), tDev = !times || isDevicePtr(times);
  if (ptsDev && outDev && tDev) {
    launchSampleTemporal(g, filter, N, (const float *)pts, times, M, attrs, (float *)out, grad, d->stream);
    return;
  }
  std::lock_guard<std::mutex> lock(d->stagingMutex);
  d->stageIn.reserve(N * 16);
  d->stageOut.reserve(N * outStride);
  const float *dp = (const float *)pts, *dt = times;
  if (!ptsDev) {
    cudaCheck(cudaMemcpyAsync(d->stageIn.ptr, pts, N * 12, cudaMemcpyHostToDevice, d->stream), "stage in");
    dp = d->stageIn.as<float>();
  }
  if (!tDev) {
    float *slot = (float *)(d->stageIn.as<uint8_t>() + N * 12);
    cudaCheck(cudaMemcpyAsync(slot, times, N * 4, cudaMemcpyHostToDevice, d->stream), "stage in");
    dt = slot;
  }
  float *dout = outDev ? (float *)out : d->stageOut.as<float>();
  launchSampleTemporal(g, filter, N, dp, dt, M, attrs, dout, grad, d->stream);
  if (!outDev)
    cudaCheck(cudaMemcpyAsync(out, dout, N * outStride, cudaMemcpyDeviceToHost, d->stream), "stage out");
  cudaCheck(cudaStreamSynchronize(d->stream), "synchronize");
}

// `times`: one time per point (host or device memory), or NULL for time 0;
// only temporally varying volumes read them (the reference's temporally
// constant volumes ignore the time as well).
// Ray-run sampling (k_sample_rays.cu) of large dense float trilinear calls
// whose points come as runs of samples per ray; the run length is detected
// once per call (on its first chunk).  Returns false where the ordinary
// launch is to run.
bool rayRuns(Device *d, Sampler *s, int filter, uint64_t n, const float *pts, uint32_t attr, float *out, bool grad,
             int &runS)
{
  const DevGrid &g = s->volume->grid;
  if (!d->rayRuns || !rayRunsApply(g, filter, attr) || n < (1u << 20) || s->s.maxSamplingDepth < kNumLevels - 1)
    return false;
  std::lock_guard<std::mutex> lock(d->runMutex);
  if (runS < 0) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaCheck(cudaStreamIsCapturing(d->stream, &cs), "capture status");
    // the detector reads back its counters: not while the stream is captured
    runS = cs == cudaStreamCaptureStatusNone ? detectRayRuns(g, n, pts, d->runScratch, d->stream) : 0;
    if (runS > 0)
      d->log(VKL_LOG_DEBUG, "sampling " + std::to_string(n) + " points as runs of " + std::to_string(runS) +
                                " samples per ray\n");
  }
  if (runS <= 0)
    return false;
  launchSampleRays(s->launchGrid(), s->s.maxSamplingDepth, n, pts, attr, out, grad, runS, d->runScratch,
                   d->stream);
  return true;
}

void sampleN(const VKLSampler *sampler, uint64_t N, const vkl_vec3f *pts, float *out,
             uint32_t M, const uint32_t *attrs, const float *times = nullptr)
{
  Sampler *s = committedSampler(sampler);
  if (M == 0 || M > kMaxAttributes)
    fail("invalid number of attributes", VKL_INVALID_ARGUMENT);
  for (uint32_t m = 0; m < M; ++m)
    if (attrs[m] >= s->volume->grid.numAttributes)
      fail("invalid attribute index", VKL_INVALID_ARGUMENT);
  if (N == 0)
    return;
  if (!pts || !out)
    fail("NULL coordinates or output", VKL_INVALID_ARGUMENT);
  Device *d = s->device;
  if (s->volume->grid.temporal) {
    sampleTemporal(d, s, N, pts, times, out, M, attrs, false);
    return;
  }
  int runS = -1;
  staged(d, N, 12, pts, 4 * M, out, [&](uint64_t n, const void *din, void *dout) {
    if (M == 1 && binned(d, s, s->s.filter, n, (const float *)din, attrs[0], (float *)dout, false))
      return;
    if (M == 1 && rayRuns(d, s, s->s.filter, n, (const float *)din, attrs[0], (float *)dout, false, runS))
      return;
    launchSample(s->launchGrid(), s->s.filter, s->s.maxSamplingDepth, n, (const float *)din, M,
                 attrs, (float *)dout, d->stream);
  });
}

void gradientN(const VKLSampler *sampler, uint64_t N, const vkl_vec3f *pts, vkl_vec3f *out,
               uint32_t attr, const float *times = nullptr)
{
  Sampler *s = committedSampler(sampler);
  if (attr >= s->volume->grid.numAttributes)
    fail("invalid attribute index", VKL_INVALID_ARGUMENT);
  if (N == 0)
    return;
  if (!pts || !out)
    fail("NULL coordinates or output", VKL_INVALID_ARGUMENT);
  Device *d = s->device;
  if (s->volume->grid.temporal) {
    sampleTemporal(d, s, N, pts, times, out, 1, &attr, true);
    return;
  }
  int runS = -1;
  staged(d, N, 12, pts, 12, out, [&](uint64_t n, const void *din, void *dout) {
    if (binned(d, s, s->s.gradientFilter, n, (const float *)din, attr, (float *)dout, true))
      return;
    if (rayRuns(d, s, s->s.gradientFilter, n, (const float *)din, attr, (float *)dout, true, runS))
      return;
    launchGradient(s->launchGrid(), s->s.gradientFilter, s->s.maxSamplingDepth, n,
                   (const float *)din, attr, (float *)dout, d->stream);
  });
}

template <int W, class V>
void sampleW(const int *valid, const VKLSampler *sampler, const V *oc, float *samples,
             uint32_t M, const uint32_t *attrs, const float *times)
{
  vkl_vec3f pts[W];
  float tm[W];
  int idx[W];
  int n = 0;
  for (int i = 0; i < W; ++i)
    if (!valid || valid[i]) {
      pts[n] = {oc->x[i], oc->y[i], oc->z[i]};
      tm[n]  = times ? times[i] : 0.f;
      idx[n++] = i;
    }
  std::vector<float> out((size_t)W * M);
  sampleN(sampler, (uint64_t)n, pts, out.data(), M, attrs, tm);
  for (int k = 0; k < n; ++k)
    for (uint32_t m = 0; m < M; ++m)
      samples[m * W + idx[k]] = out[k * M + m];
}

template <int W, class V>
void gradientW(const int *valid, const VKLSampler *sampler, const V *oc, V *grads, uint32_t attr,
               const float *times)
{
  vkl_vec3f pts[W], out[W];
  float tm[W];
  int idx[W];
  int n = 0;
  for (int i = 0; i < W; ++i)
    if (!valid || valid[i]) {
      pts[n] = {oc->x[i], oc->y[i], oc->z[i]};
      tm[n]  = times ? times[i] : 0.f;
      idx[n++] = i;
    }
  gradientN(sampler, (uint64_t)n, pts, out, attr, tm);
  for (int k = 0; k < n; ++k) {
    grads->x[idx[k]] = out[k].x;
    grads->y[idx[k]] = out[k].y;
    grads->z[idx[k]] = out[k].z;
  }
}

// Layout of a per-ray iterator inside the caller's buffer.
constexpr uint32_t kIntervalMagic = 0x564b4c49u;  // "IKLV"
constexpr uint32_t kHitMagic      = 0x564b4c48u;
struct IterHeader {
  uint32_t magic;
  uint32_t pad;
  ManagedObject *context;
};

// The reference device's default callbacks (Device.cpp:27-54): log
// messages go to stdout as they are, errors to stderr as
// "OPENVKL ERROR [<code>]: <message>".
void logToStdout(void *, const char *msg) { std::fputs(msg, stdout); }
void logToStderr(void *, const char *msg) { std::fputs(msg, stderr); }
void logToNowhere(void *, const char *) {}
void errorToStderr(void *, VKLError e, const char *msg)
{
  std::fprintf(stderr, "OPENVKL ERROR [%d]: %s\n", (int)e, msg);
}
void errorToStdout(void *, VKLError e, const char *msg)
{
  std::fprintf(stdout, "OPENVKL ERROR [%d]: %s\n", (int)e, msg);
  std::fflush(stdout);
}
void errorToNowhere(void *, VKLError, const char *) {}

std::string lowerCase(std::string s)
{
  for (char &c : s)
    c = (char)std::tolower((unsigned char)c);
  return s;
}

// Device::commit (Device.cpp:135-199): the logLevel / logOutput /
// errorOutput parameters, each overridden by its OPENVKL_* environment
// variable.  OPENVKL_THREADS / numThreads and OPENVKL_FLUSH_DENORMALS /
// flushDenormals configure the reference's host tasking system; the cuda
// device has none, so they are read and ignored.
void configureFromEnvironment(Device *d)
{
  auto ip = d->intParams.find("logLevel");
  d->logLevel = ip != d->intParams.end() ? ip->second : VKL_LOG_INFO;
  if (const char *e = std::getenv("OPENVKL_LOG_LEVEL")) {
    const std::string v = lowerCase(e);
    if (v == "debug")
      d->logLevel = VKL_LOG_DEBUG;
    else if (v == "info")
      d->logLevel = VKL_LOG_INFO;
    else if (v == "warning")
      d->logLevel = VKL_LOG_WARNING;
    else if (v == "error")
      d->logLevel = VKL_LOG_ERROR;
    else if (v == "none")
      d->logLevel = VKL_LOG_NONE;
    else if (!v.empty())
      d->log(VKL_LOG_ERROR, "unknown OPENVKL_LOG_LEVEL env value; must be debug, info, warning, error or none");
  }
  auto param = [&](const char *name) {
    auto it = d->stringParams.find(name);
    return it == d->stringParams.end() ? std::string() : it->second;
  };
  const char *lo = std::getenv("OPENVKL_LOG_OUTPUT");
  const std::string logDst = lo ? std::string(lo) : param("logOutput");
  if (logDst == "cout") {
    d->logCb   = logToStdout;
    d->logUser = nullptr;
  } else if (logDst == "cerr") {
    d->logCb   = logToStderr;
    d->logUser = nullptr;
  } else if (logDst == "none") {
    d->logCb   = logToNowhere;
    d->logUser = nullptr;
  }
  const char *eo = std::getenv("OPENVKL_ERROR_OUTPUT");
  const std::string errDst = eo ? std::string(eo) : param("errorOutput");
  if (errDst == "cout") {
    d->errorCb   = errorToStdout;
    d->errorUser = nullptr;
  } else if (errDst == "cerr") {
    d->errorCb   = errorToStderr;
    d->errorUser = nullptr;
  } else if (errDst == "none") {
    d->errorCb   = errorToNowhere;
    d->errorUser = nullptr;
  }
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// Device.
// ---------------------------------------------------------------------------
void vklInit(void) {}

VKLDevice vklNewDevice(const char *name)
{
  try {
    if (!name || (std::strcmp(name, "cuda") != 0 && std::strcmp(name, "cuda_b200") != 0))
      return nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      cudaGetLastError();
      return nullptr;
    }
    Device *d = new Device();
    cudaGetDevice(&d->cudaDevice);
    d->logCb   = logToStdout;
    d->errorCb = errorToStderr;
    std::lock_guard<std::mutex> lock(g_devicesMutex);
    g_lastDevice = d;
    return (VKLDevice)d;
  } catch (...) {
    return nullptr;
  }
}

void vklDeviceSetLogCallback(VKLDevice dev, VKLLogCallback cb, void *user)
{
  if (!dev)
    return;
  ((Device *)dev)->logCb   = cb;
  ((Device *)dev)->logUser = user;
}

void vklDeviceSetErrorCallback(VKLDevice dev, VKLErrorCallback cb, void *user)
{
  if (!dev)
    return;
  ((Device *)dev)->errorCb   = cb;
  ((Device *)dev)->errorUser = user;
}

void vklDeviceSetInt(VKLDevice dev, const char *name, int x)
{
  if (!dev || !name)
    return;
  Device *d = (Device *)dev;
  d->intParams[name] = x;
  if (!std::strcmp(name, "logLevel"))
    d->logLevel = x;
  if (!std::strcmp(name, "binnedSampling"))
    d->binning = x != 0;
  if (!std::strcmp(name, "textureSampling"))
    d->textureSampling = x != 0;
  if (!std::strcmp(name, "rayRunSampling"))
    d->rayRuns = x != 0;
}

void vklDeviceSetString(VKLDevice dev, const char *name, const char *s)
{
  if (!dev || !name)
    return;
  ((Device *)dev)->stringParams[name] = s ? s : "";
}

void vklDeviceSetVoidPtr(VKLDevice dev, const char *name, void *v)
{
  if (!dev || !name)
    return;
  Device *d = (Device *)dev;
  if (!std::strcmp(name, "cudaStream"))
    d->stream = (cudaStream_t)v;
  else if (!std::strcmp(name, "errorUserData"))
    d->errorUser = v;
  else if (!std::strcmp(name, "logUserData"))
    d->logUser = v;
}

void vklCommitDevice(VKLDevice dev)
{
  if (!dev)
    return;
  Device *d = (Device *)dev;
  guardedVoid(d, [&]() {
    auto it = d->intParams.find("cudaDevice");
    if (it != d->intParams.end()) {
      d->cudaDevice = it->second;
      cudaCheck(cudaSetDevice(d->cudaDevice), "cudaSetDevice");
    }
    configureFromEnvironment(d);
    d->committed = true;
  });
}

VKLError vklDeviceGetLastErrorCode(VKLDevice dev)
{
  return dev ? ((Device *)dev)->lastErrorCode : VKL_INVALID_ARGUMENT;
}

const char *vklDeviceGetLastErrorMsg(VKLDevice dev)
{
  return dev ? ((Device *)dev)->lastErrorMsg.c_str() : "invalid device";
}

int vklGetNativeSIMDWidth(VKLDevice) { return 32; }

void vklCommit(VKLObject object)
{
  Device *d = deviceOf(object);
  guardedVoid(d, [&]() {
    if (!object.host)
      fail("vklCommit: NULL handle", VKL_INVALID_ARGUMENT);
    ManagedObject *o = (ManagedObject *)object.host;
    o->commit();
  });
}

void vklRelease(VKLObject object)
{
  Device *d = deviceOf(object);
  guardedVoid(d, [&]() {
    if (object.host)
      ((ManagedObject *)object.host)->refDec();
  });
}

void vklReleaseDevice(VKLDevice dev)
{
  if (!dev)
    return;
  {
    std::lock_guard<std::mutex> lock(g_devicesMutex);
    if (g_lastDevice == (Device *)dev)
      g_lastDevice = nullptr;
  }
  ((Device *)dev)->refDec();  // freed when its last object goes (vklReleaseDevice, API.cpp:298-303)
}

// ---------------------------------------------------------------------------
// Data.
// ---------------------------------------------------------------------------
VKLData vklNewData(VKLDevice dev, size_t numItems, VKLDataType type, const void *source,
                   VKLDataCreationFlags flags, size_t byteStride)
{
  Device *d = (Device *)dev;
  return guarded(
      d,
      [&]() -> VKLData {
        if (!d)
          fail("vklNewData: NULL device", VKL_INVALID_ARGUMENT);
        if (numItems && !source)
          fail("vklNewData: NULL source", VKL_INVALID_ARGUMENT);
        Data *data     = new Data();
        data->device   = d;
        data->type     = type;
        data->numItems = numItems;
        if (type & VKL_OBJECT) {
          const size_t stride = byteStride ? byteStride : sizeof(VKLObject);
          data->itemSize      = sizeof(VKLObject);
          for (size_t i = 0; i < numItems; ++i) {
            const VKLObject *o = (const VKLObject *)((const uint8_t *)source + i * stride);
            ManagedObject *m   = (ManagedObject *)o->host;
            if (m)
              m->refInc();
            data->objects.push_back(m);
          }
          return handleOf(data);
        }
        const size_t isz = sizeOfType(type);
        if (!isz) {
          delete data;
          fail("vklNewData: unsupported data type", VKL_INVALID_ARGUMENT);
        }
        data->itemSize      = isz;
        const size_t stride = byteStride ? byteStride : isz;
        const size_t bytes  = numItems * isz;
        const bool devSrc   = isDevicePtr(source);
        if (devSrc && stride == isz && (flags & VKL_DATA_SHARED_BUFFER)) {
          data->dev = source;  // shared device buffer: used in place
        } else if (devSrc) {
          data->owned.alloc(bytes);
          if (stride == isz)
            cudaCheck(cudaMemcpyAsync(data->owned.ptr, source, bytes, cudaMemcpyDeviceToDevice,
                                      d->stream),
                      "data copy");
          else
            cudaCheck(cudaMemcpy2DAsync(data->owned.ptr, isz, source, stride, isz, numItems,
                                        cudaMemcpyDeviceToDevice, d->stream),
                      "data copy");
          cudaCheck(cudaStreamSynchronize(d->stream), "data copy");
          data->dev = data->owned.ptr;
        } else if (stride == isz) {
          // compact host source: uploaded from the caller's memory (a DMA
          // when it is pinned); small arrays also keep a host copy
          data->owned.alloc(bytes);
          cudaCheck(cudaMemcpyAsync(data->owned.ptr, source, bytes, cudaMemcpyHostToDevice, d->stream),
                    "data upload");
          if (bytes <= (64u << 20))
            data->host.assign((const uint8_t *)source, (const uint8_t *)source + bytes);
          cudaCheck(cudaStreamSynchronize(d->stream), "data upload");
          data->dev = data->owned.ptr;
        } else {
          // strided host source: compacted on the host first
          std::vector<uint8_t> compact(bytes);
          for (size_t i = 0; i < numItems; ++i)
            std::memcpy(&compact[i * isz], (const uint8_t *)source + i * stride, isz);
          data->owned.alloc(bytes);
          cudaCheck(cudaMemcpy(data->owned.ptr, compact.data(), bytes, cudaMemcpyHostToDevice),
                    "data upload");
          data->dev = data->owned.ptr;
          if (bytes <= (64u << 20))
            data->host.swap(compact);
        }
        return handleOf(data, (void *)data->dev);
      },
      VKLData{nullptr, nullptr});
}

// ---------------------------------------------------------------------------
// Volumes and parameters.
// ---------------------------------------------------------------------------
VKLVolume vklNewVolume(VKLDevice dev, const char *type)
{
  Device *d = (Device *)dev;
  return guarded(
      d,
      [&]() -> VKLVolume {
        if (!d)
          fail("vklNewVolume: NULL device", VKL_INVALID_ARGUMENT);
        const std::string t = type ? type : "";
        if (t != "structuredRegular" && t != "vdb")
          fail("unsupported volume type '" + t + "' on the cuda device", VKL_INVALID_ARGUMENT);
        Volume *v  = new Volume();
        v->device  = d;
        v->isDense = (t == "structuredRegular");
        return handleOf(v);
      },
      VKLVolume{nullptr, nullptr});
}

vkl_box3f vklGetBoundingBox(VKLVolume volume)
{
  return guarded(
      deviceOf(volume),
      [&]() -> vkl_box3f {
        Volume *v = objectAs<Volume>(volume, "volume");
        if (!v->committed)
          fail("volume is not committed", VKL_INVALID_OPERATION);
        return v->bounds;
      },
      vkl_box3f{{kNaN, kNaN, kNaN}, {kNaN, kNaN, kNaN}});
}

unsigned int vklGetNumAttributes(VKLVolume volume)
{
  return guarded(
      deviceOf(volume),
      [&]() -> unsigned int {
        Volume *v = objectAs<Volume>(volume, "volume");
        return v->committed ? v->grid.numAttributes : 0u;
      },
      0u);
}

vkl_range1f vklGetValueRange(VKLVolume volume, unsigned int attr)
{
  return guarded(
      deviceOf(volume),
      [&]() -> vkl_range1f {
        Volume *v = objectAs<Volume>(volume, "volume");
        if (!v->committed || attr >= v->grid.numAttributes)
          fail("invalid attribute index or uncommitted volume", VKL_INVALID_ARGUMENT);
        return vkl_range1f{v->rangeLo[attr], v->rangeHi[attr]};
      },
      vkl_range1f{kNaN, kNaN});
}

void vklSetParam(VKLObject object, const char *name, VKLDataType type, const void *mem)
{
  guardedVoid(deviceOf(object), [&]() {
    if (!object.host)
      fail("vklSetParam: NULL handle", VKL_INVALID_ARGUMENT);
    ((ManagedObject *)object.host)->setParam(name, type, mem);
  });
}

void vklSetBool(VKLObject o, const char *name, int b)
{
  const int v = b ? 1 : 0;
  vklSetParam(o, name, VKL_BOOL, &v);
}
void vklSetFloat(VKLObject o, const char *name, float x) { vklSetParam(o, name, VKL_FLOAT, &x); }
void vklSetInt(VKLObject o, const char *name, int x) { vklSetParam(o, name, VKL_INT, &x); }
void vklSetVec3f(VKLObject o, const char *name, float x, float y, float z)
{
  const float v[3] = {x, y, z};
  vklSetParam(o, name, VKL_VEC3F, v);
}
void vklSetVec3i(VKLObject o, const char *name, int x, int y, int z)
{
  const int v[3] = {x, y, z};
  vklSetParam(o, name, VKL_VEC3I, v);
}
void vklSetData(VKLObject o, const char *name, VKLData data) { vklSetParam(o, name, VKL_DATA, &data); }
void vklSetString(VKLObject o, const char *name, const char *s) { vklSetParam(o, name, VKL_STRING, s); }
void vklSetVoidPtr(VKLObject o, const char *name, void *v) { vklSetParam(o, name, VKL_VOID_PTR, &v); }

// ---------------------------------------------------------------------------
// Samplers.
// ---------------------------------------------------------------------------
VKLSampler vklNewSampler(VKLVolume volume)
{
  return guarded(
      deviceOf(volume),
      [&]() -> VKLSampler {
        Volume *v = objectAs<Volume>(volume, "volume");
        if (!v->committed)
          fail("vklNewSampler: volume is not committed", VKL_INVALID_OPERATION);
        Sampler *s = new Sampler();
        s->device  = v->device;
        s->volume  = Ref<Volume>(v);
        s->commit();
        return handleOf(s, s->devState.ptr);
      },
      VKLSampler{nullptr, nullptr});
}

VKLFeatureFlags vklGetFeatureFlags(VKLSampler sampler)
{
  return guarded(
      deviceOf(sampler),
      [&]() -> VKLFeatureFlags {
        Sampler *s = objectAs<Sampler>(sampler, "sampler");
        VKLFeatureFlags ff = s->volume->isDense ? (1u << 0) : (1u << 5);
        auto filterBit = [](int f, int base) -> VKLFeatureFlags {
          return f == VKL_FILTER_NEAREST ? (1u << base)
                 : f == VKL_FILTER_LINEAR ? (1u << (base + 1))
                                          : (1u << (base + 2));
        };
        ff |= filterBit(s->s.filter, 6) | filterBit(s->s.gradientFilter, 9);
        // temporal format (VKLFeatureFlagsInternal.h:32-34): constant,
        // structured or unstructured
        const uint32_t tf = s->volume->grid.temporal;
        ff |= tf == 1 ? (1u << 13) : tf == 2 ? (1u << 14) : (1u << 12);
        ff |= (s->volume->isDense || !s->volume->has("nodesPackedDense")) ? (1u << 20) : (1u << 19);
        return ff;
      },
      (VKLFeatureFlags)0);
}

// ---------------------------------------------------------------------------
// Sampling.
// ---------------------------------------------------------------------------
float vklComputeSample(const VKLSampler *sampler, const vkl_vec3f *oc, unsigned int attr,
                       float time)
{
  return guarded(
      sampler ? deviceOf(*sampler) : g_lastDevice,
      [&]() -> float {
        float out = kNaN;
        sampleN(sampler, 1, oc, &out, 1, &attr, &time);
        return out;
      },
      kNaN);
}

void vklComputeSample4(const int *valid, const VKLSampler *s, const vkl_vvec3f4 *oc,
                       float *samples, unsigned int attr, const float *times)
{
  guardedVoid(s ? deviceOf(*s) : g_lastDevice,
              [&]() { sampleW<4>(valid, s, oc, samples, 1, &attr, times); });
}
void vklComputeSample8(const int *valid, const VKLSampler *s, const vkl_vvec3f8 *oc,
                       float *samples, unsigned int attr, const float *times)
{
  guardedVoid(s ? deviceOf(*s) : g_lastDevice,
              [&]() { sampleW<8>(valid, s, oc, samples, 1, &attr, times); });
}
void vklComputeSample16(const int *valid, const VKLSampler *s, const vkl_vvec3f16 *oc,
                        float *samples, unsigned int attr, const float *times)
{
  guardedVoid(s ? deviceOf(*s) : g_lastDevice,
              [&]() { sampleW<16>(valid, s, oc, samples, 1, &attr, times); });
}

void vklComputeSampleM4(const int *valid, const VKLSampler *s, const vkl_vvec3f4 *oc, float *samples,
                        unsigned int M, const unsigned int *attrs, const float *times)
{
  guardedVoid(s ? deviceOf(*s) : g_lastDevice, [&]() { sampleW<4>(valid, s, oc, samples, M, attrs, times); });
}
void vklComputeSampleM8(const int *valid, const VKLSampler *s, const vkl_vvec3f8 *oc, float *samples,
                        unsigned int M, const unsigned int *attrs, const float *times)
{
  guardedVoid(s ? deviceOf(*s) : g_lastDevice, [&]() { sampleW<8>(valid, s, oc, samples, M, attrs, times); });
}
void vklComputeSampleM16(const int *valid, const VKLSampler *s, const vkl_vvec3f16 *oc, float *samples,
                         unsigned int M, const unsigned int *attrs, const float *times)
{
  guardedVoid(s ? deviceOf(*s) : g_lastDevice, [&]() { sampleW<16>(valid, s, oc, samples, M, attrs, times); });
}

void vklComputeGradient4(const int *valid, const VKLSampler *s, const vkl_vvec3f4 *oc, vkl_vvec3f4 *grads,
                         unsigned int attr, const float *times)
{
  guardedVoid(s ? deviceOf(*s) : g_lastDevice, [&]() { gradientW<4>(valid, s, oc, grads, attr, times); });
}
void vklComputeGradient8(const int *valid, const VKLSampler *s, const vkl_vvec3f8 *oc, vkl_vvec3f8 *grads,
                         unsigned int attr, const float *times)
{
  guardedVoid(s ? deviceOf(*s) : g_lastDevice, [&]() { gradientW<8>(valid, s, oc, grads, attr, times); });
}
void vklComputeGradient16(const int *valid, const VKLSampler *s, const vkl_vvec3f16 *oc,
                          vkl_vvec3f16 *grads, unsigned int attr, const float *times)
{
  guardedVoid(s ? deviceOf(*s) : g_lastDevice, [&]() { gradientW<16>(valid, s, oc, grads, attr, times); });
}

void vklComputeSampleN(const VKLSampler *sampler, unsigned int N, const vkl_vec3f *oc,
                       float *samples, unsigned int attr, const float *times)
{
  guardedVoid(sampler ? deviceOf(*sampler) : g_lastDevice,
              [&]() { sampleN(sampler, N, oc, samples, 1, &attr, times); });
}

void vklComputeSampleM(const VKLSampler *sampler, const vkl_vec3f *oc, float *samples,
                       unsigned int M, const unsigned int *attrs, float time)
{
  guardedVoid(sampler ? deviceOf(*sampler) : g_lastDevice,
              [&]() { sampleN(sampler, 1, oc, samples, M, attrs, &time); });
}

void vklComputeSampleMN(const VKLSampler *sampler, unsigned int N, const vkl_vec3f *oc,
                        float *samples, unsigned int M, const unsigned int *attrs,
                        const float *times)
{
  guardedVoid(sampler ? deviceOf(*sampler) : g_lastDevice,
              [&]() { sampleN(sampler, N, oc, samples, M, attrs, times); });
}

vkl_vec3f vklComputeGradient(const VKLSampler *sampler, const vkl_vec3f *oc, unsigned int attr,
                             float time)
{
  return guarded(
      sampler ? deviceOf(*sampler) : g_lastDevice,
      [&]() -> vkl_vec3f {
        vkl_vec3f g{kNaN, kNaN, kNaN};
        gradientN(sampler, 1, oc, &g, attr, &time);
        return g;
      },
      vkl_vec3f{kNaN, kNaN, kNaN});
}

void vklComputeGradientN(const VKLSampler *sampler, unsigned int N, const vkl_vec3f *oc,
                         vkl_vec3f *gradients, unsigned int attr, const float *times)
{
  guardedVoid(sampler ? deviceOf(*sampler) : g_lastDevice,
              [&]() { gradientN(sampler, N, oc, gradients, attr, times); });
}

// ---------------------------------------------------------------------------
// Iterator contexts.
// ---------------------------------------------------------------------------
VKLIntervalIteratorContext vklNewIntervalIteratorContext(VKLSampler sampler)
{
  return guarded(
      deviceOf(sampler),
      [&]() -> VKLIntervalIteratorContext {
        Sampler *s         = objectAs<Sampler>(sampler, "sampler");
        IntervalContext *c = new IntervalContext();
        c->device          = s->device;
        c->sampler         = Ref<Sampler>(s);
        c->commit();
        return handleOf(c, c->devState.ptr);
      },
      VKLIntervalIteratorContext{nullptr, nullptr});
}

VKLHitIteratorContext vklNewHitIteratorContext(VKLSampler sampler)
{
  return guarded(
      deviceOf(sampler),
      [&]() -> VKLHitIteratorContext {
        Sampler *s    = objectAs<Sampler>(sampler, "sampler");
        HitContext *c = new HitContext();
        c->device     = s->device;
        c->sampler    = Ref<Sampler>(s);
        c->commit();
        return handleOf(c, c->devState.ptr);
      },
      VKLHitIteratorContext{nullptr, nullptr});
}

size_t vklGetIntervalIteratorSize(const VKLIntervalIteratorContext *)
{
  return sizeof(IterHeader) + intervalIterStateSize();
}

size_t vklGetHitIteratorSize(const VKLHitIteratorContext *)
{
  return sizeof(IterHeader) + hitIterStateSize();
}

VKLIntervalIterator vklInitIntervalIterator(const VKLIntervalIteratorContext *context,
                                            const vkl_vec3f *origin, const vkl_vec3f *direction,
                                            const vkl_range1f *tRange, float /*time*/,
                                            void *buffer)
{
  return guarded(
      context ? deviceOf(*context) : g_lastDevice,
      [&]() -> VKLIntervalIterator {
        if (!context || !buffer || !origin || !direction || !tRange)
          fail("vklInitIntervalIterator: NULL argument", VKL_INVALID_ARGUMENT);
        IntervalContext *c = objectAs<IntervalContext>(*context, "interval iterator context");
        if (c->macrocells)
          fail("vklInitIntervalIterator: macrocell intervals (context parameter \"macrocells\") are "
               "produced by vklIterateIntervalsN",
               VKL_INVALID_OPERATION);
        Device *d          = c->device;
        IterHeader *h      = (IterHeader *)buffer;
        h->magic           = kIntervalMagic;
        h->context         = c;
        const float ray[8] = {origin->x, origin->y, origin->z, direction->x, direction->y,
                              direction->z, tRange->lower, tRange->upper};
        std::lock_guard<std::mutex> lock(d->stagingMutex);
        const size_t ss = intervalIterStateSize();
        d->stageAux.reserve(ss + 64);
        cudaCheck(cudaMemcpyAsync(d->stageAux.as<uint8_t>() + ss, ray, sizeof(ray),
                                  cudaMemcpyHostToDevice, d->stream),
                  "iterator init");
        launchIntervalIterInit(c->sampler->volume->grid, c->attr, c->depth,
                               (const float *)(d->stageAux.as<uint8_t>() + ss), d->stageAux.ptr,
                               d->stream);
        cudaCheck(cudaMemcpyAsync(h + 1, d->stageAux.ptr, ss, cudaMemcpyDeviceToHost, d->stream),
                  "iterator init");
        cudaCheck(cudaStreamSynchronize(d->stream), "iterator init");
        return (VKLIntervalIterator)buffer;
      },
      (VKLIntervalIterator) nullptr);
}

int vklIterateInterval(VKLIntervalIterator iterator, VKLInterval *interval)
{
  IterHeader *h = (IterHeader *)iterator;
  Device *d     = (h && h->magic == kIntervalMagic) ? h->context->device : g_lastDevice;
  return guarded(
      d,
      [&]() -> int {
        if (!h || h->magic != kIntervalMagic || !interval)
          fail("vklIterateInterval: invalid iterator", VKL_INVALID_ARGUMENT);
        IntervalContext *c = (IntervalContext *)h->context;
        std::lock_guard<std::mutex> lock(d->stagingMutex);
        const size_t ss = intervalIterStateSize();
        d->stageAux.reserve(ss + 64);
        uint8_t *base = d->stageAux.as<uint8_t>();
        cudaCheck(cudaMemcpyAsync(base, h + 1, ss, cudaMemcpyHostToDevice, d->stream), "iterate");
        DevInterval *dOut = (DevInterval *)(base + ((ss + 15) & ~size_t(15)));
        int *dRes         = (int *)(dOut + 1);
        launchIntervalIterNext(c->sampler->volume->grid, c->devValueRanges(), base, dOut, dRes,
                               d->stream);
        struct {
          DevInterval iv;
          int res;
        } out;
        cudaCheck(cudaMemcpyAsync(h + 1, base, ss, cudaMemcpyDeviceToHost, d->stream), "iterate");
        cudaCheck(cudaMemcpyAsync(&out, dOut, sizeof(out), cudaMemcpyDeviceToHost, d->stream),
                  "iterate");
        cudaCheck(cudaStreamSynchronize(d->stream), "iterate");
        if (out.res) {
          interval->tRange        = {out.iv.t0, out.iv.t1};
          interval->valueRange    = {out.iv.v0, out.iv.v1};
          interval->nominalDeltaT = out.iv.nominalDeltaT;
        }
        return out.res;
      },
      0);
}

VKLHitIterator vklInitHitIterator(const VKLHitIteratorContext *context, const vkl_vec3f *origin,
                                  const vkl_vec3f *direction, const vkl_range1f *tRange,
                                  float time, void *buffer)
{
  return guarded(
      context ? deviceOf(*context) : g_lastDevice,
      [&]() -> VKLHitIterator {
        if (!context || !buffer || !origin || !direction || !tRange)
          fail("vklInitHitIterator: NULL argument", VKL_INVALID_ARGUMENT);
        HitContext *c      = objectAs<HitContext>(*context, "hit iterator context");
        Device *d          = c->device;
        IterHeader *h      = (IterHeader *)buffer;
        h->magic           = kHitMagic;
        h->context         = c;
        // the ray, its t range and the time its samples are taken at
        // (temporally varying volumes)
        const float ray[9] = {origin->x, origin->y, origin->z, direction->x, direction->y,
                              direction->z, tRange->lower, tRange->upper, time};
        std::lock_guard<std::mutex> lock(d->stagingMutex);
        const size_t ss = hitIterStateSize();
        d->stageAux.reserve(ss + 64);
        cudaCheck(cudaMemcpyAsync(d->stageAux.as<uint8_t>() + ss, ray, sizeof(ray),
                                  cudaMemcpyHostToDevice, d->stream),
                  "iterator init");
        launchHitIterInit(c->sampler->launchGrid(), c->attr, c->depth,
                          (const float *)(d->stageAux.as<uint8_t>() + ss), d->stageAux.ptr,
                          d->stream);
        cudaCheck(cudaMemcpyAsync(h + 1, d->stageAux.ptr, ss, cudaMemcpyDeviceToHost, d->stream),
                  "iterator init");
        cudaCheck(cudaStreamSynchronize(d->stream), "iterator init");
        return (VKLHitIterator)buffer;
      },
      (VKLHitIterator) nullptr);
}

int vklIterateHit(VKLHitIterator iterator, VKLHit *hit)
{
  IterHeader *h = (IterHeader *)iterator;
  Device *d     = (h && h->magic == kHitMagic) ? h->context->device : g_lastDevice;
  return guarded(
      d,
      [&]() -> int {
        if (!h || h->magic != kHitMagic || !hit)
          fail("vklIterateHit: invalid iterator", VKL_INVALID_ARGUMENT);
        HitContext *c = (HitContext *)h->context;
        std::lock_guard<std::mutex> lock(d->stagingMutex);
        const size_t ss = hitIterStateSize();
        d->stageAux.reserve(ss + 64);
        uint8_t *base = d->stageAux.as<uint8_t>();
        cudaCheck(cudaMemcpyAsync(base, h + 1, ss, cudaMemcpyHostToDevice, d->stream), "iterate");
        DevHit *dOut = (DevHit *)(base + ((ss + 15) & ~size_t(15)));
        int *dRes    = (int *)(dOut + 1);
        launchHitIterNext(c->sampler->launchGrid(), c->sampler->s.filter, c->devValueRanges(),
                          (uint32_t)c->values.size(), c->devValues.as<float>(), base, dOut, dRes,
                          d->stream);
        struct {
          DevHit hit;
          int res;
        } out;
        cudaCheck(cudaMemcpyAsync(h + 1, base, ss, cudaMemcpyDeviceToHost, d->stream), "iterate");
        cudaCheck(cudaMemcpyAsync(&out, dOut, sizeof(out), cudaMemcpyDeviceToHost, d->stream),
                  "iterate");
        cudaCheck(cudaStreamSynchronize(d->stream), "iterate");
        if (out.res) {
          hit->t       = out.hit.t;
          hit->sample  = out.hit.sample;
          hit->epsilon = out.hit.epsilon;
        }
        return out.res;
      },
      0);
}

void vklIterateIntervalsN(const VKLIntervalIteratorContext *context, unsigned int N,
                          const vkl_vec3f *origins, const vkl_vec3f *directions,
                          const vkl_range1f *tRanges, unsigned int maxPerRay,
                          VKLInterval *intervals, unsigned int *counts)
{
  guardedVoid(context ? deviceOf(*context) : g_lastDevice, [&]() {
    if (!context)
      fail("NULL context", VKL_INVALID_ARGUMENT);
    IntervalContext *c = objectAs<IntervalContext>(*context, "interval iterator context");
    Device *d          = c->device;
    if (!N)
      return;
    const bool dev = isDevicePtr(origins) && isDevicePtr(directions) && isDevicePtr(tRanges) &&
                     isDevicePtr(counts) && (maxPerRay == 0 || isDevicePtr(intervals));
    const DevGrid &g = c->sampler->volume->grid;
    const float *macro = c->macrocells ? c->sampler->volume->macrocellRanges(c->attr, d->stream) : nullptr;
    auto launch = [&](const float *o, const float *dr, const float *t, DevInterval *iv, uint32_t *cnt) {
      if (macro)
        launchMacrocellIntervals(g, macro, c->devValueRanges(), N, o, dr, t, maxPerRay, iv, cnt, d->stream);
      else
        launchIntervals(g, c->attr, c->depth, c->devValueRanges(), N, o, dr, t, maxPerRay, iv, cnt, d->stream);
    };
    if (dev) {
      launch((const float *)origins, (const float *)directions, (const float *)tRanges, (DevInterval *)intervals,
             counts);
      return;
    }
    std::lock_guard<std::mutex> lock(d->stagingMutex);
    const size_t inB = (size_t)N * 32, outB = (size_t)N * maxPerRay * 20 + (size_t)N * 4;
    d->stageIn.reserve(inB);
    d->stageOut.reserve(outB);
    uint8_t *in = d->stageIn.as<uint8_t>(), *out = d->stageOut.as<uint8_t>();
    cudaCheck(cudaMemcpyAsync(in, origins, N * 12, cudaMemcpyHostToDevice, d->stream), "stage");
    cudaCheck(cudaMemcpyAsync(in + N * 12, directions, N * 12, cudaMemcpyHostToDevice, d->stream),
              "stage");
    cudaCheck(cudaMemcpyAsync(in + N * 24, tRanges, N * 8, cudaMemcpyHostToDevice, d->stream),
              "stage");
    DevInterval *dIv = (DevInterval *)out;
    uint32_t *dCnt   = (uint32_t *)(out + (size_t)N * maxPerRay * 20);
    launch((const float *)in, (const float *)(in + N * 12), (const float *)(in + N * 24), dIv, dCnt);
    if (maxPerRay)
      cudaCheck(cudaMemcpyAsync(intervals, dIv, (size_t)N * maxPerRay * 20, cudaMemcpyDeviceToHost,
                                d->stream),
                "stage");
    cudaCheck(cudaMemcpyAsync(counts, dCnt, (size_t)N * 4, cudaMemcpyDeviceToHost, d->stream),
              "stage");
    cudaCheck(cudaStreamSynchronize(d->stream), "synchronize");
  });
}

void vklIterateHitsN(const VKLHitIteratorContext *context, unsigned int N,
                     const vkl_vec3f *origins, const vkl_vec3f *directions,
                     const vkl_range1f *tRanges, unsigned int maxPerRay, VKLHit *hits,
                     unsigned int *counts)
{
  guardedVoid(context ? deviceOf(*context) : g_lastDevice, [&]() {
    if (!context)
      fail("NULL context", VKL_INVALID_ARGUMENT);
    HitContext *c = objectAs<HitContext>(*context, "hit iterator context");
    Device *d     = c->device;
    if (!N)
      return;
    const bool dev = isDevicePtr(origins) && isDevicePtr(directions) && isDevicePtr(tRanges) &&
                     isDevicePtr(counts) && (maxPerRay == 0 || isDevicePtr(hits));
    const DevGrid g = c->sampler->launchGrid();
    const int filter = c->sampler->s.filter;
    if (dev) {
      launchHits(g, c->attr, filter, c->depth, c->devValueRanges(), (uint32_t)c->values.size(),
                 c->devValues.as<float>(), N, (const float *)origins, (const float *)directions,
                 (const float *)tRanges, maxPerRay, (DevHit *)hits, counts, d->stream);
      return;
    }
    std::lock_guard<std::mutex> lock(d->stagingMutex);
    const size_t inB = (size_t)N * 32, outB = (size_t)N * maxPerRay * 12 + (size_t)N * 4;
    d->stageIn.reserve(inB);
    d->stageOut.reserve(outB);
    uint8_t *in = d->stageIn.as<uint8_t>(), *out = d->stageOut.as<uint8_t>();
    cudaCheck(cudaMemcpyAsync(in, origins, N * 12, cudaMemcpyHostToDevice, d->stream), "stage");
    cudaCheck(cudaMemcpyAsync(in + N * 12, directions, N * 12, cudaMemcpyHostToDevice, d->stream),
              "stage");
    cudaCheck(cudaMemcpyAsync(in + N * 24, tRanges, N * 8, cudaMemcpyHostToDevice, d->stream),
              "stage");
    DevHit *dHit   = (DevHit *)out;
    uint32_t *dCnt = (uint32_t *)(out + (size_t)N * maxPerRay * 12);
    launchHits(g, c->attr, filter, c->depth, c->devValueRanges(), (uint32_t)c->values.size(),
               c->devValues.as<float>(), N, (const float *)in, (const float *)(in + N * 12),
               (const float *)(in + N * 24), maxPerRay, dHit, dCnt, d->stream);
    if (maxPerRay)
      cudaCheck(cudaMemcpyAsync(hits, dHit, (size_t)N * maxPerRay * 12, cudaMemcpyDeviceToHost,
                                d->stream),
                "stage");
    cudaCheck(cudaMemcpyAsync(counts, dCnt, (size_t)N * 4, cudaMemcpyDeviceToHost, d->stream),
              "stage");
    cudaCheck(cudaStreamSynchronize(d->stream), "synchronize");
  });
}

// ---------------------------------------------------------------------------
// Observers.
// ---------------------------------------------------------------------------
VKLObserver vklNewVolumeObserver(VKLVolume volume, const char *type)
{
  return guarded(
      deviceOf(volume),
      [&]() -> VKLObserver {
        Volume *v = objectAs<Volume>(volume, "volume");
        if (!v->committed)
          fail("Trying to create an observer on a vdb volume that was not committed.",
               VKL_INVALID_OPERATION);
        const std::string t = type ? type : "";
        if (t != "InnerNode")
          fail("unsupported volume observer type '" + t + "'", VKL_INVALID_ARGUMENT);
        Observer *o = new Observer();
        o->device   = v->device;
        o->volume   = Ref<Volume>(v);
        o->kind     = t;
        return handleOf(o);
      },
      VKLObserver{nullptr, nullptr});
}

VKLObserver vklNewSamplerObserver(VKLSampler sampler, const char *type)
{
  return guarded(
      deviceOf(sampler),
      [&]() -> VKLObserver {
        Sampler *s          = objectAs<Sampler>(sampler, "sampler");
        const std::string t = type ? type : "";
        // VdbSampler::newObserver (VdbSampler.cpp:280-290): LeafNodeAccess on
        // vdb volumes; a uint32 per leaf, set to 1 where sampling reached it
        if (t != "LeafNodeAccess" || s->volume->isDense)
          fail("unsupported sampler observer type '" + t + "'", VKL_INVALID_ARGUMENT);
        if (s->leafObservers.size() >= kMaxLeafObservers)
          fail("too many LeafNodeAccess observers on one sampler", VKL_INVALID_OPERATION);
        Observer *o    = new Observer();
        o->device      = s->device;
        o->sampler     = Ref<Sampler>(s);
        o->kind        = t;
        o->numElements = s->volume->grid.numLeaves;
        o->devCounters.alloc(std::max<size_t>(4, o->numElements * 4));
        cudaCheck(cudaMemset(o->devCounters.ptr, 0, o->devCounters.bytes), "memset");
        s->leafObservers.push_back(o);
        s->uploadState();
        return handleOf(o);
      },
      VKLObserver{nullptr, nullptr});
}

const void *vklMapObserver(VKLObserver observer)
{
  return guarded(
      deviceOf(observer),
      [&]() -> const void * {
        Observer *o = objectAs<Observer>(observer, "observer");
        o->commit();
        if (o->kind == "LeafNodeAccess")
          return (const void *)o->leafAccess.data();
        return (const void *)o->buffer.data();
      },
      (const void *)nullptr);
}

void vklUnmapObserver(VKLObserver) {}

VKLDataType vklGetObserverElementType(VKLObserver observer)
{
  return guarded(
      deviceOf(observer),
      [&]() -> VKLDataType {
        return objectAs<Observer>(observer, "observer")->kind == "LeafNodeAccess" ? VKL_UINT : VKL_OBJECT;
      },
      VKL_UNKNOWN);
}

size_t vklGetObserverElementSize(VKLObserver observer)
{
  return guarded(
      deviceOf(observer),
      [&]() -> size_t {
        const Observer *o = objectAs<Observer>(observer, "observer");
        return o->kind == "LeafNodeAccess" ? sizeof(uint32_t) : o->elementFloats * 4;
      },
      (size_t)0);
}

size_t vklGetObserverNumElements(VKLObserver observer)
{
  return guarded(
      deviceOf(observer),
      [&]() -> size_t { return objectAs<Observer>(observer, "observer")->numElements; },
      (size_t)0);
}

uint64_t vklCudaGetTreeLevel(VKLVolume volume, unsigned int level, uint64_t *voxels,
                             float *valueRanges, uint32_t *origins)
{
  return guarded(
      deviceOf(volume),
      [&]() -> uint64_t {
        Volume *v = objectAs<Volume>(volume, "volume");
        if (!v->committed)
          fail("volume is not committed", VKL_INVALID_OPERATION);
        if (level >= kNumLevels)
          fail("invalid level", VKL_INVALID_ARGUMENT);
        if (level == kNumLevels - 1)
          return v->grid.numLeaves;
        const DevLevel &L = v->grid.levels[level];
        const uint64_t nv = L.numNodes * levelNumVoxels(level);
        if (voxels)
          cudaCheck(cudaMemcpy(voxels, L.voxels, nv * 8, cudaMemcpyDeviceToHost), "readback");
        if (valueRanges)
          cudaCheck(cudaMemcpy(valueRanges, L.valueRange, nv * 8 * v->grid.numAttributes,
                               cudaMemcpyDeviceToHost),
                    "readback");
        if (origins)
          cudaCheck(cudaMemcpy(origins, L.origin, L.numNodes * 12, cudaMemcpyDeviceToHost),
                    "readback");
        return L.numNodes;
      },
      (uint64_t)0);
}

}  // extern "C"
