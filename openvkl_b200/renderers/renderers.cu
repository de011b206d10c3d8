// The reference's example renderers as CUDA consumers of the cuda device's
// __device__ API (include/openvkl_cuda_device.h), headless: each kernel
// writes one RGBA float4 per pixel into a device framebuffer (the windowed
// GLFW/OpenGL display of the reference examples does not exist here).
//
//   ray march iterator       examples/interactive/renderer/ray_march_iterator/
//                            RayMarchIteratorGpuKernel.cpp:9-88
//   interval iterator debug  interval_iterator_debug/
//                            IntervalIteratorDebugGpuKernel.cpp:9-77
//   hit iterator renderer    hit_iterator_renderer/HitIteratorRendererGpuKernel.cpp:9-114
//   camera                   Camera.ih (Camera_createRay)
//   transfer function        RendererGpuKernel.h:64-93 (sampleTransferFunction)
//   box clip                 RendererGpuKernel.h:142-155 (intersectBox)
//   density path tracer      density_path_tracer/DensityPathTracerGpuKernel.cpp:
//                            9-170 (Woodcock tracking, isotropic scattering,
//                            progressive accumulation), Random.ih (RandomTEA)
//
// One ray per pixel, through the pixel centre.  The reference's approximate
// reciprocals and rsqrt (ISPC rcp / rsqrt, sycl::native::recip) are written
// as exact divisions and square roots, as in the oracle's restatement of the
// same renderers (oracle/vkl_oracle.cpp, orc_render).  Built with the
// library's --fmad=false, the images are bit-identical to it.
#include <cstdint>

#include "../../include/openvkl_cuda_device.h"
#include "pt_math.h"

extern "C" {

// Camera (Camera.ih): sensor width and focal length in world units, the
// rows of the camera-to-world rotation and its translation.
typedef struct {
  float sensorWidth, focalLength;
  float ctwR[9];
  float ctwT[3];
} VKLExampleCamera;

// Piecewise-linear transfer function over valueRange (TransferFunction.h).
#define VKL_EXAMPLE_MAX_TF 256
typedef struct {
  float valueRange[2];
  int numValues;
  float colorsAndOpacities[4 * VKL_EXAMPLE_MAX_TF];
} VKLExampleTransferFunction;

typedef struct {
  int width, height;
  unsigned int attributeIndex;
  float time;
  unsigned long long featureFlags;  // the sampler's (vklGetFeatureFlags)
  float bounds[6];  // volume bounding box (lower xyz, upper xyz)
  float samplingRate;                       // ray march iterator
  float intervalColorScale, intervalOpacity;  // interval iterator debug
  int firstIntervalOnly, showIntervalBorders;
} VKLExampleParams;

// Density path tracer parameters (DensityPathTracerParams.h) and the frame
// index that seeds each pixel's random sequence.
typedef struct {
  float shutter;
  int motionBlur;
  float sigmaTScale, sigmaSScale;
  int maxNumScatters;
  float ambientLightIntensity;
  int showBbox;
  unsigned int frame;
} VKLExamplePathTracerParams;

}  // extern "C"

namespace {

struct v3 {
  float x, y, z;
};
struct v4 {
  float x, y, z, w;
};
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 operator*(float s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 normalize(v3 a)
{
  const float l = sqrtf(dot(a, a));
  return {a.x / l, a.y / l, a.z / l};
}
__device__ __forceinline__ float clamp01(float x) { return fminf(fmaxf(x, 0.f), 1.f); }

// Camera_createRay (Camera.ih) at film position (px, py).
__device__ __forceinline__ void createRay(const VKLExampleCamera &c, int resX, int resY, float px, float py, v3 &org,
                                          v3 &dir)
{
  const float irx    = 1.f / (float)resX;
  const float sx     = (px - 0.5f * (float)resX) * irx;
  const float sy     = -(py - 0.5f * (float)resY) * irx;
  const v3 pCamera   = {c.sensorWidth * sx, c.sensorWidth * sy, 0.f};
  const v3 pAperture = {0.f, 0.f, -c.focalLength};
  const v3 dCamera   = pAperture - pCamera;
  const v3 R0 = {c.ctwR[0], c.ctwR[1], c.ctwR[2]}, R1 = {c.ctwR[3], c.ctwR[4], c.ctwR[5]},
           R2 = {c.ctwR[6], c.ctwR[7], c.ctwR[8]};
  org = {dot(R0, pCamera) + c.ctwT[0], dot(R1, pCamera) + c.ctwT[1], dot(R2, pCamera) + c.ctwT[2]};
  dir = normalize({dot(R0, dCamera), dot(R1, dCamera), dot(R2, dCamera)});
}

// intersectBox (RendererGpuKernel.h:142-155): [max of the slab entries and
// 0, min of the slab exits and +inf].
__device__ __forceinline__ vkl_range1f intersectBox(v3 o, v3 d, const float *b)
{
  const float rx = 1.f / d.x, ry = 1.f / d.y, rz = 1.f / d.z;
  const float x0 = (b[0] - o.x) * rx, y0 = (b[1] - o.y) * ry, z0 = (b[2] - o.z) * rz;
  const float x1 = (b[3] - o.x) * rx, y1 = (b[4] - o.y) * ry, z1 = (b[5] - o.z) * rz;
  vkl_range1f r;
  r.lower = fmaxf(fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fminf(z0, z1)), 0.f);
  r.upper = fminf(fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fmaxf(z0, z1)), __int_as_float(0x7f800000));
  return r;
}

// sampleTransferFunction (RendererGpuKernel.h:64-93).
__device__ __forceinline__ v4 transfer(const VKLExampleTransferFunction &tf, float value)
{
  const float *c = tf.colorsAndOpacities;
  if (isnan(value) || tf.numValues == 0)
    return {0.f, 0.f, 0.f, 0.f};
  if (value <= tf.valueRange[0])
    return {c[0], c[1], c[2], c[3]};
  const int last = tf.numValues - 1;
  if (value >= tf.valueRange[1])
    return {c[4 * last], c[4 * last + 1], c[4 * last + 2], c[4 * last + 3]};
  value                 = (value - tf.valueRange[0]) / (tf.valueRange[1] - tf.valueRange[0]) * (float)last;
  const int index       = (int)floorf(value);
  const float remainder = value - (float)index;
  const int next        = min(index + 1, last);
  const float a         = 1.f - remainder;
  return {a * c[4 * index] + remainder * c[4 * next], a * c[4 * index + 1] + remainder * c[4 * next + 1],
          a * c[4 * index + 2] + remainder * c[4 * next + 2], a * c[4 * index + 3] + remainder * c[4 * next + 3]};
}

constexpr int kThreads = 128;

__device__ __forceinline__ void pixelRay(const VKLExampleCamera &cam, const VKLExampleParams &prm, int idx, v3 &org,
                                         v3 &dir)
{
  createRay(cam, prm.width, prm.height, (float)(idx % prm.width) + 0.5f, (float)(idx / prm.width) + 0.5f, org, dir);
}

__global__ void __launch_bounds__(kThreads) kRayMarch(VKLSampler sampler, VKLIntervalIteratorContext context,
                                                      const __grid_constant__ VKLExampleCamera cam,
                                                      const __grid_constant__ VKLExampleTransferFunction tf,
                                                      const __grid_constant__ VKLExampleParams prm, float4 *out)
{
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= prm.width * prm.height)
    return;
  const VKLFeatureFlags ff = prm.featureFlags;
  v3 org, dir;
  pixelRay(cam, prm, idx, org, dir);
  const vkl_range1f tRange = intersectBox(org, dir, prm.bounds);
  alignas(16) char buffer[VKL_CUDA_INTERVAL_ITERATOR_SIZE];
  const vkl_vec3f o{org.x, org.y, org.z}, d{dir.x, dir.y, dir.z};
  VKLIntervalIterator it = vklInitIntervalIterator(&context, &o, &d, &tRange, prm.time, buffer, ff);
  VKLInterval interval;
  v3 color    = {0.f, 0.f, 0.f};
  float alpha = 0.f;
  while (vklIterateInterval(it, &interval, ff) && alpha < 0.99f) {
    const float nominalSamplingDt = interval.nominalDeltaT / prm.samplingRate;
    float lo = interval.tRange.lower;
    float hi = fminf(interval.tRange.lower + nominalSamplingDt, interval.tRange.upper);
    while (hi - lo > 0.f && alpha < 0.99f) {
      const float t  = 0.5f * (lo + hi);
      const float dt = hi - lo;
      const v3 c     = org + t * dir;
      const vkl_vec3f cv{c.x, c.y, c.z};
      const float sample         = vklComputeSample(&sampler, &cv, prm.attributeIndex, prm.time, ff);
      v4 sc                      = transfer(tf, sample);
      const float clampedOpacity = clamp01(sc.w * dt);
      sc    = {sc.x * clampedOpacity, sc.y * clampedOpacity, sc.z * clampedOpacity, sc.w * clampedOpacity};
      color = color + (1.f - alpha) * v3{sc.x, sc.y, sc.z};
      alpha = alpha + (1.f - alpha) * clampedOpacity;
      lo    = hi;
      hi    = fminf(lo + nominalSamplingDt, interval.tRange.upper);
    }
  }
  out[idx] = make_float4(color.x, color.y, color.z, 1.f);
}

__global__ void __launch_bounds__(kThreads) kIntervalDebug(VKLIntervalIteratorContext context,
                                                           const __grid_constant__ VKLExampleCamera cam,
                                                           const __grid_constant__ VKLExampleTransferFunction tf,
                                                           const __grid_constant__ VKLExampleParams prm, float4 *out)
{
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= prm.width * prm.height)
    return;
  const VKLFeatureFlags ff = prm.featureFlags;
  v3 org, dir;
  pixelRay(cam, prm, idx, org, dir);
  const vkl_range1f tRange = intersectBox(org, dir, prm.bounds);
  alignas(16) char buffer[VKL_CUDA_INTERVAL_ITERATOR_SIZE];
  const vkl_vec3f o{org.x, org.y, org.z}, d{dir.x, dir.y, dir.z};
  VKLIntervalIterator it = vklInitIntervalIterator(&context, &o, &d, &tRange, prm.time, buffer, ff);
  VKLInterval interval;
  int count   = 0;
  v3 color    = {0.f, 0.f, 0.f};
  float alpha = 0.f;
  while (vklIterateInterval(it, &interval, ff) && alpha < 0.99f) {
    count++;
    const float dt = interval.tRange.upper - interval.tRange.lower;
    const float normalizedValue =
        tf.valueRange[0] + (float)count / prm.intervalColorScale * (tf.valueRange[1] - tf.valueRange[0]);
    v4 sc                = transfer(tf, normalizedValue);
    sc.w                 = prm.intervalOpacity;
    float clampedOpacity = clamp01(sc.w * dt);
    sc = {sc.x * clampedOpacity, sc.y * clampedOpacity, sc.z * clampedOpacity, sc.w * clampedOpacity};
    if (prm.showIntervalBorders && dt < interval.nominalDeltaT) {
      sc             = {1.f, 1.f, 1.f, 1.f};
      clampedOpacity = 1.f;
    }
    color = color + (1.f - alpha) * v3{sc.x, sc.y, sc.z};
    alpha = alpha + (1.f - alpha) * clampedOpacity;
    if (prm.firstIntervalOnly)
      break;
  }
  out[idx] = make_float4(color.x, color.y, color.z, 1.f);
}

__global__ void __launch_bounds__(kThreads) kHitRenderer(VKLSampler sampler, VKLHitIteratorContext context,
                                                         const __grid_constant__ VKLExampleCamera cam,
                                                         const __grid_constant__ VKLExampleTransferFunction tf,
                                                         const __grid_constant__ VKLExampleParams prm, float4 *out)
{
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= prm.width * prm.height)
    return;
  const VKLFeatureFlags ff = prm.featureFlags;
  v3 org, dir;
  pixelRay(cam, prm, idx, org, dir);
  const vkl_range1f tRange = intersectBox(org, dir, prm.bounds);
  alignas(16) char buffer[VKL_CUDA_HIT_ITERATOR_SIZE];
  alignas(16) char shadowBuffer[VKL_CUDA_HIT_ITERATOR_SIZE];
  const vkl_vec3f o{org.x, org.y, org.z}, d{dir.x, dir.y, dir.z};
  VKLHitIterator it = vklInitHitIterator(&context, &o, &d, &tRange, prm.time, buffer, ff);
  VKLHit hit;
  const float surfaceAlpha = 0.6f;
  const float emission[2]  = {1.f, 0.8f};
  const v3 lightDir[2]     = {normalize({1.f, 1.f, 1.f}), normalize({1.f, 1.f, -1.f})};
  v3 color                 = {0.f, 0.f, 0.f};
  float alpha              = 0.f;
  while (vklIterateHit(it, &hit, ff) && alpha < 0.99f) {
    const v3 c = org + hit.t * dir;
    const vkl_vec3f cv{c.x, c.y, c.z};
    const vkl_vec3f grad = vklComputeGradient(&sampler, &cv, prm.attributeIndex, prm.time, ff);
    v3 N                 = normalize({grad.x, grad.y, grad.z});
    if (isnan(N.x) || isnan(N.y) || isnan(N.z))
      N = {0.f, 0.f, 0.f};
    const v3 wi    = normalize({-1.f * dir.x, -1.f * dir.y, -1.f * dir.z});
    const float ci = dot(N, wi);
    float illum    = 0.f;
    if (sqrtf(dot(N, N)) > 0.f) {
      illum = 0.1f;  // ambient
      for (int i = 0; i < 2; ++i) {
        const v3 wo    = lightDir[i];
        const float co = dot(N, wo);
        // shadow test only when the light is not behind the surface we hit
        if ((co > 0.f) == (ci > 0.f)) {
          vkl_range1f shadowRange;
          shadowRange.lower = hit.epsilon;
          shadowRange.upper = __int_as_float(0x7f800000);
          const vkl_vec3f wov{wo.x, wo.y, wo.z};
          VKLHitIterator sit = vklInitHitIterator(&context, &cv, &wov, &shadowRange, prm.time, shadowBuffer, ff);
          VKLHit shadowHit;
          if (!vklIterateHit(sit, &shadowHit, ff))
            illum += fabsf(co) * emission[i];
        }
      }
    } else {
      illum = 1.f;  // no normal: unshaded
    }
    const v4 sc = transfer(tf, hit.sample);
    color       = color + ((1.f - alpha) * illum) * v3{sc.x, sc.y, sc.z};
    alpha       = alpha + (1.f - alpha) * surfaceAlpha;
  }
  out[idx] = make_float4(color.x, color.y, color.z, 1.f);
}

// RandomTEA (Random.ih): 8 rounds of the tiny encryption algorithm per draw
// of two floats in [0, 1).
struct Tea {
  uint32_t v0, v1;
};
__device__ __forceinline__ void teaFloats(Tea &r, float &a, float &b)
{
  uint32_t v0 = r.v0, v1 = r.v1, sum = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    sum += 0x9e3779b9u;
    v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + sum) ^ ((v1 >> 5) + 0xc8013ea4u);
    v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + sum) ^ ((v0 >> 5) + 0x7e95761eu);
  }
  r.v0 = v0;
  r.v1 = v1;
  const float tofloat = 2.3283064365386962890625e-10f;  // 2^-32
  a                   = (float)v0 * tofloat;
  b                   = (float)v1 * tofloat;
}

// Woodcock steps one tracking call may take: the tracking ends long before
// on any volume (each step moves on by an exponential distance), the bound
// only keeps a degenerate transfer function from looping.
constexpr int kMaxWoodcockSteps = 1 << 16;

// sampleWoodcock (DensityPathTracerGpuKernel.cpp:25-75): distance tracking
// against the majorant sigmaTScale; true with the sample at the event.
__device__ __forceinline__ bool sampleWoodcock(VKLSampler sampler, const VKLExampleTransferFunction &tf,
                                               const VKLExampleParams &prm, const VKLExamplePathTracerParams &pt,
                                               Tea &rng, v3 org, v3 dir, vkl_range1f hits, float &t, float &sample,
                                               float &transmittance)
{
  t                    = hits.lower;
  const float sigmaMax = pt.sigmaTScale;
  if (sigmaMax <= 0.f) {
    transmittance = 1.f;
    return false;
  }
  for (int step = 0; step < kMaxWoodcockSteps; ++step) {
    float r0, r1, s0, s1;
    teaFloats(rng, r0, r1);
    teaFloats(rng, s0, s1);
    t = t + (-pt_log(1.f - r0)) / sigmaMax;
    if (t > hits.upper) {
      transmittance = 1.f;
      return false;
    }
    const v3 c  = org + t * dir;
    float time  = prm.time;
    if (pt.motionBlur)
      time = time + (s0 - 0.5f) * pt.shutter;
    time = fminf(fmaxf(time, 0.f), 1.f);
    const vkl_vec3f cv{c.x, c.y, c.z};
    sample                   = vklComputeSample(&sampler, &cv, prm.attributeIndex, time, prm.featureFlags);
    const v4 sc              = transfer(tf, sample);
    const float sigmaTSample = sigmaMax * sc.w;
    if (r1 < sigmaTSample / sigmaMax)
      break;
  }
  transmittance = 0.f;
  return true;
}

// integrate + renderPixel (DensityPathTracerGpuKernel.cpp:77-163): scatter
// until the path leaves the volume or maxNumScatters, ambient light picked
// up by secondary paths, accumulated into rgba / weight.
__global__ void __launch_bounds__(kThreads) kDensityPathTracer(VKLSampler sampler,
                                                               const __grid_constant__ VKLExampleCamera cam,
                                                               const __grid_constant__ VKLExampleTransferFunction tf,
                                                               const __grid_constant__ VKLExampleParams prm,
                                                               const __grid_constant__ VKLExamplePathTracerParams pt,
                                                               float4 *rgba, float *weight)
{
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= prm.width * prm.height)
    return;
  v3 org, dir;
  pixelRay(cam, prm, idx, org, dir);
  Tea rng{pt.frame, (uint32_t)idx};
  int maxScatterIndex      = 0;
  bool primaryRayIntersect = false;
  v3 Le = {0.f, 0.f, 0.f}, sigmaS = {0.f, 0.f, 0.f};
  for (int scatterIndex = 0; true; scatterIndex++) {
    float sample    = 0.f;
    maxScatterIndex = max(scatterIndex, maxScatterIndex);
    const vkl_range1f rt = intersectBox(org, dir, prm.bounds);
    const bool empty     = rt.lower > rt.upper;
    if (scatterIndex == 0 && !empty)
      primaryRayIntersect = true;
    if (empty)
      break;
    float t = 0.f, transmittance = 0.f;
    if (!sampleWoodcock(sampler, tf, prm, pt, rng, org, dir, rt, t, sample, transmittance)) {
      if (scatterIndex > 0) {
        const float a = transmittance * pt.ambientLightIntensity;
        Le            = Le + v3{a * sigmaS.x, a * sigmaS.y, a * sigmaS.z};
      }
      break;
    }
    if (scatterIndex >= pt.maxNumScatters)
      break;
    const v4 sc = transfer(tf, sample);
    sigmaS      = {pt.sigmaSScale * sc.x * sc.w, pt.sigmaSScale * sc.y * sc.w, pt.sigmaSScale * sc.z * sc.w};
    org         = org + t * dir;
    // uniformSampleSphere(1, s) (Random.ih:57-63)
    float s0, s1;
    teaFloats(rng, s0, s1);
    const float phi      = 6.28318530717958647692f * s0;
    const float cosTheta = 1.f * (1.f - 2.f * s1);
    const float sinTheta = 2.f * 1.f * sqrtf(s1 * (1.f - s1));
    float sinPhi, cosPhi;
    pt_sincos(phi, &sinPhi, &cosPhi);
    dir = {cosPhi * sinTheta, sinPhi * sinTheta, cosTheta};
  }
  v3 color    = Le;
  float alpha = maxScatterIndex > 0 ? 1.f : 0.f;
  if (pt.showBbox && primaryRayIntersect) {
    const float blend = 0.2f;
    alpha             = (1.f - blend) * alpha + blend * 1.f;
    color             = (1.f - blend) * color + v3{blend * 1.f, blend * 1.f, blend * 1.f};
  }
  float4 acc  = rgba[idx];
  acc.x       = acc.x + color.x;
  acc.y       = acc.y + color.y;
  acc.z       = acc.z + color.z;
  acc.w       = acc.w + alpha;
  rgba[idx]   = acc;
  weight[idx] = weight[idx] + 1.f;
}

// User code sampling its own points with the device API: sample and
// gradient of every point (the per-point analogue of vklComputeSampleN /
// vklComputeGradientN).
__global__ void __launch_bounds__(kThreads) kSamplePoints(VKLSampler sampler, VKLFeatureFlags featureFlags,
                                                          uint64_t n, const float *pts, unsigned int attr,
                                                          float *samples, float *gradients)
{
  const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  if (i >= n)
    return;
  const vkl_vec3f p{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
  samples[i]        = vklComputeSample(&sampler, &p, attr, 0.f, featureFlags);
  const vkl_vec3f g = vklComputeGradient(&sampler, &p, attr, 0.f, featureFlags);
  gradients[3 * i]     = g.x;
  gradients[3 * i + 1] = g.y;
  gradients[3 * i + 2] = g.z;
}

}  // namespace

extern "C" {

// Renders one frame into `rgba` (device memory, width*height float4, row
// major, row 0 at the top) on `stream`.  renderer: 0 ray march iterator,
// 1 interval iterator debug, 2 hit iterator renderer.  Returns a
// cudaError_t value (0 on success).
__attribute__((visibility("default"))) int vklExampleRender(int renderer, VKLSampler sampler,
                                                            VKLIntervalIteratorContext intervalContext,
                                                            VKLHitIteratorContext hitContext,
                                                            const VKLExampleCamera *camera,
                                                            const VKLExampleTransferFunction *tf,
                                                            const VKLExampleParams *params, float *rgba,
                                                            void *stream)
{
  const int n = params->width * params->height;
  if (n <= 0)
    return 0;
  const unsigned blocks = (unsigned)((n + kThreads - 1) / kThreads);
  cudaStream_t st       = (cudaStream_t)stream;
  if (renderer == 0)
    kRayMarch<<<blocks, kThreads, 0, st>>>(sampler, intervalContext, *camera, *tf, *params, (float4 *)rgba);
  else if (renderer == 1)
    kIntervalDebug<<<blocks, kThreads, 0, st>>>(intervalContext, *camera, *tf, *params, (float4 *)rgba);
  else if (renderer == 2)
    kHitRenderer<<<blocks, kThreads, 0, st>>>(sampler, hitContext, *camera, *tf, *params, (float4 *)rgba);
  else
    return (int)cudaErrorInvalidValue;
  return (int)cudaGetLastError();
}

// One progressive frame of the density path tracer: adds each pixel's
// radiance and alpha to rgba (width*height float4) and 1 to its weight.
__attribute__((visibility("default"))) int vklExamplePathTrace(VKLSampler sampler, const VKLExampleCamera *camera,
                                                               const VKLExampleTransferFunction *tf,
                                                               const VKLExampleParams *params,
                                                               const VKLExamplePathTracerParams *pt, float *rgba,
                                                               float *weights, void *stream)
{
  const int n = params->width * params->height;
  if (n <= 0)
    return 0;
  kDensityPathTracer<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      sampler, *camera, *tf, *params, *pt, (float4 *)rgba, weights);
  return (int)cudaGetLastError();
}

// Samples and gradients of n points (device memory) through the device API,
// with the sampler's feature flags (vklGetFeatureFlags).
__attribute__((visibility("default"))) int vklExampleSamplePoints(VKLSampler sampler, VKLFeatureFlags featureFlags,
                                                                  uint64_t n, const float *points,
                                                                  unsigned int attr, float *samples,
                                                                  float *gradients, void *stream)
{
  if (n == 0)
    return 0;
  kSamplePoints<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      sampler, featureFlags, n, points, attr, samples, gradients);
  return (int)cudaGetLastError();
}

}  // extern "C"
