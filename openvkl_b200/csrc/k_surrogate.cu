// Learned surrogate of a volume (extension; no reference counterpart).
//
// A multi-resolution hash-grid encoding (16 levels, 2 FP16 features per
// entry, per-level resolution floor(base * growth^l), direct indexing while
// (res+1)^3 fits the table, else the spatial hash) feeds a 32-64-64-64-1 ReLU
// MLP without biases, FP16 weights and activations, FP32 accumulation.  It
// is trained on samples of the plain sampler (the caller supplies points and
// the plain samples as targets), with the loss sum (y - target)^2 / n over
// the points with a finite target, and Adam.  The plain sampler also
// measures the error: calibration evaluates both on caller-supplied points
// and flags every 32^3-voxel region whose largest error exceeds a threshold
// (or that no calibration point reached); sampling with fallback returns the
// plain sample there and outside the volume's domain.
//
// Inference fuses the encoding and the MLP: each 128-point group encodes its
// points into shared memory and runs every hidden layer as one tcgen05
// product (M = 128 points, N = 64) into tensor memory.  Training runs
// forward and backward per 128-point tile in one kernel: forward and the
// backward signals on mma.sync m16n8k16 tiles with the activations in
// registers, the weight gradients (G^T H over the tile's points) as tcgen05
// products from transposed, swizzled copies of the activations and signals,
// encoding gradients scattered into the table's gradient with float2
// atomics; a separate kernel applies Adam to the FP32 master parameters and
// refreshes their FP16 copies.
#include <cuda_fp16.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "kernels.h"
#include "objects.h"
#include "sampling.cuh"
#include "tcgen05.cuh"

namespace vklcuda {

namespace {

constexpr int kLv = 16;
constexpr int kIn = 2 * kLv;  // 32 encoded features
constexpr int kH  = 64;
constexpr int kOffW1 = 0, kOffW2 = kH * kIn, kOffW3 = kOffW2 + kH * kH, kOffW4 = kOffW3 + kH * kH;
constexpr int kNumW  = kOffW4 + kH;  // 10304
constexpr int kTile  = 128;          // points per CTA tile
constexpr int kThr   = 128;          // 4 warps x 32 points
constexpr int kRegionLog = 5;        // 32^3-voxel calibration regions

struct Encoding {
  float lo[3], inv[3];
  uint32_t res[kLv];
  uint32_t dense[kLv];
  uint32_t tableMask;
  uint32_t tableSize;
};

struct Judge {
  // plain-sampler fallback and calibration regions (index space)
  uint32_t regionDims[3];
  const uint8_t *flags;
  float *regionErr;
  uint32_t *regionSeen;
  uint32_t attr;
};

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1)
{
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld32(const __half *p) { return *reinterpret_cast<const uint32_t *>(p); }

__device__ __forceinline__ uint32_t pack(float lo, float hi)
{
  const __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&h);
}

// A fragment of the 16x16 block at (m0, k0) of row-major A (leading dim ld).
__device__ __forceinline__ void loadA(uint32_t a[4], const __half *A, int ld, int m0, int k0, int g, int t)
{
  a[0] = ld32(A + (m0 + g) * ld + k0 + 2 * t);
  a[1] = ld32(A + (m0 + g + 8) * ld + k0 + 2 * t);
  a[2] = ld32(A + (m0 + g) * ld + k0 + 8 + 2 * t);
  a[3] = ld32(A + (m0 + g + 8) * ld + k0 + 8 + 2 * t);
}

// B fragment of the 16x8 block (k0, n0) given B transposed, Bt[n][k] row-major.
__device__ __forceinline__ void loadB(uint32_t &b0, uint32_t &b1, const __half *Bt, int ld, int n0, int k0,
                                      int g, int t)
{
  b0 = ld32(Bt + (n0 + g) * ld + k0 + 2 * t);
  b1 = ld32(Bt + (n0 + g) * ld + k0 + 8 + 2 * t);
}

// ReLU'd accumulators of 8 n-tiles (64 columns) -> A fragments of 4 k-steps.
__device__ __forceinline__ void chain(const float acc[8][4], uint32_t a[4][4])
{
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    a[kk][0] = pack(fmaxf(acc[2 * kk][0], 0.f), fmaxf(acc[2 * kk][1], 0.f));
    a[kk][1] = pack(fmaxf(acc[2 * kk][2], 0.f), fmaxf(acc[2 * kk][3], 0.f));
    a[kk][2] = pack(fmaxf(acc[2 * kk + 1][0], 0.f), fmaxf(acc[2 * kk + 1][1], 0.f));
    a[kk][3] = pack(fmaxf(acc[2 * kk + 1][2], 0.f), fmaxf(acc[2 * kk + 1][3], 0.f));
  }
}

// Per-level cell of a point in [0,1]^3: integer corner and fraction.
__device__ __forceinline__ void levelCell(const Encoding &E, int l, const float u[3], uint32_t i[3], float f[3])
{
  const float r = (float)E.res[l];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float x = u[a] * r;
    const float fl = fminf(floorf(x), r - 1.f);
    i[a]           = (uint32_t)fl;
    f[a]           = x - fl;
  }
}

__device__ __forceinline__ uint32_t entryOf(const Encoding &E, int l, uint32_t cx, uint32_t cy, uint32_t cz)
{
  if (E.dense[l]) {
    const uint32_t r1 = E.res[l] + 1;
    return cx + cy * r1 + cz * r1 * r1;
  }
  return (cx ^ (cy * 2654435761u) ^ (cz * 805459861u)) & E.tableMask;
}

__device__ __forceinline__ float cornerWeight(int c, const float f[3])
{
  const float wx = (c & 4) ? f[0] : 1.f - f[0];
  const float wy = (c & 2) ? f[1] : 1.f - f[1];
  const float wz = (c & 1) ? f[2] : 1.f - f[2];
  return (wx * wy) * wz;
}

__device__ __forceinline__ void unitPosition(const Encoding &E, f3 p, float u[3])
{
  const float q[3] = {p.x, p.y, p.z};
#pragma unroll
  for (int a = 0; a < 3; ++a)
    u[a] = fminf(fmaxf((q[a] - E.lo[a]) * E.inv[a], 0.f), 1.f);
}

// Encodes one point into 32 FP16 features (out: 16 half2 slots).
// UNROLL levels are encoded at once: all 16 (128 table gathers in flight per
// thread) in inference, 2 in training, whose kernel needs the registers for
// its backward pass (measured: full unrolling speeds inference 1.9x and
// slows training 1.2x).
template <int UNROLL>
__device__ __forceinline__ void encodePoint(const Encoding &E, const __half2 *__restrict__ table, const float u[3],
                                            __half2 *out)
{
#pragma unroll UNROLL
  for (int l = 0; l < kLv; ++l) {
    uint32_t i[3];
    float f[3];
    levelCell(E, l, u, i, f);
    const __half2 *tl = table + (size_t)l * E.tableSize;
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const uint32_t e = entryOf(E, l, i[0] + ((c >> 2) & 1), i[1] + ((c >> 1) & 1), i[2] + (c & 1));
      const float w    = cornerWeight(c, f);
      const float2 v   = __half22float2(__ldg(tl + e));
      s0 += w * v.x;
      s1 += w * v.y;
    }
    out[l] = __floats2half2_rn(s0, s1);
  }
}

// Index-space region of an object-space point, or -1 outside the domain.
__device__ __forceinline__ int64_t regionOf(const DevGrid &g, const Judge &J, f3 p)
{
  const f3 q = xfmPoint(g.objectToIndex, p);
  const uint32_t ox = (uint32_t)(ifloor(q.x) - g.rootOrigin[0]), oy = (uint32_t)(ifloor(q.y) - g.rootOrigin[1]),
                 oz = (uint32_t)(ifloor(q.z) - g.rootOrigin[2]);
  if (!(ox < g.activeSize[0] && oy < g.activeSize[1] && oz < g.activeSize[2]))
    return -1;
  return ((int64_t)(oz >> kRegionLog) * J.regionDims[1] + (oy >> kRegionLog)) * J.regionDims[0] +
         (ox >> kRegionLog);
}

template <class Field>
__device__ __forceinline__ float plainSample(const DevGrid &g, const Judge &J, f3 p)
{
  const Field F = [&]() {
    if constexpr (std::is_same<Field, DenseField<float>>::value)
      return DenseField<float>(g, J.attr);
    else
      return SparseField<float>(g, J.attr, kNumLevels - 1);
  }();
  return sampleLinear(F, xfmPoint(g.objectToIndex, p));
}

// Shared weights of the forward pass (row-major [out][in], padded rows).
struct FwdWeights {
  __half w1[kH][kIn + 8];
  __half w2[kH][kH + 8];
  __half w3[kH][kH + 8];
  __half w4[8][kH + 8];  // row 0 = W4, rows 1..7 zero (n8 tile)
};

__device__ __forceinline__ void loadFwdWeights(FwdWeights &W, const __half *__restrict__ w16)
{
  for (int k = threadIdx.x; k < kH * kIn; k += blockDim.x)
    W.w1[k / kIn][k % kIn] = w16[kOffW1 + k];
  for (int k = threadIdx.x; k < kH * kH; k += blockDim.x) {
    W.w2[k / kH][k % kH] = w16[kOffW2 + k];
    W.w3[k / kH][k % kH] = w16[kOffW3 + k];
  }
  for (int k = threadIdx.x; k < 8 * kH; k += blockDim.x)
    W.w4[k / kH][k % kH] = k < kH ? w16[kOffW4 + k] : __float2half(0.f);
}

// Transposed operands of the training kernel's tensor-core weight gradients
// (dW = G^T H over a tile's 128 points): unit u is a row, point p the K
// index, in the 128-byte-swizzled K-major layout (tcgen05.cuh), as two atoms
// of 64 points; an atom holds `rows` rows of 128 bytes.  Byte offset of
// element (u, p):
__device__ __forceinline__ uint32_t tOff(uint32_t rows, uint32_t u, uint32_t p)
{
  return (p >> 6) * (rows * 128u) + tc::swizzledChunk(u, (p & 63u) >> 3) + (p & 7u) * 2u;
}
constexpr uint32_t kTBytes64 = 2 * 64 * 128;  // 64 units x 128 points
constexpr uint32_t kTBytes32 = 2 * 32 * 128;  // 32 units x 128 points

// Forward of one 16-row chunk (rows m0..m0+15 of X); returns the outputs of
// rows m0+g and m0+g+8 in lanes with t == 0.  When HT is given, the FP16
// activations of each hidden layer l are also stored transposed at
// HT + l * kTBytes64 (tOff layout).
__device__ __forceinline__ void forwardChunk(const FwdWeights &W, const __half *X, int ldx, int m0, int g, int t,
                                             float &y0, float &y1, unsigned char *HT)
{
  uint32_t a[4][4];
  float acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j)
    acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
#pragma unroll
  for (int kk = 0; kk < 2; ++kk) {
    uint32_t ax[4];
    loadA(ax, X, ldx, m0, 16 * kk, g, t);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      uint32_t b0, b1;
      loadB(b0, b1, &W.w1[0][0], kIn + 8, 8 * j, 16 * kk, g, t);
      mma16816(acc[j], ax, b0, b1);
    }
  }
#pragma unroll
  for (int layer = 0; layer < 3; ++layer) {
    chain(acc, a);
    if (HT) {
      unsigned char *H = HT + (size_t)layer * kTBytes64;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = 8 * j + 2 * t;
        const __half2 lo = *reinterpret_cast<const __half2 *>(&a[j >> 1][(j & 1) ? 2 : 0]);
        const __half2 hi = *reinterpret_cast<const __half2 *>(&a[j >> 1][(j & 1) ? 3 : 1]);
        *reinterpret_cast<__half *>(H + tOff(64, c, m0 + g))         = __low2half(lo);
        *reinterpret_cast<__half *>(H + tOff(64, c + 1, m0 + g))     = __high2half(lo);
        *reinterpret_cast<__half *>(H + tOff(64, c, m0 + g + 8))     = __low2half(hi);
        *reinterpret_cast<__half *>(H + tOff(64, c + 1, m0 + g + 8)) = __high2half(hi);
      }
    }
    if (layer == 2)
      break;
    const __half *Wl = layer == 0 ? &W.w2[0][0] : &W.w3[0][0];
#pragma unroll
    for (int j = 0; j < 8; ++j)
      acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        uint32_t b0, b1;
        loadB(b0, b1, Wl, kH + 8, 8 * j, 16 * kk, g, t);
        mma16816(acc[j], a[kk], b0, b1);
      }
  }
  float o[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    uint32_t b0, b1;
    loadB(b0, b1, &W.w4[0][0], kH + 8, 0, 16 * kk, g, t);
    mma16816(o, a[kk], b0, b1);
  }
  y0 = o[0];
  y1 = o[2];
}

// ---------------------------------------------------------------------------
// Inference (optionally with the plain fallback) and calibration.
// MODE 0: samples; MODE 1: calibration (region error of the network).
//
// A CTA of 256 threads runs two independent groups of 128 (own named
// barrier, mbarrier and TMEM columns); a group owns a 128-point tile:
// thread r encodes point r into row r of the group's operand buffer in
// shared memory; each hidden layer is then one 128 x 64 tensor-core product
// (tcgen05.mma, M = 128, N = 64, K = 32 or 64, FP16 operands, FP32
// accumulator in tensor memory) issued by the group's first thread, and
// thread r reads its row back from TMEM lane r (tcgen05.ld), applies ReLU,
// rounds to FP16 and writes the next layer's operand row into the same
// buffer (the product that read it has completed).  The 64 -> 1 output layer
// is a dot product on the CUDA cores.  The weights stay in shared memory for
// the CTA's lifetime (persistent over tiles).
// ---------------------------------------------------------------------------
constexpr int kInferThr   = 256;  // two groups of 128 threads
constexpr int kInferCtasPerSM = 3;
constexpr uint32_t kTcCols = 128;  // TMEM columns per CTA: one 64-column accumulator per group

struct TcInferSmem {                // operand buffers on 1024-byte boundaries
  unsigned char act[2][kTile * 128];  // per group: layer-1 operand (K = 32 of 64), then hidden activations
  unsigned char w1[kH * 128];         // K = 32 of 64 used
  unsigned char w2[kH * 128];
  unsigned char w3[kH * 128];
  float w4[kH];
  uint64_t bar[2];
  uint32_t tmem;
};
constexpr size_t kTcInferSmemBytes = sizeof(TcInferSmem) + 1024;  // + alignment slack
static_assert(kInferCtasPerSM * (kTcInferSmemBytes + 1024) <= 228 * 1024, "inference CTAs per SM exceed shared memory");

// Rows of a row-major [rows][k] FP16 matrix into the swizzled K-major layout.
__device__ __forceinline__ void loadSwizzledRows(unsigned char *dst, const __half *__restrict__ src, int rows, int k)
{
  const int cpr = k / 8;
  for (int idx = threadIdx.x; idx < rows * cpr; idx += blockDim.x) {
    const int r = idx / cpr, c = idx - r * cpr;
    *reinterpret_cast<uint4 *>(dst + tc::swizzledChunk(r, c)) =
        __ldg(reinterpret_cast<const uint4 *>(src + (size_t)r * k) + c);
  }
}

__device__ __forceinline__ uint32_t reluPack(uint32_t lo, uint32_t hi)
{
  return pack(fmaxf(__uint_as_float(lo), 0.f), fmaxf(__uint_as_float(hi), 0.f));
}

// Barrier of one 128-thread group; returns whether any thread passed true.
__device__ __forceinline__ bool groupSyncOr(uint32_t id, bool v)
{
  uint32_t r;
  asm volatile(
      "{ .reg .pred p, q; setp.ne.u32 q, %1, 0; bar.red.or.pred p, %2, 128, q; selp.u32 %0, 1, 0, p; }"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id)
      : "memory");
  return r != 0;
}

template <class Field, int MODE>
__global__ void __launch_bounds__(kInferThr, kInferCtasPerSM)
    kSurrogateInfer(const __grid_constant__ Encoding E, const __half2 *__restrict__ table,
                    const __half *__restrict__ w16, const __grid_constant__ DevGrid g,
                    const __grid_constant__ Judge J, uint64_t n, const float *__restrict__ pts,
                    float *__restrict__ out, int fallback, uint32_t *__restrict__ err)
{
  extern __shared__ unsigned char smemRaw[];
  TcInferSmem &S = *reinterpret_cast<TcInferSmem *>(smemRaw + ((1024u - (tc::smemAddr(smemRaw) & 1023u)) & 1023u));
  const int warp = threadIdx.x >> 5;
  const int grp  = threadIdx.x >> 7;
  const uint32_t row = threadIdx.x & 127u;
  loadSwizzledRows(S.w1, w16 + kOffW1, kH, kIn);
  loadSwizzledRows(S.w2, w16 + kOffW2, kH, kH);
  loadSwizzledRows(S.w3, w16 + kOffW3, kH, kH);
  for (int k = threadIdx.x; k < kH; k += kInferThr)
    S.w4[k] = __half2float(w16[kOffW4 + k]);
  if (threadIdx.x == 0) {
    tc::mbarInit(&S.bar[0], 1);
    tc::mbarInit(&S.bar[1], 1);
  }
  if (warp == 0)
    tc::tmemAlloc(&S.tmem, kTcCols);
  tc::fenceProxyAsync();
  tc::fenceBeforeSync();
  __syncthreads();
  tc::fenceAfterSync();
  // this group's accumulator: columns 64 grp..; this warp's lanes 32 (warp % 4)..
  const uint32_t acc   = S.tmem + 64u * grp;
  const uint32_t myRow = acc + ((uint32_t)(32 * (warp & 3)) << 16);
  constexpr uint32_t idesc = tc::f16InstrDesc(kTile, kH);
  unsigned char *buf   = S.act[grp];
  const uint32_t bufA  = tc::smemAddr(buf);
  uint64_t *bar        = &S.bar[grp];
  const uint32_t barId = 1u + grp;
  uint32_t phase = 0;
  bool ok        = true;
  for (uint64_t base = ((uint64_t)blockIdx.x * 2 + grp) * kTile; base < n && ok;
       base += (uint64_t)gridDim.x * 2 * kTile) {
    const uint64_t i = base + row;
    f3 p             = {0.f, 0.f, 0.f};
    __half2 feat[kLv];
    if (i < n) {
      p = {__ldg(pts + 3 * i), __ldg(pts + 3 * i + 1), __ldg(pts + 3 * i + 2)};
      float u[3];
      unitPosition(E, p, u);
      encodePoint<kLv>(E, table, u, feat);
    } else {
#pragma unroll
      for (int k = 0; k < kLv; ++k)
        feat[k] = __floats2half2_rn(0.f, 0.f);
    }
#pragma unroll
    for (int c = 0; c < kIn / 8; ++c) {
      uint4 v;
      v.x = *reinterpret_cast<const uint32_t *>(&feat[4 * c]);
      v.y = *reinterpret_cast<const uint32_t *>(&feat[4 * c + 1]);
      v.z = *reinterpret_cast<const uint32_t *>(&feat[4 * c + 2]);
      v.w = *reinterpret_cast<const uint32_t *>(&feat[4 * c + 3]);
      *reinterpret_cast<uint4 *>(buf + tc::swizzledChunk(row, c)) = v;
    }
    float y = 0.f;
#pragma unroll 1
    for (int layer = 0; layer < 3; ++layer) {
      // every thread's operand row is written -> one thread issues the layer
      tc::fenceProxyAsync();
      tc::fenceBeforeSync();
      groupSyncOr(barId, false);
      if (row == 0) {
        tc::fenceAfterSync();
        const uint32_t w = tc::smemAddr(layer == 0 ? S.w1 : layer == 1 ? S.w2 : S.w3);
        const int ks     = layer == 0 ? kIn / 16 : kH / 16;
        for (int k = 0; k < ks; ++k)
          tc::mmaF16(acc, tc::sw128Desc(bufA + 32u * k), tc::sw128Desc(w + 32u * k), idesc, k > 0);
        tc::commitTo(bar);
      }
      const bool done = tc::mbarWait(bar, phase);
      phase ^= 1u;
      if (groupSyncOr(barId, !done)) {
        ok = false;
        break;
      }
      tc::fenceAfterSync();
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        uint32_t r[32];
        tc::tmemLoad32(myRow + 32u * half, r);
        tc::tmemLoadWait();
        if (layer < 2) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            uint4 v;
            v.x = reluPack(r[8 * q], r[8 * q + 1]);
            v.y = reluPack(r[8 * q + 2], r[8 * q + 3]);
            v.z = reluPack(r[8 * q + 4], r[8 * q + 5]);
            v.w = reluPack(r[8 * q + 6], r[8 * q + 7]);
            *reinterpret_cast<uint4 *>(buf + tc::swizzledChunk(row, 4 * half + q)) = v;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j)
            y += __half2float(__float2half_rn(fmaxf(__uint_as_float(r[j]), 0.f))) * S.w4[32 * half + j];
        }
      }
    }
    if (!ok)
      break;
    if (i < n) {
      if (MODE == 0) {
        if (fallback) {
          const int64_t r = regionOf(g, J, p);
          if (r < 0 || J.flags[r])
            y = plainSample<Field>(g, J, p);
        }
        out[i] = y;
      } else {
        const int64_t r = regionOf(g, J, p);
        const float ref = plainSample<Field>(g, J, p);
        if (r >= 0 && !isnan(ref)) {
          const float e = fabsf(y - ref);
          atomicMax(reinterpret_cast<unsigned int *>(J.regionErr) + r, __float_as_uint(isnan(e) ? INFINITY : e));
          J.regionSeen[r] = 1u;
        }
      }
    }
  }
  tc::fenceBeforeSync();
  __syncthreads();
  if (warp == 0)
    tc::tmemDealloc(S.tmem, kTcCols);
  if (!ok && row == 0)
    atomicExch(err, 1u);
}

__global__ void kRegionFlags(uint64_t n, const float *regionErr, const uint32_t *seen, float threshold,
                             uint8_t *flags, unsigned int *flagged)
{
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const bool f = !seen[i] || !(regionErr[i] <= threshold);
  flags[i]     = f ? 1 : 0;
  if (f)
    atomicAdd(flagged, 1u);
}

// ---------------------------------------------------------------------------
// Training: forward + backward of 128-point tiles.
// ---------------------------------------------------------------------------
constexpr int kLdR = kH + 8;     // row-major [row][64]

struct TrainSmem {  // GT, HT, XT on 1024-byte boundaries (the struct is placed so)
  unsigned char GT[kTBytes64];     // backward signal, transposed (A of the weight gradients)
  unsigned char HT[3][kTBytes64];  // hidden activations, transposed (B)
  unsigned char XT[kTBytes32];     // encoded inputs, transposed (B of dW1)
  FwdWeights W;
  __half w1t[kIn][kH + 8];   // W1 transposed [in][out]
  __half w2t[kH][kH + 8];
  __half w3t[kH][kH + 8];
  float w4[kH];
  __half X[kTile][kIn + 8];
  __half G[kTile][kLdR];     // backward signal, row-major
  float u[kTile][3];
  float dy[kTile];
  float loss[kThr / 32];
  uint64_t bar;
  uint32_t tmem;
};
constexpr size_t kTrainSmemBytes = sizeof(TrainSmem) + 1024;  // + alignment slack
constexpr uint32_t kTrainCols    = 64;                         // TMEM columns: one 64-wide accumulator
static_assert(kTrainSmemBytes <= 227 * 1024, "training tile exceeds the shared memory of one CTA");

// Weight gradient dW (64 x N) += G^T (64 x 128 points) * B^T on the tensor
// cores: one thread issues 8 K-steps of M = 128 (rows 64..127 of the A
// operand read the next 8 KB of shared memory and land in TMEM lanes
// 64..127, which nobody reads), N = 64 or 32, then every thread waits for the
// commit; warps 0 and 1 read lanes 0..63 (output units) and add them to the
// FP32 gradient in global memory.  Returns false if the wait gave up.
template <int N>
__device__ __forceinline__ bool weightGradTc(TrainSmem &S, const unsigned char *B, uint32_t &phase,
                                             float *__restrict__ gW)
{
  constexpr uint32_t idesc = tc::f16InstrDesc(128, N);
  const uint32_t aBase = tc::smemAddr(S.GT), bBase = tc::smemAddr(B);
  if (threadIdx.x == 0) {
    tc::fenceAfterSync();
#pragma unroll
    for (int k = 0; k < kTile / 16; ++k) {
      const uint32_t off = (uint32_t)(k >> 2), in = 32u * (uint32_t)(k & 3);
      tc::mmaF16(S.tmem, tc::sw128Desc(aBase + off * (64u * 128u) + in),
                 tc::sw128Desc(bBase + off * ((uint32_t)N * 128u) + in), idesc, k > 0);
    }
    tc::commitTo(&S.bar);
  }
  const bool done = tc::mbarWait(&S.bar, phase);
  phase ^= 1u;
  if (__syncthreads_or(!done))
    return false;
  tc::fenceAfterSync();
  const int warp = threadIdx.x >> 5;
  if (warp < 2) {
    const uint32_t o = threadIdx.x;  // output unit = TMEM lane
#pragma unroll
    for (int h = 0; h < N / 32; ++h) {
      uint32_t r[32];
      tc::tmemLoad32(S.tmem + ((uint32_t)(32 * warp) << 16) + 32u * h, r);
      tc::tmemLoadWait();
      float4 *dst = reinterpret_cast<float4 *>(gW + (size_t)o * N + 32 * h);
#pragma unroll
      for (int q = 0; q < 8; ++q)
        atomicAdd(dst + q, make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                       __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3])));
    }
  }
  tc::fenceBeforeSync();
  return true;
}

// Backward signal of the previous layer for this warp's 32 rows:
// acc[c][j] = (G * Wt^T) restricted to rows 32w+16c.., NT n-tiles.
template <int NT>
__device__ __forceinline__ void signalGrad(const TrainSmem &S, const __half *Wt, int warp, int g, int t,
                                           float acc[2][NT][4])
{
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll
    for (int j = 0; j < NT; ++j)
      acc[c][j][0] = acc[c][j][1] = acc[c][j][2] = acc[c][j][3] = 0.f;
#pragma unroll
    for (int kk = 0; kk < kH / 16; ++kk) {
      uint32_t a[4];
      loadA(a, &S.G[0][0], kLdR, 32 * warp + 16 * c, 16 * kk, g, t);
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        uint32_t b0, b1;
        loadB(b0, b1, Wt, kH + 8, 8 * j, 16 * kk, g, t);
        mma16816(acc[c][j], a, b0, b1);
      }
    }
  }
}

// G <- ReLU-masked signal (mask from the stored transposed activations H).
__device__ __forceinline__ void storeSignal(TrainSmem &S, const float acc[2][8][4], const unsigned char *H,
                                            int warp, int g, int t)
{
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int r = 32 * warp + 16 * c + g, col = 8 * j + 2 * t;
      auto hv = [&](int u, int p) { return __half2float(*reinterpret_cast<const __half *>(H + tOff(64, u, p))); };
      const float v0 = hv(col, r) > 0.f ? acc[c][j][0] : 0.f;
      const float v1 = hv(col + 1, r) > 0.f ? acc[c][j][1] : 0.f;
      const float v2 = hv(col, r + 8) > 0.f ? acc[c][j][2] : 0.f;
      const float v3 = hv(col + 1, r + 8) > 0.f ? acc[c][j][3] : 0.f;
      const __half2 lo = __floats2half2_rn(v0, v1), hi = __floats2half2_rn(v2, v3);
      *reinterpret_cast<__half2 *>(&S.G[r][col])     = lo;
      *reinterpret_cast<__half2 *>(&S.G[r + 8][col]) = hi;
      *reinterpret_cast<__half *>(S.GT + tOff(64, col, r))         = __low2half(lo);
      *reinterpret_cast<__half *>(S.GT + tOff(64, col + 1, r))     = __high2half(lo);
      *reinterpret_cast<__half *>(S.GT + tOff(64, col, r + 8))     = __low2half(hi);
      *reinterpret_cast<__half *>(S.GT + tOff(64, col + 1, r + 8)) = __high2half(hi);
    }
}

__global__ void __launch_bounds__(kThr) kSurrogateTrain(const __grid_constant__ Encoding E,
                                                        const __half2 *__restrict__ table,
                                                        const __half *__restrict__ w16, uint64_t n,
                                                        const float *__restrict__ pts,
                                                        const float *__restrict__ targets,
                                                        float2 *__restrict__ gTable, float *__restrict__ gW,
                                                        float *__restrict__ lossOut, uint32_t *__restrict__ err)
{
  extern __shared__ unsigned char smemRaw[];
  TrainSmem &S = *reinterpret_cast<TrainSmem *>(smemRaw + ((1024u - (tc::smemAddr(smemRaw) & 1023u)) & 1023u));
  loadFwdWeights(S.W, w16);
  for (int k = threadIdx.x; k < kH * kIn; k += kThr)
    S.w1t[k % kIn][k / kIn] = w16[kOffW1 + k];
  for (int k = threadIdx.x; k < kH * kH; k += kThr) {
    S.w2t[k % kH][k / kH] = w16[kOffW2 + k];
    S.w3t[k % kH][k / kH] = w16[kOffW3 + k];
  }
  for (int k = threadIdx.x; k < kH; k += kThr)
    S.w4[k] = __half2float(w16[kOffW4 + k]);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  if (threadIdx.x == 0)
    tc::mbarInit(&S.bar, 1);
  if (warp == 0)
    tc::tmemAlloc(&S.tmem, kTrainCols);
  tc::fenceBeforeSync();
  __syncthreads();
  tc::fenceAfterSync();
  uint32_t phase = 0;
  bool ok        = true;
  float lossAcc = 0.f;
  for (uint64_t base = (uint64_t)blockIdx.x * kTile; base < n && ok; base += (uint64_t)gridDim.x * kTile) {
    const uint64_t i = base + threadIdx.x;
    float u[3]       = {0.f, 0.f, 0.f};
    __half2 *row     = reinterpret_cast<__half2 *>(&S.X[threadIdx.x][0]);
    if (i < n) {
      const f3 p = {__ldg(pts + 3 * i), __ldg(pts + 3 * i + 1), __ldg(pts + 3 * i + 2)};
      unitPosition(E, p, u);
      encodePoint<2>(E, table, u, row);
    } else {
      for (int k = 0; k < kLv; ++k)
        row[k] = __floats2half2_rn(0.f, 0.f);
    }
    S.u[threadIdx.x][0] = u[0];
    S.u[threadIdx.x][1] = u[1];
    S.u[threadIdx.x][2] = u[2];
    __syncthreads();
    for (int k = 0; k < kIn; ++k)
      *reinterpret_cast<__half *>(S.XT + tOff(32, k, threadIdx.x)) = S.X[threadIdx.x][k];
    // forward; output and d(loss)/dy per row
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int m0 = 32 * warp + 16 * c;
      float y0, y1;
      forwardChunk(S.W, &S.X[0][0], kIn + 8, m0, g, t, y0, y1, &S.HT[0][0]);
      if (t == 0) {
        const uint64_t r0 = base + m0 + g, r1 = r0 + 8;
        // points whose target is not finite (outside the data, where a
        // sampler with an undefined background returns NaN) are ignored
        const float t0 = r0 < n ? __ldg(targets + r0) : 0.f, t1 = r1 < n ? __ldg(targets + r1) : 0.f;
        const float d0 = (r0 < n && isfinite(t0)) ? y0 - t0 : 0.f;
        const float d1 = (r1 < n && isfinite(t1)) ? y1 - t1 : 0.f;
        S.dy[m0 + g]     = 2.f * d0;
        S.dy[m0 + g + 8] = 2.f * d1;
        lossAcc += d0 * d0 + d1 * d1;
      }
    }
    __syncthreads();
    // layer 4: dW4 and the signal into layer 3
    auto ht = [&](int l, int u, int p) {
      return __half2float(*reinterpret_cast<const __half *>(S.HT[l] + tOff(64, u, p)));
    };
    if (threadIdx.x < kH) {
      float s = 0.f;
      for (int r = 0; r < kTile; ++r)
        s += S.dy[r] * ht(2, threadIdx.x, r);
      atomicAdd(gW + kOffW4 + threadIdx.x, s);
    }
    {
      const int r = threadIdx.x;
      for (int col = 0; col < kH; ++col) {
        const float v = ht(2, col, r) > 0.f ? S.dy[r] * S.w4[col] : 0.f;
        const __half h = __float2half_rn(v);
        S.G[r][col] = h;
        *reinterpret_cast<__half *>(S.GT + tOff(64, col, r)) = h;
      }
    }
    // the transposed operands are read by the tensor cores (async proxy)
    tc::fenceProxyAsync();
    tc::fenceBeforeSync();
    __syncthreads();
    // layers 3 and 2: weight gradient (tensor cores) beside the signal into
    // the layer below (mma.sync), then the new signal
#pragma unroll 1
    for (int layer = 2; layer >= 1 && ok; --layer) {
      float acc[2][8][4];
      signalGrad<8>(S, layer == 2 ? &S.w3t[0][0] : &S.w2t[0][0], warp, g, t, acc);
      ok = weightGradTc<64>(S, S.HT[layer - 1], phase, gW + (layer == 2 ? kOffW3 : kOffW2));
      if (!ok)
        break;
      __syncthreads();
      storeSignal(S, acc, S.HT[layer - 1], warp, g, t);
      tc::fenceProxyAsync();
      tc::fenceBeforeSync();
      __syncthreads();
    }
    if (!ok)
      break;
    // layer 1: weight gradient and the encoding gradient
    ok = weightGradTc<kIn>(S, S.XT, phase, gW + kOffW1);
    if (!ok)
      break;
    {
      float acc[2][4][4];
      signalGrad<4>(S, &S.w1t[0][0], warp, g, t, acc);
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          const int r = 32 * warp + 16 * c + g + 8 * half;
          if (base + r >= n)
            continue;
          const float uu[3] = {S.u[r][0], S.u[r][1], S.u[r][2]};
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int l = 4 * j + t;  // columns 8j+2t, 8j+2t+1 = level l's two features
            const float d0 = acc[c][j][2 * half], d1 = acc[c][j][2 * half + 1];
            uint32_t ci[3];
            float f[3];
            levelCell(E, l, uu, ci, f);
            float2 *gl = gTable + (size_t)l * E.tableSize;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const uint32_t e = entryOf(E, l, ci[0] + ((k >> 2) & 1), ci[1] + ((k >> 1) & 1), ci[2] + (k & 1));
              const float w    = cornerWeight(k, f);
              atomicAdd(gl + e, make_float2(w * d0, w * d1));
            }
          }
        }
    }
    __syncthreads();  // shared buffers are reused by the next tile
  }
  tc::fenceBeforeSync();
  __syncthreads();
  if (warp == 0)
    tc::tmemDealloc(S.tmem, kTrainCols);
  if (!ok && threadIdx.x == 0)
    atomicExch(err, 1u);
  // loss of this CTA
  for (int o = 16; o > 0; o >>= 1)
    lossAcc += __shfl_xor_sync(0xffffffffu, lossAcc, o);
  if (lane == 0)
    S.loss[warp] = lossAcc;
  __syncthreads();
  if (threadIdx.x == 0 && lossOut)
    atomicAdd(lossOut, S.loss[0] + S.loss[1] + S.loss[2] + S.loss[3]);
}

// Adam on FP32 master parameters; refreshes the FP16 copies and clears the
// gradient.
__global__ void kAdam(uint64_t n, float *__restrict__ p, float *__restrict__ grad, float *__restrict__ m,
                      float *__restrict__ v, __half *__restrict__ p16, float gradScale, float lr, float b1,
                      float b2, float eps, float c1, float c2)
{
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const float gr = grad[i] * gradScale;
  const float mi = b1 * m[i] + (1.f - b1) * gr;
  const float vi = b2 * v[i] + (1.f - b2) * gr * gr;
  m[i]           = mi;
  v[i]           = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i]           = pi;
  p16[i]         = __float2half_rn(pi);
  grad[i]        = 0.f;
}

__global__ void kToHalf(uint64_t n, const float *__restrict__ p, __half *__restrict__ p16)
{
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    p16[i] = __float2half_rn(p[i]);
}

inline unsigned blocks(uint64_t n, unsigned b) { return (unsigned)((n + b - 1) / b); }

bool onDevice(const void *p)
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

struct Surrogate {
  Device *device = nullptr;
  Ref<Sampler> sampler;
  Encoding E{};
  Judge J{};
  uint64_t tableFloats = 0;  // levels * T * 2
  uint64_t numRegions  = 0;
  DeviceBuffer table32, table16, w32, w16, gTable, gW, mTable, vTable, mW, vW;
  DeviceBuffer flags, regionErr, regionSeen, scalars;
  int step    = 0;
  int numSMs  = 0;
  bool dense  = false;
  uint32_t *errHost = nullptr;  // host-mapped timeout flag of the inference kernel
  uint32_t *errDev  = nullptr;

  void zeroGrads(cudaStream_t st)
  {
    cudaCheck(cudaMemsetAsync(gTable.ptr, 0, tableFloats * 4, st), "memset");
    cudaCheck(cudaMemsetAsync(gW.ptr, 0, kNumW * 4, st), "memset");
  }

  void train(uint64_t n, const float *pts, const float *targets, float *lossDev, cudaStream_t st)
  {
    // the dynamic shared-memory limit is raised once per device (bit = ordinal)
    static std::atomic<uint64_t> configured{0};
    const uint64_t bit = 1ull << (device->cudaDevice & 63);
    if (!(configured.load() & bit)) {
      cudaCheck(cudaFuncSetAttribute(kSurrogateTrain, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kTrainSmemBytes),
                "smem attribute");
      configured.fetch_or(bit);
    }
    // one CTA per SM fits (the tile's activations, signals and weights)
    const unsigned grid = (unsigned)std::min<uint64_t>(blocks(n, kTile), (uint64_t)numSMs);
    kSurrogateTrain<<<grid, kThr, kTrainSmemBytes, st>>>(E, table16.as<__half2>(), w16.as<__half>(), n, pts,
                                                         targets, gTable.as<float2>(), gW.as<float>(), lossDev,
                                                         errDev);
    cudaCheck(cudaGetLastError(), "surrogate train kernel");
  }

  void adam(uint64_t n, float lr, cudaStream_t st)
  {
    ++step;
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-10f;
    const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
    const float scale = 1.f / (float)n;
    kAdam<<<blocks(tableFloats, 256), 256, 0, st>>>(tableFloats, table32.as<float>(), gTable.as<float>(),
                                                    mTable.as<float>(), vTable.as<float>(), table16.as<__half>(),
                                                    scale, lr, b1, b2, eps, c1, c2);
    kAdam<<<blocks(kNumW, 256), 256, 0, st>>>(kNumW, w32.as<float>(), gW.as<float>(), mW.as<float>(),
                                              vW.as<float>(), w16.as<__half>(), scale, lr, b1, b2, eps, c1, c2);
    cudaCheck(cudaGetLastError(), "adam kernel");
  }

  template <class Field, int MODE>
  void inferWith(uint64_t n, const float *pts, float *out, int fallback, cudaStream_t st)
  {
    // the dynamic shared-memory limit is raised once per instantiation and
    // device (bit = device ordinal)
    static std::atomic<uint64_t> configured{0};
    const uint64_t bit = 1ull << (device->cudaDevice & 63);
    if (!(configured.load() & bit)) {
      cudaCheck(cudaFuncSetAttribute(kSurrogateInfer<Field, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kTcInferSmemBytes),
                "smem attribute");
      configured.fetch_or(bit);
    }
    const unsigned grid = (unsigned)std::min<uint64_t>(blocks(n, 2 * kTile), (uint64_t)numSMs * kInferCtasPerSM);
    kSurrogateInfer<Field, MODE><<<grid, kInferThr, kTcInferSmemBytes, st>>>(
        E, table16.as<__half2>(), w16.as<__half>(), sampler->volume->grid, J, n, pts, out, fallback, errDev);
    cudaCheck(cudaGetLastError(), "surrogate kernel");
  }

  template <int MODE>
  void infer(uint64_t n, const float *pts, float *out, int fallback, cudaStream_t st)
  {
    if (dense)
      inferWith<DenseField<float>, MODE>(n, pts, out, fallback, st);
    else
      inferWith<SparseField<float>, MODE>(n, pts, out, fallback, st);
  }

  // A tensor-core wait of an earlier inference or training launch that gave
  // up sets a word of host-mapped memory; the next call reports it.
  void checkTimeout()
  {
    if (errHost && *(volatile uint32_t *)errHost) {
      *(volatile uint32_t *)errHost = 0u;
      fail("surrogate: a tensor-core completion wait of an earlier launch timed out", VKL_UNKNOWN_ERROR);
    }
  }

  ~Surrogate()
  {
    if (errHost)
      cudaFreeHost(errHost);
  }
};

}  // namespace vklcuda

using namespace vklcuda;

namespace {

template <class F>
VKLError surrogateCall(Surrogate *s, F &&f)
{
  if (!s)
    return VKL_INVALID_ARGUMENT;
  try {
    f();
    return VKL_NO_ERROR;
  } catch (const VklError &e) {
    s->device->setError(e.code, e.what());
    return e.code;
  } catch (const std::exception &e) {
    s->device->setError(VKL_UNKNOWN_ERROR, e.what());
    return VKL_UNKNOWN_ERROR;
  }
}

void requireDevice(const void *p, const char *what)
{
  if (!onDevice(p))
    fail(std::string("surrogate: ") + what + " must be device memory", VKL_INVALID_ARGUMENT);
}

}  // namespace

extern "C" OPENVKL_CUDA_INTERFACE VKLCudaSurrogate vklCudaNewSurrogate(VKLSampler sampler,
                                                                      unsigned int log2TableSize,
                                                                      float baseResolution, float growth)
{
  Sampler *sp = dynamic_cast<Sampler *>((ManagedObject *)sampler.host);
  if (!sp)
    return nullptr;
  Device *d    = sp->device;
  Surrogate *s = nullptr;
  try {
    if (!sp->volume || !sp->volume->committed)
      fail("surrogate: the sampler's volume is not committed", VKL_INVALID_OPERATION);
    const DevGrid &g = sp->volume->grid;
    if (sp->s.filter != kFilterLinear || g.type[0] != kFloat || g.compress != kCompressNone)
      fail("surrogate: needs a trilinear sampler over float voxels", VKL_INVALID_ARGUMENT);
    if (log2TableSize < 4 || log2TableSize > 24 || !(baseResolution >= 1.f) || !(growth >= 1.f))
      fail("surrogate: invalid hash grid configuration", VKL_INVALID_ARGUMENT);
    s          = new Surrogate();
    s->device  = d;
    s->sampler = Ref<Sampler>(sp);
    s->dense   = g.dense != 0;
    const uint32_t T = 1u << log2TableSize;
    s->E.tableSize   = T;
    s->E.tableMask   = T - 1;
    for (int l = 0; l < kLv; ++l) {
      const float r  = std::floor(baseResolution * std::pow(growth, (float)l));
      s->E.res[l]    = (uint32_t)std::max(1.f, r);
      const double r1 = (double)s->E.res[l] + 1.0;
      s->E.dense[l]  = r1 * r1 * r1 <= (double)T ? 1u : 0u;
    }
    const vkl_box3f &b = sp->volume->bounds;
    const float lo[3] = {b.lower.x, b.lower.y, b.lower.z}, hi[3] = {b.upper.x, b.upper.y, b.upper.z};
    for (int a = 0; a < 3; ++a) {
      s->E.lo[a]      = lo[a];
      const float ext = hi[a] - lo[a];
      s->E.inv[a]     = 1.f / (ext > 0.f ? ext : 1.f);
    }
    s->tableFloats = (uint64_t)kLv * T * 2;
    for (DeviceBuffer *buf : {&s->table32, &s->gTable, &s->mTable, &s->vTable})
      buf->alloc(s->tableFloats * 4);
    s->table16.alloc(s->tableFloats * 2);
    for (DeviceBuffer *buf : {&s->w32, &s->gW, &s->mW, &s->vW})
      buf->alloc(kNumW * 4);
    s->w16.alloc(kNumW * 2);
    for (DeviceBuffer *buf : {&s->table32, &s->gTable, &s->mTable, &s->vTable, &s->w32, &s->gW, &s->mW, &s->vW})
      cudaCheck(cudaMemset(buf->ptr, 0, buf->bytes), "memset");
    s->J.attr = 0;
    uint64_t nr = 1;
    for (int a = 0; a < 3; ++a) {
      s->J.regionDims[a] = (g.activeSize[a] + (1u << kRegionLog) - 1) >> kRegionLog;
      nr *= s->J.regionDims[a];
    }
    s->numRegions = nr;
    s->flags.alloc(nr);
    s->regionErr.alloc(nr * 4);
    s->regionSeen.alloc(nr * 4);
    s->scalars.alloc(16);
    cudaCheck(cudaMemset(s->flags.ptr, 1, nr), "memset");  // everything falls back until calibrated
    s->J.flags      = s->flags.as<uint8_t>();
    s->J.regionErr  = s->regionErr.as<float>();
    s->J.regionSeen = s->regionSeen.as<uint32_t>();
    cudaCheck(cudaDeviceGetAttribute(&s->numSMs, cudaDevAttrMultiProcessorCount, d->cudaDevice), "attribute");
    cudaCheck(cudaHostAlloc((void **)&s->errHost, 4, cudaHostAllocMapped), "surrogate error flag");
    *s->errHost = 0u;
    cudaCheck(cudaHostGetDevicePointer((void **)&s->errDev, s->errHost, 0), "surrogate error flag");
    return (VKLCudaSurrogate)s;
  } catch (const VklError &e) {
    delete s;
    d->setError(e.code, e.what());
  } catch (const std::exception &e) {
    delete s;
    d->setError(VKL_UNKNOWN_ERROR, e.what());
  }
  return nullptr;
}

extern "C" OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateSetParameters(VKLCudaSurrogate surrogate,
                                                                        const float *table,
                                                                        const float *weights)
{
  Surrogate *s = (Surrogate *)surrogate;
  return surrogateCall(s, [&]() {
    cudaStream_t st = s->device->stream;
    if (table) {
      cudaCheck(cudaMemcpyAsync(s->table32.ptr, table, s->tableFloats * 4, cudaMemcpyDefault, st), "copy");
      kToHalf<<<blocks(s->tableFloats, 256), 256, 0, st>>>(s->tableFloats, s->table32.as<float>(),
                                                           s->table16.as<__half>());
    }
    if (weights) {
      cudaCheck(cudaMemcpyAsync(s->w32.ptr, weights, kNumW * 4, cudaMemcpyDefault, st), "copy");
      kToHalf<<<blocks(kNumW, 256), 256, 0, st>>>(kNumW, s->w32.as<float>(), s->w16.as<__half>());
    }
    for (DeviceBuffer *buf : {&s->mTable, &s->vTable, &s->mW, &s->vW})
      cudaCheck(cudaMemsetAsync(buf->ptr, 0, buf->bytes, st), "memset");
    s->step = 0;
    cudaCheck(cudaStreamSynchronize(st), "surrogate parameters");
  });
}

extern "C" OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateGetParameters(VKLCudaSurrogate surrogate,
                                                                        float *table, float *weights)
{
  Surrogate *s = (Surrogate *)surrogate;
  return surrogateCall(s, [&]() {
    cudaStream_t st = s->device->stream;
    if (table)
      cudaCheck(cudaMemcpyAsync(table, s->table32.ptr, s->tableFloats * 4, cudaMemcpyDefault, st), "copy");
    if (weights)
      cudaCheck(cudaMemcpyAsync(weights, s->w32.ptr, kNumW * 4, cudaMemcpyDefault, st), "copy");
    cudaCheck(cudaStreamSynchronize(st), "surrogate parameters");
  });
}

extern "C" OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateGradient(VKLCudaSurrogate surrogate, unsigned int n,
                                                                   const vkl_vec3f *points, const float *targets,
                                                                   float *loss, float *tableGrad,
                                                                   float *weightGrad)
{
  Surrogate *s = (Surrogate *)surrogate;
  return surrogateCall(s, [&]() {
    requireDevice(points, "points");
    requireDevice(targets, "targets");
    s->checkTimeout();
    cudaStream_t st = s->device->stream;
    s->zeroGrads(st);
    cudaCheck(cudaMemsetAsync(s->scalars.ptr, 0, 4, st), "memset");
    s->train(n, (const float *)points, targets, s->scalars.as<float>(), st);
    if (loss)
      cudaCheck(cudaMemcpyAsync(loss, s->scalars.ptr, 4, cudaMemcpyDefault, st), "copy");
    if (tableGrad)
      cudaCheck(cudaMemcpyAsync(tableGrad, s->gTable.ptr, s->tableFloats * 4, cudaMemcpyDefault, st), "copy");
    if (weightGrad)
      cudaCheck(cudaMemcpyAsync(weightGrad, s->gW.ptr, kNumW * 4, cudaMemcpyDefault, st), "copy");
    cudaCheck(cudaStreamSynchronize(st), "surrogate gradient");
    s->checkTimeout();
    s->zeroGrads(st);
  });
}

extern "C" OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateTrainStep(VKLCudaSurrogate surrogate, unsigned int n,
                                                                    const vkl_vec3f *points, const float *targets,
                                                                    float learningRate, float *loss)
{
  Surrogate *s = (Surrogate *)surrogate;
  return surrogateCall(s, [&]() {
    requireDevice(points, "points");
    requireDevice(targets, "targets");
    s->checkTimeout();
    if (n == 0)
      return;
    cudaStream_t st = s->device->stream;
    if (loss) {
      requireDevice(loss, "loss");
      cudaCheck(cudaMemsetAsync(loss, 0, 4, st), "memset");
    }
    s->train(n, (const float *)points, targets, loss, st);
    s->adam(n, learningRate, st);
  });
}

extern "C" OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateCalibrate(VKLCudaSurrogate surrogate, unsigned int n,
                                                                    const vkl_vec3f *points, float threshold,
                                                                    unsigned int *flaggedRegions)
{
  Surrogate *s = (Surrogate *)surrogate;
  return surrogateCall(s, [&]() {
    requireDevice(points, "points");
    s->checkTimeout();
    cudaStream_t st = s->device->stream;
    cudaCheck(cudaMemsetAsync(s->regionErr.ptr, 0, s->numRegions * 4, st), "memset");
    cudaCheck(cudaMemsetAsync(s->regionSeen.ptr, 0, s->numRegions * 4, st), "memset");
    cudaCheck(cudaMemsetAsync(s->scalars.ptr, 0, 4, st), "memset");
    if (n)
      s->infer<1>(n, (const float *)points, nullptr, 0, st);
    kRegionFlags<<<blocks(s->numRegions, 256), 256, 0, st>>>(s->numRegions, s->regionErr.as<float>(),
                                                             s->regionSeen.as<uint32_t>(), threshold,
                                                             s->flags.as<uint8_t>(), s->scalars.as<unsigned int>());
    unsigned int f = 0;
    cudaCheck(cudaMemcpyAsync(&f, s->scalars.ptr, 4, cudaMemcpyDeviceToHost, st), "copy");
    cudaCheck(cudaStreamSynchronize(st), "surrogate calibration");
    s->checkTimeout();
    if (flaggedRegions)
      *flaggedRegions = f;
  });
}

extern "C" OPENVKL_CUDA_INTERFACE VKLError vklCudaSurrogateSample(VKLCudaSurrogate surrogate, unsigned int n,
                                                                 const vkl_vec3f *points, float *samples,
                                                                 int fallback)
{
  Surrogate *s = (Surrogate *)surrogate;
  return surrogateCall(s, [&]() {
    requireDevice(points, "points");
    requireDevice(samples, "samples");
    s->checkTimeout();
    if (n)
      s->infer<0>(n, (const float *)points, samples, fallback, s->device->stream);
  });
}

extern "C" OPENVKL_CUDA_INTERFACE void vklCudaGetSurrogateInfo(VKLCudaSurrogate surrogate, uint64_t *tableEntries,
                                                              unsigned int *numWeights, uint64_t *numRegions,
                                                              unsigned int *levelResolutions)
{
  Surrogate *s = (Surrogate *)surrogate;
  if (!s)
    return;
  if (tableEntries)
    *tableEntries = s->tableFloats / 2;
  if (numWeights)
    *numWeights = kNumW;
  if (numRegions)
    *numRegions = s->numRegions;
  if (levelResolutions)
    for (int l = 0; l < kLv; ++l)
      levelResolutions[l] = s->E.res[l];
}

extern "C" OPENVKL_CUDA_INTERFACE void vklCudaReleaseSurrogate(VKLCudaSurrogate surrogate)
{
  delete (Surrogate *)surrogate;
}
