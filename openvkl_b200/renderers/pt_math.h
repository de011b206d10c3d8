// Elementary functions of the density path tracer, written out so that the
// CUDA renderer and its CPU restatement (the oracle) round identically: the
// same source, every operation a single IEEE float add, multiply or divide
// in source order (the renderer is built with --fmad=false, the oracle with
// -ffp-contract=off), so the images compare bit for bit.  The reference's
// renderer calls its platform's log / sin / cos (ISPC stdlib, SYCL
// native::), whose results differ between platforms in the last bits.
//
// pt_log: natural logarithm by the method of Cody and Waite ("Software
// Manual for the Elementary Functions", 1980): x = 2^e * m with m in
// [sqrt(1/2), sqrt(2)), log(m) = 2 atanh(s) with s = (m - 1) / (m + 1),
// |s| <= 0.1716, summed as the series s + s^3/3 + ... + s^13/13 (truncation
// below 1e-12 relative), and e * ln 2 added from a two-part split of ln 2
// (a high part with few significant bits, so e * high is exact).
//
// pt_sincos: Cody-Waite argument reduction by pi/2 (k = nearest integer to
// x * 2/pi, r = (x - k * C1) - k * C2 with pi/2 = C1 + C2, C1 exact in few
// bits) to r in about [-pi/4, pi/4], then the Taylor polynomials of sin
// (through r^13/13!) and cos (through r^12/12!) in Horner form, and the
// quadrant's swap and signs.  Meant for the arguments the path tracer
// passes (0 <= x < 2 pi); the reduction stays accurate for |x| up to a few
// thousand.
//
// Both are accurate to a few float ulps (checked against double precision
// in tests/test_pt_math.py); NaN and the special cases of log return NaN /
// -inf / +inf as log does.
#pragma once

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define PT_HD __host__ __device__ __forceinline__
#else
#define PT_HD static inline
#endif

PT_HD uint32_t pt_float_bits(float x)
{
  uint32_t u;
  memcpy(&u, &x, 4);
  return u;
}
PT_HD float pt_bits_float(uint32_t u)
{
  float x;
  memcpy(&x, &u, 4);
  return x;
}

PT_HD float pt_log(float x)
{
  const uint32_t u = pt_float_bits(x);
  if (x != x || (u >> 31) != 0u) {  // NaN, negative values and -0
    if (x == 0.f)
      return -pt_bits_float(0x7f800000u);
    return pt_bits_float(0x7fc00000u);
  }
  if (x == 0.f)
    return -pt_bits_float(0x7f800000u);
  if (u == 0x7f800000u)
    return x;
  // x = 2^e * m, m in [1, 2) (denormals scaled up first)
  int e        = 0;
  uint32_t b   = u;
  if ((b >> 23) == 0u) {
    b = pt_float_bits(x * 8388608.f);  // 2^23
    e = -23;
  }
  e += (int)(b >> 23) - 127;
  float m = pt_bits_float((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421356f) {  // m in [sqrt(1/2), sqrt(2))
    m = m * 0.5f;
    e = e + 1;
  }
  const float s  = (m - 1.f) / (m + 1.f);
  const float s2 = s * s;
  float p        = 1.f / 13.f;
  p              = p * s2 + 1.f / 11.f;
  p              = p * s2 + 1.f / 9.f;
  p              = p * s2 + 1.f / 7.f;
  p              = p * s2 + 1.f / 5.f;
  p              = p * s2 + 1.f / 3.f;
  const float lm = 2.f * s + 2.f * s * (s2 * p);
  // ln 2 = 0.693145751953125 + 1.42860682030941723212e-6
  const float fe = (float)e;
  return fe * 0.693145751953125f + (lm + fe * 1.42860682030941723212e-6f);
}

PT_HD void pt_sincos(float x, float *sinx, float *cosx)
{
  // k = round(x * 2/pi)
  const float kf = x * 0.636619772f;
  const float k  = (float)(int)(kf + (kf >= 0.f ? 0.5f : -0.5f));
  // pi/2 = 1.5703125 + 4.83826794896619231321691639751442e-4
  const float r  = (x - k * 1.5703125f) - k * 4.83826794896619231321691639751442e-4f;
  const float r2 = r * r;
  float sp       = 1.f / 6227020800.f;  // 1/13!
  sp             = sp * r2 - 1.f / 39916800.f;
  sp             = sp * r2 + 1.f / 362880.f;
  sp             = sp * r2 - 1.f / 5040.f;
  sp             = sp * r2 + 1.f / 120.f;
  sp             = sp * r2 - 1.f / 6.f;
  const float sr = r + r * (r2 * sp);
  float cp       = 1.f / 479001600.f;  // 1/12!
  cp             = cp * r2 - 1.f / 3628800.f;
  cp             = cp * r2 + 1.f / 40320.f;
  cp             = cp * r2 - 1.f / 720.f;
  cp             = cp * r2 + 1.f / 24.f;
  cp             = cp * r2 - 0.5f;
  const float cr = 1.f + r2 * cp;
  const int q    = ((int)k) & 3;
  *sinx          = q == 0 ? sr : q == 1 ? cr : q == 2 ? -sr : -cr;
  *cosx          = q == 0 ? cr : q == 1 ? -sr : q == 2 ? -cr : sr;
}
