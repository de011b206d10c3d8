// Fifth-generation tensor core (tcgen05) building blocks for sm_100a, in
// inline PTX: tensor-memory (TMEM) allocation, shared-memory matrix
// descriptors for 128-byte-swizzled K-major operands, the single-thread
// kind::f16 MMA with its completion on an mbarrier, and TMEM loads.
//
// Operand layout (both A and B, K-major, 16-bit elements): rows of 128 bytes
// (64 elements of K), 8-row groups of 1024 bytes, the 16-byte chunk c of row
// r stored at chunk c ^ (r & 7) -- the 128-byte swizzle the descriptor's
// layout field names.  A buffer holding such rows must start on a 1024-byte
// boundary.  One MMA consumes K = 16 (32 bytes of each row); the K step is
// taken by advancing the descriptor's start address by 32 bytes inside the
// 128-byte row, the hardware applying the swizzle to the final address.
#pragma once

#include <stdint.h>

namespace vklcuda {
namespace tc {

__device__ __forceinline__ uint32_t smemAddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of 16-byte chunk c of row r in a 128-byte-swizzled K-major
// operand.
__device__ __forceinline__ uint32_t swizzledChunk(uint32_t r, uint32_t c)
{
  return (r >> 3) * 1024u + (r & 7u) * 128u + ((c ^ (r & 7u)) << 4);
}

// Shared-memory matrix descriptor: start address, leading byte offset
// (unused by swizzled K-major layouts; 16 bytes), stride byte offset 1024
// (between 8-row groups), descriptor version 1, 128-byte swizzle.
__device__ __forceinline__ uint64_t sw128Desc(uint32_t addr)
{
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(16u >> 4) << 16) | ((uint64_t)(1024u >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16: F16 A and B, F32 accumulator, both
// operands K-major, M x N.
__host__ __device__ constexpr uint32_t f16InstrDesc(int M, int N)
{
  return (1u << 4)                      // D format: F32
         | (0u << 7) | (0u << 10)       // A, B format: F16
         | (0u << 15) | (0u << 16)      // A, B K-major
         | ((uint32_t)(N >> 3) << 17)   // N / 8
         | ((uint32_t)(M >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mbarInit(uint64_t *bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the mbarrier phase with the given parity to complete, at most
// 2^22 polls; false if it gave up.
__device__ __forceinline__ bool mbarWait(uint64_t *bar, uint32_t parity)
{
  for (uint32_t it = 0; it < (1u << 22); ++it) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    if (ok)
      return true;
  }
  return false;
}

// TMEM allocation of `cols` columns (a power of two >= 32) by one whole warp;
// the base address is written to *dst (shared memory).
__device__ __forceinline__ void tmemAlloc(uint32_t *dst, uint32_t cols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(dst)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmemDealloc(uint32_t base, uint32_t cols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's generic-proxy shared-memory writes visible to the
// tensor core's (async proxy) reads.
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mmaF16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc,
                                       bool accumulate)
{
  asm volatile(
      "{ .reg .pred p; setp.ne.u32 p, %4, 0; "
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }" ::"r"(dTmem),
      "l"(aDesc), "l"(bDesc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}

// Arrives once on the mbarrier when every MMA this thread issued before has
// completed.
__device__ __forceinline__ void commitTo(uint64_t *bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddr(bar))
               : "memory");
}

// 32 consecutive 32-bit columns of this thread's TMEM lane (warp w of the
// CTA reads lanes 32 (w % 4) ..; taddr carries the lane in its upper half).
__device__ __forceinline__ void tmemLoad32(uint32_t taddr, uint32_t (&r)[32])
{
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void tmemLoadWait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace tc
}  // namespace vklcuda
