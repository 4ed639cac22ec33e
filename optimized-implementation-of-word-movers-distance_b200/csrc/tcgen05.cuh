// tcgen05 / TMA / mbarrier primitives shared by the tensor-core kernels
// (sm_100a inline PTX).  Descriptor bit layouts follow the PTX ISA's
// shared-memory matrix descriptor and kind::f16 instruction descriptor.
#pragma once
#include <cuda.h>
#include <stdint.h>

#include "wmd_internal.cuh"

namespace wmd {
namespace tc {

constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s bound per wait
constexpr uint32_t kSuspendNs = 100000;  // try_wait suspend hint (upper bound)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// Waits for the phase of parity `par` to complete.  Bounded: returns false
// (and flags the error word) after limit_ns of wall-clock time.  Each
// try_wait carries a suspend-time hint, so a waiting thread sleeps in
// hardware until the phase completes instead of spinning on issue slots that
// the MMA-issuing and converting warps of the same SM sub-partition need.
__device__ __forceinline__ bool mbar_wait_ns(uint64_t* bar, uint32_t par,
                                             unsigned* err,
                                             unsigned long long limit_ns) {
  const uint32_t a = smem_u32(bar);
  unsigned long long t0 = 0;
  for (uint32_t i = 0;; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(par), "r"(kSuspendNs)
        : "memory");
    if (done) return true;
    if ((i & 63) == 0) {
      const unsigned long long t = gtime();
      if (t0 == 0) t0 = t;
      else if (t - t0 > limit_ns) {
        atomicOr(err, ERR_TIMEOUT);
        return false;
      }
    }
  }
}
// The kernels' wait: bounded by kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t par,
                                          unsigned* err) {
  return mbar_wait_ns(bar, par, err, kWaitNs);
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm,
                                            uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (tile rows are 128 bytes, stored back to back).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;               // leading byte offset (unused, SW128 K-major)
  d |= (uint64_t)(1024u >> 4) << 32;     // stride byte offset: next 8-row group
  d |= (uint64_t)1u << 46;               // descriptor version (sm_100)
  d |= (uint64_t)2u << 61;               // SWIZZLE_128B
  return d;
}
// Instruction descriptor of kind::f16 / kind::tf32: FP32 accumulate, A/B
// K-major, fmt 0 = FP16, 1 = BF16, 2 = TF32 (both operands), M x N tile.
__host__ __device__ constexpr uint32_t make_idesc(int fmt, int M, int N) {
  return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b,
                                        uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
          d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b,
                                         uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
          d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
        "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
        "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace wmd
