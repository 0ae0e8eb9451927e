// tcgen05 / mbarrier helpers shared by the tensor-core gradient kernels
// (k_grad_tc.cu, k_grad_cov.cu): shared-memory matrix descriptors in the
// SWIZZLE_NONE K-major canonical layout, kind::tf32 MMA issue and commit,
// TMEM loads, and bounded mbarrier waits.
#pragma once
#include <cstdint>

namespace fem25 {

// A bounded wait gives up after this many SM clocks (about half a second)
// unless the launch passes another limit.
constexpr long long kTcSpinCycles = 1000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// tcgen05 shared-memory matrix descriptor, SWIZZLE_NONE, K-major:
// LBO = distance between the two 16-byte K chunks of an MMA, SBO = distance
// between 8-row groups
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                 // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor of a kind::tf32 MMA: D f32, A/B tf32, both K-major
constexpr uint32_t tf32_idesc(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(mbar)
      : "memory");
}

// try_wait with a suspend-time hint (ns): the thread sleeps in hardware until
// the phase completes or the hint expires instead of re-polling shared memory
__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(phase), "r"(1000000u)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase.  Returns at once in drain mode; on
// running out (after `limit` SM clocks) it sets the error word and puts the
// CTA in drain mode.
__device__ __forceinline__ void mbar_wait(uint32_t mbar, uint32_t phase, volatile int *drain,
                                          int *err, int code, long long limit) {
  if (mbar_try_wait(mbar, phase)) return;  // the common case: already complete
  if (*drain) return;
  const long long t0 = clock64();
  while (!mbar_try_wait(mbar, phase)) {
    if (*drain) return;
    if (clock64() - t0 > limit) {
      atomicCAS(err, 0, code);
      *drain = 1;
      return;
    }
  }
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float *v) {
  uint32_t r0, r1, r2, r3;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(taddr));
  v[0] = __uint_as_float(r0);
  v[1] = __uint_as_float(r1);
  v[2] = __uint_as_float(r2);
  v[3] = __uint_as_float(r3);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// one TMEM column of the warp's 32 lanes
__device__ __forceinline__ uint32_t tmem_ld1(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
  return r;
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// byte offset of element (row, k) in a K-major SWIZZLE_NONE tile with the
// given distance between K chunks (LBO); core matrices of 8 rows x 16 bytes
__host__ __device__ __forceinline__ uint32_t kmajor_off(int row, int k, uint32_t lbo) {
  return (uint32_t)((row >> 3) * 128 + (row & 7) * 16 + (k >> 2) * lbo + (k & 3) * 4);
}

}  // namespace fem25
