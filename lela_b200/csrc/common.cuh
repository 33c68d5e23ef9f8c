// lela_b200/csrc/common.cuh -- shared device helpers for the sm_100a kernels:
// modular arithmetic (Barrett reduction), bounded mbarrier waits, TMA and
// tcgen05 (5th-generation tensor core) inline-PTX wrappers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace lela {

// ------------------------------------------------------------ status codes
enum : int {
  ST_OK = 0,
  ST_ARG = 1,          // invalid argument (dimension, modulus, pointer)
  ST_CUDA = 2,         // CUDA runtime error
  ST_NOMEM = 3,        // device allocation failed
  ST_DIAG = 4,         // DiagonalEntryNotInvertible (trsm)
  ST_WRONG_FORM = 5,   // WrongMatrixForm (Faugere-Lachartre input)
  ST_PIVOT = 6,        // pivot not invertible in the ring (echelon)
  ST_TIMEOUT = 7,      // a bounded device-side wait expired
  ST_UNSUPPORTED = 8,  // configuration not supported by this build
  ST_CAPACITY = 9,     // an output array is too small (the result is kept)
};

// Device-side error flags written by kernels (bit mask, OR-ed).
enum : uint32_t {
  DEVERR_TIMEOUT = 1u,
};

// ------------------------------------------------------ modular arithmetic
//
// Barrett reduction (P. Barrett, CRYPTO '86) of a 64-bit value by a modulus
// p in [2, 2^32): with mu = floor((2^64 - 1) / p) the quotient estimate
// q = floor(v * mu / 2^64) satisfies floor(v/p) - 2 <= q <= floor(v/p), so at
// most two corrections follow.
struct Modulus {
  uint64_t p;
  uint64_t mu;
};

__host__ __device__ inline Modulus make_modulus(uint32_t p) {
  Modulus m;
  m.p = p;
  m.mu = ~0ull / (uint64_t)p;
  return m;
}

__device__ __forceinline__ uint32_t mod_reduce(uint64_t v, const Modulus &m) {
  uint64_t q = __umul64hi(v, m.mu);
  uint64_t r = v - q * m.p;
  if (r >= m.p) r -= m.p;
  if (r >= m.p) r -= m.p;
  return (uint32_t)r;
}

__device__ __forceinline__ uint32_t mod_mul(uint32_t a, uint32_t b, const Modulus &m) {
  return mod_reduce((uint64_t)a * b, m);
}

// (a*x + b*y) mod p for a, x, b, y < p < 2^32.
__device__ __forceinline__ uint32_t mod_axpby(uint32_t a, uint32_t x, uint32_t b, uint32_t y,
                                              const Modulus &m) {
  uint32_t s = mod_mul(a, x, m);
  uint32_t t = mod_mul(b, y, m);
  uint64_t u = (uint64_t)s + t;
  return (uint32_t)(u >= m.p ? u - m.p : u);
}

// Modular inverse with the semantics of Modular<uint32>::inv
// (lela/ring/modular.h:460-474, eea at :540-557): the extended Euclidean
// algorithm runs in 32-bit signed ints (ModularTraits<uint32>::EEAElement,
// modular.h:210), so all coefficient arithmetic wraps modulo 2^32.  The
// iterative form below yields the same Bezout coefficient modulo 2^32 as the
// reference's recursion (both are ring operations on the same quotient
// sequence).  Exact for p < 2^31; for p >= 2^31 it reproduces the reference's
// wrapped result, normally a failure.  Returns 0 when the reference reports
// "not invertible".
__host__ __device__ inline uint32_t lela_inv_u32(uint32_t p, uint32_t x) {
  int32_t r0 = (int32_t)x, r1 = (int32_t)p;
  int32_t s0 = 1, s1 = 0;
  while (r1 != 0) {
    int32_t q, r;
    if (r1 == -1) {
      q = (int32_t)(0u - (uint32_t)r0);
      r = 0;
    } else {
      q = r0 / r1;
      r = r0 % r1;
    }
    r0 = r1;
    r1 = r;
    int32_t s = (int32_t)((uint32_t)s0 - (uint32_t)q * (uint32_t)s1);
    s0 = s1;
    s1 = s;
  }
  if (r0 != 1) return 0;
  int32_t ty = s0;
  if (ty < 0) ty = (int32_t)((uint32_t)ty + p);
  uint32_t out = (uint32_t)ty;
  if ((uint64_t)out >= (uint64_t)p) out -= p;
  return out;
}

// 2^64 mod p (the delayed-reduction correction of ZpModule<uint32>,
// lela/ring/modular.h:604-626).
__host__ __device__ inline uint32_t two64_mod(uint32_t p) {
  uint64_t t = 2;
  for (int i = 0; i < 6; ++i) t = (t * t) % p;
  return (uint32_t)t;
}

// ------------------------------------------------------ bounded waiting
//
// Every spin-wait in these kernels is bounded: after WAIT_LIMIT_NS of
// global time the waiter records DEVERR_TIMEOUT in the kernel's error word
// and gives up, so a broken pipeline ends the kernel instead of hanging the
// GPU.  Waiters also poll the error word so that one role's failure
// releases the others.
constexpr uint64_t WAIT_LIMIT_NS = 4000000000ull;  // 4 s

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Asynchronous global -> shared copies of 4 or 8 bytes (cp.async; the
// source is read only when `valid`, else the destination is zero-filled),
// completed by cp_async_wait_all().
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait until the phase with the given parity has completed.  Returns false
// (after setting DEVERR_TIMEOUT) when the wait limit expires or another
// role has already reported an error.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t *err) {
  if (mbar_try_wait(bar, parity)) return true;
  uint64_t t0 = globaltimer_ns();
  uint32_t spins = 0;
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((++spins & 63u) == 0) {
      if (*(volatile uint32_t *)err != 0) return false;
      if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
        atomicOr(err, DEVERR_TIMEOUT);
        return false;
      }
    }
  }
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// ------------------------------------------------------------------ TMA
// 3-D tiled bulk tensor load global -> shared of this CTA only, completion
// counted on an mbarrier.
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, uint64_t *bar, int c0,
                                            int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)tmap), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// Prefetch the 128-byte line holding ptr into L2 (a hint; no data moves to
// registers).
__device__ __forceinline__ void prefetch_l2(const void *ptr) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

__device__ __forceinline__ void prefetch_tmap(const void *tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)tmap) : "memory");
}

// ------------------------------------------------------------- tcgen05
// Tensor-memory allocation is warp-wide; the allocated base column address
// is written to shared memory.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor for a K-major operand laid out by a TMA
// load with 128-byte swizzling: rows of 128 bytes, 8-row (1024-byte) swizzle
// atoms stacked at a stride of 1024 bytes.  Fields: start address >> 4
// (bits 0-13), leading byte offset >> 4 (16-29, unused for swizzled K-major
// layouts, set to 1), stride byte offset >> 4 (32-45), descriptor version 1
// (46-47), layout 2 = 128-byte swizzle (61-63).
__device__ __forceinline__ uint64_t smem_desc_sw128(const void *smem) {
  uint64_t addr = (uint64_t)(smem_u32(smem) & 0x3FFFFu) >> 4;
  uint64_t d = 0;
  d |= addr;
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// Instruction descriptor for tcgen05.mma .kind::i8: unsigned 8-bit A and B
// (format 0), signed 32-bit accumulator (format 2), both K-major, shape
// M x N.  Bits: D format 4-5, A format 7-9, B format 10-12, A/B major 15/16,
// N >> 3 at 17-22, M >> 4 at 24-28.
__host__ __device__ constexpr uint32_t idesc_u8_s32(int M, int N) {
  return (2u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_u8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Signal an mbarrier once all previously issued tcgen05 operations of this
// thread have completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// Load 16 consecutive 32-bit accumulator columns of this warp's 32 TMEM
// lanes (thread i gets lane i of the warp's quadrant).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace lela
