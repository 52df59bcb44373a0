// Inline-PTX helpers for the sm_100a kernels of the row-block (Chebyshev-filtered subspace) path:
// mbarriers, 2-D TMA tile loads, and the tcgen05 tensor-core instructions (TMEM allocation,
// shared-memory operand descriptors, MMA issue, commit, TMEM loads).
//
// Operand layout used here: an MN-major TF32 operand, for which the tensor cores accept one
// shared-memory layout only, the 128-byte swizzle with 32-byte atomicity (descriptor layout type
// SWIZZLE_128B_BASE32B); a TMA tile load with CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B and a 128-byte
// inner box writes exactly that.  An "MN block" is 32 elements (128 bytes) wide; a tile of R rows
// (the K dimension) of one MN block is R x 128 bytes, row r at byte 128 r with its four 32-byte
// chunks permuted by r mod 4, so a swizzle atom is 4 rows (512 bytes, the SBO between K atoms).  One
// MMA of kind::tf32 consumes K = 8 rows (two atoms, 1024 bytes); the MN blocks of a wider operand
// sit LBO bytes apart.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "common.h"

namespace b200 {
namespace ptx {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait on a phase: false when it did not complete within kSpinLimit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (long long it = 0; it < kSpinLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 2-D tile load through a tensor map: box at (x = inner coordinate, y = outer coordinate).
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tmap, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// ---- tcgen05 (one CTA, cta_group::1)

// Allocate ncols TMEM columns (a power of two >= 32); the address is written to *dst (shared).
// Issued by one full warp.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: start address, leading and stride byte offsets, descriptor
// version 1 (sm_100), base offset 0 (atoms aligned to their swizzle period), layout type 1 =
// 128-byte swizzle with 32-byte atomicity (the layout of MN-major TF32 operands).
__device__ __forceinline__ uint64_t smem_desc_sw128_32b(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // version
  d |= (uint64_t)1 << 61;  // SWIZZLE_128B_BASE32B
  return d;
}

// Instruction descriptor of kind::tf32 with FP32 accumulation, both operands MN-major, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32_mn(int M, int N) {
  return (1u << 4)                      // D format F32
         | (2u << 7) | (2u << 10)       // A, B format TF32
         | (1u << 15) | (1u << 16)      // A, B MN-major
         | ((uint32_t)(N >> 3) << 17)   // N / 8
         | ((uint32_t)(M >> 4) << 24);  // M / 16
}

// D (TMEM) += A * B (shared-memory descriptors); accumulate = false overwrites D.
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
// Arrive on an mbarrier once every tcgen05 operation issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// Eight consecutive 32-bit TMEM columns of this thread's lane (32x32b shape; warp w of the four
// sub-partitions reads lanes 32 w .. 32 w + 31).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace ptx
}  // namespace b200
