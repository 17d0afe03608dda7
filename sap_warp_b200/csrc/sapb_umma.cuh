// sapb_umma.cuh -- thin inline-PTX wrappers for the sm_100a 5th-generation
// tensor core path (tcgen05): shared-memory matrix descriptors, the kind::f16
// MMA with TMEM accumulators, TMEM allocation and loads, mbarriers with
// bounded waits, and the proxy / thread-sync fences that order them.
//
// Operand images used by every caller: a matrix with R rows (R % 8 == 0) and
// K columns of bf16 is stored as 8x8 core matrices (8 rows x 16 bytes), core
// (row group rg, column group kg) at byte ((kg * R/8) + rg) * 128, each core
// row-major.  Read as a K-major operand (rows = M or N) the descriptor takes
// LBO = R/8 * 128 (next column group) and SBO = 128 (next row group); read
// as an MN-major operand (columns = M or N, rows = K) it takes LBO = 128 (next
// K group) and SBO = R/8 * 128 (next MN group).  No swizzle.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sapb {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Element offset of (row r, column k) in the core-matrix image of a matrix
// with `rows` rows.
__host__ __device__ __forceinline__ int core_off(int r, int k, int rows) {
  return ((k >> 3) * (rows >> 3) + (r >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

// Shared-memory matrix descriptor (no swizzle, version 1, base offset 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of tcgen05.mma kind::f16: BF16 A and B, FP32 D,
// dense, no negation; a_mn / b_mn select MN-major operands.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T over one K = 16 slice; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

// K-loop of MMAs over operand images: step s reads A at a + s*a_step and B at
// b + s*b_step.  `acc_first` = 0 overwrites D on the first slice.
__device__ __forceinline__ void mma_chain(uint32_t d_tmem, uint32_t a, uint32_t a_lbo, uint32_t a_sbo, uint32_t a_step,
                                          uint32_t b, uint32_t b_lbo, uint32_t b_sbo, uint32_t b_step, int ksteps,
                                          uint32_t idesc, uint32_t acc_first) {
  for (int s = 0; s < ksteps; ++s)
    mma_bf16(d_tmem, smem_desc(a + s * a_step, a_lbo, a_sbo), smem_desc(b + s * b_step, b_lbo, b_sbo), idesc,
             s > 0 ? 1u : acc_first);
}

// Arrive on `bar` when every tcgen05 operation issued so far by this thread
// has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of `bar` with at most `polls` polls (each try_wait
// suspends for a bounded, hardware-defined time).  False on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t polls) {
  for (uint32_t i = 0; i < polls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// TMEM allocation (one full warp), permit release and deallocation.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this warp's 32 TMEM lanes (lane = row),
// waited for before returning.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace sapb
