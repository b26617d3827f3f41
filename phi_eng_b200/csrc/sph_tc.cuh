// 5th-generation tensor core (tcgen05) building blocks for sm_100a: tensor
// memory (TMEM) allocation, shared-memory matrix descriptors, the MMA issue,
// its completion through an mbarrier, and TMEM loads. PTX ISA 8.6+,
// "Tensor Core 5th Generation Family Instructions".
//
// Conventions used here:
//   - one CTA of 128 threads (4 warps) owns an M = 128 tile; row m of the
//     tile lives in TMEM lane m, and warp w reads lanes 32w..32w+31;
//   - operands are bf16 / fp16 in shared memory, K-major, no swizzle: a
//     "core matrix" is 8 rows x 16 bytes stored contiguously (row r of the
//     core matrix at byte 16 r). Element (row, k) of a matrix with K columns
//     sits at byte  (row / 8) * (K * 16) + (k / 8) * 128 + (row % 8) * 16
//     + (k % 8) * 2: the K-direction core matrices of an 8-row group are
//     adjacent (128 bytes apart, the descriptor's leading byte offset) and
//     8-row groups are K * 16 bytes apart (its stride byte offset). One MMA
//     consumes K = 16, i.e. two core matrices per row group; the k-th slice
//     starts 256 k bytes into the matrix.
//   - accumulators are f32; D = A B^T with A [M][K] (activations) and B
//     [N][K] (weights W[out][in]), so D[m][n] = sum_k A[m][k] W[n][k].
// Every wait is bounded: a caller that sees a wait run out records an error,
// gives the in-flight MMA one more bounded wait, frees its TMEM and returns.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace phieng {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (tcgen05 "matrix descriptor"): start
// address, leading / stride byte offsets (all >> 4, 14 bits), descriptor
// version 1 at bits 46-47, base offset 0, no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16 with f32 accumulation, both operands
// K-major, M = 128: D format f32 (bits 4-5 = 1), A and B format (bits 7-9,
// 10-12: 0 = f16, 1 = bf16, the same for both), N >> 3 at bits 17-22,
// M >> 4 at bits 24-28.
constexpr uint32_t kFmtF16 = 0, kFmtBF16 = 1;
__host__ __device__ constexpr uint32_t idesc_f16(uint32_t ab_format, uint32_t n) {
  return (1u << 4) | (ab_format << 7) | (ab_format << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

// D (+)= A B^T, issued by one thread; acc = 0 overwrites D.
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                        uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(acc)
      : "memory");
}

// The mbarrier's next phase completes once every tcgen05 operation this
// thread issued before has completed (its shared-memory reads included).
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for the phase of parity `parity` to complete, at most `limit` polls
// (each poll may suspend the thread for a hardware-defined interval).
// Returns false if the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t i = 0; i < limit; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Generic-proxy shared-memory writes made visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation of `cols` columns (a power of two >= 32) by one whole warp;
// the address lands in *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// 16 consecutive f32 columns of this thread's lane (warp w: lanes 32w + lane).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld2(uint32_t taddr, float (&v)[2]) {
  uint32_t r0, r1;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(taddr) : "memory");
  v[0] = __uint_as_float(r0);
  v[1] = __uint_as_float(r1);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset of element (row, k) in the no-swizzle K-major layout above,
// for a matrix with kcols columns.
__host__ __device__ constexpr uint32_t kmajor_offset(uint32_t row, uint32_t k, uint32_t kcols) {
  return (row >> 3) * (kcols * 16u) + (k >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

// One CTA-wide MMA step: every thread's operand writes (generic proxy) are
// made visible to the tensor core, thread 0 issues `issue` and commits to
// `bar`, and every thread waits for the completion (at most `limit` polls).
// The caller's TMEM reads must have completed (tmem_wait_ld) before. Returns
// false for every thread if the wait ran out; `phase` then stays at the
// incomplete phase.
template <class F>
__device__ __forceinline__ bool mma_step(uint64_t* bar, uint32_t& phase, uint32_t limit, F&& issue) {
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_after_sync();
    issue();
    commit(bar);
  }
  const bool done = mbar_wait(bar, phase, limit);
  if (__syncthreads_or(!done)) return false;
  phase ^= 1u;
  fence_after_sync();
  return true;
}

}  // namespace tc
}  // namespace phieng
