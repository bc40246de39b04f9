// Fifth-generation tensor-core primitives (tcgen05, sm_100a) in inline PTX:
// tensor-memory allocation, shared-memory matrix descriptors, the BF16 MMA
// with an FP32 accumulator in tensor memory, its commit to an mbarrier, and
// tensor-memory loads.  Written from the PTX ISA (version 8.6+) description
// of tcgen05; the descriptor bit layouts are those of the ISA's "shared memory
// descriptor" and "instruction descriptor" tables.
//
// Shared-memory operands use the K-major layout without swizzling: a tile of
// R rows x K bf16 is made of 8-row x 16-byte core matrices (8 rows x 8
// elements, rows 16 bytes apart); core matrices adjacent along K are LBO
// bytes apart and those adjacent along the rows SBO bytes apart.  Here every
// tile stores row r, element k at
//     (r / 8) * (16 K) + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// bytes, i.e. LBO = 128 and SBO = 16 K; the K-slice [16 s, 16 s + 16) of such
// a tile starts 256 s bytes after its base.  The same bytes read as an
// MN-major operand whose MN index is k and whose K index is r (the transposed
// matrix: 8 consecutive k contiguous, 8 r per core matrix) have LBO = 16 K
// (r groups) and SBO = 128 (k groups); its K-slice of rows [16 s, 16 s + 16)
// starts 32 K s bytes after the base.
//
// Every wait on an mbarrier is bounded (a clock budget): the kernels record a
// timeout in a status word instead of spinning forever.
#pragma once

#include <stdint.h>

namespace sns {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of (row, k) in a K-major, unswizzled tile of K columns.
__host__ __device__ constexpr int kmajor_off(int r, int k, int K) {
  return (r >> 3) * (16 * K) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// Shared-memory matrix descriptor: start address >> 4 (bits 0-13), leading
// byte offset >> 4 (16-29), stride byte offset >> 4 (32-45), descriptor
// version 1 (bits 46-47), base offset 0, absolute LBO mode 0, no swizzling
// (bits 61-63 = 0).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of tcgen05.mma kind::f16: dense, D in F32 (bits
// 4-5 = 1), A and B in BF16 (bits 7-9, 10-12 = 1), A and B K-major (bits 15,
// 16 = 0) or MN-major (= 1), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn = false,
                                                  bool b_mn = false) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// Arrive on the mbarrier once every MMA issued so far by this thread is done.
__device__ __forceinline__ void commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(mbar))
               : "memory");
}

// Tensor-memory allocation of ncols columns (a power of two >= 32) by one
// full warp; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes become visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 32 lanes x 16 columns of 32-bit accumulators: thread t of the warp gets
// lane (taddr lane + t), columns taddr..taddr+15.  The wait is in the same
// statement, so the registers are complete when it returns.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for the completion of the phase with parity `parity`; false once
// max_cycles SM clocks have passed without it.
__device__ __forceinline__ bool mbar_wait(uint64_t* m, uint32_t parity, long long max_cycles) {
  const uint32_t a = smem_u32(m);
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > max_cycles) return false;
  }
}

// About half a second at the B200's SM clock.
constexpr long long kWaitCycles = 1000000000ll;

}  // namespace tc
}  // namespace sns
