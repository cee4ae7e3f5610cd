// tcgen05 (fifth-generation tensor core) building blocks for sm_100a: the
// split-BF16 product of the precision form.
//
// Operands live in shared memory in the K-major layout without swizzle: for
// every 8-element step of K ("k column"), a row-major array [rows][8] of BF16
// (16 bytes per row). In the tcgen05 matrix descriptor that is
//   core matrix      = 8 rows x 16 bytes, rows 16 bytes apart,
//   stride (SBO)     = 128 bytes between core matrices adjacent in M (or N),
//   leading (LBO)    = rows * 16 bytes between core matrices adjacent in K.
// An MMA of M = 128 reads 16 row groups per k column. When an operand has
// fewer real rows than the MMA's M (or N), the missing rows are "virtual":
// their addresses fall into the next k columns (finite data of this tile) or
// into the padding after the tile, and they only feed accumulator rows (or
// columns) that are never read. Every buffer is followed by enough padding
// that those reads stay inside the block's shared memory.
//
// The accumulator D (FP32) is in tensor memory: M = 128 rows = TMEM lanes,
// N columns. The product of two FP64-accurate operands is recovered from three
// BF16 slices of each, x = x0 + x1 + x2 (each slice the BF16 rounding of the
// remainder, 24 significant bits in all), and the six products
// x_i y_j with i + j <= 2 (the dropped ones are below 2^-24 of the result).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace pa {
namespace umma {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Matrix descriptor: K-major, no swizzle (layout type 0), descriptor version 1.
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  return d;
}

// Instruction descriptor of tcgen05.mma kind::f16: D FP32 (bits 4-5 = 1), A and
// B BF16 (bits 7-9 and 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at
// bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

// D (+)= A B^T for one K = 16 step, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrives on the mbarrier once every tcgen05 operation issued so far by this
// thread is complete.
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's shared-memory writes visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Tensor-memory allocation by one whole warp; the address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 8 consecutive FP32 columns of this warp's 32 TMEM lanes (lane quarter
// warp % 4), one column per register; followed by wait_ld before use.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_async_smem();
}

// Waits for the phase with the given parity to complete; gives up after about
// 2^32 clock cycles (about two seconds) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > (1LL << 32)) return false;
  }
}

// x = s0 + s1 + s2 with every slice the BF16 rounding of the remainder.
__device__ __forceinline__ void split3(float x, __nv_bfloat16& s0, __nv_bfloat16& s1, __nv_bfloat16& s2) {
  s0 = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(s0);
  s1 = __float2bfloat16_rn(r1);
  s2 = __float2bfloat16_rn(r1 - __bfloat162float(s1));
}
__device__ __forceinline__ void split3(double x, __nv_bfloat16& s0, __nv_bfloat16& s1, __nv_bfloat16& s2) {
  s0 = __double2bfloat16(x);
  const double r1 = x - static_cast<double>(__bfloat162float(s0));
  s1 = __double2bfloat16(r1);
  s2 = __double2bfloat16(r1 - static_cast<double>(__bfloat162float(s1)));
}

// Byte offset of element (row, k) in one slice of an operand with `rows` real
// rows per k column.
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int rows) {
  return static_cast<uint32_t>((k >> 3) * rows * 16 + row * 16 + (k & 7) * 2);
}

// The six slice pairs (i, j), i + j <= 2, smallest first.
__device__ __forceinline__ int pair_a(int p) { return p == 0 ? 2 : (p == 1 ? 1 : (p == 2 ? 0 : (p == 3 ? 1 : 0))); }
__device__ __forceinline__ int pair_b(int p) { return p == 0 ? 0 : (p == 1 ? 1 : (p == 2 ? 2 : (p == 3 ? 0 : (p == 4 ? 1 : 0)))); }

// D[128 x N] = sum over the K columns of A (arows real rows) x B (brows real
// rows), all six slice pairs; issued by one thread. a_slice / b_slice: byte
// distance between the slices of an operand.
__device__ __forceinline__ void issue_split_product(uint32_t tmem_d, uint32_t a0, uint32_t a_slice, int arows,
                                                    uint32_t b0, uint32_t b_slice, int brows, int K,
                                                    uint32_t idesc) {
  const uint32_t lbo_a = static_cast<uint32_t>(arows) * 16, lbo_b = static_cast<uint32_t>(brows) * 16;
  for (int k16 = 0; k16 < K / 16; ++k16) {
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int i = pair_a(p), j = pair_b(p);
      const uint64_t ad = desc_kmajor(a0 + i * a_slice + k16 * 2 * lbo_a, lbo_a, 128);
      const uint64_t bd = desc_kmajor(b0 + j * b_slice + k16 * 2 * lbo_b, lbo_b, 128);
      mma_bf16(tmem_d, ad, bd, idesc, (k16 | p) != 0);
    }
  }
}

}  // namespace umma
}  // namespace pa
