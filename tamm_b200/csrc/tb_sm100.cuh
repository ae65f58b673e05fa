// sm_100a primitives used by the tensor-core kernels: mbarriers with bounded waits,
// untiled bulk copies (cp.async.bulk, no multicast), UMMA shared-memory and
// instruction descriptors, tcgen05 MMA / commit / TMEM load / TMEM allocation.
#pragma once

#include <cstdint>

namespace tb::sm100 {

// Iteration cap of every device-side wait: a wait that exceeds it records an error
// code in *err and returns false instead of spinning forever.
constexpr uint32_t kWaitLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbarrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(
                 smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
    : "=r"(ok)
    : "r"(smem_u32(bar)), "r"(parity)
    : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase; on timeout sets *err (atomically, first code
// wins) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code) {
  for(uint32_t i = 0; i < kWaitLimit; i++)
    if(mbar_try_wait(bar, parity)) return true;
  atomicCAS(err, 0, code);
  return false;
}

// Global -> shared bulk copy completing on an mbarrier (no cluster multicast).
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
      smem_u32(smem_dst)),
    "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
    : "memory");
}

// UMMA shared-memory descriptor, K-major, no swizzle ("interleaved" canonical
// layout): 8-row x 16-byte core matrices; lbo = byte distance between the two
// 16-byte K halves of a 32-byte K step, sbo = byte distance between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t smem_addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t) ((smem_addr & 0x3FFFF) >> 4);
  d |= (uint64_t) ((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t) ((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t) 1 << 46; // descriptor version for sm_100
  // base offset 0, LBO mode 0, layout type 0 (no swizzle)
  return d;
}

// Instruction descriptor of tcgen05.mma kind::i8: S32 accumulator, K-major A and B,
// a_signed / b_signed pick s8 or u8 per operand, shape M x N.
__host__ __device__ constexpr uint32_t idesc_i8(int m, int n, bool a_signed, bool b_signed) {
  return (2u << 4)                          // D format: S32
         | ((a_signed ? 1u : 0u) << 7)      // A: 1 = s8, 0 = u8
         | ((b_signed ? 1u : 0u) << 10)     // B: 1 = s8, 0 = u8
         | (0u << 15) | (0u << 16)          // A, B K-major
         | ((uint32_t) (n >> 3) << 17)      // N / 8
         | ((uint32_t) (m >> 4) << 24);     // M / 16
}

// Instruction descriptor of tcgen05.mma kind::f16 with BF16 A/B and F32 accumulator.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4)                      // D format: F32
         | (1u << 7) | (1u << 10)       // A, B: BF16
         | ((uint32_t) (n >> 3) << 17) | ((uint32_t) (m >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       bool accumulate) {
  asm volatile(
    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
    "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t) accumulate));
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        bool accumulate) {
  asm volatile(
    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
    "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t) accumulate));
}

// Arrive on `bar` when every tcgen05.mma issued so far by this thread has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                 smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

// Warp-wide: allocate `ncols` TMEM columns, base address written to *dst (smem).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(dst)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols));
}

// Warp-wide: 16 consecutive 32-bit TMEM columns of this warp's 32 lanes (one lane
// per thread); complete with tmem_wait_ld() before use.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
    : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
}
// N consecutive columns (N a multiple of 4) into r[0..N), as x16 / x8 / x4 loads.
template<int N>
__device__ __forceinline__ void tmem_ld_cols(uint32_t taddr, uint32_t* r) {
  static_assert(N % 4 == 0, "columns in multiples of 4");
#pragma unroll
  for(int l = 0; l + 16 <= N; l += 16) tmem_ld16(taddr + l, *reinterpret_cast<uint32_t(*)[16]>(r + l));
  constexpr int R16 = N / 16 * 16;
  if constexpr((N - R16) >= 8) tmem_ld8(taddr + R16, *reinterpret_cast<uint32_t(*)[8]>(r + R16));
  constexpr int R8 = R16 + ((N - R16) >= 8 ? 8 : 0);
  if constexpr((N - R8) == 4) tmem_ld4(taddr + R8, *reinterpret_cast<uint32_t(*)[4]>(r + R8));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

__device__ __forceinline__ bool elect_one() {
  uint32_t pred = 0;
  asm volatile(
    "{\n\t.reg .b32 rx;\n\t.reg .pred px;\n\telect.sync rx|px, %1;\n\tselp.u32 %0, 1, 0, px;\n\t}\n"
    : "=r"(pred)
    : "r"(0xffffffffu));
  return pred != 0;
}

// 2^n as a double, n in [-1022, 1023], built from the IEEE-754 exponent field.
__device__ __forceinline__ double pow2i(int n) {
  return __longlong_as_double((long long) (n + 1023) << 52);
}

} // namespace tb::sm100
