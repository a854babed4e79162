// sm_100a building blocks for the tensor-core (tcgen05) kernels: shared-memory
// matrix descriptors, the BF16 -> FP32 instruction descriptor, TMEM
// allocation / loads, mbarriers with bounded waits and bulk copies.
//
// Operand layout used throughout: K-major with the 128-byte swizzle.  A tile of
// R rows x 64 BF16 (128 bytes per row) starts on a 1024-byte boundary; row r
// sits at (r / 8) * 1024 + (r % 8) * 128 and its 16-byte chunk j (elements
// 8j .. 8j+7) at chunk position j ^ (r % 8).  The descriptor of such a tile has
// stride 1024 bytes between 8-row groups; stepping K by 16 elements moves the
// start address by 32 bytes.
#pragma once

#include <cstdint>

namespace ftb {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void * p) { return (uint32_t) __cvta_generic_to_shared(p); }

// byte offset of element (row r, k) inside a swizzled K-major tile (BF16, 64 per row)
__host__ __device__ __forceinline__ uint32_t sw128_offset(int r, int k) {
    return (uint32_t) ((r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 3) ^ (r & 7)) & 7) << 4) + (k & 7) * 2);
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t) ((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t) 1 << 16;                          // leading byte offset (unused with this swizzle)
    d |= (uint64_t) (1024 >> 4) << 32;                // stride byte offset
    d |= (uint64_t) 1 << 46;                          // descriptor version (sm_100)
    d |= (uint64_t) 2 << 61;                          // 128-byte swizzle
    return d;
}

// instruction descriptor: BF16 x BF16 -> FP32, A and B K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (N >> 3) << 17) | ((uint32_t) (M >> 4) << 24);
}

// instruction descriptor: S8 x S8 -> S32 (exact integer accumulation), A and B K-major, M x N
__host__ __device__ constexpr uint32_t idesc_s8(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (N >> 3) << 17) | ((uint32_t) (M >> 4) << 24);
}

// byte offset of byte k of row r inside a K-major tile with the 64-byte swizzle (64 one-byte
// elements a row): the 16-byte chunk index XOR address bits 7-8, 8-row groups 512 bytes apart
__host__ __device__ __forceinline__ uint32_t sw64_byte(int r, int k) {
    return (uint32_t) ((r >> 3) * 512 + (r & 7) * 64 + ((((k >> 4) ^ (r >> 1)) & 3) << 4) + (k & 15));
}

// shared-memory matrix descriptor: K-major, 64-byte swizzle, 8-row groups 512 bytes apart
__device__ __forceinline__ uint64_t desc_sw64(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t) ((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t) 1 << 16;                          // leading byte offset (unused with this swizzle)
    d |= (uint64_t) (512 >> 4) << 32;                 // stride byte offset
    d |= (uint64_t) 1 << 46;                          // descriptor version (sm_100)
    d |= (uint64_t) 4 << 61;                          // 64-byte swizzle
    return d;
}

// D[tmem] (+)= A[smem] * B[smem]^T over 8-bit signed integers, 32-bit integer accumulation, one thread
__device__ __forceinline__ void mma_s8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t) accumulate));
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t) accumulate));
}

// arrive on an mbarrier once every tcgen05 operation this thread issued so far has completed
__device__ __forceinline__ void commit(uint64_t * bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                 :: "r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// generic-proxy shared-memory writes visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// TMEM allocation (whole warp); the base address is written to *dst
__device__ __forceinline__ void tmem_alloc(uint32_t * dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" :: "r"(smem_addr(dst)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(base), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32 (w % 4) ..)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float * v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float * v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns without waiting: several loads can be in flight
// before one tmem_wait_ld()
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t * r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld8_async(uint32_t taddr, uint32_t * r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// ---- integer slices at the full FP32 rate ----
// Nearest integer, ties to even, for |t| < 2^22: adding 1.5 * 2^23 leaves a value whose unit in
// the last place is 1, so the addition rounds t to an integer; subtracting it back is exact.
// (rintf gives the same value, up to the sign of a zero result, through a conversion-class
// instruction that runs at an eighth of the FP32 rate.)
__device__ __forceinline__ float round_small(float t) {
    return __fsub_rn(__fadd_rn(t, 12582912.0f), 12582912.0f);
}
// Two integer-valued floats with at most 8 significant bits (|i| <= 256) as a BF16 pair (lo in
// the low half): their FP32 words end in 16 zero bits, so the BF16 values are the high halves
// exactly; a byte permute instead of a conversion-class instruction.
__device__ __forceinline__ uint32_t pack_bf16_ints(float lo, float hi) {
    return __byte_perm(__float_as_uint(lo), __float_as_uint(hi), 0x7632);
}

// ---- mbarriers ----
__device__ __forceinline__ void mbar_init(uint64_t * bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t * bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" :: "r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t * bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// The waiting thread may be suspended (up to the hint, 0.1 ms) until the phase
// completes, which leaves its issue slots to the warps doing work.
__device__ __forceinline__ bool mbar_try_wait(uint64_t * bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity), "r"(100000u) : "memory");
    return ok != 0;
}

// Wait for the phase of the given parity to complete.  Gives up after about
// 2^32 SM cycles (two seconds at full clock) or when *abort is set, and then
// returns false; no wait in these kernels is unbounded.
__device__ __forceinline__ bool mbar_wait(uint64_t * bar, uint32_t parity, volatile int * abort) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > (1LL << 32)) return false;
    }
    return true;
}

// bring bytes (a multiple of 16, 16-byte aligned) of global memory into L2
__device__ __forceinline__ void prefetch_l2(const void * src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" :: "l"(src), "r"(bytes) : "memory");
}

// bulk copy global -> shared, completing `bytes` on the mbarrier (both addresses
// 16-byte aligned, bytes a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void * dst, const void * src, uint32_t bytes, uint64_t * bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

}  // namespace tc
}  // namespace ftb
