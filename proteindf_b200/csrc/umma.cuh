// Blackwell (sm_100a) tensor-core building blocks: mbarriers, bulk async
// copies, TMEM allocation, tcgen05.mma (kind::f16, BF16 in, FP32 accumulate)
// and tcgen05.ld, written as inline PTX.
//
// Operand layout ("packed K-major"): a matrix of R rows (R % 128 == 0) and K
// columns (K % 64 == 0) of BF16 is stored as tiles of 128 rows; a tile is a
// sequence of 64-column slabs (16 KiB each); inside a slab the 8x8 core
// matrices are ordered [k8][r8] with 8 rows of 16 bytes each:
//   off(r, k) = (r / 128) * 128 * K * 2 + (k / 64) * 16384
//             + (((k % 64) / 8) * 16 + (r % 128) / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// A slab is contiguous, so one cp.async.bulk moves it into shared memory, where
// it is the canonical SWIZZLE_NONE K-major layout of the UMMA shared-memory
// descriptor: 8-row groups SBO = 128 B apart, 8-column groups LBO = 2048 B
// apart; the K = 16 step kk of a slab starts at kk * 4096 B.
#pragma once

#include <cstdint>

namespace pdfxc {
namespace umma {

constexpr int TILE_ROWS = 128;
constexpr int SLAB_K = 64;
constexpr uint32_t SLAB_BYTES = TILE_ROWS * SLAB_K * 2;  // 16 KiB
constexpr uint32_t LBO = 2048;                           // next 8-column group
constexpr uint32_t SBO = 128;                            // next 8-row group
constexpr uint32_t WAIT_LIMIT = 1u << 26;                // bounded spin (several seconds)

__host__ __device__ inline size_t packed_offset(int r, int k, int K) {
    return (size_t)(r / 128) * 128 * K * 2 + (size_t)(k / 64) * 16384 +
           (size_t)((((k % 64) / 8) * 16 + (r % 128) / 8) * 128 + (r % 8) * 16 + (k % 8) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Named barrier over n threads (a multiple of 32, whole warps).
__device__ __forceinline__ void named_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

// Named barrier over n threads that also returns the AND of every thread's flag, so that all
// of them take the same branch after it.
__device__ __forceinline__ bool named_and(int id, int n, bool flag) {
    uint32_t out;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(out)
        : "r"((uint32_t)flag), "r"(id), "r"(n)
        : "memory");
    return out != 0;
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: gives up (returns false, and the caller records an error)
// after limit_ns (about one second by default), or at once when another CTA has
// already recorded an error in *err.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, const int* err,
                                          uint64_t limit_ns = 1000000000ull) {
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255) == 255) {
            if (*reinterpret_cast<const volatile int*>(err) != 0) return false;
            if (globaltimer_ns() - t0 > limit_ns) return false;
        }
    }
    return false;
}

// 1-D bulk copy global -> shared, completing tx bytes on `bar`.
// dst, src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// 4-D tensor copy global -> shared through a tensor map (no multicast), completing its bytes
// on `bar`. The map lives in kernel-parameter space; c0 is the innermost coordinate.
__device__ __forceinline__ void tensor4_g2s(void* dst, const void* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, SWIZZLE_NONE, K-major.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    // base offset 0, LBO mode 0, layout type 0 (no swizzle)
    return d;
}

// Instruction descriptor, kind::f16: BF16 x BF16 -> FP32, both K-major.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N) {
    return (1u << 4)                      // D format F32
           | (1u << 7)                    // A format BF16
           | (1u << 10)                   // B format BF16
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(M >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// ---- INT8 operands (kind::i8, exact int32 accumulation) -------------------
// Packed layout of an int8 matrix (R % 128 == 0 rows, K % 64 == 0 columns):
// 128-row tiles, 64-byte K slabs (8 KiB), core matrices of 8 rows x 16 bytes
// ordered [k16][r8] inside a slab. LBO = 2048 B, SBO = 128 B as for BF16;
// one MMA consumes K = 32 (two 16-byte groups), step kk at kk * 4096 B.
constexpr uint32_t I8_SLAB_K = 64;
constexpr uint32_t I8_SLAB_BYTES = TILE_ROWS * I8_SLAB_K;  // 8 KiB

__host__ __device__ inline size_t packed_offset_i8(int r, int k, int K) {
    return (size_t)(r / 128) * 128 * K + (size_t)(k / 64) * I8_SLAB_BYTES +
           (size_t)((((k % 64) / 16) * 16 + (r % 128) / 8) * 128 + (r % 8) * 16 + (k % 16));
}

// kind::i8: signed INT8 x signed INT8 -> S32, both K-major.
__host__ __device__ constexpr uint32_t instr_desc_s8(int M, int N) {
    return (2u << 4)                      // D format S32
           | (1u << 7)                    // A format signed 8-bit
           | (1u << 10)                   // B format signed 8-bit
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(M >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma_s8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// 32 lanes x 16 consecutive 32-bit columns per thread, raw bits.
__device__ __forceinline__ void tmem_ld16_raw(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// 32 lanes x 8 consecutive 32-bit columns per thread, raw bits.
__device__ __forceinline__ void tmem_ld8_raw(uint32_t taddr, uint32_t* r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}

// 32 lanes x 1 32-bit column per thread, raw bits.
__device__ __forceinline__ void tmem_ld1_raw(uint32_t taddr, uint32_t& r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 lanes x 16 consecutive 32-bit columns per thread.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace pdfxc
