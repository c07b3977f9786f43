// tcgen05.cuh -- small helpers for hand-written sm_100a tensor-core kernels:
// shared-memory matrix descriptors (canonical layouts, no swizzle), the INT8
// MMA issue with a caller-given instruction descriptor, commits, bounded
// mbarrier waits, TMEM loads and 8-byte cp.async copies.
//
// Layout conventions (no swizzle, 16-byte core-matrix rows):
//   K-major operand (rows x K bytes): element (row, k) at
//       (row / 8) * SBO + (k / 16) * LBO + (row % 8) * 16 + k % 16
//   MN-major operand (K x MN bytes): element (k, mn) at
//       (k / 8) * LBO + (mn / 16) * SBO + (k % 8) * 16 + mn % 16
// Instruction descriptor of kind::i8 (u8 x u8 -> s32): D type s32 at bits 4-5,
// A and B unsigned (bits 7-12 zero), A major at bit 15 (0 = K-major), B major at
// bit 16 (1 = MN-major), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
#pragma once
#include <cstdint>

namespace tcg {

typedef uint32_t u32;

constexpr u32 idesc_i8(u32 m, u32 n, bool b_mn_major) {
    return (2u << 4) | ((b_mn_major ? 1u : 0u) << 16) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

// A waiting thread sleeps in mbarrier.try_wait (woken when the phase completes,
// at the latest after kSuspendNs) and gives up after kWaitCycles (about a second).
constexpr u32 kSuspendNs = 20000;
constexpr long long kWaitCycles = 1ll << 31;

__device__ __forceinline__ u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t sdesc(u32 saddr, u32 lbo, u32 sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version (sm_100); base offset 0, no swizzle
    return d;
}

__device__ __forceinline__ void mma_i8(u32 d_tmem, uint64_t a, uint64_t b, u32 idesc, u32 accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit(u32 bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void arrive(u32 bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_init(u32 bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool try_parity(u32 bar, u32 parity) {
    u32 done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return done != 0;
}

// true once the phase with the given parity has completed (bounded; the clock
// is read only when the first try finds the phase open)
__device__ __forceinline__ bool wait_parity(u32 bar, u32 parity) {
    if (try_parity(bar, parity)) return true;
    const long long t0 = clock64();
    do {
        if (try_parity(bar, parity)) return true;
    } while (clock64() - t0 < kWaitCycles);
    return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void named_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
// barrier over the n threads of group `id` that returns the OR of v (one decision for the group)
__device__ __forceinline__ bool group_any(int id, int n, bool v) {
    u32 r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\t"
                 "selp.u32 %0, 1, 0, q;\n\t}\n"
                 : "=r"(r)
                 : "r"((u32)v), "r"(id), "r"(n)
                 : "memory");
    return r != 0;
}

// 8-byte asynchronous global -> shared copy; src_bytes 0 stores zeros
__device__ __forceinline__ void cp8(u32 dst, const void* src, u32 src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Untiled bulk copy global -> shared that completes `bytes` of the transaction
// count of mbarrier `bar` (16-byte aligned addresses, size a multiple of 16).
// The barrier's expected count is raised first by expect_tx (one arrival).
__device__ __forceinline__ void expect_tx(u32 bar, u32 bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(bar),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(u32 dst, const void* src, u32 bytes, u32 bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// 32 TMEM lanes x 8 columns (with the wait, as below)
__device__ __forceinline__ void tmem_ld8(u32 taddr, u32 (&r)[8]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr));
}

// 32 TMEM lanes x 32 columns: lane L of the warp gets columns 0 .. 31 of lane L.
// The wait is part of the same statement, so no use of r is scheduled before it.
__device__ __forceinline__ void tmem_ld32(u32 taddr, u32 (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

}  // namespace tcg
