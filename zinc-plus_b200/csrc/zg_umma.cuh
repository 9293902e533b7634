// sm_100a building blocks for the 5th-generation tensor cores: mbarriers,
// bulk copies global -> shared, tensor-memory (TMEM) allocation, tcgen05.mma
// issue and commit, TMEM loads, and the shared-memory and instruction
// descriptors they take.  Inline PTX, one instruction per wrapper.
//
// Every wait is bounded: mbar_wait gives up after a cycle limit and
// returns false, so that a kernel can record the failure, release its tensor
// memory and return instead of spinning.
#pragma once
#include <cstdint>

namespace zg {
namespace umma {

// Upper bound of one mbarrier wait, in SM clock cycles (clock64: a cheap
// per-SM counter; 2^31 cycles is about a second at the B200's clocks).
constexpr long long kWaitLimitCycles = 1ll << 31;

// Codes written to the device status word (device_status_word) by a kernel
// whose wait ran out.
enum : uint32_t { kStatusLoadTimeout = 1, kStatusMmaTimeout = 2, kStatusProbeTimeout = 4 };

// Records a timed-out wait in the device status word (mapped pinned host
// memory): a plain system-scope store, which every host link supports (device
// atomics on host memory need native host atomics).  Concurrent reporters may
// overwrite each other's code; the word is nonzero either way.
__device__ __forceinline__ void report_status(uint32_t *status, uint32_t code) {
    *reinterpret_cast<volatile uint32_t *>(status) = code;
    __threadfence_system();
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes initialised mbarriers visible to the async proxy (bulk copies, tcgen05).
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy reads (tcgen05.mma operands).
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Waits for the completion of the phase with parity `parity`; false when the
// time limit passed first.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kWaitLimitCycles) return false;
    }
}

// mbar_wait that also gives up once *abort (shared memory) is set, and sets it
// on its own timeout: the roles of a warp-specialised kernel then leave their
// loops together instead of each waiting out its own limit.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t *bar, uint32_t parity, volatile uint32_t *abort) {
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (*abort) return false;
        if (clock64() - t0 > kWaitLimitCycles) {
            *abort = 1;
            return false;
        }
    }
}

// Named barrier over `nthreads` threads (a multiple of 32) of the CTA.
__device__ __forceinline__ void named_bar_sync(uint32_t id, uint32_t nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from
// global to this CTA's shared memory; completion is counted on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// TMEM allocation (one full warp): writes the base address to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[adesc] x B[bdesc]^T, 8-bit integer operands, s32 accumulator.
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrives on `bar` when every tcgen05.mma this thread issued so far completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 consecutive 32-bit columns of this thread's TMEM lane (warp-wide; the
// warp's lanes are 32 * (warp % 4) + lane).  Complete after tmem_wait_ld.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory descriptor of a K-major operand in the 128-byte swizzle: rows
// of 128 bytes, eight-row atoms of 1024 bytes (1024-byte aligned), row r's
// 16-byte chunk j stored at chunk j ^ (r % 8).  `addr` is the operand's first
// byte for this K step (an atom base plus 0, 32, 64 or 96).
__device__ __forceinline__ uint64_t sdesc_k_sw128(uint32_t addr) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);  // start address, 16-byte units
    d |= (uint64_t)1 << 16;                           // leading byte offset (unused here)
    d |= (uint64_t)(1024 >> 4) << 32;                 // stride byte offset: next 8-row group
    d |= (uint64_t)1 << 46;                           // descriptor version of sm_100
    d |= (uint64_t)2 << 61;                           // 128-byte swizzle
    return d;
}

// Instruction descriptor of kind::i8 with an s32 accumulator, both operands
// K-major.  M in {64, 128}, N a multiple of 16 in [16, 256].
__host__ __device__ constexpr uint32_t idesc_i8(uint32_t M, uint32_t N, bool a_signed, bool b_signed) {
    return (2u << 4)                      // D format: s32
           | ((a_signed ? 1u : 0u) << 7)  // A: u8 / s8
           | ((b_signed ? 1u : 0u) << 10) // B: u8 / s8
           | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// Byte offset of (row, k) in a K-major 128-byte-swizzled tile of `rows` rows:
// [k / 128 atoms][rows][128 bytes].
__host__ __device__ inline uint32_t sw128_offset(uint32_t row, uint32_t k, uint32_t rows) {
    const uint32_t kin = k & 127u;
    return (k >> 7) * rows * 128u + row * 128u + ((((kin >> 4) ^ (row & 7u)) << 4) | (kin & 15u));
}

}  // namespace umma
}  // namespace zg
