// Blackwell (sm_100a) tensor-core helpers: one CTA computes a 128 x N tile of
// dot products G[i][j] = sum_k A[i][k] * B[j][k] with tcgen05.mma kind::tf32,
// operands in shared memory, accumulator in tensor memory (TMEM).
//
// Shared-memory operand layout (K-major, no swizzle): the tile is stored as
// K/4 "column chunks" of 16 bytes (4 tf32 values) per row.  Chunk c of row r
// lives at   base + c * (ROWS * 16) + r * 16,
// so each 8-row x 16-byte core matrix is 128 contiguous bytes.  In the
// descriptor terms: stride-dimension byte offset (between 8-row groups) = 128,
// leading-dimension byte offset (between the two K chunks one MMA consumes)
// = ROWS * 16.  One MMA consumes K = 8 (two chunks); step s starts at chunk 2s.
//
// Accumulator: M = 128 rows map to TMEM lanes 0..127, column j of the tile to
// TMEM column (tmem_base + j).  Warp w of the CTA's first warpgroup reads
// lanes 32w..32w+31 (tcgen05.ld 32x32b).
//
// Every wait is bounded: after kSpinLimit polls the wait gives up, the caller
// records an error and skips the work that depended on it.
#pragma once

#include <cstdint>

namespace knng {
namespace tc {

constexpr uint32_t kSpinLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---------------------------------------------------------------- mbarrier

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrives once on the barrier and raises its expected transaction bytes.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Arrives once on the barrier.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bulk copy (the TMA engine's untiled form, this CTA's shared memory, no
// multicast) of `bytes` from global memory; completes `bytes` transactions on
// the barrier.  Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem_dst)),
                 "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Poll limit of the waits for work in progress (mbar_wait_limited) in this
// translation unit's kernels.  A diagnostic entry point may shorten it so a
// test can make such a wait run out; waits that drain a kernel's own copies
// before it exits always use kSpinLimit.
static __device__ uint32_t g_wait_limit = kSpinLimit;

__device__ __forceinline__ bool mbar_poll(uint32_t addr, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Waits for phase `parity` with this translation unit's poll limit.
__device__ __forceinline__ bool mbar_wait_limited(uint64_t* bar, uint32_t parity) {
    return mbar_poll(smem_u32(bar), parity, g_wait_limit);
}

// Polls phase `parity` of the barrier; returns false if the poll limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// ------------------------------------------------------------------- TMEM

// Allocates `ncols` TMEM columns (power of two >= 32); one whole warp calls it.
// The TMEM address is written to *slot (shared memory).
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

__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Generic-proxy shared-memory writes become visible to the tensor core.
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 8 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---------------------------------------------------------- cp.async

// 16-byte global -> shared copy that does not pass through registers; with
// `valid` false it writes 16 zero bytes and reads nothing.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc, bool valid) {
    const uint32_t d = smem_u32(smem_dst);
    const uint32_t sz = valid ? 16u : 0u;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gsrc), "r"(sz) : "memory");
}

// Waits until every cp.async this thread issued has landed (visible to this
// thread; other threads need a barrier after it).
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ---------------------------------------------------------------- MMA

// Shared-memory matrix descriptor, K-major, no swizzle (see the file comment).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);             // start address, bits [0,14)
    d |= static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16;   // leading byte offset, bits [16,30)
    d |= static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32;   // stride byte offset, bits [32,46)
    d |= static_cast<uint64_t>(1) << 46;                           // descriptor version 1 (sm_100)
    // base offset 0, leading-offset mode 0, layout type 0 (no swizzle)
    return d;
}

// Instruction descriptor: kind::tf32, F32 accumulate, A and B K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(uint32_t M, uint32_t N) {
    return (1u << 4)                // D format: F32
           | (2u << 7)              // A format: TF32
           | (2u << 10)             // B format: TF32
           | ((N >> 3) << 17)       // N / 8
           | ((M >> 4) << 24);      // M / 16
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t desc_a, uint64_t desc_b, uint32_t idesc,
                                         bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u;
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(desc_a), "l"(desc_b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

// Arrives on the mbarrier once every MMA this thread issued has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// Issues the K/8 MMAs of one 128 x N tile (call from a single thread).
// a_base / b_base: shared addresses of the chunk-major operand tiles with
// a_rows (= 128) and b_rows (= N) rows; kpad: K rounded up to 8.
__device__ __forceinline__ void issue_tile_tf32(uint32_t tmem_d, uint32_t a_base, uint32_t b_base, uint32_t a_rows,
                                                uint32_t b_rows, uint32_t kpad, uint32_t idesc) {
    for (uint32_t s = 0; s < kpad / 8; ++s) {
        const uint64_t da = smem_desc(a_base + 2 * s * a_rows * 16, a_rows * 16, 128);
        const uint64_t db = smem_desc(b_base + 2 * s * b_rows * 16, b_rows * 16, 128);
        mma_tf32(tmem_d, da, db, idesc, s > 0);
    }
}

// Instruction descriptor: kind::f16 with BF16 A and B, F32 accumulate, both
// K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N) {
    return (1u << 4)                // D format: F32
           | (1u << 7)              // A format: BF16
           | (1u << 10)             // B format: BF16
           | ((N >> 3) << 17)       // N / 8
           | ((M >> 4) << 24);      // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t desc_a, uint64_t desc_b, uint32_t idesc,
                                         bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u;
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(desc_a), "l"(desc_b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

// Instruction descriptor: kind::f16 with FP16 A and B, F32 accumulate, both
// K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_f16(uint32_t M, uint32_t N) {
    return (1u << 4)                // D format: F32
           | (0u << 7)              // A format: F16
           | (0u << 10)             // B format: F16
           | ((N >> 3) << 17)       // N / 8
           | ((M >> 4) << 24);      // M / 16
}

// Issues the K/16 MMAs of one 128 x N 16-bit tile (call from a single thread).
// The operand tiles (FP16 or BF16, as idesc says) use the same chunk-major
// layout as the TF32 ones, a 16-byte chunk holding 8 values; one MMA consumes
// K = 16 (two chunks).
__device__ __forceinline__ void issue_tile_16bit(uint32_t tmem_d, uint32_t a_base, uint32_t b_base, uint32_t a_rows,
                                                 uint32_t b_rows, uint32_t kpad, uint32_t idesc) {
    for (uint32_t s = 0; s < kpad / 16; ++s) {
        const uint64_t da = smem_desc(a_base + 2 * s * a_rows * 16, a_rows * 16, 128);
        const uint64_t db = smem_desc(b_base + 2 * s * b_rows * 16, b_rows * 16, 128);
        mma_bf16(tmem_d, da, db, idesc, s > 0);
    }
}

// Byte offset of element (row r, k) in a chunk-major tile with `rows` rows.
__host__ __device__ constexpr uint32_t chunk_offset(uint32_t r, uint32_t k, uint32_t rows) {
    return (k >> 2) * rows * 16 + r * 16 + (k & 3) * 4;
}

}  // namespace tc
}  // namespace knng
