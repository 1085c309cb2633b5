// Precision form of the bucket pass (KNNG_PRECISION_BF16_RERANK): the
// reference's addCandidatesLessThan (src/KnnSets.hpp:131-160) offers every
// other bucket member to a point's set with its exact FP32 distance.  Here the
// bucket's distances are first estimated on the tensor cores and only each
// point's 128 best candidates are offered, with exact distances:
//
//   1. the bucket's rows, centred on its first point, are rounded to BF16 and
//      multiplied on the tensor cores (tcgen05.mma kind::f16, FP32
//      accumulation): approx(i, j) = |x_i'|^2 + |x_j'|^2 - 2 bf16(x_i').bf16(x_j'),
//      with the norms of the FP32 centred rows; a block of 128 rows against the
//      whole bucket lands in TMEM (at most 512 columns);
//   2. one thread per row finds the 128th smallest estimate by bisection over
//      its bit pattern (non-negative floats order like their bits) and keeps
//      the candidates at or below it, ties in bucket order, 128 in all;
//   3. each kept candidate gets the exact FP32 distance in the reference's
//      order and is offered to the point's set in bucket position order (the
//      order of the FP32 form), through the same warp-resident set update.
//
// Buckets of at most 512 points (max_leaf <= 513).  The result differs from the
// FP32 form only where a candidate outside a point's 128 best estimates would
// have entered its set.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "context.hpp"
#include "dispatch.hpp"
#include "tc.cuh"

namespace knng {
namespace {

constexpr int kBfThreads = 256;
constexpr int kBfRows = 128;   // MMA M: rows per block
constexpr int kBfCols = 128;   // MMA N: columns per tile
constexpr int kKeep = 128;     // candidates re-ranked per point
constexpr int kBfMaxBucket = 512;

template <int D>
struct BfLayout {
    static constexpr int KP = (D + 15) / 16 * 16;  // K padded to the MMA step (16 BF16)
    static constexpr int CH = KP / 8;              // 16-byte chunks per row
    static constexpr uint32_t tile_bytes = kBfRows * KP * 2;
    // A tile, B tile, norms of every bucket row, the centre, bucket ids, and
    // every row's kept candidates (bucket positions, ascending)
    static constexpr uint32_t a = 0;
    static constexpr uint32_t b = a + tile_bytes;
    static constexpr uint32_t norms = b + tile_bytes;
    static constexpr uint32_t centre = norms + kBfMaxBucket * 4;
    static constexpr uint32_t ids = centre + (D + 3) / 4 * 16;
    static constexpr uint32_t keep = ids + kBfMaxBucket * 4;
    static constexpr uint32_t bytes = keep + kBfRows * kKeep * 2;
};

// Rows ids[r] (r < count) minus `centre`, rounded to BF16, into a chunk-major
// tile of 128 rows (rows past `count` and dims past D are zero).  Threads with
// consecutive indices take consecutive rows of one chunk.
template <int D>
__device__ __forceinline__ void stage_bf16(unsigned char* __restrict__ tile, const uint32_t* __restrict__ ids,
                                           uint32_t count, const float* __restrict__ pts, int ld,
                                           const float* __restrict__ centre) {
    constexpr int CH = BfLayout<D>::CH;
    for (int f = threadIdx.x; f < kBfRows * CH; f += kBfThreads) {
        const int r = f % kBfRows, ch = f / kBfRows;
        uint32_t packed[4] = {0u, 0u, 0u, 0u};
        if (static_cast<uint32_t>(r) < count) {
            const float* row = pts + static_cast<size_t>(ids[r]) * ld;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int k0 = 8 * ch + 4 * q;
                if (k0 < D) {
                    const float4 v = __ldg(reinterpret_cast<const float4*>(row + k0));
                    const float4 m = reinterpret_cast<const float4*>(centre)[k0 / 4];
                    const __nv_bfloat162 lo = __floats2bfloat162_rn(__fsub_rn(v.x, m.x), __fsub_rn(v.y, m.y));
                    const __nv_bfloat162 hi = __floats2bfloat162_rn(__fsub_rn(v.z, m.z), __fsub_rn(v.w, m.w));
                    packed[2 * q] = *reinterpret_cast<const uint32_t*>(&lo);
                    packed[2 * q + 1] = *reinterpret_cast<const uint32_t*>(&hi);
                }
            }
        }
        *reinterpret_cast<uint4*>(tile + static_cast<uint32_t>(ch) * kBfRows * 16 + static_cast<uint32_t>(r) * 16) =
            make_uint4(packed[0], packed[1], packed[2], packed[3]);
    }
}

// Squared norm of row `id` minus `centre` in FP32 (dims in order).
template <int D>
__device__ __forceinline__ float centred_norm(const float* __restrict__ pts, int ld, uint32_t id,
                                              const float* __restrict__ centre) {
    const float* row = pts + static_cast<size_t>(id) * ld;
    float s = 0.f;
#pragma unroll 4
    for (int k = 0; k < D; ++k) {
        const float t = __fsub_rn(__ldg(row + k), centre[k]);
        s = __fmaf_rn(t, t, s);
    }
    return s;
}

template <int D>
__global__ void __launch_bounds__(kBfThreads, 1)
    k_leaf_bf16(const uint32_t* __restrict__ starts, const uint32_t* __restrict__ ends,
                const uint32_t* __restrict__ idx, const float* __restrict__ pts, int ld, float* __restrict__ set_dist,
                uint32_t* __restrict__ set_id, uint32_t* __restrict__ set_size, uint32_t* __restrict__ set_maxslot,
                float* __restrict__ set_bound, int K, uint32_t tmem_cols, uint32_t* __restrict__ error_flag) {
    using L = BfLayout<D>;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* A = smem + L::a;
    unsigned char* B = smem + L::b;
    float* norms = reinterpret_cast<float*>(smem + L::norms);
    float* centre = reinterpret_cast<float*>(smem + L::centre);
    uint32_t* ids = reinterpret_cast<uint32_t*>(smem + L::ids);
    uint16_t* keep = reinterpret_cast<uint16_t*>(smem + L::keep);
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    const uint32_t s0 = starts[blockIdx.x];
    const uint32_t b = ends[blockIdx.x] - s0;
    if (b < 2) return;
    const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
    for (uint32_t t = tid; t < b; t += kBfThreads) ids[t] = idx[s0 + t];
    if (warp == 0) tc::tmem_alloc(&tmem_slot, tmem_cols);
    if (tid == 0) {
        tc::mbar_init(&mbar, 1);
        tc::fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    for (int k = tid; k < D; k += kBfThreads) centre[k] = pts[static_cast<size_t>(ids[0]) * ld + k];
    __syncthreads();
    for (uint32_t t = tid; t < b; t += kBfThreads) norms[t] = centred_norm<D>(pts, ld, ids[t], centre);
    uint32_t phase = 0;
    bool healthy = true;
    const uint32_t idesc = tc::idesc_bf16(kBfRows, kBfCols);
    for (uint32_t rb = 0; rb < b && healthy; rb += kBfRows) {
        const uint32_t cnt = min(static_cast<uint32_t>(kBfRows), b - rb);
        stage_bf16<D>(A, ids + rb, cnt, pts, ld, centre);
        // The bucket's columns, one 128-column tile at a time, into TMEM
        // columns [cb, cb + 128).
        for (uint32_t cb = 0; cb < b; cb += kBfCols) {
            stage_bf16<D>(B, ids + cb, min(static_cast<uint32_t>(kBfCols), b - cb), pts, ld, centre);
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                tc::issue_tile_bf16(tmem + cb, tc::smem_u32(A), tc::smem_u32(B), kBfRows, kBfCols, L::KP, idesc);
                tc::mma_commit(&mbar);
            }
            const bool done = tc::mbar_wait(&mbar, phase);
            phase ^= 1u;
            if (__syncthreads_or(!done)) {
                if (tid == 0) atomicExch(error_flag, 1u);
                healthy = false;
                break;
            }
            tc::fence_after_sync();
        }
        if (!healthy) break;
        // Selection: thread r of the first four warps owns row r (its TMEM lane).
        if (warp < 4) {
            const uint32_t r = static_cast<uint32_t>(warp * kWarp + lane);
            const uint32_t i = rb + r;  // bucket position of the row's point
            const float na = r < cnt ? norms[i] : 0.f;
            const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * kWarp) << 16);
            // Estimate bits of column j (+inf for the point itself and past b).
            auto bits_of = [&](uint32_t j, float g) -> uint32_t {
                if (j >= b || j == i) return 0x7F800000u;
                const float v = fmaxf(0.f, na + norms[j] - 2.0f * g);
                return __float_as_uint(v);
            };
            uint32_t thr = 0x7F800000u;  // keep every column below this, and ties in order
            if (b - 1 > static_cast<uint32_t>(kKeep)) {
                // Smallest bit pattern with at least 128 estimates at or below
                // it; 31 halvings cover [0, +inf] (a fixed count: the TMEM
                // loads are warp-collective).
                uint32_t lo = 0, hi = 0x7F800000u;
                for (int it = 0; it < 31; ++it) {
                    const uint32_t mid = lo + (hi - lo) / 2;
                    uint32_t c = 0;
                    for (uint32_t j0 = 0; j0 < b; j0 += 16) {
                        float g[16];
                        tc::tmem_ld16(taddr + j0, g);
                        tc::tmem_wait_ld();
#pragma unroll
                        for (int u = 0; u < 16; ++u) c += bits_of(j0 + u, g[u]) <= mid ? 1u : 0u;
                    }
                    if (c >= static_cast<uint32_t>(kKeep)) hi = mid; else lo = mid + 1;
                }
                thr = lo;
            }
            // Kept candidates in column order: every estimate below thr, then
            // ties at thr until 128.
            uint32_t below = 0;
            if (b - 1 > static_cast<uint32_t>(kKeep)) {
                for (uint32_t j0 = 0; j0 < b; j0 += 16) {
                    float g[16];
                    tc::tmem_ld16(taddr + j0, g);
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int u = 0; u < 16; ++u) below += bits_of(j0 + u, g[u]) < thr ? 1u : 0u;
                }
            }
            uint32_t ties_left = static_cast<uint32_t>(kKeep) - min(below, static_cast<uint32_t>(kKeep));
            uint32_t n_keep = 0;
            uint16_t* mine = keep + r * kKeep;
            for (uint32_t j0 = 0; j0 < b; j0 += 16) {
                float g[16];
                tc::tmem_ld16(taddr + j0, g);
                tc::tmem_wait_ld();
#pragma unroll
                for (int u = 0; u < 16; ++u) {
                    const uint32_t j = j0 + u;
                    const uint32_t v = bits_of(j, g[u]);
                    bool take;
                    if (b - 1 <= static_cast<uint32_t>(kKeep))
                        take = j < b && j != i;
                    else if (v < thr)
                        take = true;
                    else if (v == thr && ties_left > 0 && j < b && j != i) {
                        take = true;
                        --ties_left;
                    } else
                        take = false;
                    if (take && r < cnt && n_keep < static_cast<uint32_t>(kKeep)) mine[n_keep++] = static_cast<uint16_t>(j);
                }
            }
            for (uint32_t t = n_keep; t < static_cast<uint32_t>(kKeep); ++t) mine[t] = 0xFFFFu;
        }
        tc::fence_before_sync();
        __syncthreads();
        // Offers: warp w takes rows w, w + 8, ...; lanes take 32 kept
        // candidates at a time, in bucket order.
        for (uint32_t r = static_cast<uint32_t>(warp); r < cnt; r += kBfThreads / kWarp) {
            const uint32_t p = ids[rb + r];
            WarpSet s;
            set_load(s, set_dist, set_id, set_size, set_maxslot, set_bound, p, K, lane);
            const float4* prow = reinterpret_cast<const float4*>(pts + static_cast<size_t>(p) * ld);
            for (int g0 = 0; g0 < kKeep; g0 += kWarp) {
                const uint16_t j = keep[r * kKeep + g0 + lane];
                const bool valid = j != 0xFFFFu;
                const uint32_t cand = valid ? ids[j] : 0u;
                float d = 0.f;
                if (valid)
                    d = canonical_distance4_lean<D>(
                        reinterpret_cast<const float4*>(pts + static_cast<size_t>(cand) * ld), prow);
                set_offer_batch(s, cand, d, valid, K, lane);
            }
            set_store(s, set_dist, set_id, set_size, set_maxslot, set_bound, p, K, lane);
        }
        __syncthreads();
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, tmem_cols);
    }
}

// One 128 x 128 BF16 tile of a(m x D) . b(n x D)^T with FP32 accumulation
// (rows past m / n are zero); the diagnostic behind knng_debug_tile_gram_bf16.
template <int D>
__global__ void __launch_bounds__(kBfThreads, 1)
    k_tile_gram_bf16(const float* __restrict__ a, uint32_t m, const float* __restrict__ b, uint32_t n,
                     float* __restrict__ out, uint32_t* __restrict__ error_flag) {
    using L = BfLayout<D>;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* A = smem + L::a;
    unsigned char* B = smem + L::b;
    uint32_t* ids = reinterpret_cast<uint32_t*>(smem + L::ids);
    float* zero = reinterpret_cast<float*>(smem + L::centre);
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
    if (tid < kBfRows) ids[tid] = tid;
    for (int k = tid; k < D; k += kBfThreads) zero[k] = 0.0f;
    if (warp == 0) tc::tmem_alloc(&tmem_slot, kBfCols);
    if (tid == 0) {
        tc::mbar_init(&mbar, 1);
        tc::fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    stage_bf16<D>(A, ids, m, a, D, zero);
    stage_bf16<D>(B, ids, n, b, D, zero);
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        tc::fence_after_sync();
        tc::issue_tile_bf16(tmem, tc::smem_u32(A), tc::smem_u32(B), kBfRows, kBfCols, L::KP,
                            tc::idesc_bf16(kBfRows, kBfCols));
        tc::mma_commit(&mbar);
    }
    const bool done = tc::mbar_wait(&mbar, 0);
    if (__syncthreads_or(!done)) {
        if (tid == 0) atomicExch(error_flag, 1u);
    } else if (warp < 4) {
        tc::fence_after_sync();
        const uint32_t row = static_cast<uint32_t>(warp * kWarp + lane);
        for (uint32_t j0 = 0; j0 < kBfCols; j0 += 16) {
            float g[16];
            tc::tmem_ld16(tmem + (static_cast<uint32_t>(warp * kWarp) << 16) + j0, g);
            tc::tmem_wait_ld();
#pragma unroll
            for (int u = 0; u < 16; ++u)
                if (row < m && j0 + u < n) out[static_cast<size_t>(row) * n + j0 + u] = g[u];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kBfCols);
    }
}

}  // namespace

void run_tile_gram_bf16(Context& c, uint32_t d, const float* d_a, uint32_t m, const float* d_b, uint32_t n,
                        float* d_out) {
    auto* err = static_cast<uint32_t*>(scratch(c, "gram_error", sizeof(uint32_t)));
    KNNG_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), c.stream));
    KNNG_DISPATCH_D(d, {
        auto kern = k_tile_gram_bf16<D>;
        allow_max_smem(c, kern);
        kern<<<1, kBfThreads, BfLayout<D>::bytes, c.stream>>>(d_a, m, d_b, n, d_out, err);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    uint32_t h = 0;
    download(c, &h, err, 1);
    if (h) fail(KNNG_ERR_CUDA, "BF16 tile: the MMA completion wait timed out");
}

void launch_leaves_bf16(Context& c, uint32_t count, const uint32_t* d_starts, const uint32_t* d_ends,
                        uint32_t max_bucket) {
    if (count == 0) return;
    if (max_bucket > static_cast<uint32_t>(kBfMaxBucket))
        fail(KNNG_ERR_INVALID_ARGUMENT, "the BF16 bucket pass takes buckets of at most 512 points");
    auto* err = static_cast<uint32_t*>(scratch(c, "bf16_error", sizeof(uint32_t)));
    KNNG_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), c.stream));
    // TMEM for a whole row of the bucket: 256 columns up to 256 points (two
    // CTAs per SM), 512 above (one CTA per SM: the shared memory asked for
    // keeps a second one off the SM, so no CTA waits for TMEM).
    const uint32_t tmem_cols = max_bucket <= 256 ? 256u : 512u;
    KNNG_DISPATCH_D(c.d, {
        using L = BfLayout<D>;
        uint32_t smem = L::bytes;
        if (tmem_cols == 512u) smem = std::max<uint32_t>(smem, 120u * 1024u);
        auto kern = k_leaf_bf16<D>;
        allow_max_smem(c, kern);
        kern<<<count, kBfThreads, smem, c.stream>>>(d_starts, d_ends, c.indices, c.points, c.ld, c.set_dist, c.set_id,
                                                    c.set_size, c.set_maxslot, c.set_bound, static_cast<int>(c.k),
                                                    tmem_cols, err);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    uint32_t h = 0;
    download(c, &h, err, 1);
    if (h) fail(KNNG_ERR_CUDA, "BF16 bucket pass: the MMA completion wait timed out");
}

}  // namespace knng
