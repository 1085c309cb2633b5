// Precision form of the bucket pass (KNNG_PRECISION_BF16_RERANK): the
// reference's addCandidatesLessThan (src/KnnSets.hpp:131-160) offers every
// other bucket member to a point's set with its exact FP32 distance.  Here the
// bucket's distances are first estimated on the tensor cores and only each
// point's 128 best candidates are offered, with exact distances:
//
//   1. the bucket's rows, centred on its first point, are rounded to BF16 and
//      multiplied on the tensor cores (tcgen05.mma kind::f16, FP32
//      accumulation): approx(i, j) = |x_i'|^2 + |x_j'|^2 - 2 bf16(x_i').bf16(x_j'),
//      with the norms of the FP32 centred rows; a block of 128 rows against a
//      tile of 128 columns at a time lands in TMEM;
//   2. one thread per row keeps the 128 smallest (estimate, bucket position)
//      keys seen so far in a max-heap in shared memory, reading every TMEM
//      column once: the kept set is every candidate whose estimate is below
//      the 128th smallest, then ties in bucket order;
//   3. each kept candidate gets the exact FP32 distance in the reference's
//      order and is offered to the point's set in bucket position order (the
//      order of the FP32 form), through the same warp-resident set update.
//
// Buckets of at most 1024 points (max_leaf <= 1025).  The result differs from
// the FP32 form only where a candidate outside a point's 128 best estimates
// would have entered its set.
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
constexpr int kBfMaxBucket = 1024;

template <int D>
struct BfLayout {
    static constexpr int KP = (D + 15) / 16 * 16;  // K padded to the MMA step (16 BF16)
    static constexpr int CH = KP / 8;              // 16-byte chunks per row
    static constexpr uint32_t tile_bytes = kBfRows * KP * 2;
    // A tile, B tile, every block row's heap of kept keys ([slot][row]),
    // norms of every bucket row, the centre, bucket ids.  Once a row block's
    // selection is done its kept bucket positions (ascending) take the tiles'
    // space.
    static constexpr uint32_t a = 0;
    static constexpr uint32_t b = a + tile_bytes;
    static constexpr uint32_t keep = a;
    static constexpr uint32_t heap = b + tile_bytes;
    static constexpr uint32_t norms = heap + kKeep * kBfRows * 8;
    static constexpr uint32_t centre = norms + kBfMaxBucket * 4;
    static constexpr uint32_t ids = centre + (D + 3) / 4 * 16;
    static constexpr uint32_t bytes = ids + kBfMaxBucket * 4;
    static_assert(kBfRows * kKeep * 2 <= 2 * tile_bytes, "kept positions fit the tiles' space");
};

// Max-heap of `n` keys in column `r` of a [slot][kBfRows] array: restores the
// heap order below slot i.
__device__ __forceinline__ void heap_sift_down(unsigned long long* __restrict__ h, uint32_t r, uint32_t n, uint32_t i) {
    const unsigned long long key = h[i * kBfRows + r];
    for (;;) {
        const uint32_t l = 2 * i + 1;
        if (l >= n) break;
        uint32_t c = l;
        unsigned long long cv = h[l * kBfRows + r];
        if (l + 1 < n) {
            const unsigned long long rv = h[(l + 1) * kBfRows + r];
            if (rv > cv) {
                c = l + 1;
                cv = rv;
            }
        }
        if (cv <= key) break;
        h[i * kBfRows + r] = cv;
        i = c;
    }
    h[i * kBfRows + r] = key;
}

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
                float* __restrict__ set_bound, int K, uint32_t* __restrict__ error_flag,
                const uint32_t* __restrict__ dcount, uint32_t* __restrict__ work) {
    using L = BfLayout<D>;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* A = smem + L::a;
    unsigned char* B = smem + L::b;
    unsigned long long* heap = reinterpret_cast<unsigned long long*>(smem + L::heap);
    uint16_t* keep = reinterpret_cast<uint16_t*>(smem + L::keep);
    float* norms = reinterpret_cast<float*>(smem + L::norms);
    float* centre = reinterpret_cast<float*>(smem + L::centre);
    uint32_t* ids = reinterpret_cast<uint32_t*>(smem + L::ids);
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ uint32_t next_s;
    const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
    if (warp == 0) tc::tmem_alloc(&tmem_slot, kBfCols);
    if (tid == 0) {
        tc::mbar_init(&mbar, 1);
        tc::fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    uint32_t phase = 0;
    bool healthy = true;
    const uint32_t idesc = tc::idesc_bf16(kBfRows, kBfCols);
    // One bucket per CTA, or (with `work`) buckets [0, *dcount) taken one at a
    // time from the work counter by a persistent grid.
    for (uint32_t round = 0; healthy; ++round) {
    uint32_t leaf;
    if (work) {
        if (tid == 0) next_s = atomicAdd(work, 1u);
        __syncthreads();
        leaf = next_s;
        __syncthreads();
        if (leaf >= *dcount) break;
    } else {
        if (round > 0) break;
        leaf = blockIdx.x;
    }
    const uint32_t s0 = starts[leaf];
    const uint32_t b = ends[leaf] - s0;
    if (b < 2) continue;
    for (uint32_t t = tid; t < b; t += kBfThreads) ids[t] = idx[s0 + t];
    __syncthreads();
    for (int k = tid; k < D; k += kBfThreads) centre[k] = pts[static_cast<size_t>(ids[0]) * ld + k];
    __syncthreads();
    // Buckets of at most 129 points keep every other member: no estimates,
    // and the tiles' space holds only the kept positions.
    const bool keep_all = b - 1 <= static_cast<uint32_t>(kKeep);
    if (!keep_all)
        for (uint32_t t = tid; t < b; t += kBfThreads) norms[t] = centred_norm<D>(pts, ld, ids[t], centre);
    for (uint32_t rb = 0; rb < b && healthy; rb += kBfRows) {
        const uint32_t cnt = min(static_cast<uint32_t>(kBfRows), b - rb);
        // The A tile overlays `keep`: staged only when estimates are made,
        // and read (by the MMA) only behind the column loop's barriers.
        if (!keep_all) stage_bf16<D>(A, ids + rb, cnt, pts, ld, centre);
        // Selection state of the row this thread owns (warps 0-3: TMEM lane r).
        const uint32_t r = static_cast<uint32_t>(warp * kWarp + lane);
        const uint32_t i = rb + r;  // bucket position of the row's point
        uint32_t n_in = 0;
        // The bucket's columns, one 128-column tile at a time.
        for (uint32_t cb = 0; cb < b && !keep_all; cb += kBfCols) {
            stage_bf16<D>(B, ids + cb, min(static_cast<uint32_t>(kBfCols), b - cb), pts, ld, centre);
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                tc::issue_tile_16bit(tmem, tc::smem_u32(A), tc::smem_u32(B), kBfRows, kBfCols, L::KP, idesc);
                tc::mma_commit(&mbar);
            }
            const bool done = tc::mbar_wait(&mbar, phase);
            phase ^= 1u;
            if (__syncthreads_or(!done)) {
                if (tid == 0) atomicExch(error_flag, 1u);
                tc::mbar_wait(&mbar, phase ^ 1u);
                healthy = false;
                break;
            }
            tc::fence_after_sync();
            if (warp < 4) {
                const float na = r < cnt ? norms[i] : 0.f;
                const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * kWarp) << 16);
                for (uint32_t j0 = 0; j0 < kBfCols && cb + j0 < b; j0 += 16) {  // warp-uniform
                    float g[16];
                    tc::tmem_ld16(taddr + j0, g);
                    tc::tmem_wait_ld();
                    if (r >= cnt) continue;
#pragma unroll 4
                    for (int u = 0; u < 16; ++u) {
                        const uint32_t j = cb + j0 + u;
                        if (j >= b || j == i) continue;
                        const float v = fmaxf(0.f, na + norms[j] - 2.0f * g[u]);
                        const unsigned long long key =
                            (static_cast<unsigned long long>(__float_as_uint(v)) << 32) | j;
                        if (n_in < static_cast<uint32_t>(kKeep)) {
                            heap[n_in * kBfRows + r] = key;
                            if (++n_in == static_cast<uint32_t>(kKeep))
                                for (int h = kKeep / 2 - 1; h >= 0; --h) heap_sift_down(heap, r, kKeep, h);
                        } else if (key < heap[r]) {
                            heap[r] = key;
                            heap_sift_down(heap, r, kKeep, 0);
                        }
                    }
                }
            }
            tc::fence_before_sync();
            __syncthreads();
        }
        if (!healthy) break;
        // Kept bucket positions of each row, ascending: every other member
        // when the bucket has at most 129 points, else the heap's.
        if (warp < 4 && r < cnt) {
            uint16_t* mine = keep + r * kKeep;
            uint32_t nk = 0;
            if (keep_all) {
                for (uint32_t j = 0; j < b; ++j)
                    if (j != i) mine[nk++] = static_cast<uint16_t>(j);
            } else {
                for (uint32_t h = 0; h < n_in; ++h) mine[nk++] = static_cast<uint16_t>(heap[h * kBfRows + r] & 0xFFFFu);
                for (uint32_t a2 = 1; a2 < nk; ++a2) {  // insertion sort of at most 128 positions
                    const uint16_t v = mine[a2];
                    uint32_t z = a2;
                    while (z > 0 && mine[z - 1] > v) {
                        mine[z] = mine[z - 1];
                        --z;
                    }
                    mine[z] = v;
                }
            }
            for (uint32_t t = nk; t < static_cast<uint32_t>(kKeep); ++t) mine[t] = 0xFFFFu;
        }
        __syncthreads();
        // Offers: warp w takes rows w, w + 8, ...; lanes take 32 kept
        // candidates at a time, in bucket order.
        for (uint32_t rr = static_cast<uint32_t>(warp); rr < cnt; rr += kBfThreads / kWarp) {
            const uint32_t p = ids[rb + rr];
            WarpSet s;
            set_load(s, set_dist, set_id, set_size, set_maxslot, set_bound, p, K, lane);
            const float4* prow = reinterpret_cast<const float4*>(pts + static_cast<size_t>(p) * ld);
            for (int g0 = 0; g0 < kKeep; g0 += kWarp) {
                const uint16_t j = keep[rr * kKeep + g0 + lane];
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
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kBfCols);
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
        tc::issue_tile_16bit(tmem, tc::smem_u32(A), tc::smem_u32(B), kBfRows, kBfCols, L::KP,
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
    if (h) fail(KNNG_ERR_CUDA, "BF16 tile: the MMA completion wait gave up");
}

void launch_leaves_bf16(Context& c, uint32_t count, const uint32_t* d_starts, const uint32_t* d_ends,
                        uint32_t max_bucket) {
    if (count == 0) return;
    if (max_bucket > static_cast<uint32_t>(kBfMaxBucket))
        fail(KNNG_ERR_INVALID_ARGUMENT, "the BF16 bucket pass takes buckets of at most 1024 points");
    auto* err = static_cast<uint32_t*>(scratch(c, "bf16_error", sizeof(uint32_t)));
    KNNG_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), c.stream));
    // One CTA per SM (the heaps take most of the shared memory), 128 TMEM
    // columns each.
    KNNG_DISPATCH_D(c.d, {
        auto kern = k_leaf_bf16<D>;
        allow_max_smem(c, kern);
        kern<<<count, kBfThreads, BfLayout<D>::bytes, c.stream>>>(d_starts, d_ends, c.indices, c.points, c.ld,
                                                                  c.set_dist, c.set_id, c.set_size, c.set_maxslot,
                                                                  c.set_bound, static_cast<int>(c.k), err, nullptr,
                                                                  nullptr);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    uint32_t h = 0;
    download(c, &h, err, 1);
    if (h) fail(KNNG_ERR_CUDA, "BF16 bucket pass: the MMA completion wait gave up");
}

void prepare_leaves_bf16_list(Context& c) {
    KNNG_DISPATCH_D(c.d, { allow_max_smem(c, k_leaf_bf16<D>); });
}

void launch_leaves_bf16_list(Context& c, const uint32_t* d_starts, const uint32_t* d_ends, const uint32_t* d_count,
                             uint32_t* d_work, uint32_t* d_error) {
    const int sms = c.sms;
    KNNG_DISPATCH_D(c.d, {
        auto kern = k_leaf_bf16<D>;
        allow_max_smem(c, kern);
        // Persistent: one CTA per SM takes the buckets from the work counter.
        kern<<<sms, kBfThreads, BfLayout<D>::bytes, c.stream>>>(d_starts, d_ends, c.indices, c.points, c.ld,
                                                                c.set_dist, c.set_id, c.set_size, c.set_maxslot,
                                                                c.set_bound, static_cast<int>(c.k), d_error, d_count,
                                                                d_work);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

}  // namespace knng
