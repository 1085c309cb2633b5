// Bucket all-pairs kernel: addCandidatesLessThan (src/KnnSets.hpp:131-160)
// for every bucket of a repetition at once, one CTA per bucket.
//
// The reference offers, for a point at bucket position q, the other members
// in position order (0..q-1 from the outer loop, then q+1..b-1 from its own
// inner loop), each offer gated by dist < bound and applied with
// KnnSetScannableSimd::addCandidateLessThan.  This kernel keeps that order
// exactly: for a block of 64 points (4 per warp, sets held in registers) it
// walks the bucket in 64-point column blocks in ascending order, computes the
// 64x64 distance block in the reference's FP32 order from dim-major shared
// memory tiles, then each warp replays its points' 64 offers in column order
// (set_offer_batch).  Distances are computed for the full b x b matrix (both
// triangles); each (i, j) and (j, i) evaluation gives the same bits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "common.cuh"
#include "context.hpp"
#include "dispatch.hpp"

namespace knng {
namespace {

constexpr int kLeafThreads = 512;
constexpr int kLeafWarps = kLeafThreads / kWarp;  // 16
constexpr int kBI = 64;                            // points updated per row block
constexpr int kBJ = 64;                            // candidates per column block
constexpr int kPtsPerWarp = kBI / kLeafWarps;      // 4
constexpr int kJPerThread = kBI * kBJ / kLeafThreads;  // 8
constexpr int kDmStride = kBJ + 1;

// rows [base, base+64) of the bucket -> tile[dim][r] (zeros past the bucket end)
template <int D>
__device__ __forceinline__ void load_tile(float* __restrict__ tile, const uint32_t* __restrict__ ids, uint32_t base,
                                          uint32_t b, const float* __restrict__ pts, int ld) {
    constexpr int Q = D / 4;
    for (int f = threadIdx.x; f < kBI * Q; f += kLeafThreads) {
        const int r = f % kBI, q = f / kBI;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (base + r < b) v = __ldg(reinterpret_cast<const float4*>(pts + static_cast<size_t>(ids[base + r]) * ld) + q);
        tile[(4 * q + 0) * kBI + r] = v.x;
        tile[(4 * q + 1) * kBI + r] = v.y;
        tile[(4 * q + 2) * kBI + r] = v.z;
        tile[(4 * q + 3) * kBI + r] = v.w;
    }
}

// Dm[i][j] = canonical distance(I row i, J row j), thread -> (i, 8 columns).
template <int D>
__device__ __forceinline__ void distance_block(const float* __restrict__ I, const float* __restrict__ J,
                                               float* __restrict__ Dm) {
    constexpr int M = D / 8 * 8;
    const int i = threadIdx.x % kBI;
    const int jg = threadIdx.x / kBI;  // 0..7
    const float4* J4 = reinterpret_cast<const float4*>(J);
    float tot[kJPerThread];
#pragma unroll
    for (int q = 0; q < kJPerThread; ++q) tot[q] = 0.0f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        float ch[kJPerThread];
#pragma unroll
        for (int q = 0; q < kJPerThread; ++q) ch[q] = 0.0f;
#pragma unroll
        for (int dim = c; dim < M; dim += 8) {
            const float a = I[dim * kBI + i];
            const float4 v0 = J4[dim * (kBJ / 4) + jg * 2 + 0];
            const float4 v1 = J4[dim * (kBJ / 4) + jg * 2 + 1];
            const float bv[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
#pragma unroll
            for (int q = 0; q < kJPerThread; ++q) {
                const float diff = __fsub_rn(a, bv[q]);
                ch[q] = __fmaf_rn(diff, diff, ch[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < kJPerThread; ++q) tot[q] = __fadd_rn(tot[q], ch[q]);
    }
#pragma unroll
    for (int dim = M; dim < D; ++dim) {
        const float a = I[dim * kBI + i];
        const float4 v0 = J4[dim * (kBJ / 4) + jg * 2 + 0];
        const float4 v1 = J4[dim * (kBJ / 4) + jg * 2 + 1];
        const float bv[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
#pragma unroll
        for (int q = 0; q < kJPerThread; ++q) {
            const float diff = __fsub_rn(a, bv[q]);
            tot[q] = __fadd_rn(tot[q], __fmul_rn(diff, diff));
        }
    }
#pragma unroll
    for (int q = 0; q < kJPerThread; ++q) Dm[i * kDmStride + jg * kJPerThread + q] = tot[q];
}

template <int D>
__global__ void __launch_bounds__(kLeafThreads, 2)
    k_leaf(const uint32_t* __restrict__ starts, const uint32_t* __restrict__ ends, const uint32_t* __restrict__ idx,
           const float* __restrict__ pts, int ld, float* __restrict__ set_dist, uint32_t* __restrict__ set_id,
           uint32_t* __restrict__ set_size, uint32_t* __restrict__ set_maxslot, float* __restrict__ set_bound,
           int K, const uint32_t* __restrict__ dcount, uint32_t* __restrict__ work) {
    extern __shared__ float4 smem4[];
    float* I = reinterpret_cast<float*>(smem4);
    float* J = I + D * kBI;
    float* Dm = J + D * kBJ;
    uint32_t* ids = reinterpret_cast<uint32_t*>(Dm + kBI * kDmStride);
    __shared__ uint32_t next_s;
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    // One bucket per CTA, or (with `work`) buckets [0, *dcount) taken one at a
    // time from the work counter by a persistent grid.
    for (uint32_t round = 0;; ++round) {
    uint32_t leaf;
    if (work) {
        if (threadIdx.x == 0) next_s = atomicAdd(work, 1u);
        __syncthreads();
        leaf = next_s;
        __syncthreads();
        if (leaf >= *dcount) break;
    } else {
        if (round > 0) break;
        leaf = blockIdx.x;
    }
    const uint32_t s = starts[leaf];
    const uint32_t b = ends[leaf] - s;
    if (b < 2) continue;
    for (uint32_t t = threadIdx.x; t < b; t += kLeafThreads) ids[t] = idx[s + t];
    __syncthreads();
    for (uint32_t ib = 0; ib < b; ib += kBI) {
        load_tile<D>(I, ids, ib, b, pts, ld);
        WarpSet sets[kPtsPerWarp];
#pragma unroll
        for (int u = 0; u < kPtsPerWarp; ++u) {
            const uint32_t p = ib + warp * kPtsPerWarp + u;
            if (p < b) set_load(sets[u], set_dist, set_id, set_size, set_maxslot, set_bound, ids[p], K, lane);
        }
        for (uint32_t jb = 0; jb < b; jb += kBJ) {
            __syncthreads();  // previous block's readers of J / Dm are done; I is written
            load_tile<D>(J, ids, jb, b, pts, ld);
            __syncthreads();
            distance_block<D>(I, J, Dm);
            __syncthreads();
#pragma unroll
            for (int u = 0; u < kPtsPerWarp; ++u) {
                const int row = warp * kPtsPerWarp + u;
                const uint32_t p = ib + row;
                if (p < b) {
#pragma unroll
                    for (int h = 0; h < kBJ / kWarp; ++h) {
                        const int jj = h * kWarp + lane;
                        const uint32_t j = jb + jj;
                        const bool valid = j < b && j != p;
                        const float d = Dm[row * kDmStride + jj];
                        const uint32_t cand = valid ? ids[j] : 0u;
                        set_offer_batch(sets[u], cand, d, valid, K, lane);
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kPtsPerWarp; ++u) {
            const uint32_t p = ib + warp * kPtsPerWarp + u;
            if (p < b) set_store(sets[u], set_dist, set_id, set_size, set_maxslot, set_bound, ids[p], K, lane);
        }
        __syncthreads();  // everyone is done with I before it is reloaded
    }
    }
}

// ------------------------------------------------- sample k-NN (estimator)
//
// The k nearest points of a sample of query points, by the same FP32
// distances and set update as the bucket kernel, for the build's recall
// estimate: CTA (query block of 64, column range) offers its range's points
// to the 64 queries' sets in point order; k_sample_merge keeps each query's k
// best (distance, id) over the ranges.

// rows [first, first+64) of [first, last) -> tile[dim][r] (zeros past last)
template <int D>
__device__ __forceinline__ void load_range_tile(float* __restrict__ tile, uint32_t first, uint32_t last,
                                                const float* __restrict__ pts, int ld) {
    constexpr int Q = D / 4;
    for (int f = threadIdx.x; f < kBI * Q; f += kLeafThreads) {
        const int r = f % kBI, q = f / kBI;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (first + r < last) v = __ldg(reinterpret_cast<const float4*>(pts + static_cast<size_t>(first + r) * ld) + q);
        tile[(4 * q + 0) * kBI + r] = v.x;
        tile[(4 * q + 1) * kBI + r] = v.y;
        tile[(4 * q + 2) * kBI + r] = v.z;
        tile[(4 * q + 3) * kBI + r] = v.w;
    }
}

template <int D>
__global__ void __launch_bounds__(kLeafThreads, 2)
    k_sample_knn(const uint32_t* __restrict__ queries, uint32_t nq, const float* __restrict__ pts, int ld, uint32_t n,
                 uint32_t splits, int K, float* __restrict__ part_dist, uint32_t* __restrict__ part_id,
                 uint32_t* __restrict__ part_size) {
    extern __shared__ float4 smem4[];
    float* I = reinterpret_cast<float*>(smem4);
    float* J = I + D * kBI;
    float* Dm = J + D * kBJ;
    uint32_t* qid = reinterpret_cast<uint32_t*>(Dm + kBI * kDmStride);
    const uint32_t qb = blockIdx.x / splits, sp = blockIdx.x % splits;
    const uint32_t chunk = (n + splits - 1) / splits;
    const uint32_t c0 = min(n, sp * chunk), c1 = min(n, c0 + chunk);
    const uint32_t q0 = qb * kBI, rows = min(static_cast<uint32_t>(kBI), nq - q0);
    for (uint32_t t = threadIdx.x; t < static_cast<uint32_t>(kBI); t += kLeafThreads) qid[t] = t < rows ? queries[q0 + t] : 0u;
    __syncthreads();
    load_tile<D>(I, qid, 0, rows, pts, ld);
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    WarpSet sets[kPtsPerWarp];
#pragma unroll
    for (int u = 0; u < kPtsPerWarp; ++u) {
#pragma unroll
        for (int r = 0; r < kSlotsPerLane; ++r) {
            sets[u].dist[r] = 0.0f;
            sets[u].id[r] = 0u;
        }
        sets[u].size = 0;
        sets[u].maxslot = 0;
        sets[u].bound = FLT_MAX;
    }
    for (uint32_t jb = c0; jb < c1; jb += kBJ) {
        __syncthreads();
        load_range_tile<D>(J, jb, c1, pts, ld);
        __syncthreads();
        distance_block<D>(I, J, Dm);
        __syncthreads();
#pragma unroll
        for (int u = 0; u < kPtsPerWarp; ++u) {
            const int row = warp * kPtsPerWarp + u;
            if (static_cast<uint32_t>(row) < rows) {
#pragma unroll
                for (int h = 0; h < kBJ / kWarp; ++h) {
                    const uint32_t j = jb + h * kWarp + lane;
                    const bool valid = j < c1 && j != qid[row];
                    set_offer_batch(sets[u], valid ? j : 0u, Dm[row * kDmStride + h * kWarp + lane], valid, K, lane);
                }
            }
        }
    }
#pragma unroll
    for (int u = 0; u < kPtsPerWarp; ++u) {
        const uint32_t row = warp * kPtsPerWarp + u;
        if (row < rows) {
            const size_t at = static_cast<size_t>(q0 + row) * splits + sp;
#pragma unroll
            for (int r = 0; r < kSlotsPerLane; ++r) {
                const int slot = lane + r * kWarp;
                if (slot < K) {
                    part_dist[at * K + slot] = sets[u].dist[r];
                    part_id[at * K + slot] = sets[u].id[r];
                }
            }
            if (lane == 0) part_size[at] = sets[u].size;
        }
    }
}

// Per query (one warp): the k smallest (distance, id) over its ranges' sets,
// ids ascending by (distance, id) into truth[q * K ...] (kNone past the end).
__global__ void k_sample_merge(uint32_t nq, uint32_t splits, int K, const float* __restrict__ part_dist,
                               const uint32_t* __restrict__ part_id, const uint32_t* __restrict__ part_size,
                               unsigned long long* __restrict__ keys, uint32_t cap, uint32_t* __restrict__ truth) {
    const int lane = threadIdx.x % kWarp;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
    if (w >= nq) return;
    unsigned long long* buf = keys + static_cast<size_t>(w) * cap;
    const uint32_t total = splits * static_cast<uint32_t>(K);
    for (uint32_t t = lane; t < cap; t += kWarp) {
        unsigned long long key = ~0ull;
        if (t < total) {
            const uint32_t sp = t / K, slot = t % K;
            const size_t at = static_cast<size_t>(w) * splits + sp;
            if (slot < part_size[at])
                key = (static_cast<unsigned long long>(__float_as_uint(part_dist[at * K + slot])) << 32) |
                      part_id[at * K + slot];
        }
        buf[t] = key;
    }
    __syncwarp();
    warp_bitonic_sort(buf, cap, lane);
    for (int t = lane; t < K; t += kWarp)
        truth[static_cast<size_t>(w) * K + t] = buf[t] == ~0ull ? kNone : static_cast<uint32_t>(buf[t] & 0xFFFFFFFFu);
}

// Matches between each sampled point's set and its true k nearest, summed.
__global__ void k_sample_recall(const uint32_t* __restrict__ queries, uint32_t nq, int K,
                                const uint32_t* __restrict__ truth, const uint32_t* __restrict__ set_id,
                                const uint32_t* __restrict__ set_size, unsigned long long* __restrict__ hits) {
    const int lane = threadIdx.x % kWarp;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
    if (w >= nq) return;
    const uint32_t p = queries[w];
    const uint32_t size = set_size[p];
    uint32_t mine = 0;
    for (int a = lane; a < K; a += kWarp) {
        const uint32_t t = truth[static_cast<size_t>(w) * K + a];
        if (t == kNone) continue;
        for (uint32_t b = 0; b < size; ++b)
            if (set_id[static_cast<size_t>(p) * K + b] == t) {
                ++mine;
                break;
            }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(kFull, mine, o);
    if (lane == 0 && mine) atomicAdd(hits, static_cast<unsigned long long>(mine));
}

}  // namespace

void sample_knn(Context& c, const uint32_t* d_queries, uint32_t nq, uint32_t* d_truth) {
    if (nq == 0) return;
    const int K = static_cast<int>(c.k);
    const uint32_t qblocks = (nq + kBI - 1) / kBI;
    const uint32_t splits = std::max<uint32_t>(1, std::min<uint32_t>((2u * c.sms + qblocks - 1) / qblocks,
                                                                      (c.n + kBJ - 1) / kBJ));
    auto* pd = static_cast<float*>(scratch(c, "sknn_dist", static_cast<size_t>(nq) * splits * K * sizeof(float)));
    auto* pi = static_cast<uint32_t*>(scratch(c, "sknn_id", static_cast<size_t>(nq) * splits * K * sizeof(uint32_t)));
    auto* ps = static_cast<uint32_t*>(scratch(c, "sknn_size", static_cast<size_t>(nq) * splits * sizeof(uint32_t)));
    uint32_t cap = 2;
    while (cap < splits * static_cast<uint32_t>(K)) cap <<= 1;
    auto* keys = static_cast<unsigned long long*>(
        scratch(c, "sknn_keys", static_cast<size_t>(nq) * cap * sizeof(unsigned long long)));
    KNNG_DISPATCH_D(c.d, {
        const size_t smem = static_cast<size_t>(D) * (kBI + kBJ) * sizeof(float) +
                            static_cast<size_t>(kBI) * kDmStride * sizeof(float) + kBI * sizeof(uint32_t);
        auto kern = k_sample_knn<D>;
        allow_max_smem(c, kern);
        kern<<<qblocks * splits, kLeafThreads, smem, c.stream>>>(d_queries, nq, c.points, c.ld, c.n, splits, K, pd,
                                                                  pi, ps);
    });
    k_sample_merge<<<(nq + 7) / 8, 256, 0, c.stream>>>(nq, splits, K, pd, pi, ps, keys, cap, d_truth);
    c.launches += 2;
    KNNG_CUDA(cudaGetLastError());
}

double sample_recall(Context& c, const uint32_t* d_queries, uint32_t nq, const uint32_t* d_truth) {
    if (nq == 0) return 0.0;
    auto* hits = static_cast<unsigned long long*>(scratch(c, "sknn_hits", sizeof(unsigned long long)));
    KNNG_CUDA(cudaMemsetAsync(hits, 0, sizeof(unsigned long long), c.stream));
    k_sample_recall<<<(nq + 7) / 8, 256, 0, c.stream>>>(d_queries, nq, static_cast<int>(c.k), d_truth, c.set_id,
                                                        c.set_size, hits);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    download(c, &h, hits, 1);
    return static_cast<double>(h) / (static_cast<double>(nq) * c.k);
}

void launch_leaves(Context& c, uint32_t count, const uint32_t* d_starts, const uint32_t* d_ends,
                   uint32_t max_bucket, uint64_t* evals) {
    if (count == 0) return;
    KNNG_DISPATCH_D(c.d, {
        const size_t smem = static_cast<size_t>(D) * (kBI + kBJ) * sizeof(float) +
                            static_cast<size_t>(kBI) * kDmStride * sizeof(float) +
                            static_cast<size_t>(std::max<uint32_t>(max_bucket, 1)) * sizeof(uint32_t);
        if (smem > 227 * 1024) fail(KNNG_ERR_INVALID_ARGUMENT, "bucket too large for the bucket kernel");
        auto kern = k_leaf<D>;
        allow_max_smem(c, kern);
        kern<<<count, kLeafThreads, smem, c.stream>>>(d_starts, d_ends, c.indices, c.points, c.ld, c.set_dist,
                                                      c.set_id, c.set_size, c.set_maxslot, c.set_bound,
                                                      static_cast<int>(c.k), nullptr, nullptr);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    (void)evals;
}

void prepare_leaves_list(Context& c) {
    KNNG_DISPATCH_D(c.d, { allow_max_smem(c, k_leaf<D>); });
}

void launch_leaves_list(Context& c, const uint32_t* d_starts, const uint32_t* d_ends, const uint32_t* d_count,
                        uint32_t* d_work, uint32_t max_bucket) {
    KNNG_DISPATCH_D(c.d, {
        const size_t smem = static_cast<size_t>(D) * (kBI + kBJ) * sizeof(float) +
                            static_cast<size_t>(kBI) * kDmStride * sizeof(float) +
                            static_cast<size_t>(std::max<uint32_t>(max_bucket, 1)) * sizeof(uint32_t);
        if (smem > 227 * 1024) fail(KNNG_ERR_INVALID_ARGUMENT, "bucket too large for the bucket kernel");
        auto kern = k_leaf<D>;
        allow_max_smem(c, kern);
        const int sms = c.sms;
        // Persistent: two CTAs per SM take the buckets from the work counter.
        kern<<<2 * sms, kLeafThreads, smem, c.stream>>>(d_starts, d_ends, c.indices, c.points, c.ld, c.set_dist,
                                                        c.set_id, c.set_size, c.set_maxslot, c.set_bound,
                                                        static_cast<int>(c.k), d_count, d_work);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

}  // namespace knng
