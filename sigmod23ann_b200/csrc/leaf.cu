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
// k_leaf_tc makes the same offers but computes distances only for the pairs
// a tensor-core filter cannot rule out (see below); it is the slower of the
// two at 10M points, where the sequential set updates dominate.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "common.cuh"
#include "context.hpp"
#include "dispatch.hpp"
#include "tc.cuh"

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

// ------------------------------------------- bucket pass, tensor-core filter
//
// The same offers in the same order as k_leaf, with the distances of pairs
// that cannot be accepted left out.  Per 64 x 64 block (row block I, column
// block J) the rows, centred on the bucket's first point and rounded to FP16,
// are multiplied on the tensor cores (tcgen05.mma kind::f16, FP32
// accumulation; the A tile has 128 rows, the row block's 64 and zeros):
// approx = |x'|^2 + |y'|^2 - 2 x'.y'.  A pair is left out when
// approx - margin >= bound(p) at the start of the column block, with the
// margin of the neighbour-of-neighbour join's filter
//   2^-8 (|x'|^2 + |y'|^2) + 2^-16 |approx| + 2^-19 (|x'| + |y'|)
// (+inf for a row with a value outside FP16's range): its FP32 distance is
// then >= the bound at the time of its offer (bounds only fall), so the
// reference rejects it too.  The other pairs of each row are compacted in
// column order, their exact distances computed in the reference's FP32 order
// from the dim-major FP32 tiles, and offered through the same warp-resident
// set update.  While a set is not full its bound is FLT_MAX and nothing is
// left out.

constexpr int kTcRows = 128;  // MMA M: the A tile's rows

template <int D>
struct LeafTc {
    static constexpr int KP = (D + 15) / 16 * 16;  // K padded to the MMA step of 16
    static constexpr int CH = KP / 8;              // 16-byte chunks per FP16 row
    static constexpr uint32_t I = 0;                                     // FP32 [D][kBI]
    static constexpr uint32_t J = I + D * kBI * 4;                       // FP32 [D][kBJ]
    static constexpr uint32_t A = (J + D * kBJ * 4 + 127) / 128 * 128;  // FP16 chunk-major, kTcRows rows
    static constexpr uint32_t B = A + kTcRows * KP * 2;                  // FP16 chunk-major, kBJ rows
    static constexpr uint32_t norm_a = B + kBJ * KP * 2;
    static constexpr uint32_t rt_a = norm_a + kBI * 4;
    static constexpr uint32_t norm_b = rt_a + kBI * 4;
    static constexpr uint32_t rt_b = norm_b + kBJ * 4;
    static constexpr uint32_t bnd = rt_b + kBJ * 4;         // bound of each row at the column block's start
    static constexpr uint32_t pass = bnd + kBI * 4;         // u16 pass masks [kBI rows][4 groups of 16 columns]
    static constexpr uint32_t cols = pass + kBI * 4 * 2;    // per warp: compacted columns of one row (u8 [kBJ])
    static constexpr uint32_t centre = cols + kLeafWarps * kBJ;
    static constexpr uint32_t ids = centre + (D + 3) / 4 * 16;
    static constexpr size_t bytes(uint32_t max_bucket) {
        return ids + static_cast<size_t>(max_bucket > 1 ? max_bucket : 1) * 4;
    }
};

// Rows r < count of a dim-major FP32 tile (`src`, kBI == kBJ columns) minus
// `centre`, rounded to FP16, into a chunk-major tile of R rows (chunk c of row
// r at c*R*16 + r*16); rows past count are zeros.  Also each row's squared
// norm (FP32 of the centred values) and absolute error term 2^-19 |x'| (+inf
// when a value does not fit FP16).  Threads 0..127 (warps 0-3, all lanes):
// two per row.
template <int D>
__device__ __forceinline__ void convert_dm(const float* __restrict__ src, uint32_t count, uint32_t R,
                                           unsigned char* __restrict__ tile, const float* __restrict__ centre,
                                           float* __restrict__ norm, float* __restrict__ rt, int t) {
    constexpr int CH = LeafTc<D>::CH;
    constexpr int HALF = (CH + 1) / 2;
    const uint32_t r = static_cast<uint32_t>(t) >> 1;
    const int h = t & 1;
    const bool live = r < count;
    float s = 0.0f, mx = 0.0f;
#pragma unroll 1
    for (int i = 0; i < HALF; ++i) {
        const int c = h * HALF + i;
        if (c >= CH) break;
        float v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int k = 8 * c + e;
            v[e] = live && k < D ? __fsub_rn(src[k * kBJ + r], centre[k]) : 0.0f;
            s = fmaf(v[e], v[e], s);
            mx = fmaxf(mx, fabsf(v[e]));
        }
        uint4 packed;
        uint32_t* pk = reinterpret_cast<uint32_t*>(&packed);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const __half2 hv = __floats2half2_rn(v[2 * e], v[2 * e + 1]);
            pk[e] = *reinterpret_cast<const uint32_t*>(&hv);
        }
        *reinterpret_cast<uint4*>(tile + static_cast<size_t>(c) * R * 16 + static_cast<size_t>(r) * 16) = packed;
    }
    const float so = __shfl_xor_sync(kFull, s, 1);
    const float mo = __shfl_xor_sync(kFull, mx, 1);
    if (h == 0) {
        const float nrm = s + so;
        norm[r] = nrm;
        rt[r] = fmaxf(mx, mo) >= 32768.0f ? __int_as_float(0x7f800000) : 1.9073486328125e-06f * sqrtf(nrm);
    }
}

// Canonical FP32 distance (the reference's order) between row `i` of the
// dim-major I tile and column `j` of the dim-major J tile; the same
// arithmetic as distance_block.
template <int D>
__device__ __forceinline__ float distance_dm(const float* __restrict__ I, uint32_t i, const float* __restrict__ J,
                                             uint32_t j) {
    constexpr int M = D / 8 * 8;
    float tot = 0.0f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        float ch = 0.0f;
#pragma unroll
        for (int dim = c; dim < M; dim += 8) {
            const float diff = __fsub_rn(I[dim * kBI + i], J[dim * kBJ + j]);
            ch = __fmaf_rn(diff, diff, ch);
        }
        tot = __fadd_rn(tot, ch);
    }
#pragma unroll
    for (int dim = M; dim < D; ++dim) {
        const float diff = __fsub_rn(I[dim * kBI + i], J[dim * kBJ + j]);
        tot = __fadd_rn(tot, __fmul_rn(diff, diff));
    }
    return tot;
}

template <int D>
__global__ void __launch_bounds__(kLeafThreads, 2)
    k_leaf_tc(const uint32_t* __restrict__ starts, const uint32_t* __restrict__ ends,
              const uint32_t* __restrict__ idx, const float* __restrict__ pts, int ld, float* __restrict__ set_dist,
              uint32_t* __restrict__ set_id, uint32_t* __restrict__ set_size, uint32_t* __restrict__ set_maxslot,
              float* __restrict__ set_bound, int K, const uint32_t* __restrict__ dcount, uint32_t* __restrict__ work,
              uint32_t* __restrict__ error_flag) {
    using L = LeafTc<D>;
    extern __shared__ __align__(1024) unsigned char smem[];
    float* I = reinterpret_cast<float*>(smem + L::I);
    float* J = reinterpret_cast<float*>(smem + L::J);
    unsigned char* A = smem + L::A;
    unsigned char* Bt = smem + L::B;
    float* norm_a = reinterpret_cast<float*>(smem + L::norm_a);
    float* rt_a = reinterpret_cast<float*>(smem + L::rt_a);
    float* norm_b = reinterpret_cast<float*>(smem + L::norm_b);
    float* rt_b = reinterpret_cast<float*>(smem + L::rt_b);
    float* bnd = reinterpret_cast<float*>(smem + L::bnd);
    uint16_t* pass = reinterpret_cast<uint16_t*>(smem + L::pass);
    uint8_t* cols = smem + L::cols;
    float* centre = reinterpret_cast<float*>(smem + L::centre);
    uint32_t* ids = reinterpret_cast<uint32_t*>(smem + L::ids);
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ uint32_t next_s;
    const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
    const unsigned lt = (1u << lane) - 1u;
    uint8_t* my_cols = cols + warp * kBJ;
    if (warp == 0) tc::tmem_alloc(&tmem_slot, kBJ);
    if (tid == 0) {
        tc::mbar_init(&mbar, 1);
        tc::fence_barrier_init();
    }
    // A tile rows kBI..kTcRows-1 stay zero.
    for (int f = tid; f < L::CH * (kTcRows - kBI); f += kLeafThreads) {
        const int c = f / (kTcRows - kBI), r = kBI + f % (kTcRows - kBI);
        *reinterpret_cast<uint4*>(A + static_cast<size_t>(c) * kTcRows * 16 + static_cast<size_t>(r) * 16) =
            make_uint4(0u, 0u, 0u, 0u);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = tc::idesc_f16(kTcRows, kBJ);
    uint32_t phase = 0;
    bool healthy = true;
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
        for (uint32_t t = tid; t < b; t += kLeafThreads) ids[t] = idx[s0 + t];
        __syncthreads();
        for (int k = tid; k < D; k += kLeafThreads) centre[k] = pts[static_cast<size_t>(ids[0]) * ld + k];
        for (uint32_t ib = 0; ib < b && healthy; ib += kBI) {
            __syncthreads();  // the centre is written; the last row block's readers of I are done
            load_tile<D>(I, ids, ib, b, pts, ld);
            WarpSet sets[kPtsPerWarp];
#pragma unroll
            for (int u = 0; u < kPtsPerWarp; ++u) {
                const uint32_t row = warp * kPtsPerWarp + u;
                const uint32_t p = ib + row;
                if (p < b) set_load(sets[u], set_dist, set_id, set_size, set_maxslot, set_bound, ids[p], K, lane);
                if (lane == 0) bnd[row] = p < b ? sets[u].bound : -FLT_MAX;
            }
            __syncthreads();
            if (tid < 2 * kBI) convert_dm<D>(I, min(static_cast<uint32_t>(kBI), b - ib), kTcRows, A, centre, norm_a,
                                             rt_a, tid);
            for (uint32_t jb = 0; jb < b; jb += kBJ) {
                __syncthreads();  // the last column block's readers of J, B and the masks are done
                load_tile<D>(J, ids, jb, b, pts, ld);
                __syncthreads();
                if (tid < 2 * kBJ)
                    convert_dm<D>(J, min(static_cast<uint32_t>(kBJ), b - jb), kBJ, Bt, centre, norm_b, rt_b, tid);
                tc::fence_proxy_async();
                tc::fence_before_sync();
                __syncthreads();
                if (tid == 0) {
                    tc::fence_after_sync();
                    tc::issue_tile_16bit(tmem, tc::smem_u32(A), tc::smem_u32(Bt), kTcRows, kBJ, L::KP, idesc);
                    tc::mma_commit(&mbar);
                }
                // Thread 0 polls; the others wait in the barrier.
                const bool done = tid == 0 ? tc::mbar_wait_limited(&mbar, phase) : true;
                phase ^= 1u;
                if (__syncthreads_or(!done)) {
                    if (tid == 0) {
                        atomicExch(error_flag, 1u);
                        tc::mbar_wait(&mbar, phase ^ 1u);
                    }
                    healthy = false;
                    break;
                }
                tc::fence_after_sync();
                // Filter: warps whose TMEM lane quarter holds rows 0..63 read
                // 16 accumulator columns each.
                if ((warp & 3) < kBI / kWarp) {
                    const int row = (warp & 3) * kWarp + lane;
                    const int g0 = (warp >> 2) * 16;
                    const float na = norm_a[row], ra = rt_a[row], bp = bnd[row];
                    uint32_t m = 0;
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh) {  // two loads of 8 columns: fewer live registers
                        float g[8];
                        tc::tmem_ld8(tmem + (static_cast<uint32_t>((warp & 3) * kWarp) << 16) + g0 + 8 * hh, g);
                        tc::tmem_wait_ld();
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            const int j = g0 + 8 * hh + u;
                            const float nb = norm_b[j];
                            const float approx = na + nb - 2.0f * g[u];
                            const float margin =
                                0.00390625f * (na + nb) + 1.52587890625e-5f * fabsf(approx) + ra + rt_b[j];
                            // NaN-safe: a pair is left out only when the bound provably holds.
                            if (!(approx - margin >= bp)) m |= 1u << (8 * hh + u);
                        }
                    }
                    pass[row * 4 + (warp >> 2)] = static_cast<uint16_t>(m);
                }
                tc::fence_before_sync();
                __syncthreads();
                // Offers: each warp its four rows, the passing columns in order.
#pragma unroll
                for (int u = 0; u < kPtsPerWarp; ++u) {
                    const uint32_t row = warp * kPtsPerWarp + u;
                    const uint32_t p = ib + row;
                    if (p >= b) continue;  // warp-uniform
                    const uint32_t ncols = min(static_cast<uint32_t>(kBJ), b - jb);
                    unsigned long long m = static_cast<unsigned long long>(pass[row * 4 + 0]) |
                                           static_cast<unsigned long long>(pass[row * 4 + 1]) << 16 |
                                           static_cast<unsigned long long>(pass[row * 4 + 2]) << 32 |
                                           static_cast<unsigned long long>(pass[row * 4 + 3]) << 48;
                    if (ncols < 64) m &= (1ull << ncols) - 1ull;
                    if (p >= jb && p < jb + kBJ) m &= ~(1ull << (p - jb));
                    uint32_t n = 0;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const bool bit = (m >> (h * kWarp + lane)) & 1ull;
                        const unsigned bal = __ballot_sync(kFull, bit);
                        if (bit) my_cols[n + __popc(bal & lt)] = static_cast<uint8_t>(h * kWarp + lane);
                        n += __popc(bal);
                    }
                    __syncwarp();
                    for (uint32_t t0 = 0; t0 < n; t0 += kWarp) {
                        const bool valid = t0 + lane < n;
                        const uint32_t j = valid ? my_cols[t0 + lane] : 0u;
                        const float d = valid ? distance_dm<D>(I, row, J, j) : 0.0f;
                        const uint32_t cand = valid ? ids[jb + j] : 0u;
                        set_offer_batch(sets[u], cand, d, valid, K, lane);
                    }
                    __syncwarp();
                    if (lane == 0) bnd[row] = sets[u].bound;
                }
            }
#pragma unroll
            for (int u = 0; u < kPtsPerWarp; ++u) {
                const uint32_t p = ib + warp * kPtsPerWarp + u;
                if (p < b) set_store(sets[u], set_dist, set_id, set_size, set_maxslot, set_bound, ids[p], K, lane);
            }
        }
        __syncthreads();  // every warp is done with ids before the next bucket
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kBJ);
    }
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
    (void)evals;
    if (c.leaf_tc) {
        auto* err = static_cast<uint32_t*>(scratch(c, "leaf_error", sizeof(uint32_t)));
        KNNG_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), c.stream));
        KNNG_DISPATCH_D(c.d, {
            const size_t smem = LeafTc<D>::bytes(max_bucket);
            if (smem > 227 * 1024) fail(KNNG_ERR_INVALID_ARGUMENT, "bucket too large for the bucket kernel");
            auto kern = k_leaf_tc<D>;
            allow_max_smem(c, kern);
            kern<<<count, kLeafThreads, smem, c.stream>>>(d_starts, d_ends, c.indices, c.points, c.ld, c.set_dist,
                                                          c.set_id, c.set_size, c.set_maxslot, c.set_bound,
                                                          static_cast<int>(c.k), nullptr, nullptr, err);
        });
        ++c.launches;
        KNNG_CUDA(cudaGetLastError());
        uint32_t h = 0;
        download(c, &h, err, 1);
        if (h) fail(KNNG_ERR_CUDA, "bucket pass: the MMA completion wait gave up");
        return;
    }
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
}

void prepare_leaves_list(Context& c) {
    KNNG_DISPATCH_D(c.d, {
        allow_max_smem(c, k_leaf<D>);
        allow_max_smem(c, k_leaf_tc<D>);
    });
}

void launch_leaves_list(Context& c, const uint32_t* d_starts, const uint32_t* d_ends, const uint32_t* d_count,
                        uint32_t* d_work, uint32_t max_bucket, uint32_t* d_error) {
    if (c.leaf_tc) {
        KNNG_DISPATCH_D(c.d, {
            const size_t smem = LeafTc<D>::bytes(max_bucket);
            if (smem > 227 * 1024) fail(KNNG_ERR_INVALID_ARGUMENT, "bucket too large for the bucket kernel");
            auto kern = k_leaf_tc<D>;
            allow_max_smem(c, kern);
            // Persistent: leaf_ctas CTAs per SM take the buckets from the work counter.
            kern<<<c.leaf_ctas * c.sms, kLeafThreads, smem, c.stream>>>(
                d_starts, d_ends, c.indices, c.points, c.ld, c.set_dist, c.set_id, c.set_size, c.set_maxslot,
                c.set_bound, static_cast<int>(c.k), d_count, d_work, d_error);
        });
        ++c.launches;
        KNNG_CUDA(cudaGetLastError());
        return;
    }
    KNNG_DISPATCH_D(c.d, {
        const size_t smem = static_cast<size_t>(D) * (kBI + kBJ) * sizeof(float) +
                            static_cast<size_t>(kBI) * kDmStride * sizeof(float) +
                            static_cast<size_t>(std::max<uint32_t>(max_bucket, 1)) * sizeof(uint32_t);
        if (smem > 227 * 1024) fail(KNNG_ERR_INVALID_ARGUMENT, "bucket too large for the bucket kernel");
        auto kern = k_leaf<D>;
        allow_max_smem(c, kern);
        const int sms = c.sms;
        // Persistent: leaf_ctas CTAs per SM take the buckets from the work counter.
        kern<<<c.leaf_ctas * sms, kLeafThreads, smem, c.stream>>>(d_starts, d_ends, c.indices, c.points, c.ld, c.set_dist,
                                                        c.set_id, c.set_size, c.set_maxslot, c.set_bound,
                                                        static_cast<int>(c.k), d_count, d_work);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

}  // namespace knng
