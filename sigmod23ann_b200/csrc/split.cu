// Tree construction kernels: the recursive 2-means split of
// SolutionKmeans::splitKmeansBinaryProcess (src/SolutionKmeans.hpp:142-311),
// run level-synchronously over every node of a tree level at once.
//
//   k_draw_positions   sample / seed positions from the counter RNG
//                      (getSampleFromPercent :55-66, kmeansStartVecs :103-111)
//   k_farthest_pair    farthest pair among the seed positions (:68-101, :113-127)
//   k_plane            between / coefs / offset from two centres (:162-164)
//   k_side             side test of a node's Lloyd set (:170-175, :227-238) or
//                      of its whole range (:195-197, :273-278), eight lanes
//                      per point in the reference's FMA-chain order
//   k_lloyd_seq        per-side double sums in the Lloyd set's order and the
//                      new centres (:170-186, :227-259), one CTA per node fed
//                      by bulk copies
//   k_scan_items       exclusive scan of per-tile side-true counts
//   k_scatter          stable partition, side-true first (std::stable_partition
//                      at :195, the group memcpy at :301-304)
//
// Layout in HBM: points n x ld float32 rows (ld = d rounded up to 4, 16-byte
// aligned); indices u32[n]; one byte of side flag per position.  The side
// test reads each row once per tree level (ld*4 + 4 + 1 bytes per position);
// the scatter moves 4-byte indices, never rows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <limits>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"
#include "context.hpp"
#include "dispatch.hpp"
#include "tc.cuh"

namespace knng {
namespace {

constexpr int kSideThreads = 256;
constexpr int kSidePer = 8;  // positions per thread in the side / scatter kernels
constexpr int kChunk = kSideThreads * kSidePer;
constexpr int kPairThreads = 256;
constexpr uint32_t kListItem = 0x80000000u;  // Item::node flag: entries come from a position list

// A chunk of one node's entries: positions begin .. begin+count (range item)
// or list[begin .. begin+count) (list item, kListItem set in `node`).  The
// side kernel writes entry r's flag at fbase + r.
struct Item {
    uint32_t node;
    uint32_t count;
    uint64_t begin;
    uint64_t fbase;
};

__global__ void k_iota(uint32_t* __restrict__ idx, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) idx[i] = i;
}

// Node i draws draws[i] positions; the first seed_len[i] go to its seed list
// and the first lloyd_len[i] to its Lloyd list (both CSR).
// Node [start, end) of a set starting at `base` draws with keys relative to
// the set, so a set's tree is the same alone and in a batch.
// With `dcount` the nodes are [0, *dcount) (a grid-stride loop) and seed / rep
// come from rep_params[0] / [1]; else one node per CTA.
__global__ void k_draw_positions(const uint32_t* __restrict__ starts, const uint32_t* __restrict__ ends,
                                 const uint32_t* __restrict__ bases, const uint32_t* __restrict__ attempts,
                                 const uint64_t* __restrict__ draw_off,
                                 const uint64_t* __restrict__ seed_off, const uint64_t* __restrict__ lloyd_off,
                                 uint64_t seed, uint32_t rep, uint32_t* __restrict__ seeds_out,
                                 uint32_t* __restrict__ lloyd_out, const uint32_t* __restrict__ dcount,
                                 const uint64_t* __restrict__ rep_params) {
    const uint32_t count = dcount ? *dcount : gridDim.x;
    if (rep_params) {
        seed = rep_params[0];
        rep = static_cast<uint32_t>(rep_params[1]);
    }
    for (uint32_t node = blockIdx.x; node < count; node += gridDim.x) {
        const uint64_t cnt = draw_off[node + 1] - draw_off[node];
        const uint64_t sb = seed_off[node], sl = seed_off[node + 1] - sb;
        const uint64_t lb = lloyd_off[node], ll = lloyd_off[node + 1] - lb;
        const uint32_t s = starts[node], t = ends[node], a = attempts[node], b = bases[node];
        for (uint64_t i = threadIdx.x; i < cnt; i += blockDim.x) {
            const uint32_t pos = b + counter_position(seed, rep, s - b, t - b, a, static_cast<uint32_t>(i));
            if (i < sl) seeds_out[sb + i] = pos;
            if (i < ll) lloyd_out[lb + i] = pos;
        }
    }
}

// dst[u] = src[pick[u]] for rows of `ld` floats, plus the matching offsets.
__global__ void k_gather_planes(const float* __restrict__ src, const float* __restrict__ src_off,
                                const uint32_t* __restrict__ pick, uint32_t count, int ld, float* __restrict__ dst,
                                float* __restrict__ dst_off) {
    const uint32_t u = blockIdx.x;
    if (u >= count) return;
    const uint32_t p = pick[u];
    for (int j = threadIdx.x; j < ld; j += blockDim.x)
        dst[static_cast<size_t>(u) * ld + j] = src[static_cast<size_t>(p) * ld + j];
    if (threadIdx.x == 0) dst_off[u] = src_off[p];
}

// One CTA per node.  Rows of the listed positions are staged in shared memory;
// every pair (i < j) is evaluated and the maximum is taken with the
// reference's rule: strictly greater than a running maximum that starts at
// FLT_MIN, first pair in (i, j) order winning ties.
template <int D>
__global__ void k_farthest_pair(const uint64_t* __restrict__ offsets, const uint32_t* __restrict__ positions,
                                const uint32_t* __restrict__ idx, const float* __restrict__ pts, int ld,
                                uint32_t* __restrict__ out_first, uint32_t* __restrict__ out_second,
                                int32_t* __restrict__ out_ok, float* __restrict__ c1, float* __restrict__ c2,
                                const uint32_t* __restrict__ dcount) {
    extern __shared__ float4 smem4[];
    float* rows = reinterpret_cast<float*>(smem4);
    __shared__ float sv[kPairThreads / kWarp];
    __shared__ uint32_t si[kPairThreads / kWarp], sj[kPairThreads / kWarp];
    const uint32_t count = dcount ? *dcount : gridDim.x;
    for (uint32_t node = blockIdx.x; node < count; node += gridDim.x) {
    const uint64_t b = offsets[node];
    const uint32_t m = static_cast<uint32_t>(offsets[node + 1] - b);
    constexpr int Q = (D + 3) / 4;
    for (uint32_t f = threadIdx.x; f < m * Q; f += blockDim.x) {
        const uint32_t r = f / Q, q = f % Q;
        const uint32_t id = idx[positions[b + r]];
        reinterpret_cast<float4*>(rows)[r * Q + q] =
            reinterpret_cast<const float4*>(pts + static_cast<size_t>(id) * ld)[q];
    }
    __syncthreads();
    float best = FLT_MIN;
    uint32_t bi = kNone, bj = kNone;
    for (uint32_t i = 0; i + 1 < m; ++i) {
        for (uint32_t j = i + 1 + threadIdx.x; j < m; j += blockDim.x) {
            const float dd = canonical_distance<D>(rows + i * Q * 4, rows + j * Q * 4);
            // Within one thread pairs arrive in increasing (i, j) order.
            if (dd > best) {
                best = dd;
                bi = i;
                bj = j;
            }
        }
    }
    // Block arg-max: larger distance wins; equal distances -> smaller (i, j).
    auto better = [](float v, uint32_t i, uint32_t j, float bv, uint32_t bi2, uint32_t bj2) {
        if (i == kNone) return false;
        if (bi2 == kNone) return true;
        if (v != bv) return v > bv;
        return i < bi2 || (i == bi2 && j < bj2);
    };
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        float ov = __shfl_xor_sync(kFull, best, off);
        uint32_t oi = __shfl_xor_sync(kFull, bi, off), oj = __shfl_xor_sync(kFull, bj, off);
        if (better(ov, oi, oj, best, bi, bj)) {
            best = ov;
            bi = oi;
            bj = oj;
        }
    }
    if (lane == 0) {
        sv[warp] = best;
        si[warp] = bi;
        sj[warp] = bj;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < static_cast<int>(blockDim.x / kWarp); ++w) {
            if (better(sv[w], si[w], sj[w], best, bi, bj)) {
                best = sv[w];
                bi = si[w];
                bj = sj[w];
            }
        }
        si[0] = bi;
        sj[0] = bj;
        out_first[node] = bi;
        out_second[node] = bj;
        out_ok[node] = bi != kNone ? 1 : 0;
    }
    __syncthreads();
    bi = si[0];
    bj = sj[0];
    for (int q = threadIdx.x; q < Q * 4; q += blockDim.x) {
        c1[static_cast<size_t>(node) * ld + q] = bi != kNone ? rows[bi * Q * 4 + q] : 0.0f;
        c2[static_cast<size_t>(node) * ld + q] = bj != kNone ? rows[bj * Q * 4 + q] : 0.0f;
    }
    __syncthreads();  // rows and the arg-max slots are reused by the next node
    }
}

// between = 0.5f * (c1 + c2); coefs = c1 - between; offset = dot(between, coefs).
template <int D>
__global__ void k_plane(const float* __restrict__ c1, const float* __restrict__ c2, int ld, uint32_t count,
                        float* __restrict__ coefs, float* __restrict__ offsets, const uint32_t* __restrict__ dcount) {
    if (dcount) count = *dcount;
    const int lane = threadIdx.x % kWarp;
    __shared__ float between_s[8][(D + 3) / 4 * 4];
    float* between = between_s[threadIdx.x / kWarp];
    for (uint32_t node = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp; node < count;
         node += gridDim.x * (blockDim.x / kWarp)) {
    const size_t base = static_cast<size_t>(node) * ld;
    for (int j = lane; j < ld; j += kWarp) {
        if (j < D) {
            const float bt = __fmul_rn(0.5f, __fadd_rn(c1[base + j], c2[base + j]));
            between[j] = bt;
            coefs[base + j] = __fsub_rn(c1[base + j], bt);
        } else {
            coefs[base + j] = 0.0f;
        }
    }
    __syncwarp();
    if (lane == 0) offsets[node] = canonical_dot<D>(between, coefs + base);
    __syncwarp();
    }
}

// ------------------------------------------------------------ side test
//
// Eight lanes test one point: lane l of the group runs FMA chain l of the
// reference's dot (dims l, l+8, ... below the largest multiple of 8), the
// group's lanes are then summed left to right into 0.0f and the tail dims
// added as separately rounded products -- the order of `dot`
// (src/LinearAlgebra.hpp:179-200).  A warp tests four points at a time; each
// of its scalar loads reads a whole 32-byte sector of each point's row.

// The hyperplane values FMA chain l needs (chain steps, then the tail).
template <int D>
struct ChainPlane {
    static constexpr int M = D / 8 * 8;
    float c[M / 8 > 0 ? M / 8 : 1];
    float4 tail;
};

template <int D>
__device__ __forceinline__ void load_chain_plane(ChainPlane<D>& p, const float* __restrict__ coefs_row, int l) {
    constexpr int M = ChainPlane<D>::M;
#pragma unroll
    for (int i = 0; i < M / 8; ++i) p.c[i] = coefs_row[8 * i + l];
    p.tail = make_float4(0.f, 0.f, 0.f, 0.f);
    if constexpr (D > M) p.tail = *reinterpret_cast<const float4*>(coefs_row + M);
}

// dot(coefs, row) in the reference's order, by the eight lanes of the group
// whose first lane is `g0`; every lane of the group returns the result.  All
// 32 lanes must call it together.
template <int D>
__device__ __forceinline__ float group_dot(const ChainPlane<D>& p, const float* __restrict__ row, int l, int g0) {
    constexpr int M = ChainPlane<D>::M;
    static_assert(D - M == 0 || D - M == 4, "tail of 0 or 4 dims");
    float chain = 0.0f;
#pragma unroll
    for (int i = 0; i < M / 8; ++i) chain = __fmaf_rn(__ldg(row + 8 * i + l), p.c[i], chain);
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) acc = __fadd_rn(acc, __shfl_sync(kFull, chain, g0 + j));
    if constexpr (D > M) {
        const float4 x = __ldg(reinterpret_cast<const float4*>(row + M));
        acc = __fadd_rn(acc, __fmul_rn(p.tail.x, x.x));
        acc = __fadd_rn(acc, __fmul_rn(p.tail.y, x.y));
        acc = __fadd_rn(acc, __fmul_rn(p.tail.z, x.z));
        acc = __fadd_rn(acc, __fmul_rn(p.tail.w, x.w));
    }
    return acc;
}

// Side flags of one item (up to kChunk entries of one node): entry r reads
// position begin + r, or list[begin + r] for a list item; its flag goes to
// flags[fbase + r] and, when `ids_out` is given, its point id to
// ids_out[fbase + r].  item_true[item] = the item's side-true count.
template <int D>
__global__ void __launch_bounds__(kSideThreads) k_side(const Item* __restrict__ items, const uint32_t* __restrict__ list,
                                                       const uint32_t* __restrict__ idx, const float* __restrict__ pts,
                                                       int ld, const float* __restrict__ coefs,
                                                       const float* __restrict__ offsets, uint8_t* __restrict__ flags,
                                                       uint32_t* __restrict__ ids_out,
                                                       uint32_t* __restrict__ item_true,
                                                       const uint32_t* __restrict__ dcount) {
    __shared__ uint32_t warp_sum[kSideThreads / kWarp];
    const uint32_t n_items = dcount ? *dcount : gridDim.x;
    for (uint32_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const Item it = items[item];
    const bool from_list = (it.node & kListItem) != 0;
    const uint32_t node = it.node & ~kListItem;
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    const int l = lane & 7, grp = lane >> 3, g0 = lane & ~7;
    ChainPlane<D> plane;
    load_chain_plane<D>(plane, coefs + static_cast<size_t>(node) * ld, l);
    const float off = offsets[node];
    uint32_t cnt = 0;
    // Each warp takes 32 consecutive entries at a time.
    for (uint32_t r0 = warp * kWarp; r0 < it.count; r0 += kSideThreads) {
        const uint32_t r = r0 + lane;
        uint32_t id = 0;
        if (r < it.count) {
            const uint64_t e = it.begin + r;
            id = idx[from_list ? list[e] : static_cast<uint32_t>(e)];
        }
        uint32_t mask = 0;  // bit j: entry r0 + j is side-true
#pragma unroll 1
        for (int b = 0; b < 8; ++b) {
            const int j = 4 * b + grp;
            const uint32_t pid = __shfl_sync(kFull, id, j);
            const float v = group_dot<D>(plane, pts + static_cast<size_t>(pid) * ld, l, g0);
            const bool f = r0 + j < it.count && v >= off;
            const unsigned bal = __ballot_sync(kFull, f && l == 0);
#pragma unroll
            for (int q = 0; q < 4; ++q) mask |= ((bal >> (8 * q)) & 1u) << (4 * b + q);
        }
        if (r < it.count) {
            const uint8_t f = (mask >> lane) & 1u;
            flags[it.fbase + r] = f;
            if (ids_out) ids_out[it.fbase + r] = id;
        }
        cnt += __popc(mask);  // warp-uniform
    }
    if (lane == 0) warp_sum[warp] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int w = 0; w < kSideThreads / kWarp; ++w) s += warp_sum[w];
        item_true[item] = s;
    }
    __syncthreads();  // warp_sum is reused by the next item
    }
}

// ------------------------------------------------------------- Lloyd sums
//
// The new centres are the per-side means of the node's Lloyd set, summed in
// double one point at a time in the set's order (src/SolutionKmeans.hpp:
// 170-175, :227-238 -- under a serial scheduler the large-node combinable
// holds one partial, so that order is the sample's).  Rounding makes that
// sum order-dependent, so it is not split: one CTA per node walks the set in
// order.  A producer warp streams the rows into shared memory with bulk
// copies (one per row, into a ring of kSeqStages tiles on mbarriers); warp 0
// sums the side-true rows and warp 1 the side-false rows, each lane owning
// dims lane, lane+32, ... so a node's 2*D sums advance together.
constexpr int kSeqRows = 64;
constexpr int kSeqStages = 4;
constexpr int kSeqThreads = 3 * kWarp;

struct SeqNode {
    uint64_t fbase;  // first entry of the node in the flag / id arrays (16-byte aligned)
    uint32_t len;    // entries
    uint32_t pad;
};

__host__ __device__ constexpr size_t seq_smem_bytes(int D) {
    return static_cast<size_t>(kSeqStages) * kSeqRows * D * sizeof(float) + kSeqStages * kSeqRows;
}

template <int D>
__global__ void __launch_bounds__(kSeqThreads) k_lloyd_seq(const SeqNode* __restrict__ nodes,
                                                           const uint8_t* __restrict__ flags,
                                                           const uint32_t* __restrict__ ids,
                                                           const float* __restrict__ pts, int ld, float* __restrict__ c1,
                                                           float* __restrict__ c2, int32_t* __restrict__ ok,
                                                           int32_t* __restrict__ error_flag,
                                                           const uint32_t* __restrict__ dcount) {
    extern __shared__ __align__(128) unsigned char smem[];
    float* tiles = reinterpret_cast<float*>(smem);                                   // [stage][row][D]
    uint8_t* tflags = smem + static_cast<size_t>(kSeqStages) * kSeqRows * D * 4;  // [stage][row]
    __shared__ uint64_t full[kSeqStages], empty[kSeqStages];
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    // Nodes blockIdx.x, blockIdx.x + gridDim.x, ... of [0, count); their
    // tiles run through one ring, tile g of the CTA in stage g % kSeqStages.
    const uint32_t count = dcount ? *dcount : gridDim.x;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kSeqStages; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 2);
        }
        tc::fence_barrier_init();
    }
    __syncthreads();
    constexpr uint32_t kRowBytes = D * sizeof(float);
    if (warp == 2) {
        // Producer: a node's ids of the next tile are loaded while this one is issued.
        uint32_t g = 0;
        bool failed = false;
        for (uint32_t node = blockIdx.x; node < count && !failed; node += gridDim.x) {
            const SeqNode nd = nodes[node];
            const uint32_t ntiles = (nd.len + kSeqRows - 1) / kSeqRows;
            uint32_t next[kSeqRows / kWarp];
            auto load_ids = [&](uint32_t t) {
#pragma unroll
                for (int u = 0; u < kSeqRows / kWarp; ++u) {
                    const uint32_t e = t * kSeqRows + lane + u * kWarp;
                    next[u] = (t < ntiles && e < nd.len) ? ids[nd.fbase + e] : 0u;
                }
            };
            load_ids(0);
            for (uint32_t t = 0; t < ntiles; ++t, ++g) {
                uint32_t cur[kSeqRows / kWarp];
#pragma unroll
                for (int u = 0; u < kSeqRows / kWarp; ++u) cur[u] = next[u];
                load_ids(t + 1);
                const uint32_t s = g % kSeqStages;
                if (g >= kSeqStages && !tc::mbar_wait_limited(&empty[s], ((g / kSeqStages) - 1) & 1u)) {
                    if (lane == 0) atomicExch(error_flag, 1);
                    failed = true;
                    break;
                }
                const uint32_t rows = min(static_cast<uint32_t>(kSeqRows), nd.len - t * kSeqRows);
                const uint32_t fbytes = (rows + 15u) & ~15u;
                if (lane == 0) tc::mbar_arrive_expect_tx(&full[s], rows * kRowBytes + fbytes);
                __syncwarp();
#pragma unroll
                for (int u = 0; u < kSeqRows / kWarp; ++u) {
                    const uint32_t r = lane + u * kWarp;
                    if (r < rows)
                        tc::bulk_g2s(tiles + (static_cast<size_t>(s) * kSeqRows + r) * D,
                                     pts + static_cast<size_t>(cur[u]) * ld, kRowBytes, &full[s]);
                }
                if (lane == 0) tc::bulk_g2s(tflags + s * kSeqRows, flags + nd.fbase + t * kSeqRows, fbytes, &full[s]);
            }
        }
        // No copy may be in flight when the CTA exits.
        const uint32_t first = g > kSeqStages ? g - kSeqStages : 0u;
        for (uint32_t t = first; t < g; ++t)
            if (!tc::mbar_wait(&full[t % kSeqStages], (t / kSeqStages) & 1u) && lane == 0) atomicExch(error_flag, 1);
        return;
    }
    // Consumers: warp 0 sums the side-true rows, warp 1 the side-false rows.
    const uint8_t want = warp == 0 ? 1 : 0;
    constexpr int PER = (D + kWarp - 1) / kWarp;
    uint32_t g = 0;
    for (uint32_t node = blockIdx.x; node < count; node += gridDim.x) {
        const SeqNode nd = nodes[node];
        const uint32_t ntiles = (nd.len + kSeqRows - 1) / kSeqRows;
        double acc[PER];
#pragma unroll
        for (int j = 0; j < PER; ++j) acc[j] = 0.0;
        uint32_t cnt = 0;
        for (uint32_t t = 0; t < ntiles; ++t, ++g) {
            const uint32_t s = g % kSeqStages;
            if (!tc::mbar_wait_limited(&full[s], (g / kSeqStages) & 1u)) {
                if (lane == 0) atomicExch(error_flag, 1);
                return;
            }
            const uint32_t rows = min(static_cast<uint32_t>(kSeqRows), nd.len - t * kSeqRows);
            const float* tile = tiles + static_cast<size_t>(s) * kSeqRows * D;
            const uint8_t* tf = tflags + s * kSeqRows;
#pragma unroll 4
            for (uint32_t r = 0; r < rows; ++r) {
                if (tf[r] == want) {
#pragma unroll
                    for (int j = 0; j < PER; ++j)
                        if (lane + j * kWarp < D)
                            acc[j] = __dadd_rn(acc[j], static_cast<double>(tile[r * D + lane + j * kWarp]));
                    ++cnt;
                }
            }
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&empty[s]);
        }
        if (cnt == 0) {
            if (lane == 0) ok[node] = 0;
            continue;
        }
        float* c = (warp == 0 ? c1 : c2) + static_cast<size_t>(node) * ld;
        const double nn = static_cast<double>(cnt);
#pragma unroll
        for (int j = 0; j < PER; ++j)
            if (lane + j * kWarp < D) c[lane + j * kWarp] = __double2float_rn(__ddiv_rn(acc[j], nn));
    }
}

// Exclusive scan of n values into out[0..n] (out[n] = total); one CTA.
__global__ void k_scan_items(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ out,
                             const uint32_t* __restrict__ dn) {
    __shared__ uint32_t part[1024];
    if (dn) n = *dn;
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t b = threadIdx.x * per, e = min(n, b + per);
    uint32_t s = 0;
    for (uint32_t i = b; i < e; ++i) s += in[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t w = 0; w < blockDim.x; ++w) {
            const uint32_t v = part[w];
            part[w] = run;
            run += v;
        }
        out[n] = run;
    }
    __syncthreads();
    uint32_t run = part[threadIdx.x];
    for (uint32_t i = b; i < e; ++i) {
        out[i] = run;
        run += in[i];
    }
}

__global__ void k_node_true(const uint32_t* __restrict__ item_begin, const uint32_t* __restrict__ item_end,
                            const uint32_t* __restrict__ prefix, uint32_t count, uint32_t* __restrict__ out_true,
                            const uint32_t* __restrict__ dcount) {
    if (dcount) count = *dcount;
    for (uint32_t node = blockIdx.x * blockDim.x + threadIdx.x; node < count; node += gridDim.x * blockDim.x)
        out_true[node] = prefix[item_end[node]] - prefix[item_begin[node]];
}

// Stable partition scatter of one chunk: side-true positions go to
// start + (true before), side-false to start + T + (false before).
__global__ void __launch_bounds__(kSideThreads) k_scatter(const Item* __restrict__ items,
                                                          const uint32_t* __restrict__ node_start,
                                                          const uint32_t* __restrict__ node_item_begin,
                                                          const uint32_t* __restrict__ node_true,
                                                          const uint32_t* __restrict__ prefix,
                                                          const uint8_t* __restrict__ flags,
                                                          const uint32_t* __restrict__ idx,
                                                          uint32_t* __restrict__ idx_out,
                                                          const uint32_t* __restrict__ dcount) {
    __shared__ uint32_t warp_tot[kSideThreads / kWarp];
    const uint32_t n_items = dcount ? *dcount : gridDim.x;
    for (uint32_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const Item it = items[item];
    const uint32_t s = node_start[it.node];
    const uint32_t T = node_true[it.node];
    const uint32_t before_item = prefix[item] - prefix[node_item_begin[it.node]];
    // Thread t owns positions [t*kSidePer, (t+1)*kSidePer) of the chunk.
    const uint32_t first = threadIdx.x * kSidePer;
    uint8_t f[kSidePer];
    uint32_t mine = 0;
#pragma unroll
    for (int u = 0; u < kSidePer; ++u) {
        const uint32_t r = first + u;
        f[u] = r < it.count ? flags[it.begin + r] : 0;
        mine += f[u];
    }
    // Block exclusive scan of `mine`.
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    uint32_t incl = mine;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
        uint32_t v = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == kWarp - 1) warp_tot[warp] = incl;
    __syncthreads();
    uint32_t warp_base = 0;
    for (int w = 0; w < warp; ++w) warp_base += warp_tot[w];
    uint32_t t_before = before_item + warp_base + incl - mine;
#pragma unroll
    for (int u = 0; u < kSidePer; ++u) {
        const uint32_t r = first + u;
        if (r < it.count) {
            const uint64_t pos = it.begin + r;
            const uint32_t rel = static_cast<uint32_t>(pos - s);
            uint32_t dst;
            if (f[u]) {
                dst = s + t_before;
                ++t_before;
            } else {
                dst = s + T + (rel - t_before);
            }
            idx_out[dst] = idx[pos];
        }
    }
    __syncthreads();  // warp_tot is reused by the next item
    }
}

__global__ void k_copy_back(const Item* __restrict__ items, const uint32_t* __restrict__ src,
                            uint32_t* __restrict__ dst, const uint32_t* __restrict__ dcount) {
    const uint32_t n_items = dcount ? *dcount : gridDim.x;
    for (uint32_t item = blockIdx.x; item < n_items; item += gridDim.x) {
        const Item it = items[item];
        for (uint32_t r = threadIdx.x; r < it.count; r += blockDim.x) dst[it.begin + r] = src[it.begin + r];
    }
}

// ------------------------------------------------- device-side repetition
//
// The tree of one repetition built without host round trips: the node list
// of a level, its sampling plan, work items, split outcomes and the next
// level's list all stay in device memory, so one tree level is a fixed
// sequence of launches whose sizes come from device counters -- the body of
// a CUDA-graph WHILE node that runs until no node is left to split.
// Results equal the host-sequenced repetition's: the counter RNG is keyed by
// node, nodes of a level are disjoint, and a node that fails (no seed pair,
// an empty cluster or side) is retried with the next attempt index in the
// next level instead of at once, which changes nothing but the order.

constexpr uint32_t kPlanThreads = 1024;
constexpr uint32_t kMaxSplitAttempts = 64;
// Level iterations a repetition may take: far above any real tree (depth
// <= 32, each node retried at most kMaxSplitAttempts times); past it the
// loop stops and reports an error instead of running on.
constexpr uint32_t kMaxLevelIterations = 8192;

struct LevelCounts {
    uint32_t cur, next, leaves, lloyd_items, part_items, iterations, restarts, fallbacks, nodes, leaf_work;
    unsigned long long pairs;  // sum of b (b - 1) / 2 over the leaves
};

// Exclusive prefix sum of one value per thread over a CTA of kPlanThreads;
// *total receives the sum.  Every thread calls it.
__device__ __forceinline__ unsigned long long plan_scan(unsigned long long v, unsigned long long* __restrict__ wt,
                                                        unsigned long long* total) {
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    unsigned long long incl = v;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == kWarp - 1) wt[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned long long t = wt[lane];
#pragma unroll
        for (int o = 1; o < kWarp; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, t, o);
            if (lane >= o) t += y;
        }
        wt[lane] = t;
    }
    __syncthreads();
    const unsigned long long base = warp > 0 ? wt[warp - 1] : 0ull;
    *total = wt[kWarp - 1];
    __syncthreads();
    return base + incl - v;
}

// The level's sampling plan (rules of getSampleFromPercent / kmeansStartVecs,
// as the host-sequenced level applies them; `table[n]` = sample count << 8 |
// seed count): per node the CSR offsets of its draws, seeds and Lloyd list,
// its Lloyd set (list or whole range) in the flag / id arrays, and its first
// Lloyd work item.
__global__ void __launch_bounds__(kPlanThreads)
    k_level_plan(const uint32_t* __restrict__ start, const uint32_t* __restrict__ end, LevelCounts* __restrict__ cnt,
                 const uint32_t* __restrict__ table, uint32_t small_threshold, uint64_t* __restrict__ draw_off,
                 uint64_t* __restrict__ seed_off, uint64_t* __restrict__ lloyd_off, SeqNode* __restrict__ seq,
                 uint64_t* __restrict__ lbegin, uint32_t* __restrict__ lfrom, uint32_t* __restrict__ item_off) {
    __shared__ unsigned long long wt[kWarp];
    const uint32_t count = cnt->cur;
    const uint32_t per = (count + kPlanThreads - 1) / kPlanThreads;
    const uint32_t b = threadIdx.x * per, e = min(count, b + per);
    auto plan = [&](uint32_t i, uint32_t& draws, uint32_t& seeds, uint32_t& list, uint32_t& entries) {
        const uint32_t n = end[i] - start[i];
        const uint32_t packed = table[n];
        const uint32_t S = packed & 0xFFu, samp = packed >> 8;
        const bool large = n >= small_threshold;
        draws = large ? samp : S;
        seeds = min(draws, S);
        list = large ? draws : 0u;
        entries = list > 0 ? list : n;
    };
    unsigned long long sd = 0, ss = 0, sl = 0, sf = 0, si = 0;
    for (uint32_t i = b; i < e; ++i) {
        uint32_t draws, seeds, list, entries;
        plan(i, draws, seeds, list, entries);
        sd += draws;
        ss += seeds;
        sl += list;
        sf += (entries + 15u) / 16u * 16u;
        si += (entries + kChunk - 1) / kChunk;
    }
    unsigned long long td, ts, tl, tf, ti;
    unsigned long long od = plan_scan(sd, wt, &td), os = plan_scan(ss, wt, &ts), ol = plan_scan(sl, wt, &tl);
    unsigned long long of = plan_scan(sf, wt, &tf), oi = plan_scan(si, wt, &ti);
    for (uint32_t i = b; i < e; ++i) {
        uint32_t draws, seeds, list, entries;
        plan(i, draws, seeds, list, entries);
        draw_off[i] = od;
        seed_off[i] = os;
        lloyd_off[i] = ol;
        seq[i] = {of, entries, 0u};
        lbegin[i] = list > 0 ? ol : start[i];
        lfrom[i] = list > 0 ? 1u : 0u;
        item_off[i] = static_cast<uint32_t>(oi);
        od += draws;
        os += seeds;
        ol += list;
        of += (entries + 15u) / 16u * 16u;
        oi += (entries + kChunk - 1) / kChunk;
    }
    if (threadIdx.x == 0) {
        draw_off[count] = td;
        seed_off[count] = ts;
        lloyd_off[count] = tl;
        item_off[count] = static_cast<uint32_t>(ti);
        cnt->lloyd_items = static_cast<uint32_t>(ti);
        cnt->nodes += count;
    }
}

// Largest i in [0, count) with off[i] <= t (off non-decreasing, off[0] = 0).
__device__ __forceinline__ uint32_t owner_of(const uint32_t* __restrict__ off, uint32_t count, uint32_t t) {
    uint32_t lo = 0, hi = count - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Lloyd work items of the level (chunks of kChunk entries of a node's set).
__global__ void k_lloyd_items(const LevelCounts* __restrict__ cnt, const uint32_t* __restrict__ item_off,
                              const SeqNode* __restrict__ seq, const uint64_t* __restrict__ lbegin,
                              const uint32_t* __restrict__ lfrom, Item* __restrict__ items) {
    const uint32_t count = cnt->cur, total = cnt->lloyd_items;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const uint32_t i = owner_of(item_off, count, t);
        const uint64_t o = static_cast<uint64_t>(t - item_off[i]) * kChunk;
        const uint64_t left = seq[i].len - o;
        items[t] = {i | (lfrom[i] ? kListItem : 0u), static_cast<uint32_t>(left < kChunk ? left : kChunk),
                    lbegin[i] + o, seq[i].fbase + o};
    }
}

// Partition plan: the nodes that seeded and converged (ok) are cut into
// kChunk-position items; ib / ie bound each node's items.
__global__ void __launch_bounds__(kPlanThreads)
    k_part_plan(const uint32_t* __restrict__ start, const uint32_t* __restrict__ end, LevelCounts* __restrict__ cnt,
                const int32_t* __restrict__ ok, uint32_t* __restrict__ ib, uint32_t* __restrict__ ie) {
    __shared__ unsigned long long wt[kWarp];
    const uint32_t count = cnt->cur;
    const uint32_t per = (count + kPlanThreads - 1) / kPlanThreads;
    const uint32_t b = threadIdx.x * per, e = min(count, b + per);
    unsigned long long si = 0;
    for (uint32_t i = b; i < e; ++i) si += ok[i] ? (end[i] - start[i] + kChunk - 1) / kChunk : 0u;
    unsigned long long ti;
    unsigned long long oi = plan_scan(si, wt, &ti);
    for (uint32_t i = b; i < e; ++i) {
        ib[i] = static_cast<uint32_t>(oi);
        oi += ok[i] ? (end[i] - start[i] + kChunk - 1) / kChunk : 0u;
        ie[i] = static_cast<uint32_t>(oi);
    }
    if (threadIdx.x == 0) cnt->part_items = static_cast<uint32_t>(ti);
}

__global__ void k_part_items(const LevelCounts* __restrict__ cnt, const uint32_t* __restrict__ start,
                             const uint32_t* __restrict__ end, const uint32_t* __restrict__ ib,
                             Item* __restrict__ items) {
    const uint32_t count = cnt->cur, total = cnt->part_items;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const uint32_t i = owner_of(ib, count, t);
        const uint64_t o = static_cast<uint64_t>(start[i]) + static_cast<uint64_t>(t - ib[i]) * kChunk;
        const uint64_t left = end[i] - o;
        items[t] = {i, static_cast<uint32_t>(left < kChunk ? left : kChunk), o, o};
    }
}

// Outcome of every node of the level: split at start + (side-true count), or
// retried with the next attempt (no seed pair, an empty cluster or side), or
// after kMaxSplitAttempts failures split at its index midpoint; children below
// max_leaf points become leaves, the others the next level's nodes.
__global__ void k_level_next(const uint32_t* __restrict__ start, const uint32_t* __restrict__ end,
                             const uint32_t* __restrict__ base, const uint32_t* __restrict__ attempt,
                             LevelCounts* __restrict__ cnt, const int32_t* __restrict__ ok,
                             const uint32_t* __restrict__ node_true, const uint64_t* __restrict__ rep_params,
                             uint32_t* __restrict__ nstart, uint32_t* __restrict__ nend, uint32_t* __restrict__ nbase,
                             uint32_t* __restrict__ nattempt, uint32_t* __restrict__ leaf_start,
                             uint32_t* __restrict__ leaf_end) {
    const uint32_t count = cnt->cur;
    const uint32_t max_leaf = static_cast<uint32_t>(rep_params[2]);
    auto child = [&](uint32_t lo, uint32_t hi, uint32_t b) {
        if (hi - lo < max_leaf) {
            const uint32_t li = atomicAdd(&cnt->leaves, 1u);
            leaf_start[li] = lo;
            leaf_end[li] = hi;
            const unsigned long long m = hi - lo;
            atomicAdd(&cnt->pairs, m * (m - 1) / 2);
        } else {
            const uint32_t ni = atomicAdd(&cnt->next, 1u);
            nstart[ni] = lo;
            nend[ni] = hi;
            nbase[ni] = b;
            nattempt[ni] = 0;
        }
    };
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t s = start[i], e = end[i], b = base[i], a = attempt[i];
        const uint32_t n = e - s, t = node_true[i];
        uint32_t mid;
        if (!ok[i] || t == 0 || t == n) {
            atomicAdd(&cnt->restarts, 1u);
            if (a + 1 < kMaxSplitAttempts) {
                const uint32_t ni = atomicAdd(&cnt->next, 1u);
                nstart[ni] = s;
                nend[ni] = e;
                nbase[ni] = b;
                nattempt[ni] = a + 1;
                continue;
            }
            atomicAdd(&cnt->fallbacks, 1u);
            mid = s + n / 2;
        } else {
            mid = s + t;
        }
        child(s, mid, b);
        child(mid, e, b);
    }
}

// The next level becomes the current one; with `set_cond` the graph's WHILE
// condition becomes (nodes left to split).
__global__ void __launch_bounds__(kPlanThreads)
    k_level_swap(LevelCounts* __restrict__ cnt, const uint32_t* __restrict__ nstart,
                 const uint32_t* __restrict__ nend, const uint32_t* __restrict__ nbase,
                 const uint32_t* __restrict__ nattempt, uint32_t* __restrict__ start, uint32_t* __restrict__ end,
                 uint32_t* __restrict__ base, uint32_t* __restrict__ attempt, int32_t* __restrict__ error_flag,
                 cudaGraphConditionalHandle cond, int set_cond) {
    const bool runaway = cnt->iterations + 1 >= kMaxLevelIterations;
    const uint32_t n = runaway ? 0u : cnt->next;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        start[i] = nstart[i];
        end[i] = nend[i];
        base[i] = nbase[i];
        attempt[i] = nattempt[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (runaway) *error_flag = 1;
        cnt->cur = n;
        cnt->next = 0;
        cnt->iterations += 1;
        if (set_cond) cudaGraphSetConditional(cond, n > 0 ? 1u : 0u);
    }
}

// Start of a repetition: indices 0..n-1 (done by k_iota), every point set's
// root a node of the first level, or a leaf when it has fewer than max_leaf
// points; counters cleared.
__global__ void k_rep_init(const uint32_t* __restrict__ set_offsets, uint32_t nsets,
                           const uint64_t* __restrict__ rep_params, LevelCounts* __restrict__ cnt,
                           uint32_t* __restrict__ start, uint32_t* __restrict__ end, uint32_t* __restrict__ base,
                           uint32_t* __restrict__ attempt, uint32_t* __restrict__ leaf_start,
                           uint32_t* __restrict__ leaf_end, cudaGraphConditionalHandle cond, int set_cond) {
    __shared__ uint32_t n_cur, n_leaf;
    __shared__ unsigned long long pairs;
    const uint32_t max_leaf = static_cast<uint32_t>(rep_params[2]);
    if (threadIdx.x == 0) {
        n_cur = 0;
        n_leaf = 0;
        pairs = 0;
    }
    __syncthreads();
    for (uint32_t s = threadIdx.x; s < nsets; s += blockDim.x) {
        const uint32_t lo = set_offsets[s], hi = set_offsets[s + 1];
        if (hi - lo < max_leaf) {
            const uint32_t li = atomicAdd(&n_leaf, 1u);
            leaf_start[li] = lo;
            leaf_end[li] = hi;
            const unsigned long long m = hi - lo;
            atomicAdd(&pairs, m * (m > 0 ? m - 1 : 0) / 2);
        } else {
            const uint32_t ni = atomicAdd(&n_cur, 1u);
            start[ni] = lo;
            end[ni] = hi;
            base[ni] = lo;
            attempt[ni] = 0;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *cnt = LevelCounts{};
        cnt->cur = n_cur;
        cnt->leaves = n_leaf;
        cnt->pairs = pairs;
        if (set_cond) cudaGraphSetConditional(cond, n_cur > 0 ? 1u : 0u);
    }
}

}  // namespace

void set_split_wait_limit(uint32_t polls) { KNNG_CUDA(cudaMemcpyToSymbol(tc::g_wait_limit, &polls, sizeof(polls))); }

void launch_iota(Context& c) {
    if (c.n == 0) return;
    k_iota<<<std::min<uint32_t>((c.n + 255) / 256, 148 * 16), 256, 0, c.stream>>>(c.indices, c.n);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

void launch_draw_positions(Context& c, uint32_t count, const uint32_t* d_starts, const uint32_t* d_ends,
                           const uint32_t* d_bases, const uint32_t* d_attempts, const uint64_t* d_draw_off,
                           const uint64_t* d_seed_off, const uint64_t* d_lloyd_off, uint64_t seed, uint32_t rep,
                           uint32_t* d_seeds, uint32_t* d_lloyd) {
    if (count == 0) return;
    k_draw_positions<<<count, 256, 0, c.stream>>>(d_starts, d_ends, d_bases, d_attempts, d_draw_off, d_seed_off, d_lloyd_off,
                                                  seed, rep, d_seeds, d_lloyd, nullptr, nullptr);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

void launch_gather_planes(Context& c, const float* d_coefs, const float* d_offsets, const uint32_t* d_pick,
                          uint32_t count, float* d_out_coefs, float* d_out_offsets) {
    if (count == 0) return;
    k_gather_planes<<<count, 128, 0, c.stream>>>(d_coefs, d_offsets, d_pick, count, c.ld, d_out_coefs, d_out_offsets);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

void launch_farthest_pair(Context& c, uint32_t count, const uint64_t* d_offsets, const uint32_t* d_positions,
                          uint32_t max_list, uint32_t* d_first, uint32_t* d_second, int32_t* d_ok, float* d_c1,
                          float* d_c2) {
    if (count == 0) return;
    const size_t smem = static_cast<size_t>(std::max<uint32_t>(max_list, 1)) * c.ld * sizeof(float);
    if (smem > 200 * 1024) fail(KNNG_ERR_INVALID_ARGUMENT, "farthest-pair list too long");
    KNNG_DISPATCH_D(c.d, {
        auto kern = k_farthest_pair<D>;
        allow_max_smem(c, kern);
        kern<<<count, kPairThreads, smem, c.stream>>>(d_offsets, d_positions, c.indices, c.points, c.ld, d_first,
                                                      d_second, d_ok, d_c1, d_c2, nullptr);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

void launch_plane(Context& c, uint32_t count, const float* d_c1, const float* d_c2, float* d_coefs,
                  float* d_offsets) {
    if (count == 0) return;
    KNNG_DISPATCH_D(c.d, {
        k_plane<D><<<(count + 7) / 8, 256, 0, c.stream>>>(d_c1, d_c2, c.ld, count, d_coefs, d_offsets, nullptr);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

void launch_lloyd(Context& c, uint32_t count, const uint32_t* h_starts, const uint32_t* h_ends,
                  const uint64_t* h_lloyd_offsets, const uint32_t* d_lloyd_positions, float* d_c1, float* d_c2,
                  uint32_t iters, float* d_coefs, float* d_offsets, int32_t* d_ok) {
    if (count == 0) return;
    // Each node's Lloyd set is its list (large nodes) or its whole range
    // (small nodes).  Its entries get a 16-byte aligned block of the flag / id
    // arrays (the bulk copies of the sums kernel read whole 16-byte pieces),
    // and are cut into kChunk-entry items for the side kernel.
    std::vector<Item> items;
    std::vector<SeqNode> nodes(count);
    uint64_t fnext = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const uint64_t lb = h_lloyd_offsets[i], le = h_lloyd_offsets[i + 1];
        const bool from_list = le > lb;
        const uint64_t b = from_list ? lb : h_starts[i];
        const uint64_t len = from_list ? le - lb : static_cast<uint64_t>(h_ends[i] - h_starts[i]);
        nodes[i] = {fnext, static_cast<uint32_t>(len), 0u};
        for (uint64_t o = 0; o < len; o += kChunk)
            items.push_back({i | (from_list ? kListItem : 0u), static_cast<uint32_t>(std::min<uint64_t>(kChunk, len - o)),
                             b + o, fnext + o});
        fnext += (len + 15) / 16 * 16;
    }
    const uint32_t ni = static_cast<uint32_t>(items.size());
    const Item* d_items = upload(c, "lloyd_items", items.data(), ni);
    const SeqNode* d_nodes = upload(c, "lloyd_nodes", nodes.data(), count);
    uint8_t* flags = static_cast<uint8_t*>(scratch(c, "lloyd_flags", fnext + 64));
    uint32_t* ids = static_cast<uint32_t*>(scratch(c, "lloyd_ids", (fnext + 64) * sizeof(uint32_t)));
    uint32_t* item_true = static_cast<uint32_t*>(scratch(c, "lloyd_item_true", (ni + 1) * sizeof(uint32_t)));
    int32_t* err = d_ok + count;
    KNNG_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t), c.stream));
    KNNG_DISPATCH_D(c.d, {
        auto seq = k_lloyd_seq<D>;
        allow_max_smem(c, seq);
        for (uint32_t iter = 0; iter < iters; ++iter) {
            launch_plane(c, count, d_c1, d_c2, d_coefs, d_offsets);
            k_side<D><<<ni, kSideThreads, 0, c.stream>>>(d_items, d_lloyd_positions, c.indices, c.points, c.ld,
                                                         d_coefs, d_offsets, flags, ids, item_true, nullptr);
            seq<<<count, kSeqThreads, seq_smem_bytes(D), c.stream>>>(d_nodes, flags, ids, c.points, c.ld, d_c1, d_c2,
                                                                     d_ok, err, nullptr);
            c.launches += 2;
            KNNG_CUDA(cudaGetLastError());
        }
    });
    launch_plane(c, count, d_c1, d_c2, d_coefs, d_offsets);
}

void launch_partition(Context& c, uint32_t count, const uint32_t* h_starts, const uint32_t* h_ends,
                      const uint32_t* d_starts, const float* d_coefs, const float* d_offsets, uint32_t* d_true) {
    if (count == 0) return;
    std::vector<Item> items;
    std::vector<uint32_t> ib(count), ie(count);
    for (uint32_t i = 0; i < count; ++i) {
        ib[i] = static_cast<uint32_t>(items.size());
        for (uint64_t o = h_starts[i]; o < h_ends[i]; o += kChunk)
            items.push_back({i, static_cast<uint32_t>(std::min<uint64_t>(kChunk, h_ends[i] - o)), o, o});
        ie[i] = static_cast<uint32_t>(items.size());
    }
    const uint32_t ni = static_cast<uint32_t>(items.size());
    const Item* d_items = upload(c, "part_items", items.data(), ni);
    const uint32_t* d_ib = upload(c, "part_ib", ib.data(), count);
    const uint32_t* d_ie = upload(c, "part_ie", ie.data(), count);
    uint8_t* flags = static_cast<uint8_t*>(scratch(c, "side_flags", c.n + 16));
    uint32_t* item_true = static_cast<uint32_t*>(scratch(c, "item_true", (ni + 1) * sizeof(uint32_t)));
    uint32_t* prefix = static_cast<uint32_t*>(scratch(c, "item_prefix", (ni + 1) * sizeof(uint32_t)));
    KNNG_DISPATCH_D(c.d, {
        k_side<D><<<ni, kSideThreads, 0, c.stream>>>(d_items, nullptr, c.indices, c.points, c.ld, d_coefs, d_offsets,
                                                     flags, nullptr, item_true, nullptr);
    });
    k_scan_items<<<1, 1024, 0, c.stream>>>(item_true, ni, prefix, nullptr);
    k_node_true<<<(count + 255) / 256, 256, 0, c.stream>>>(d_ib, d_ie, prefix, count, d_true, nullptr);
    k_scatter<<<ni, kSideThreads, 0, c.stream>>>(d_items, d_starts, d_ib, d_true, prefix, flags, c.indices,
                                                 c.indices_tmp, nullptr);
    k_copy_back<<<ni, 256, 0, c.stream>>>(d_items, c.indices_tmp, c.indices, nullptr);
    c.launches += 5;
    KNNG_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------ host side

// Buffers of the device-side repetition, sized for the context's points,
// point sets and smallest bucket bound; the captured graphs (one per bucket
// bound, Lloyd count and precision, and the pointers baked into them).
struct DevRep {
    uint32_t n = 0, nsets = 0, min_leaf = 0, small_threshold = 0, max_set = 0;
    uint32_t node_cap = 0, lloyd_item_cap = 0, part_item_cap = 0, max_seed = 0;
    uint64_t draw_cap = 0, entry_cap = 0;
    std::vector<uint32_t> h_set_offsets;
    std::vector<std::pair<void*, size_t>> allocs;
    uint32_t *set_offsets, *table;
    uint32_t *start, *end, *base, *attempt, *nstart, *nend, *nbase, *nattempt, *leaf_start, *leaf_end;
    LevelCounts* cnt;
    uint64_t* params;  // seed, repetition, max_leaf, 0
    int32_t* error;    // [0] Lloyd sums, [1] BF16 bucket pass
    uint64_t *draw_off, *seed_off, *lloyd_off;
    uint32_t *seeds, *lloyd;
    SeqNode* seq;
    uint64_t* lbegin;
    uint32_t *lfrom, *item_off, *lids, *litem_true;
    Item* litems;
    uint8_t* lflags;
    uint32_t *first, *second;
    int32_t* ok;
    float *c1, *c2, *coefs, *offs;
    uint32_t *ib, *ie, *item_true, *prefix, *node_true;
    Item* pitems;
    uint8_t* side_flags;
    uint64_t* h_params = nullptr;  // pinned
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    struct Graph {
        uint32_t max_leaf, lloyd_iters, precision;
        uint32_t leaf_variant;  // bucket kernel and CTAs per SM baked into the graph
        const void* ptrs[8];
        cudaGraph_t graph;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;
};

namespace {

// Packed sizing rules for every node size up to `max_n`: sample count << 8 |
// seed count (the host's sample_count / start_count, so the device plan is
// the host plan).  Computed once per process and grown on demand.
std::mutex g_table_mutex;
std::vector<uint32_t> g_count_table;

const std::vector<uint32_t>& count_table(uint32_t max_n) {
    std::lock_guard<std::mutex> lock(g_table_mutex);
    const size_t have = g_count_table.size();
    if (have > max_n) return g_count_table;
    const size_t want = static_cast<size_t>(max_n) + 1;
    g_count_table.resize(want);
    const unsigned threads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    const size_t chunk = (want - have + threads - 1) / threads;
    bool bad = false;
    std::mutex bad_mutex;
    for (unsigned t = 0; t < threads; ++t) {
        const size_t lo = have + t * chunk, hi = std::min(want, lo + chunk);
        if (lo >= hi) break;
        pool.emplace_back([&, lo, hi] {
            for (size_t m = lo; m < hi; ++m) {
                const uint32_t v = static_cast<uint32_t>(m);
                const uint32_t S = v >= 2 ? start_count(v) : 0u;
                const uint32_t smp = v >= 2 ? sample_count(v) : 0u;
                if (S > 0xFFu || smp > 0xFFFFFFu) {
                    std::lock_guard<std::mutex> l(bad_mutex);
                    bad = true;
                }
                g_count_table[m] = (smp << 8) | (S & 0xFFu);
            }
        });
    }
    for (auto& th : pool) th.join();
    if (bad) fail(KNNG_ERR_UNSUPPORTED, "point set too large for the device-side sampling plan");
    return g_count_table;
}

template <class T>
T* upload_into(Context& c, T* dst, const T* host, size_t count) {
    if (count) KNNG_CUDA(cudaMemcpyAsync(dst, host, count * sizeof(T), cudaMemcpyHostToDevice, c.stream));
    return dst;
}

template <class T>
T* rep_alloc(Context& c, DevRep& r, size_t count) {
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    void* p = dev_alloc(c, bytes);
    r.allocs.emplace_back(p, bytes);
    return static_cast<T*>(p);
}

void release_graphs(DevRep& r) {
    for (auto& g : r.graphs) {
        cudaGraphExecDestroy(g.exec);
        cudaGraphDestroy(g.graph);
    }
    r.graphs.clear();
}

void release_buffers(Context& c, DevRep& r) {
    release_graphs(r);
    for (auto& a : r.allocs) dev_free(c, a.first, a.second);
    r.allocs.clear();
    r.n = 0;
}

// Buffers for the context's points and sets at bucket bound `max_leaf`.
DevRep& ensure_devrep(Context& c, uint32_t max_leaf, uint32_t small_threshold) {
    if (!c.devrep) {
        c.devrep = new DevRep();
        for (auto& e : c.devrep->ev) KNNG_CUDA(cudaEventCreate(&e));
        void* p = nullptr;
        KNNG_CUDA(cudaMallocHost(&p, 4 * sizeof(uint64_t)));
        c.devrep->h_params = static_cast<uint64_t*>(p);
    }
    DevRep& r = *c.devrep;
    const bool same = r.n == c.n && r.h_set_offsets == c.set_offsets && r.min_leaf <= max_leaf &&
                      r.small_threshold == small_threshold;
    if (same) return r;
    KNNG_CUDA(cudaStreamSynchronize(c.stream));
    release_buffers(c, r);
    r.n = c.n;
    r.h_set_offsets = c.set_offsets;
    r.nsets = static_cast<uint32_t>(c.set_offsets.size() - 1);
    r.min_leaf = max_leaf;
    r.small_threshold = small_threshold;
    r.max_set = 0;
    for (uint32_t s = 0; s < r.nsets; ++s) r.max_set = std::max(r.max_set, c.set_offsets[s + 1] - c.set_offsets[s]);
    const std::vector<uint32_t>& table = count_table(std::max(r.max_set, 2u));
    // Capacities: a level's nodes hold >= max_leaf points each and are
    // disjoint; draws are a large node's sample (at most r_max of its points)
    // or a small node's seeds.
    double r_max = 0.0;
    for (uint32_t m = std::max(small_threshold, 2u); m <= r.max_set; ++m)
        r_max = std::max(r_max, static_cast<double>(table[m] >> 8) / m);
    r.max_seed = 1;
    for (uint32_t m = 2; m <= r.max_set; ++m) r.max_seed = std::max(r.max_seed, table[m] & 0xFFu);
    r.node_cap = r.n / std::max(max_leaf, 2u) + r.nsets + 1;
    r.draw_cap = static_cast<uint64_t>(std::ceil(r_max * r.n)) + static_cast<uint64_t>(r.node_cap) * r.max_seed + 16;
    r.entry_cap = r.n + r.draw_cap + 16ull * r.node_cap + 64;
    r.lloyd_item_cap = static_cast<uint32_t>(r.entry_cap / kChunk) + r.node_cap + 1;
    r.part_item_cap = r.n / kChunk + r.node_cap + 1;
    const uint32_t nc = r.node_cap, ld = c.ld;
    r.set_offsets = upload_into(c, rep_alloc<uint32_t>(c, r, r.nsets + 1), c.set_offsets.data(), r.nsets + 1);
    r.table = upload_into(c, rep_alloc<uint32_t>(c, r, r.max_set + 1), table.data(), r.max_set + 1);
    r.start = rep_alloc<uint32_t>(c, r, nc);
    r.end = rep_alloc<uint32_t>(c, r, nc);
    r.base = rep_alloc<uint32_t>(c, r, nc);
    r.attempt = rep_alloc<uint32_t>(c, r, nc);
    r.nstart = rep_alloc<uint32_t>(c, r, nc);
    r.nend = rep_alloc<uint32_t>(c, r, nc);
    r.nbase = rep_alloc<uint32_t>(c, r, nc);
    r.nattempt = rep_alloc<uint32_t>(c, r, nc);
    r.leaf_start = rep_alloc<uint32_t>(c, r, r.n + r.nsets);
    r.leaf_end = rep_alloc<uint32_t>(c, r, r.n + r.nsets);
    r.cnt = rep_alloc<LevelCounts>(c, r, 1);
    r.params = rep_alloc<uint64_t>(c, r, 4);
    r.error = rep_alloc<int32_t>(c, r, 4);
    r.draw_off = rep_alloc<uint64_t>(c, r, nc + 1);
    r.seed_off = rep_alloc<uint64_t>(c, r, nc + 1);
    r.lloyd_off = rep_alloc<uint64_t>(c, r, nc + 1);
    r.seeds = rep_alloc<uint32_t>(c, r, static_cast<size_t>(nc) * r.max_seed + 1);
    r.lloyd = rep_alloc<uint32_t>(c, r, r.draw_cap);
    r.seq = rep_alloc<SeqNode>(c, r, nc);
    r.lbegin = rep_alloc<uint64_t>(c, r, nc);
    r.lfrom = rep_alloc<uint32_t>(c, r, nc);
    r.item_off = rep_alloc<uint32_t>(c, r, nc + 1);
    r.litems = rep_alloc<Item>(c, r, r.lloyd_item_cap);
    r.lflags = rep_alloc<uint8_t>(c, r, r.entry_cap);
    r.lids = rep_alloc<uint32_t>(c, r, r.entry_cap);
    r.litem_true = rep_alloc<uint32_t>(c, r, r.lloyd_item_cap + 1);
    r.first = rep_alloc<uint32_t>(c, r, nc);
    r.second = rep_alloc<uint32_t>(c, r, nc);
    r.ok = rep_alloc<int32_t>(c, r, nc);
    r.c1 = rep_alloc<float>(c, r, static_cast<size_t>(nc) * ld);
    r.c2 = rep_alloc<float>(c, r, static_cast<size_t>(nc) * ld);
    r.coefs = rep_alloc<float>(c, r, static_cast<size_t>(nc) * ld);
    r.offs = rep_alloc<float>(c, r, nc);
    r.ib = rep_alloc<uint32_t>(c, r, nc);
    r.ie = rep_alloc<uint32_t>(c, r, nc);
    r.pitems = rep_alloc<Item>(c, r, r.part_item_cap);
    r.side_flags = rep_alloc<uint8_t>(c, r, static_cast<size_t>(r.n) + 16);
    r.item_true = rep_alloc<uint32_t>(c, r, r.part_item_cap + 1);
    r.prefix = rep_alloc<uint32_t>(c, r, r.part_item_cap + 1);
    r.node_true = rep_alloc<uint32_t>(c, r, nc);
    KNNG_CUDA(cudaStreamSynchronize(c.stream));
    return r;
}

constexpr uint32_t kNodeGrid = 148 * 4;
constexpr uint32_t kItemGrid = 148 * 8;
constexpr uint32_t kThreadGrid = 148 * 2;

// Start of a repetition: the error words cleared, indices 0..n-1, the sets'
// roots as the first level.
void enqueue_prologue(Context& c, DevRep& r, cudaGraphConditionalHandle cond, int set_cond) {
    KNNG_CUDA(cudaMemsetAsync(r.error, 0, 4 * sizeof(int32_t), c.stream));
    k_iota<<<std::min<uint32_t>((c.n + 255) / 256, 148 * 16), 256, 0, c.stream>>>(c.indices, c.n);
    k_rep_init<<<1, 256, 0, c.stream>>>(r.set_offsets, r.nsets, r.params, r.cnt, r.start, r.end, r.base, r.attempt,
                                        r.leaf_start, r.leaf_end, cond, set_cond);
    c.launches += 2;
    KNNG_CUDA(cudaGetLastError());
}

// One tree level: plan, draws, seeding, Lloyd iterations, partition, outcome.
// Launch sizes do not depend on the level; no allocation, no host sync.
void enqueue_level(Context& c, DevRep& r, uint32_t lloyd_iters, cudaGraphConditionalHandle cond, int set_cond) {
    uint32_t* cur = &r.cnt->cur;
    k_level_plan<<<1, kPlanThreads, 0, c.stream>>>(r.start, r.end, r.cnt, r.table, r.small_threshold, r.draw_off,
                                                   r.seed_off, r.lloyd_off, r.seq, r.lbegin, r.lfrom, r.item_off);
    k_draw_positions<<<kNodeGrid, 256, 0, c.stream>>>(r.start, r.end, r.base, r.attempt, r.draw_off, r.seed_off,
                                                      r.lloyd_off, 0, 0, r.seeds, r.lloyd, cur, r.params);
    k_lloyd_items<<<kThreadGrid, 256, 0, c.stream>>>(r.cnt, r.item_off, r.seq, r.lbegin, r.lfrom, r.litems);
    KNNG_DISPATCH_D(c.d, {
        const size_t fp_smem = static_cast<size_t>(r.max_seed) * c.ld * sizeof(float);
        auto fp = k_farthest_pair<D>;
        allow_max_smem(c, fp);
        fp<<<kNodeGrid, kPairThreads, fp_smem, c.stream>>>(r.seed_off, r.seeds, c.indices, c.points, c.ld, r.first,
                                                           r.second, r.ok, r.c1, r.c2, cur);
        auto seqk = k_lloyd_seq<D>;
        allow_max_smem(c, seqk);
        for (uint32_t iter = 0; iter < lloyd_iters; ++iter) {
            k_plane<D><<<kNodeGrid, 256, 0, c.stream>>>(r.c1, r.c2, c.ld, 0, r.coefs, r.offs, cur);
            k_side<D><<<kItemGrid, kSideThreads, 0, c.stream>>>(r.litems, r.lloyd, c.indices, c.points, c.ld, r.coefs,
                                                                r.offs, r.lflags, r.lids, r.litem_true,
                                                                &r.cnt->lloyd_items);
            seqk<<<kThreadGrid, kSeqThreads, seq_smem_bytes(D), c.stream>>>(r.seq, r.lflags, r.lids, c.points, c.ld,
                                                                              r.c1, r.c2, r.ok, r.error, cur);
        }
        k_plane<D><<<kNodeGrid, 256, 0, c.stream>>>(r.c1, r.c2, c.ld, 0, r.coefs, r.offs, cur);
        k_part_plan<<<1, kPlanThreads, 0, c.stream>>>(r.start, r.end, r.cnt, r.ok, r.ib, r.ie);
        k_part_items<<<kThreadGrid, 256, 0, c.stream>>>(r.cnt, r.start, r.end, r.ib, r.pitems);
        k_side<D><<<kItemGrid, kSideThreads, 0, c.stream>>>(r.pitems, nullptr, c.indices, c.points, c.ld, r.coefs,
                                                            r.offs, r.side_flags, nullptr, r.item_true,
                                                            &r.cnt->part_items);
    });
    k_scan_items<<<1, 1024, 0, c.stream>>>(r.item_true, 0, r.prefix, &r.cnt->part_items);
    k_node_true<<<kThreadGrid, 256, 0, c.stream>>>(r.ib, r.ie, r.prefix, 0, r.node_true, cur);
    k_scatter<<<kItemGrid, kSideThreads, 0, c.stream>>>(r.pitems, r.start, r.ib, r.node_true, r.prefix, r.side_flags,
                                                        c.indices, c.indices_tmp, &r.cnt->part_items);
    k_copy_back<<<kItemGrid, 256, 0, c.stream>>>(r.pitems, c.indices_tmp, c.indices, &r.cnt->part_items);
    k_level_next<<<kThreadGrid, 256, 0, c.stream>>>(r.start, r.end, r.base, r.attempt, r.cnt, r.ok, r.node_true,
                                                    r.params, r.nstart, r.nend, r.nbase, r.nattempt, r.leaf_start,
                                                    r.leaf_end);
    k_level_swap<<<1, kPlanThreads, 0, c.stream>>>(r.cnt, r.nstart, r.nend, r.nbase, r.nattempt, r.start, r.end,
                                                   r.base, r.attempt, r.error + 2, cond, set_cond);
    c.launches += 14 + 3 * lloyd_iters;
    KNNG_CUDA(cudaGetLastError());
}

void enqueue_buckets(Context& c, DevRep& r, uint32_t max_leaf, uint32_t precision) {
    if (precision == KNNG_PRECISION_BF16_RERANK)
        launch_leaves_bf16_list(c, r.leaf_start, r.leaf_end, &r.cnt->leaves, &r.cnt->leaf_work,
                                reinterpret_cast<uint32_t*>(r.error + 1));
    else
        launch_leaves_list(c, r.leaf_start, r.leaf_end, &r.cnt->leaves, &r.cnt->leaf_work, max_leaf - 1,
                           reinterpret_cast<uint32_t*>(r.error + 1));
}

// The repetition as one graph: prologue, WHILE (nodes left) { level },
// buckets, with timing events between the parts.
DevRep::Graph& rep_graph(Context& c, DevRep& r, uint32_t max_leaf, uint32_t lloyd_iters, uint32_t precision) {
    const void* ptrs[8] = {c.points, c.indices, c.indices_tmp, c.set_dist, c.set_id, c.set_size, c.set_bound,
                           reinterpret_cast<const void*>(static_cast<uintptr_t>(c.k))};
    const uint32_t variant = (c.leaf_tc ? 4u : 0u) | c.leaf_ctas;
    for (auto& g : r.graphs)
        if (g.max_leaf == max_leaf && g.lloyd_iters == lloyd_iters && g.precision == precision &&
            g.leaf_variant == variant && std::equal(ptrs, ptrs + 8, g.ptrs))
            return g;
    DevRep::Graph g{max_leaf, lloyd_iters, precision, variant, {}, nullptr, nullptr};
    std::copy(ptrs, ptrs + 8, g.ptrs);
    const uint64_t launches0 = c.launches;
    // Attributes first: nothing but stream work may happen during the capture.
    KNNG_DISPATCH_D(c.d, {
        allow_max_smem(c, k_farthest_pair<D>);
        allow_max_smem(c, k_lloyd_seq<D>);
    });
    if (precision == KNNG_PRECISION_BF16_RERANK)
        prepare_leaves_bf16_list(c);
    else
        prepare_leaves_list(c);
    if (r.graphs.size() >= 4) {
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
        release_graphs(r);
    }
    struct CaptureFlag {
        Context& c;
        explicit CaptureFlag(Context& cc) : c(cc) { c.capturing = true; }
        ~CaptureFlag() { c.capturing = false; }
    } capture_flag(c);
    KNNG_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    cudaGraphConditionalHandle cond{};
    cudaGraph_t body = nullptr;
    try {
        cudaStreamCaptureStatus status;
        cudaGraph_t capg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        KNNG_CUDA(cudaStreamGetCaptureInfo(c.stream, &status, nullptr, &capg, &deps, &ndeps));
        KNNG_CUDA(cudaGraphConditionalHandleCreate(&cond, capg, 0, cudaGraphCondAssignDefault));
        KNNG_CUDA(cudaEventRecordWithFlags(r.ev[0], c.stream, cudaEventRecordExternal));
        enqueue_prologue(c, r, cond, 1);
        KNNG_CUDA(cudaStreamGetCaptureInfo(c.stream, &status, nullptr, &capg, &deps, &ndeps));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        KNNG_CUDA(cudaGraphAddNode(&node, capg, deps, ndeps, &cp));
        body = cp.conditional.phGraph_out[0];
        KNNG_CUDA(cudaStreamUpdateCaptureDependencies(c.stream, &node, 1, cudaStreamSetCaptureDependencies));
        KNNG_CUDA(cudaEventRecordWithFlags(r.ev[1], c.stream, cudaEventRecordExternal));
        enqueue_buckets(c, r, max_leaf, precision);
        KNNG_CUDA(cudaEventRecordWithFlags(r.ev[2], c.stream, cudaEventRecordExternal));
    } catch (...) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(c.stream, &junk);
        if (junk) cudaGraphDestroy(junk);
        cudaGetLastError();
        throw;
    }
    KNNG_CUDA(cudaStreamEndCapture(c.stream, &g.graph));
    // The WHILE node's body: one level, which sets the condition at its end.
    KNNG_CUDA(cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
        enqueue_level(c, r, lloyd_iters, cond, 1);
    } catch (...) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(c.stream, &junk);
        cudaGraphDestroy(g.graph);
        cudaGetLastError();
        throw;
    }
    cudaGraph_t body_out = nullptr;
    KNNG_CUDA(cudaStreamEndCapture(c.stream, &body_out));
    KNNG_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
    c.launches = launches0;  // capturing launched nothing
    r.graphs.push_back(g);
    return r.graphs.back();
}

}  // namespace

// Device time between two recorded events; NaN when the runtime cannot
// report it (the timings are diagnostics, the build's result stands).
static float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        return std::numeric_limits<float>::quiet_NaN();
    }
    return ms;
}

void devrep_release(Context& c) {
    if (!c.devrep) return;
    if (c.stream) cudaStreamSynchronize(c.stream);
    release_buffers(c, *c.devrep);
    for (auto& e : c.devrep->ev)
        if (e) cudaEventDestroy(e);
    if (c.devrep->h_params) cudaFreeHost(c.devrep->h_params);
    delete c.devrep;
    c.devrep = nullptr;
}

void run_rep_device(Context& c, uint32_t max_leaf, uint32_t lloyd_iters, uint32_t small_threshold, uint64_t seed,
                    uint32_t rep, uint32_t precision, bool graph, DevRepResult& out) {
    DevRep& r = ensure_devrep(c, max_leaf, small_threshold);
    r.h_params[0] = seed;
    r.h_params[1] = rep;
    r.h_params[2] = max_leaf;
    r.h_params[3] = 0;
    KNNG_CUDA(cudaMemcpyAsync(r.params, r.h_params, 4 * sizeof(uint64_t), cudaMemcpyHostToDevice, c.stream));
    if (graph) {
        DevRep::Graph& g = rep_graph(c, r, max_leaf, lloyd_iters, precision);
        KNNG_CUDA(cudaGraphLaunch(g.exec, c.stream));
    } else {
        KNNG_CUDA(cudaEventRecord(r.ev[0], c.stream));
        enqueue_prologue(c, r, cudaGraphConditionalHandle{}, 0);
        for (uint32_t it = 0;; ++it) {
            uint32_t cur = 0;
            download(c, &cur, &r.cnt->cur, 1);
            if (cur == 0) break;
            if (it >= kMaxLevelIterations) fail(KNNG_ERR_CUDA, "tree levels: the level loop ran past its iteration limit");
            enqueue_level(c, r, lloyd_iters, cudaGraphConditionalHandle{}, 0);
        }
        KNNG_CUDA(cudaEventRecord(r.ev[1], c.stream));
        enqueue_buckets(c, r, max_leaf, precision);
        KNNG_CUDA(cudaEventRecord(r.ev[2], c.stream));
    }
    LevelCounts h{};
    download(c, &h, r.cnt, 1);
    // Kernels the graph ran: prologue (2), every level, the bucket pass.
    if (graph) c.launches += 3 + static_cast<uint64_t>(h.iterations) * (14 + 3 * lloyd_iters);
    int32_t err[4] = {0, 0, 0, 0};
    download(c, err, r.error, 4);
    if (err[0]) fail(KNNG_ERR_CUDA, "Lloyd sums: a bulk-copy wait gave up");
    if (err[1]) fail(KNNG_ERR_CUDA, "bucket pass: the MMA completion wait gave up");
    if (err[2]) fail(KNNG_ERR_CUDA, "tree levels: the level loop ran past its iteration limit");
    out.leaf_start.resize(h.leaves);
    out.leaf_end.resize(h.leaves);
    download(c, out.leaf_start.data(), r.leaf_start, h.leaves);
    download(c, out.leaf_end.data(), r.leaf_end, h.leaves);
    out.ms_split = elapsed_ms(r.ev[0], r.ev[1]);
    out.ms_leaf = elapsed_ms(r.ev[1], r.ev[2]);
    out.levels = h.iterations;
    out.nodes = h.nodes;
    out.restarts = h.restarts;
    out.fallbacks = h.fallbacks;
    out.pairs = h.pairs;
}

}  // namespace knng
