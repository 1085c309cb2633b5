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

}  // namespace knng
