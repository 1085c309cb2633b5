// Tree construction kernels: the recursive 2-means split of
// SolutionKmeans::splitKmeansBinaryProcess (src/SolutionKmeans.hpp:142-311),
// run level-synchronously over every node of a tree level at once.
//
//   k_draw_positions   sample / seed positions from the counter RNG
//                      (getSampleFromPercent :55-66, kmeansStartVecs :103-111)
//   k_farthest_pair    farthest pair among the seed positions (:68-101, :113-127)
//   k_plane            between / coefs / offset from two centres (:162-164)
//   k_lloyd_accum      side test + per-cluster double sums over a tile
//                      (:170-175, :227-238)
//   k_lloyd_reduce     per-node sum of tile partials, new centres (:182-185, :239-259)
//   k_side             final side test of every point of a node (:195-197, :273-278)
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

namespace knng {
namespace {

constexpr int kSideThreads = 256;
constexpr int kSidePer = 8;  // positions per thread in the side / scatter kernels
constexpr int kChunk = kSideThreads * kSidePer;
constexpr int kLloydThreads = 256;
constexpr int kLloydTile = 64;
constexpr int kLloydItem = 256;  // positions per Lloyd work item
constexpr int kPairThreads = 256;

struct Item {
    uint32_t node;
    uint32_t count;
    uint64_t begin;  // first position (range items) or first list entry (list items)
};

__global__ void k_iota(uint32_t* __restrict__ idx, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) idx[i] = i;
}

// Node i draws draws[i] positions; the first seed_len[i] go to its seed list
// and the first lloyd_len[i] to its Lloyd list (both CSR).
// Node [start, end) of a set starting at `base` draws with keys relative to
// the set, so a set's tree is the same alone and in a batch.
__global__ void k_draw_positions(const uint32_t* __restrict__ starts, const uint32_t* __restrict__ ends,
                                 const uint32_t* __restrict__ bases, const uint32_t* __restrict__ attempts,
                                 const uint64_t* __restrict__ draw_off,
                                 const uint64_t* __restrict__ seed_off, const uint64_t* __restrict__ lloyd_off,
                                 uint64_t seed, uint32_t rep, uint32_t* __restrict__ seeds_out,
                                 uint32_t* __restrict__ lloyd_out) {
    const uint32_t node = blockIdx.x;
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
                                int32_t* __restrict__ out_ok, float* __restrict__ c1, float* __restrict__ c2) {
    extern __shared__ float4 smem4[];
    float* rows = reinterpret_cast<float*>(smem4);
    const uint32_t node = blockIdx.x;
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
    __shared__ float sv[kPairThreads / kWarp];
    __shared__ uint32_t si[kPairThreads / kWarp], sj[kPairThreads / kWarp];
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
}

// between = 0.5f * (c1 + c2); coefs = c1 - between; offset = dot(between, coefs).
template <int D>
__global__ void k_plane(const float* __restrict__ c1, const float* __restrict__ c2, int ld, uint32_t count,
                        float* __restrict__ coefs, float* __restrict__ offsets) {
    const uint32_t node = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
    const int lane = threadIdx.x % kWarp;
    if (node >= count) return;
    __shared__ float between_s[8][(D + 3) / 4 * 4];
    float* between = between_s[threadIdx.x / kWarp];
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
}

// Per work item: side test of up to kLloydItem points against the node's
// current hyperplane, then per-cluster double sums in point order.
// partial layout per item: [n1, n2, s1[0..D), s2[0..D)].
template <int D>
__global__ void __launch_bounds__(kLloydThreads) k_lloyd_accum(const Item* __restrict__ items,
                                                               const uint32_t* __restrict__ list,
                                                               const uint32_t* __restrict__ idx,
                                                               const float* __restrict__ pts, int ld,
                                                               const float* __restrict__ coefs,
                                                               const float* __restrict__ offsets,
                                                               double* __restrict__ partial) {
    constexpr int Q = (D + 3) / 4;
    __shared__ float4 rows[kLloydTile][Q];
    __shared__ float4 plane[Q];
    __shared__ int side[kLloydTile];
    const Item it = items[blockIdx.x];
    const bool from_list = (it.node & 0x80000000u) != 0;
    const uint32_t node = it.node & 0x7FFFFFFFu;
    for (int q = threadIdx.x; q < Q; q += blockDim.x)
        plane[q] = reinterpret_cast<const float4*>(coefs + static_cast<size_t>(node) * ld)[q];
    const float off = offsets[node];
    const int t = threadIdx.x;
    const int cluster = t / D;  // 0: side-true sums, 1: side-false sums, >= 2 idle
    const int dim = t % D;
    double acc = 0.0;
    uint32_t cnt = 0;
    for (uint32_t base = 0; base < it.count; base += kLloydTile) {
        const uint32_t rows_here = min(static_cast<uint32_t>(kLloydTile), it.count - base);
        __syncthreads();
        for (uint32_t f = threadIdx.x; f < rows_here * Q; f += blockDim.x) {
            const uint32_t r = f / Q, q = f % Q;
            const uint64_t e = it.begin + base + r;
            const uint32_t pos = from_list ? list[e] : static_cast<uint32_t>(e);
            rows[r][q] = reinterpret_cast<const float4*>(pts + static_cast<size_t>(idx[pos]) * ld)[q];
        }
        __syncthreads();
        if (t < static_cast<int>(rows_here)) side[t] = canonical_dot4<D>(plane, rows[t]) >= off ? 1 : 0;
        __syncthreads();
        if (cluster < 2) {
            const int want = cluster == 0 ? 1 : 0;
            const float* rf = reinterpret_cast<const float*>(rows);
            for (uint32_t r = 0; r < rows_here; ++r) {
                if (side[r] == want) {
                    acc = __dadd_rn(acc, static_cast<double>(rf[r * Q * 4 + dim]));
                    ++cnt;
                }
            }
        }
    }
    double* out = partial + static_cast<size_t>(blockIdx.x) * (2 * D + 2);
    if (cluster < 2) {
        out[2 + cluster * D + dim] = acc;
        if (dim == 0) out[cluster] = static_cast<double>(cnt);
    }
}

// Per node: items [item_begin, item_end) summed in order; centres updated.
template <int D>
__global__ void k_lloyd_reduce(const uint32_t* __restrict__ item_begin, const uint32_t* __restrict__ item_end,
                               const double* __restrict__ partial, int ld, float* __restrict__ c1,
                               float* __restrict__ c2, int32_t* __restrict__ ok) {
    const uint32_t node = blockIdx.x;
    const uint32_t ib = item_begin[node], ie = item_end[node];
    __shared__ double counts[2];
    if (threadIdx.x < 2) {
        double c = 0.0;
        for (uint32_t i = ib; i < ie; ++i) c = __dadd_rn(c, partial[static_cast<size_t>(i) * (2 * D + 2) + threadIdx.x]);
        counts[threadIdx.x] = c;
    }
    __syncthreads();
    const double n1 = counts[0], n2 = counts[1];
    if (threadIdx.x == 0 && (n1 == 0.0 || n2 == 0.0)) ok[node] = 0;
    for (int t = threadIdx.x; t < 2 * D; t += blockDim.x) {
        const int cluster = t / D, dim = t % D;
        double s = 0.0;
        for (uint32_t i = ib; i < ie; ++i) s = __dadd_rn(s, partial[static_cast<size_t>(i) * (2 * D + 2) + 2 + t]);
        const double nn = cluster == 0 ? n1 : n2;
        if (nn > 0.0) {
            const float v = __double2float_rn(__ddiv_rn(s, nn));
            (cluster == 0 ? c1 : c2)[static_cast<size_t>(node) * ld + dim] = v;
        }
    }
}

// Side flags for the positions of one chunk of one node; per-chunk true count.
template <int D>
__global__ void __launch_bounds__(kSideThreads) k_side(const Item* __restrict__ items, const uint32_t* __restrict__ idx,
                                                       const float* __restrict__ pts, int ld,
                                                       const float* __restrict__ coefs,
                                                       const float* __restrict__ offsets,
                                                       uint8_t* __restrict__ flags, uint32_t* __restrict__ item_true) {
    constexpr int Q = (D + 3) / 4;
    __shared__ float4 plane[Q];
    __shared__ uint32_t warp_sum[kSideThreads / kWarp];
    const Item it = items[blockIdx.x];
    for (int q = threadIdx.x; q < Q; q += blockDim.x)
        plane[q] = reinterpret_cast<const float4*>(coefs + static_cast<size_t>(it.node) * ld)[q];
    const float off = offsets[it.node];
    __syncthreads();
    uint32_t cnt = 0;
    for (uint32_t r = threadIdx.x; r < it.count; r += blockDim.x) {
        const uint64_t pos = it.begin + r;
        const float4* row = reinterpret_cast<const float4*>(pts + static_cast<size_t>(idx[pos]) * ld);
        const uint8_t f = canonical_dot4<D>(plane, row) >= off ? 1 : 0;
        flags[pos] = f;
        cnt += f;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(kFull, cnt, o);
    if (threadIdx.x % kWarp == 0) warp_sum[threadIdx.x / kWarp] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int w = 0; w < kSideThreads / kWarp; ++w) s += warp_sum[w];
        item_true[blockIdx.x] = s;
    }
}

// Exclusive scan of n values into out[0..n] (out[n] = total); one CTA.
__global__ void k_scan_items(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ out) {
    __shared__ uint32_t part[1024];
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
                            const uint32_t* __restrict__ prefix, uint32_t count, uint32_t* __restrict__ out_true) {
    const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node < count) out_true[node] = prefix[item_end[node]] - prefix[item_begin[node]];
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
                                                          uint32_t* __restrict__ idx_out) {
    __shared__ uint32_t warp_tot[kSideThreads / kWarp];
    const Item it = items[blockIdx.x];
    const uint32_t s = node_start[it.node];
    const uint32_t T = node_true[it.node];
    const uint32_t before_item = prefix[blockIdx.x] - prefix[node_item_begin[it.node]];
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
}

__global__ void k_copy_back(const Item* __restrict__ items, const uint32_t* __restrict__ src,
                            uint32_t* __restrict__ dst) {
    const Item it = items[blockIdx.x];
    for (uint32_t r = threadIdx.x; r < it.count; r += blockDim.x) dst[it.begin + r] = src[it.begin + r];
}

}  // namespace

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
                                                  seed, rep, d_seeds, d_lloyd);
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
                                                      d_second, d_ok, d_c1, d_c2);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

void launch_plane(Context& c, uint32_t count, const float* d_c1, const float* d_c2, float* d_coefs,
                  float* d_offsets) {
    if (count == 0) return;
    KNNG_DISPATCH_D(c.d, {
        k_plane<D><<<(count + 7) / 8, 256, 0, c.stream>>>(d_c1, d_c2, c.ld, count, d_coefs, d_offsets);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

void launch_lloyd(Context& c, uint32_t count, const uint32_t* h_starts, const uint32_t* h_ends,
                  const uint64_t* h_lloyd_offsets, const uint32_t* d_lloyd_positions, float* d_c1, float* d_c2,
                  uint32_t iters, float* d_coefs, float* d_offsets, int32_t* d_ok) {
    if (count == 0) return;
    // Work items: each node's Lloyd set (its list, or its whole range when the
    // list is empty) cut into kLloydItem-point items, in order.
    std::vector<Item> items;
    std::vector<uint32_t> ib(count), ie(count);
    for (uint32_t i = 0; i < count; ++i) {
        ib[i] = static_cast<uint32_t>(items.size());
        const uint64_t lb = h_lloyd_offsets[i], le = h_lloyd_offsets[i + 1];
        if (le > lb) {
            for (uint64_t o = lb; o < le; o += kLloydItem)
                items.push_back({i | 0x80000000u, static_cast<uint32_t>(std::min<uint64_t>(kLloydItem, le - o)), o});
        } else {
            for (uint64_t o = h_starts[i]; o < h_ends[i]; o += kLloydItem)
                items.push_back({i, static_cast<uint32_t>(std::min<uint64_t>(kLloydItem, h_ends[i] - o)), o});
        }
        ie[i] = static_cast<uint32_t>(items.size());
    }
    const Item* d_items = upload(c, "lloyd_items", items.data(), items.size());
    const uint32_t* d_ib = upload(c, "lloyd_ib", ib.data(), count);
    const uint32_t* d_ie = upload(c, "lloyd_ie", ie.data(), count);
    KNNG_DISPATCH_D(c.d, {
        double* partial = static_cast<double*>(scratch(c, "lloyd_partial", items.size() * (2 * D + 2) * sizeof(double)));
        for (uint32_t iter = 0; iter < iters; ++iter) {
            launch_plane(c, count, d_c1, d_c2, d_coefs, d_offsets);
            k_lloyd_accum<D><<<static_cast<uint32_t>(items.size()), kLloydThreads, 0, c.stream>>>(
                d_items, d_lloyd_positions, c.indices, c.points, c.ld, d_coefs, d_offsets, partial);
            k_lloyd_reduce<D><<<count, 256, 0, c.stream>>>(d_ib, d_ie, partial, c.ld, d_c1, d_c2, d_ok);
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
            items.push_back({i, static_cast<uint32_t>(std::min<uint64_t>(kChunk, h_ends[i] - o)), o});
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
        k_side<D><<<ni, kSideThreads, 0, c.stream>>>(d_items, c.indices, c.points, c.ld, d_coefs, d_offsets, flags,
                                                     item_true);
    });
    k_scan_items<<<1, 1024, 0, c.stream>>>(item_true, ni, prefix);
    k_node_true<<<(count + 255) / 256, 256, 0, c.stream>>>(d_ib, d_ie, prefix, count, d_true);
    k_scatter<<<ni, kSideThreads, 0, c.stream>>>(d_items, d_starts, d_ib, d_true, prefix, flags, c.indices,
                                                 c.indices_tmp);
    k_copy_back<<<ni, 256, 0, c.stream>>>(d_items, c.indices_tmp, c.indices);
    c.launches += 5;
    KNNG_CUDA(cudaGetLastError());
}

}  // namespace knng
