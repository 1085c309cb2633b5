// Neighbour-of-neighbour pass: SolutionKmeans::topUpSingle
// (src/SolutionKmeans.hpp:480-555).
//
// Snapshot: every set's k slot ids, sorted ascending, unfilled slots included
// (as the point set's first id, 0 for a single set) -- the reference reads all
// 100 current_ids (:494).  Per point p, the candidates are the union of the
// snapshot lists of p's snapshot list, minus p, each offered with the exact
// distance when dist < bound.
//
// The reference iterates its candidate set in hash order; this pass offers
// them in ascending id order.  The order can only matter between candidates
// that beat the bound p had when its pass started, so the pass collects every
// such survivor (dist < starting bound), sorts each point's survivors by id and
// replays them in that order through the sequential set update.
//
// Two ways to collect the survivors, with the same result:
//   * the local join (k_join, the default): per point q, the rows R(q) (points
//     whose list holds q) against the columns S(q) (q's list) as one block; a
//     tcgen05 tile of centred dot products (FP16 operands, FP32 accumulation)
//     rejects the pairs that provably cannot beat bound(p), members of S(p) are dropped, the rest get the exact
//     FP32 distance; survivors go to per-point slots, then to the CTA's pool
//     region (k_excess_counts / k_pool_scatter turn the pool into per-point
//     lists), and one k_apply launch sorts and replays every point's survivors;
//   * one warp per point (k_refine): the warp walks its candidates (one lane per
//     candidate, rows gathered from HBM/L2) with a shared-memory seen-set, keeps
//     the survivors in shared memory (or a per-warp global region of k*k
//     entries) and replays them.  It serves as the cross-check of the join
//     (environment KNNG_REFINE=pointwise), as the pass for the points whose
//     pool region filled up, and behind the allocation-free entry point.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "context.hpp"
#include "dispatch.hpp"
#include "tc.cuh"

namespace knng {
namespace {

constexpr int kSnapWarps = 8;
constexpr int kRefWarps = 4;
constexpr int kSurvCap = 256;

constexpr int kSeenSlots = 2048;  // per-warp open-addressing set of candidate ids
constexpr int kSeenProbes = 32;

// Inserts id into the warp's seen-set; true if it was not there.  When the
// probe limit is reached the id is reported new: a repeated offer is harmless
// (the set update rejects it), only slower.
__device__ __forceinline__ bool seen_insert(uint32_t* seen, uint32_t id) {
    uint32_t h = (id * 0x9E3779B1u) >> (32 - 11);
    for (int probe = 0; probe < kSeenProbes; ++probe) {
        const uint32_t prev = atomicCAS(&seen[h], kNone, id);
        if (prev == kNone) return true;
        if (prev == id) return false;
        h = (h + 1) & (kSeenSlots - 1);
    }
    return true;
}

__host__ __device__ uint32_t pow2_at_least(uint32_t v) {
    uint32_t p = 2;
    while (p < v) p <<= 1;
    return p;
}

// Words of a point's old-entry mask (one bit per snapshot entry).
constexpr int kOldWords = kMaxK / kWarp;  // 4

// Each point's sorted list of its set's k slot ids.  With `prev` (the sorted
// lists of the previous pass) also old[p * kOldWords + i / 32] bit i % 32 =
// entry i of the new list is in the point's previous list.
__global__ void __launch_bounds__(kSnapWarps * kWarp) k_snapshot(const uint32_t* __restrict__ set_id, uint32_t n, int K,
                                                                 uint32_t* __restrict__ snap,
                                                                 const uint32_t* __restrict__ prev,
                                                                 uint32_t* __restrict__ old) {
    __shared__ uint32_t keys_s[kSnapWarps][kMaxK];
    __shared__ uint32_t prev_s[kSnapWarps][kMaxK];
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    uint32_t* keys = keys_s[warp];
    uint32_t* pl = prev_s[warp];
    int top = 1;  // largest power of two <= K (branch-free lower bound)
    while (top * 2 <= K) top *= 2;
    for (uint32_t p = blockIdx.x * kSnapWarps + warp; p < n; p += gridDim.x * kSnapWarps) {
        const size_t base = static_cast<size_t>(p) * K;
        for (int slot = lane; slot < kMaxK; slot += kWarp) keys[slot] = slot < K ? set_id[base + slot] : ~0u;
        if (prev)
            for (int i = lane; i < K; i += kWarp) pl[i] = prev[base + i];
        __syncwarp();
        warp_bitonic_sort(keys, kMaxK, lane);
        for (int i = lane; i < K; i += kWarp) snap[base + i] = static_cast<uint32_t>(keys[i]);
        if (prev) {
#pragma unroll
            for (int w = 0; w < kOldWords; ++w) {
                const int i = w * kWarp + lane;
                bool found = false;
                if (i < K) {
                    const uint32_t id = static_cast<uint32_t>(keys[i]);
                    int pos = 0;  // first entry of pl >= id
                    for (int step = top; step > 0; step >>= 1)
                        if (pos + step <= K && pl[pos + step - 1] < id) pos += step;
                    found = pos < K && pl[pos] == id;
                }
                const unsigned m = __ballot_sync(kFull, found);
                if (lane == 0) old[static_cast<size_t>(p) * kOldWords + w] = m;
            }
        }
        __syncwarp();
    }
}

template <int D>
__global__ void __launch_bounds__(kRefWarps * kWarp)
    k_refine(const uint32_t* __restrict__ snap, const float* __restrict__ pts, int ld, float* __restrict__ set_dist,
             uint32_t* __restrict__ set_id, uint32_t* __restrict__ set_size, uint32_t* __restrict__ set_maxslot,
             float* __restrict__ set_bound, int K, uint32_t n, const uint32_t* __restrict__ plist,
             unsigned long long* __restrict__ scratch_keys, uint32_t warp_capacity,
             uint32_t* __restrict__ changed_count) {
    constexpr int Q = D / 4;
    __shared__ float4 rowp_s[kRefWarps][Q];
    __shared__ unsigned long long surv_s[kRefWarps][kSurvCap];
    __shared__ uint32_t seen_s[kRefWarps][kSeenSlots];
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    const uint32_t gw = blockIdx.x * kRefWarps + warp;
    const uint32_t nw = gridDim.x * kRefWarps;
    unsigned long long* gbuf = scratch_keys + static_cast<size_t>(gw) * warp_capacity;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (uint32_t w = gw; w < n; w += nw) {
        const uint32_t p = plist ? plist[w] : w;
        for (int q = lane; q < Q; q += kWarp)
            rowp_s[warp][q] = __ldg(reinterpret_cast<const float4*>(pts + static_cast<size_t>(p) * ld) + q);
        WarpSet s;
        set_load(s, set_dist, set_id, set_size, set_maxslot, set_bound, p, K, lane);
        // Seen-set: p itself and p's current members are pre-inserted, so
        // candidates that could only be rejected (self, already a member, or a
        // repeat from another list) skip the row gather and the distance.
        uint32_t* seen = seen_s[warp];
        for (int t = lane; t < kSeenSlots; t += kWarp) seen[t] = kNone;
        __syncwarp();
        if (lane == 0) seen_insert(seen, p);
#pragma unroll
        for (int r = 0; r < kSlotsPerLane; ++r)
            if (lane + r * kWarp < static_cast<int>(s.size)) seen_insert(seen, s.id[r]);
        __syncwarp();
        const float bound0 = s.bound;
        uint32_t S = 0;
        uint32_t prev_q = kNone;
        const uint32_t* mine = snap + static_cast<size_t>(p) * K;
        for (int a = 0; a < K; ++a) {
            const uint32_t q = mine[a];
            if (q == prev_q) continue;  // the list is sorted: repeats are adjacent
            prev_q = q;
            const uint32_t* theirs = snap + static_cast<size_t>(q) * K;
            for (int b0 = 0; b0 < K; b0 += kWarp) {
                const int bb = b0 + lane;
                const uint32_t c = bb < K ? theirs[bb] : p;
                const bool valid = c != p && seen_insert(seen, c);
                float d = 0.0f;
                if (valid)
                    d = canonical_distance4<D>(reinterpret_cast<const float4*>(pts + static_cast<size_t>(c) * ld),
                                               rowp_s[warp]);
                const bool pass = valid && d < bound0;
                const unsigned m = __ballot_sync(kFull, pass);
                if (pass) gbuf[S + __popc(m & lt_mask)] = (static_cast<unsigned long long>(c) << 32) | __float_as_uint(d);
                S += __popc(m);
            }
        }
        __syncwarp();
        // Sort the survivors by (id, dist); equal ids carry equal distances.
        const uint32_t P2 = pow2_at_least(S);
        unsigned long long* buf = gbuf;
        if (P2 <= kSurvCap) {
            buf = surv_s[warp];
            for (uint32_t t = lane; t < P2; t += kWarp) buf[t] = t < S ? gbuf[t] : ~0ull;
        } else {
            for (uint32_t t = S + lane; t < P2; t += kWarp) buf[t] = ~0ull;
        }
        __syncwarp();
        if (S > 1) warp_bitonic_sort(buf, P2, lane);
        uint32_t changed = 0;
        for (uint32_t t0 = 0; t0 < S; t0 += kWarp) {
            const uint32_t t = t0 + lane;
            const unsigned long long key = t < S ? buf[t] : ~0ull;
            const unsigned long long prev = (t > 0 && t < S) ? buf[t - 1] : ~0ull;
            const uint32_t cid = static_cast<uint32_t>(key >> 32);
            const float d = __uint_as_float(static_cast<uint32_t>(key & 0xFFFFFFFFu));
            const bool valid = t < S && (t == 0 || static_cast<uint32_t>(prev >> 32) != cid);
            changed += set_offer_batch(s, cid, d, valid, K, lane);
        }
        set_store(s, set_dist, set_id, set_size, set_maxslot, set_bound, p, K, lane);
        if (changed && lane == 0) atomicAdd(changed_count, 1u);
        __syncwarp();
    }
}

// ------------------------------------------------------------ local join
//
// The same pass, reorganised around the shared point q: p's candidates are
// the lists S(q) of every q in S(p), so for each q the block
// R(q) x S(q) (R(q) = the points whose list holds q) carries every candidate
// pair that goes through q.  Each block reads |R(q)| + |S(q)| rows instead of
// one row per (p, candidate), and its dot products run on the tensor cores:
//
//   1. k_rev_count / scan / k_rev_fill   R(q) as a CSR (counting sort; the
//                 points visited in leaf order so that the scattered writes
//                 meet in L2).  After a first pass, an entry whose edge p -> q
//                 was already in p's previous list carries bit 31.
//   2. k_join     two persistent CTAs per SM take the points q in leaf order:
//                 S(q)'s rows bulk-copied into shared memory, the rows of a
//                 128-point chunk of R(q) converted straight from global
//                 memory, both centred on q into FP16 tiles; one tcgen05
//                 128 x N tile gives approximate squared distances with a
//                 proven error bound, so a pair is dropped only when its exact
//                 distance is certainly >= bound(p), or (after a first pass)
//                 when both its edges are old (the previous pass offered it).
//                 Survivors are checked against S(p) (binary search in shared
//                 memory: members are always rejected by the set update), get
//                 the exact FP32 distance in the reference's order from the
//                 chunk's rows staged in the freed tile space, and when it
//                 beats bound(p) are appended to p's survivor slots or the
//                 CTA's pool region.
//   3. k_apply    per p: survivors sorted by id (one warp up to 1,024,
//                 k_apply_big_cta up to 8,192, k_apply_big beyond),
//                 duplicates dropped, replayed through the sequential set
//                 update in ascending id order -- the same offers, in the same
//                 order, as the per-point pass.
//   Points whose records did not fit their CTA's pool region are redone by
//   k_refine.

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanTile = kScanThreads * kScanPer;

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t* __restrict__ in, uint64_t n,
                                                              unsigned long long* __restrict__ tile_sum) {
    __shared__ unsigned long long ws[kScanThreads / kWarp];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanPer;
    unsigned long long s = 0;
#pragma unroll
    for (int u = 0; u < kScanPer; ++u)
        if (base + u < n) s += in[base + u];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (threadIdx.x % kWarp == 0) ws[threadIdx.x / kWarp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kScanThreads / kWarp; ++w) t += ws[w];
        tile_sum[blockIdx.x] = t;
    }
}

// Exclusive scan of the tile sums in place (one CTA).
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(unsigned long long* __restrict__ tile_sum, uint32_t nt) {
    __shared__ unsigned long long part[kScanThreads];
    const uint32_t per = (nt + kScanThreads - 1) / kScanThreads;
    const uint32_t b = threadIdx.x * per, e = min(nt, b + per);
    unsigned long long s = 0;
    for (uint32_t i = b; i < e; ++i) s += tile_sum[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long run = 0;
        for (int t = 0; t < kScanThreads; ++t) {
            const unsigned long long v = part[t];
            part[t] = run;
            run += v;
        }
    }
    __syncthreads();
    unsigned long long run = part[threadIdx.x];
    for (uint32_t i = b; i < e; ++i) {
        const unsigned long long v = tile_sum[i];
        tile_sum[i] = run;
        run += v;
    }
}

// out[i] = sum of in[0..i); out[n] = total.
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const uint32_t* __restrict__ in, uint64_t n,
                                                             const unsigned long long* __restrict__ tile_off,
                                                             unsigned long long* __restrict__ out) {
    __shared__ unsigned long long ws[kScanThreads / kWarp];
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanPer;
    uint32_t v[kScanPer];
    unsigned long long mine = 0;
#pragma unroll
    for (int u = 0; u < kScanPer; ++u) {
        v[u] = base + u < n ? in[base + u] : 0u;
        mine += v[u];
    }
    unsigned long long incl = mine;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == kWarp - 1) ws[warp] = incl;
    __syncthreads();
    unsigned long long wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += ws[w];
    unsigned long long run = tile_off[blockIdx.x] + wbase + incl - mine;
#pragma unroll
    for (int u = 0; u < kScanPer; ++u) {
        if (base + u < n) out[base + u] = run;
        run += v[u];
        if (base + u + 1 == n) out[n] = run;
    }
}

// One warp per point p: every distinct q of S(p) counts / receives p.
__global__ void k_rev_count(const uint32_t* __restrict__ snap, uint32_t n, int K, uint32_t* __restrict__ cnt) {
    const int lane = threadIdx.x % kWarp;
    for (uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp; p < n; p += gridDim.x * blockDim.x / kWarp) {
        const uint32_t* row = snap + static_cast<size_t>(p) * K;
        for (int a = lane; a < K; a += kWarp) {
            const uint32_t q = row[a];
            if (a == 0 || row[a - 1] != q) atomicAdd(&cnt[q], 1u);
        }
    }
}

// Bit 31 of a reverse-list entry: the edge p -> q was already in p's list of
// the previous pass (ids are below 2^31 when the marks are used).
constexpr uint32_t kOldEdge = 0x80000000u;

// Points are visited in `order` when given (the last repetition's leaf
// order): neighbouring points fill the same reverse lists close in time, so
// their 4-byte writes meet in L2 instead of each moving a DRAM sector.
__global__ void k_rev_fill(const uint32_t* __restrict__ snap, uint32_t n, int K,
                           const unsigned long long* __restrict__ off, uint32_t* __restrict__ cursor,
                           uint32_t* __restrict__ rev, const uint32_t* __restrict__ old,
                           const uint32_t* __restrict__ order) {
    const int lane = threadIdx.x % kWarp;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp; w < n; w += gridDim.x * blockDim.x / kWarp) {
        const uint32_t p = order ? order[w] : w;
        const uint32_t* row = snap + static_cast<size_t>(p) * K;
        for (int a = lane; a < K; a += kWarp) {
            const uint32_t q = row[a];
            if (a == 0 || row[a - 1] != q) {
                const bool was = old && ((old[static_cast<size_t>(p) * kOldWords + a / kWarp] >> (a % kWarp)) & 1u);
                rev[off[q] + atomicAdd(&cursor[q], 1u)] = p | (was ? kOldEdge : 0u);
            }
        }
    }
}

constexpr int kJoinThreads = 256;
constexpr int kJoinWarps = kJoinThreads / kWarp;  // 8
constexpr int kJoinPerSm = 2;                     // CTAs per SM: one's waits overlap the other's work
constexpr int kTile = 128;                        // MMA M: rows of R(q) per chunk
constexpr int kGroupCols = 64;                    // columns one thread filters (2 groups of 64)

// FP16 operand tiles, chunk-major: K padded to the MMA step of 16, a row held
// as KP / 8 chunks of 16 bytes (8 halves).
template <int D>
struct JoinLayout {
    static constexpr int KP = (D + 15) / 16 * 16;
    static constexpr int CH = KP / 8;
};

// Columns of the B tile: S(q) has at most k distinct ids; the MMA takes N in
// steps of 16.
__host__ __device__ constexpr uint32_t join_cols(uint32_t K) { return K <= 16 ? 16u : (K + 15) / 16 * 16; }

// Row stride (in ids) of the staged sorted lists: k when k is a multiple of 4
// (each list one 16-byte aligned bulk copy), else odd (searches by different
// rows spread over the banks).
__host__ __device__ constexpr uint32_t list_stride(uint32_t K) { return (K & 3u) == 0 ? K : (K | 1u); }

// Dynamic shared memory of k_join (byte offsets).  rows_b: the original FP32
// rows of S(q), row-major, bulk-copied once per q; they feed the centred B'
// tile and the column side of the exact distances.  tiles: one region used
// three times per chunk: the A' and B' operand tiles (A' converted straight
// from the rows of R(q) in global memory), once the MMA has read them the
// lists S(p) of the chunk's rows, and once the member searches are done the
// chunk's original rows (the row side of the exact distances).  Keeping only
// S(q)'s rows resident lets two CTAs share an SM.  x: per-thread pair masks,
// member masks, prefix sums.
struct JoinSmem {
    uint32_t rows_b, tiles, tile_b, norm_a, norm_b, rt_a, rt_b, bnd, pid, cid, fullrow, centre, x, bytes;
};

__host__ __device__ inline JoinSmem join_smem(int D, uint32_t K) {
    const uint32_t KP = (static_cast<uint32_t>(D) + 15) / 16 * 16;
    const uint32_t NB = join_cols(K);
    const uint32_t tiles_bytes = (kTile + NB) * KP * 2;
    const uint32_t lists_bytes = kTile * list_stride(K) * 4;
    JoinSmem s{};
    s.rows_b = 0;
    s.tiles = (s.rows_b + NB * static_cast<uint32_t>(D) * 4 + 127) / 128 * 128;
    s.tile_b = s.tiles + kTile * KP * 2;
    const uint32_t rows_bytes = kTile * static_cast<uint32_t>(D) * 4;
    uint32_t region = tiles_bytes > lists_bytes ? tiles_bytes : lists_bytes;
    region = region > rows_bytes ? region : rows_bytes;
    s.norm_a = s.tiles + (region + 15) / 16 * 16;
    s.norm_b = s.norm_a + kTile * 4;
    s.rt_a = s.norm_b + kTile * 4;
    s.rt_b = s.rt_a + kTile * 4;
    s.bnd = s.rt_b + kTile * 4;
    s.pid = s.bnd + kTile * 4;
    s.cid = s.pid + kTile * 4;
    s.fullrow = s.cid + kTile * 4;
    s.centre = s.fullrow + kTile * 4;
    s.x = s.centre + (static_cast<uint32_t>(D) + 3) / 4 * 16;
    // pair masks and member masks (u64 per thread each), prefix sums
    // (kJoinThreads + 1), warp totals
    s.bytes = s.x + 2 * kJoinThreads * 8 + (kJoinThreads + 1) * 4 + kJoinWarps * 4;
    return s;
}

// Block-wide exclusive prefix sums of the set bits of every thread's pair
// mask: call scan_masks_warp, __syncthreads, scan_masks_block,
// __syncthreads; then pref[t] is the first pair index of thread t and
// pref[kJoinThreads] the number of pairs.
__device__ __forceinline__ uint32_t scan_masks_warp(unsigned long long mask, uint32_t* __restrict__ wsum) {
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    uint32_t x = static_cast<uint32_t>(__popcll(mask));
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == kWarp - 1) wsum[warp] = x;
    return x;  // inclusive, within the warp
}

__device__ __forceinline__ void scan_masks_block(unsigned long long mask, uint32_t incl, const uint32_t* __restrict__ wsum,
                                                 uint32_t* __restrict__ pref) {
    const int warp = threadIdx.x / kWarp;
    uint32_t before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kJoinWarps; ++w) {
        const uint32_t s = wsum[w];
        before += w < warp ? s : 0u;
        total += s;
    }
    pref[threadIdx.x] = before + incl - static_cast<uint32_t>(__popcll(mask));
    if (threadIdx.x == 0) pref[kJoinThreads] = total;
}

// This thread's share [lo, hi) of the block's pairs (an even split), and the
// position of pair lo: owner thread o and the owner's mask with the pairs
// before lo cleared.
struct PairCursor {
    uint32_t lo, hi;
    int o;
    unsigned long long bits;
};

__device__ __forceinline__ PairCursor pair_share(const uint32_t* __restrict__ pref,
                                                 const unsigned long long* __restrict__ masks) {
    PairCursor c;
    const uint32_t T = pref[kJoinThreads];
    c.lo = static_cast<uint32_t>((static_cast<unsigned long long>(threadIdx.x) * T) / kJoinThreads);
    c.hi = static_cast<uint32_t>((static_cast<unsigned long long>(threadIdx.x + 1) * T) / kJoinThreads);
    c.o = 0;
    c.bits = 0;
    if (c.lo < c.hi) {
        // Owner: the last thread o with pref[o] <= lo (it has pairs left).
        int a = 0, b = kJoinThreads - 1;
        while (a < b) {
            const int mid = (a + b + 1) >> 1;
            if (pref[mid] <= c.lo) a = mid; else b = mid - 1;
        }
        c.o = a;
        c.bits = masks[a];
        for (uint32_t r = c.lo - pref[a]; r > 0; --r) c.bits &= c.bits - 1;
    }
    return c;
}

// Next pair of the cursor (call while lo < hi): owner thread and column bit.
__device__ __forceinline__ void pair_next(PairCursor& c, const unsigned long long* __restrict__ masks, int& owner,
                                          int& bit) {
    while (c.bits == 0) c.bits = masks[++c.o];
    owner = c.o;
    bit = __ffsll(c.bits) - 1;
    c.bits &= c.bits - 1;
    ++c.lo;
}

// Tile row and column of bit `bit` of thread o's mask: thread o reads TMEM
// lane (o / 32 % 4) * 32 + o % 32 (its warp's lane quarter) and filters
// columns (o / 32 / 4) * 32 + bit.
__device__ __forceinline__ int pair_row(int o) { return ((o / kWarp) % 4) * kWarp + (o % kWarp); }
__device__ __forceinline__ int pair_col(int o, int bit) { return ((o / kWarp) / 4) * kGroupCols + bit; }

// Centred FP16 operand rows.  Two threads per row (t = 2r + h; half h
// converts chunks [h*HALF, (h+1)*HALF)): row r (r < count, else zeros) minus
// `centre`, rounded to FP16, into a chunk-major tile of `R` rows (chunk c of
// row r at c*R*16 + r*16).  The FP32 source row r is rows + r * stride, or
// with kGather rows + ids[r] * stride in global memory (read through the
// read-only path, every load of the thread in flight at once).  Writes the
// row's squared norm (FP32, of the centred FP32 values; both halves summed in
// a fixed order) and its absolute error term 2^-19 |x'| (+inf when a value
// does not fit FP16's range, so that the filter keeps every pair of the row).
// All 32 lanes of a warp call it; t below 2R do work.
template <int D, bool kGather>
__device__ __forceinline__ void convert_rows(const float* __restrict__ rows, const uint32_t* __restrict__ ids,
                                             size_t stride, uint32_t count, uint32_t R,
                                             unsigned char* __restrict__ tile, const float* __restrict__ centre,
                                             float* __restrict__ norm, float* __restrict__ rt, int t) {
    constexpr int CH = JoinLayout<D>::CH;
    constexpr int HALF = (CH + 1) / 2;
    const uint32_t r = static_cast<uint32_t>(t) >> 1;
    const int h = t & 1;
    float s = 0.0f, mx = 0.0f;
    if (r < R) {
        const bool live = r < count;
        const float* row = rows + (live ? (kGather ? static_cast<size_t>(ids[r]) : r) * stride : 0);
        float4 a[2 * HALF];
#pragma unroll
        for (int i = 0; i < 2 * HALF; ++i) {
            const int k = 8 * (h * HALF + i / 2) + 4 * (i % 2);
            a[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (live && h * HALF + i / 2 < CH && k < D)
                a[i] = kGather ? __ldg(reinterpret_cast<const float4*>(row + k))
                               : *reinterpret_cast<const float4*>(row + k);
        }
#pragma unroll
        for (int i = 0; i < HALF; ++i) {
            const int c = h * HALF + i;
            if (c >= CH) break;
            float v[8];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int k = 8 * c + 4 * q;
                float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
                if (live && k < D) {
                    const float4 m = *reinterpret_cast<const float4*>(centre + k);
                    const float4 v4 = a[2 * i + q];
                    x = make_float4(__fsub_rn(v4.x, m.x), __fsub_rn(v4.y, m.y), __fsub_rn(v4.z, m.z),
                                    __fsub_rn(v4.w, m.w));
                }
                v[4 * q + 0] = x.x;
                v[4 * q + 1] = x.y;
                v[4 * q + 2] = x.z;
                v[4 * q + 3] = x.w;
            }
            uint4 packed;
            uint32_t* pk = reinterpret_cast<uint32_t*>(&packed);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const __half2 hv = __floats2half2_rn(v[2 * e], v[2 * e + 1]);
                pk[e] = *reinterpret_cast<const uint32_t*>(&hv);
            }
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                s = fmaf(v[e], v[e], s);
                mx = fmaxf(mx, fabsf(v[e]));
            }
            *reinterpret_cast<uint4*>(tile + static_cast<size_t>(c) * R * 16 + static_cast<size_t>(r) * 16) = packed;
        }
    }
    const float so = __shfl_xor_sync(kFull, s, 1);
    const float mo = __shfl_xor_sync(kFull, mx, 1);
    if (r < R && h == 0) {
        const float nrm = s + so;
        norm[r] = nrm;
        rt[r] = fmaxf(mx, mo) >= 32768.0f ? __int_as_float(0x7f800000) : 1.9073486328125e-06f * sqrtf(nrm);
    }
}

// Phase clocks of k_join (built with -DKNNG_JOIN_PHASES only): thread 0 of
// each CTA adds the clock64 time between consecutive marks to phase slot i;
// the sums land in counters[8 + i].
#ifdef KNNG_JOIN_PHASES
constexpr int kJoinPhases = 12;
#define JOIN_MARK(i)                     \
    if (tid == 0) {                      \
        const long long t1_ = clock64(); \
        ph_[i] += t1_ - t0_;             \
        t0_ = t1_;                       \
    }
#else
#define JOIN_MARK(i)
#endif

// The local join of one neighbour-of-neighbour pass.  For every point q (taken
// in `order`, the last repetition's leaf order, through the work counter):
// the rows R(q) (points whose snapshot list holds q), in chunks of 128,
// against the columns S(q) (q's snapshot list, distinct ids).
//
// Per chunk: one warp issues a bulk copy per row (R(q) rows, and S(q) rows
// when q is new) into shared memory; the CTA builds the centred FP16 tiles
// from them; one thread issues the tcgen05.mma (kind::f16, FP32 accumulate)
// into TMEM; while the lists S(p) of the chunk's rows are bulk-copied into the
// tile space, every thread filters 32 accumulator columns of its TMEM lane:
// a pair is kept unless approx - margin >= bound(p), with
//   margin = 2^-8 (|x'|^2 + |y'|^2) + 2^-16 |approx| + 2^-19 (|x'| + |y'|)
// covering FP16 rounding of both operands (2^-11 relative, 2^-25 absolute in
// the subnormal range), FP32 accumulation, the centring rounding and the
// reference's own summation order.  Members of S(p) are then dropped (branch-
// free binary searches, four in lockstep), and the remaining pairs get the
// exact FP32 distance in the reference's order from the staged rows, spread
// evenly over the CTA's threads.  Every point's survivors (distance <
// bound(p)) are counted exactly into surv_count; a point's first `slots` go to
// surv[p * slots + cursor], the rest to this CTA's pool region
// pool[blockIdx.x * pool_cap ...] as (p, candidate, distance bits, 0); when
// the region is full the record is dropped and lost[p] set; the CTA's final
// pool fill is written to pool_fill[blockIdx.x].
template <int D>
__global__ void __launch_bounds__(kJoinThreads, kJoinPerSm)
    k_join(const uint32_t* __restrict__ snap, const unsigned long long* __restrict__ rev_off,
           const uint32_t* __restrict__ rev, const float* __restrict__ pts, int ld, const float* __restrict__ bound,
           const uint32_t* __restrict__ set_size, int K, uint32_t n, uint32_t slots,
           uint32_t* __restrict__ surv_count, unsigned long long* __restrict__ surv, uint4* __restrict__ pool,
           uint32_t pool_cap, uint32_t* __restrict__ pool_fill, uint8_t* __restrict__ lost,
           uint32_t* __restrict__ error_flag, unsigned long long* __restrict__ counters,
           const uint32_t* __restrict__ order, uint32_t* __restrict__ work, const uint32_t* __restrict__ old_marks) {
    using L = JoinLayout<D>;
    extern __shared__ __align__(1024) unsigned char smem[];
    const JoinSmem S = join_smem(D, static_cast<uint32_t>(K));
    const uint32_t NB = join_cols(static_cast<uint32_t>(K));
    float* rows_b = reinterpret_cast<float*>(smem + S.rows_b);
    unsigned char* tile_a = smem + S.tiles;
    unsigned char* tile_b = smem + S.tile_b;
    uint32_t* lists = reinterpret_cast<uint32_t*>(smem + S.tiles);
    float* normA = reinterpret_cast<float*>(smem + S.norm_a);
    float* normB = reinterpret_cast<float*>(smem + S.norm_b);
    float* rtA = reinterpret_cast<float*>(smem + S.rt_a);
    float* rtB = reinterpret_cast<float*>(smem + S.rt_b);
    float* bnd = reinterpret_cast<float*>(smem + S.bnd);
    uint32_t* pid = reinterpret_cast<uint32_t*>(smem + S.pid);
    uint32_t* cid = reinterpret_cast<uint32_t*>(smem + S.cid);
    uint32_t* fullrow = reinterpret_cast<uint32_t*>(smem + S.fullrow);
    float* centre = reinterpret_cast<float*>(smem + S.centre);
    unsigned long long* todo_s = reinterpret_cast<unsigned long long*>(smem + S.x);   // [kJoinThreads]
    unsigned long long* mem_s = todo_s + kJoinThreads;                                // [kJoinThreads]
    uint32_t* pref = reinterpret_cast<uint32_t*>(smem + S.x + 2 * kJoinThreads * 8);  // [kJoinThreads + 1]
    uint32_t* wsum = pref + kJoinThreads + 1;                                          // [kJoinWarps]
    __shared__ uint64_t rows_bar, list_bar, mma_bar, arow_bar;
    __shared__ uint32_t tmem_slot;
    __shared__ uint32_t ncols_s;
    __shared__ uint32_t colold_s[4];  // old columns of the current q (bit per column)
    __shared__ uint32_t pool_cursor;
    __shared__ uint32_t work_s[2];
    const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
    if (warp == 0) tc::tmem_alloc(&tmem_slot, kTile);
    if (tid == 0) {
        pool_cursor = 0;
        tc::mbar_init(&rows_bar, 1);
        tc::mbar_init(&list_bar, 1);
        tc::mbar_init(&mma_bar, 1);
        tc::mbar_init(&arow_bar, 1);
        tc::fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = tc::idesc_f16(kTile, NB);
    const bool bulk_lists = (K & 3) == 0;
    const int KS = static_cast<int>(list_stride(static_cast<uint32_t>(K)));
    constexpr uint32_t kRowBytes = D * sizeof(float);
    uint32_t ph_rows = 0, ph_list = 0, ph_mma = 0, ph_arow = 0;
    float* arows = reinterpret_cast<float*>(smem + S.tiles);  // the chunk's R(q) rows, for the exact phase
    bool healthy = true;
    unsigned long long n_pairs = 0, n_pass = 0, n_member = 0, n_exact = 0, n_emit = 0;
    const int quarter = warp % 4, group = warp / 4;
    const int row = quarter * kWarp + lane;  // TMEM lane / tile row this thread filters
    const unsigned lt = (1u << lane) - 1u;
#ifdef KNNG_JOIN_PHASES
    long long ph_[kJoinPhases] = {};
    long long t0_ = clock64();
#endif
    int search_top = 1;  // largest power of two <= K (branch-free lower bound)
    while (search_top * 2 <= K) search_top *= 2;
    // Waits on this CTA's own copies and MMAs; a wait that gives up marks the
    // launch failed, and waits once more with the full limit (the copies in
    // flight land before the CTA exits).
    // Thread 0 alone polls; the others wait in the barrier, which takes no
    // issue slots from the CTA sharing the SM (the barrier also makes the
    // completed copies visible to them).
    auto wait_or_fail = [&](uint64_t* bar, uint32_t parity) -> bool {
        const bool done = tid == 0 ? tc::mbar_wait_limited(bar, parity) : true;
        if (__syncthreads_or(!done)) {
            if (tid == 0) {
                atomicExch(error_flag, 1u);
                tc::mbar_wait(bar, parity);
            }
            __syncthreads();
            return false;
        }
        return true;
    };
    for (uint32_t it = 0; healthy; ++it) {
        if (tid == 0) work_s[it & 1u] = atomicAdd(work, 1u);
        __syncthreads();
        const uint32_t w = work_s[it & 1u];
        JOIN_MARK(0)
        if (w >= n) break;
        const uint32_t q = order ? order[w] : w;
        const unsigned long long rb = rev_off[q], re = rev_off[q + 1];
        if (rb == re) continue;
        // Columns: the distinct ids of S(q), ascending.
        if (warp == 0) {
            const uint32_t* sq = snap + static_cast<size_t>(q) * K;
            uint32_t v[kSlotsPerLane];
#pragma unroll
            for (int i = 0; i < kSlotsPerLane; ++i) {
                const int a = i * kWarp + lane;
                v[i] = a < K ? __ldg(sq + a) : kNone;
            }
            uint32_t base = 0;
            if (lane < 4) colold_s[lane] = 0u;
            __syncwarp();
#pragma unroll
            for (int i = 0; i < kSlotsPerLane; ++i) {
                const int a = i * kWarp + lane;
                // Previous entry: from the lane below, or lane 31 of the last step.
                uint32_t prev = __shfl_up_sync(kFull, v[i], 1);
                const uint32_t wrap = i > 0 ? __shfl_sync(kFull, v[i > 0 ? i - 1 : 0], kWarp - 1) : kNone;
                if (lane == 0) prev = wrap;
                const bool keep = a < K && (a == 0 || prev != v[i]);
                const unsigned m = __ballot_sync(kFull, keep);
                if (keep) {
                    const uint32_t col = base + __popc(m & lt);
                    cid[col] = v[i];
                    // Column c of q was already in q's list of the previous pass.
                    if (old_marks && ((old_marks[static_cast<size_t>(q) * kOldWords + i] >> lane) & 1u))
                        atomicOr(&colold_s[col / kWarp], 1u << (col % kWarp));
                }
                base += __popc(m);
            }
            if (lane == 0) ncols_s = base;
        }
        for (int j = tid; j < D; j += kJoinThreads) centre[j] = pts[static_cast<size_t>(q) * ld + j];
        __syncthreads();
        JOIN_MARK(1)
        const uint32_t nc = ncols_s;
        for (unsigned long long cb = rb; cb < re && healthy; cb += kTile) {
            const uint32_t m = static_cast<uint32_t>(min(static_cast<unsigned long long>(kTile), re - cb));
            const bool with_b = cb == rb;
            if (tid < kTile) {
                const uint32_t rv = tid < static_cast<int>(m) ? rev[cb + tid] : kNone;
                // With the marks, bit 31 says the edge p -> q is old.
                const uint32_t p = rv == kNone ? kNone : (old_marks ? rv & ~kOldEdge : rv);
                const bool row_old = old_marks && rv != kNone && (rv & kOldEdge);
                pid[tid] = p;
                bnd[tid] = p != kNone ? bound[p] : 0.0f;
                fullrow[tid] = (p != kNone && set_size[p] == static_cast<uint32_t>(K) ? 1u : 0u) | (row_old ? 2u : 0u);
            }
            __syncthreads();
            JOIN_MARK(2)
            // S(q)'s rows for a new q: one bulk copy per row; meanwhile the
            // chunk's rows are converted straight from global memory.
            if (with_b && warp == 0) {
                tc::fence_proxy_async();  // the last q's reads of rows_b come before these writes
                if (lane == 0) tc::mbar_arrive_expect_tx(&rows_bar, nc * kRowBytes);
                __syncwarp();
                for (uint32_t j = lane; j < nc; j += kWarp)
                    tc::bulk_g2s(rows_b + static_cast<size_t>(j) * D, pts + static_cast<size_t>(cid[j]) * ld, kRowBytes,
                                 &rows_bar);
            }
            // Centred FP16 operand tiles, norms and error terms.
            convert_rows<D, true>(pts, pid, static_cast<size_t>(ld), m, kTile, tile_a, centre, normA, rtA, tid);
            if (with_b) {
                if (!wait_or_fail(&rows_bar, ph_rows)) {
                    healthy = false;
                    break;
                }
                ph_rows ^= 1u;
            }
            JOIN_MARK(3)
            convert_rows<D, false>(rows_b, nullptr, static_cast<size_t>(D), nc, NB, tile_b, centre, normB, rtB, tid);
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
            JOIN_MARK(4)
            if (tid == 0) {
                tc::fence_after_sync();
                tc::issue_tile_16bit(tmem, tc::smem_u32(tile_a), tc::smem_u32(tile_b), kTile, NB, L::KP, idesc);
                tc::mma_commit(&mma_bar);
            }
            if (!wait_or_fail(&mma_bar, ph_mma)) {
                healthy = false;
                break;
            }
            ph_mma ^= 1u;
            JOIN_MARK(5)
            tc::fence_after_sync();
            // The tiles are consumed: the chunk's lists S(p) go into their space
            // (one bulk copy per list) while the filter runs.
            if (bulk_lists && warp == 0) {
                if (lane == 0) tc::mbar_arrive_expect_tx(&list_bar, m * static_cast<uint32_t>(K) * 4u);
                __syncwarp();
                for (uint32_t r = lane; r < m; r += kWarp)
                    tc::bulk_g2s(lists + static_cast<size_t>(r) * KS, snap + static_cast<size_t>(pid[r]) * K,
                                 static_cast<uint32_t>(K) * 4u, &list_bar);
            }
            // Filter: bit u of `todo` marks column group*64 + u as a pair that
            // may beat bound(p).
            const uint32_t p = row < static_cast<int>(m) ? pid[row] : kNone;
            const float bp = row < static_cast<int>(m) ? bnd[row] : 0.0f;
            unsigned long long todo = 0;
            {
                const float na = normA[row], ra = rtA[row];
                const int j0 = group * kGroupCols;
                if (j0 < static_cast<int>(nc)) {  // warp-uniform
                    unsigned long long pass = 0;
#pragma unroll
                    for (int hh = 0; hh < kGroupCols / 16; ++hh) {
                        const int jb = j0 + 16 * hh;
                        if (jb >= static_cast<int>(nc)) break;  // warp-uniform
                        float g[16];
                        tc::tmem_ld16(tmem + (static_cast<uint32_t>(quarter * kWarp) << 16) + jb, g);
                        tc::tmem_wait_ld();
#pragma unroll
                        for (int u = 0; u < 16; ++u) {
                            const float nb = normB[jb + u];
                            const float approx = na + nb - 2.0f * g[u];
                            const float margin = 0.00390625f * (na + nb) + 1.52587890625e-5f * fabsf(approx) + ra +
                                                 rtB[jb + u];
                            // NaN-safe: a pair is dropped only when the bound provably holds.
                            if (!(approx - margin >= bp)) pass |= 1ull << (16 * hh + u);
                        }
                    }
                    const int valid_cols = max(0, min(kGroupCols, static_cast<int>(nc) - j0));
                    pass &= valid_cols == kGroupCols ? ~0ull : ((1ull << valid_cols) - 1ull);
                    if (p == kNone) pass = 0;
                    // A pair whose two edges (p -> q and q -> c) were both in the
                    // previous pass's lists was offered then: every offer of it
                    // now is rejected (c is in S(p), or at least as far as a
                    // bound that has only fallen since).
                    if (fullrow[row] & 2u)
                        pass &= ~(static_cast<unsigned long long>(colold_s[2 * group]) |
                                  static_cast<unsigned long long>(colold_s[2 * group + 1]) << 32);
                    if (p != kNone) {
                        n_pairs += valid_cols;
                        n_pass += __popcll(pass);
                    }
                    todo = pass;
                }
            }
            if (!bulk_lists) {
                // Lists whose rows are not 16-byte multiples: plain loads.
                __syncthreads();
                const uint32_t total = m * static_cast<uint32_t>(K);
#pragma unroll 1
                for (uint32_t f0 = tid; f0 < total; f0 += 4 * kJoinThreads) {
                    uint32_t v[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const uint32_t f = f0 + u * kJoinThreads;
                        v[u] = f < total ? __ldg(snap + static_cast<size_t>(pid[f / K]) * K + f % K) : kNone;
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const uint32_t f = f0 + u * kJoinThreads;
                        if (f < total) lists[(f / K) * KS + f % K] = v[u];
                    }
                }
            }
            // Filter-passing pairs of the chunk, then the members of S(p)
            // among them (rejected by the set update: dropped), an even share
            // of the pairs per thread, lower bounds of four at a time
            // (branch-free, in lockstep).  A set that is not full lists its
            // empty slots as its point set's first id (0 for a single set),
            // which is then its list's first entry and not taken for a member.
            JOIN_MARK(6)
            todo_s[tid] = todo;
            mem_s[tid] = 0ull;
            uint32_t incl = scan_masks_warp(todo, wsum);
            __syncthreads();
            JOIN_MARK(7)
            scan_masks_block(todo, incl, wsum, pref);
            if (bulk_lists && !wait_or_fail(&list_bar, ph_list)) {
                healthy = false;
                break;
            }
            if (bulk_lists) ph_list ^= 1u;
            __syncthreads();
            JOIN_MARK(8)
            {
                PairCursor cur = pair_share(pref, todo_s);
#pragma unroll 1
                while (cur.lo < cur.hi) {
                    int own[4], bit[4], pos[4];
                    uint32_t key[4];
                    const uint32_t* lst[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        own[u] = -1;
                        bit[u] = 0;
                        key[u] = 0;
                        pos[u] = 0;
                        lst[u] = lists;
                        if (cur.lo < cur.hi) {
                            pair_next(cur, todo_s, own[u], bit[u]);
                            key[u] = cid[pair_col(own[u], bit[u])];
                            lst[u] = lists + pair_row(own[u]) * KS;
                        }
                    }
                    for (int step = search_top; step > 0; step >>= 1) {
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int t = pos[u] + step;
                            if (t <= K && lst[u][t - 1] < key[u]) pos[u] = t;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        if (own[u] >= 0 && pos[u] < K && lst[u][pos[u]] == key[u] &&
                            (key[u] != lst[u][0] || (fullrow[pair_row(own[u])] & 1u) != 0u)) {
                            atomicOr(&mem_s[own[u]], 1ull << bit[u]);
                            ++n_member;
                        }
                    }
                }
            }
            __syncthreads();
            JOIN_MARK(9)
            // The lists are consumed: the chunk's original rows go into their
            // space (one bulk copy per row; recently read, mostly from L2).
            if (warp == 0) {
                tc::fence_proxy_async();  // the searches' reads of the lists come before these writes
                if (lane == 0) tc::mbar_arrive_expect_tx(&arow_bar, m * kRowBytes);
                __syncwarp();
                for (uint32_t r = lane; r < m; r += kWarp)
                    tc::bulk_g2s(arows + static_cast<size_t>(r) * D, pts + static_cast<size_t>(pid[r]) * ld, kRowBytes,
                                 &arow_bar);
            }
            // The remaining pairs, an even share per thread: exact distances
            // from the staged original rows.
            todo &= ~mem_s[tid];
            incl = scan_masks_warp(todo, wsum);
            todo_s[tid] = todo;
            __syncthreads();
            scan_masks_block(todo, incl, wsum, pref);
            __syncthreads();
            if (!wait_or_fail(&arow_bar, ph_arow)) {
                healthy = false;
                break;
            }
            ph_arow ^= 1u;
            JOIN_MARK(10)
            {
                // A survivor's slot comes from an atomic on its point's count,
                // whose result the record's store needs: the atomic of the
                // previous survivor is issued before the next distance, so
                // its round trip overlaps that arithmetic.
                bool held = false;
                uint32_t h_p = 0, h_c = 0;
                float h_d = 0.0f;
                auto store = [&](uint32_t slot) {
                    if (slot < slots) {
                        surv[static_cast<size_t>(h_p) * slots + slot] =
                            (static_cast<unsigned long long>(h_c) << 32) | __float_as_uint(h_d);
                    } else {
                        const uint32_t e = atomicAdd(&pool_cursor, 1u);
                        if (e < pool_cap)
                            pool[static_cast<size_t>(blockIdx.x) * pool_cap + e] =
                                make_uint4(h_p, h_c, __float_as_uint(h_d), 0u);
                        else
                            lost[h_p] = 1;
                    }
                };
                PairCursor cur = pair_share(pref, todo_s);
#pragma unroll 1
                while (cur.lo < cur.hi) {
                    int o, bit;
                    pair_next(cur, todo_s, o, bit);
                    const int prow = pair_row(o);
                    const int j = pair_col(o, bit);
                    const uint32_t pp = pid[prow];
                    const uint32_t c = cid[j];
                    if (c == pp) continue;
                    ++n_exact;
                    const uint32_t slot = held ? atomicAdd(&surv_count[h_p], 1u) : 0u;
                    const float d = canonical_distance4_lean<D>(reinterpret_cast<const float4*>(rows_b + j * D),
                                                                reinterpret_cast<const float4*>(arows + prow * D));
                    if (held) store(slot);
                    held = d < bnd[prow];
                    if (held) {
                        ++n_emit;
                        h_p = pp;
                        h_c = c;
                        h_d = d;
                    }
                }
                if (held) store(atomicAdd(&surv_count[h_p], 1u));
            }
            // Every thread is done with the rows, lists and TMEM before the
            // next chunk's copies and MMA.
            tc::fence_before_sync();
            __syncthreads();
            JOIN_MARK(11)
            tc::fence_after_sync();
        }
    }
#ifdef KNNG_JOIN_PHASES
    if (tid == 0)
        for (int i = 0; i < kJoinPhases; ++i) atomicAdd(&counters[8 + i], static_cast<unsigned long long>(ph_[i]));
#endif
    atomicAdd(&counters[0], n_pairs);
    atomicAdd(&counters[1], n_pass);
    atomicAdd(&counters[2], n_member);
    atomicAdd(&counters[3], n_exact);
    atomicAdd(&counters[4], n_emit);
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) pool_fill[blockIdx.x] = min(pool_cursor, pool_cap);
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kTile);
    }
}

// Replays one point's survivors (buf[0..S), padded to P2 with ~0 and
// sorted here) through the sequential set update in ascending id order.
// Replays a point's survivors buf[0..S), sorted by candidate id, through the
// sequential set update (a candidate repeated through several shared
// neighbours is offered once); returns 1 if the set changed.  One warp.
__device__ __forceinline__ uint32_t replay_keys(const unsigned long long* buf, uint32_t S, uint32_t p, int K,
                                                float* __restrict__ set_dist, uint32_t* __restrict__ set_id,
                                                uint32_t* __restrict__ set_size, uint32_t* __restrict__ set_maxslot,
                                                float* __restrict__ set_bound, int lane) {
    WarpSet s;
    set_load(s, set_dist, set_id, set_size, set_maxslot, set_bound, p, K, lane);
    uint32_t changed = 0;
    for (uint32_t t0 = 0; t0 < S; t0 += kWarp) {
        const uint32_t t = t0 + lane;
        const unsigned long long key = t < S ? buf[t] : ~0ull;
        const unsigned long long prev = (t > 0 && t < S) ? buf[t - 1] : ~0ull;
        const uint32_t cid = static_cast<uint32_t>(key >> 32);
        const float d = __uint_as_float(static_cast<uint32_t>(key & 0xFFFFFFFFu));
        const bool valid = t < S && (t == 0 || static_cast<uint32_t>(prev >> 32) != cid);
        changed += set_offer_batch(s, cid, d, valid, K, lane);
    }
    set_store(s, set_dist, set_id, set_size, set_maxslot, set_bound, p, K, lane);
    return changed;
}

__device__ __forceinline__ uint32_t replay_sorted(unsigned long long* buf, uint32_t S, uint32_t P2, uint32_t p, int K,
                                                  float* __restrict__ set_dist, uint32_t* __restrict__ set_id,
                                                  uint32_t* __restrict__ set_size, uint32_t* __restrict__ set_maxslot,
                                                  float* __restrict__ set_bound, int lane) {
    __syncwarp();
    warp_bitonic_sort(buf, P2, lane);
    const uint32_t changed = replay_keys(buf, S, p, K, set_dist, set_id, set_size, set_maxslot, set_bound, lane);
    __syncwarp();
    return changed;
}

constexpr int kApplyCap = 1024;  // survivors sorted in shared memory per warp

// Loads point p's S survivors into buf[0 .. P2): the first min(S, slots)
// from its slots, the rest from its list ovf[ovf_off[p] ...]; padding ~0.
__device__ __forceinline__ void gather_survivors(unsigned long long* buf, uint32_t S, uint32_t P2, uint32_t p,
                                                 uint32_t slots, const unsigned long long* __restrict__ surv,
                                                 const unsigned long long* __restrict__ ovf_off,
                                                 const unsigned long long* __restrict__ ovf, int lane) {
    const unsigned long long* direct = surv + static_cast<size_t>(p) * slots;
    const unsigned long long* rest = S > slots ? ovf + ovf_off[p] : nullptr;
    for (uint32_t t = lane; t < P2; t += kWarp)
        buf[t] = t < S ? (t < slots ? direct[t] : rest[t - slots]) : ~0ull;
}

// Every point with survivors and no lost record: gathered, sorted in shared
// memory when they fit, replayed; larger lists are queued on `big`.
__global__ void __launch_bounds__(kRefWarps * kWarp)
    k_apply(uint32_t n, int K, const uint32_t* __restrict__ surv_count, uint32_t slots,
            const unsigned long long* __restrict__ surv, const unsigned long long* __restrict__ ovf_off,
            const unsigned long long* __restrict__ ovf, const uint8_t* __restrict__ lost,
            float* __restrict__ set_dist, uint32_t* __restrict__ set_id, uint32_t* __restrict__ set_size,
            uint32_t* __restrict__ set_maxslot, float* __restrict__ set_bound, uint32_t* __restrict__ big,
            uint32_t* __restrict__ big_n, uint32_t* __restrict__ changed_count) {
    __shared__ unsigned long long keys_s[kRefWarps][kApplyCap];
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    unsigned long long* buf = keys_s[warp];
    for (uint32_t p = blockIdx.x * kRefWarps + warp; p < n; p += gridDim.x * kRefWarps) {
        const uint32_t S = surv_count[p];
        if (S == 0 || lost[p]) continue;
        if (S > kApplyCap) {
            if (lane == 0) big[atomicAdd(big_n, 1u)] = p;
            continue;
        }
        const uint32_t P2 = pow2_at_least(S);
        gather_survivors(buf, S, P2, p, slots, surv, ovf_off, ovf, lane);
        const uint32_t ch = replay_sorted(buf, S, P2, p, K, set_dist, set_id, set_size, set_maxslot, set_bound, lane);
        if (ch && lane == 0) atomicAdd(changed_count, 1u);
    }
}

constexpr int kBigCtaThreads = 256;
constexpr uint32_t kBigSmemKeys = 8192;  // survivor keys one CTA sorts in shared memory (64 KB)

// Queued points with more than kApplyCap survivors and at most kBigSmemKeys:
// one CTA per point gathers the list into shared memory, sorts it with every
// thread (bitonic), and its first warp replays it.  Longer lists are queued
// on `rest` for k_apply_big.
__global__ void __launch_bounds__(kBigCtaThreads)
    k_apply_big_cta(const uint32_t* __restrict__ big, const uint32_t* __restrict__ big_n, int K,
                    const uint32_t* __restrict__ surv_count, uint32_t slots,
                    const unsigned long long* __restrict__ surv, const unsigned long long* __restrict__ ovf_off,
                    const unsigned long long* __restrict__ ovf, float* __restrict__ set_dist,
                    uint32_t* __restrict__ set_id, uint32_t* __restrict__ set_size, uint32_t* __restrict__ set_maxslot,
                    float* __restrict__ set_bound, uint32_t* __restrict__ changed_count, uint32_t* __restrict__ rest,
                    uint32_t* __restrict__ rest_n) {
    extern __shared__ unsigned long long keys[];  // kBigSmemKeys
    const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
    const uint32_t total = *big_n;
    for (uint32_t w = blockIdx.x; w < total; w += gridDim.x) {
        const uint32_t p = big[w];
        const uint32_t S = surv_count[p];
        const uint32_t P2 = pow2_at_least(S);
        if (P2 > kBigSmemKeys) {  // uniform over the CTA
            if (tid == 0) rest[atomicAdd(rest_n, 1u)] = p;
            continue;
        }
        const unsigned long long* direct = surv + static_cast<size_t>(p) * slots;
        const unsigned long long* more = S > slots ? ovf + ovf_off[p] : nullptr;
        for (uint32_t t = tid; t < P2; t += kBigCtaThreads)
            keys[t] = t < S ? (t < slots ? direct[t] : more[t - slots]) : ~0ull;
        __syncthreads();
        for (uint32_t k = 2; k <= P2; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t t = tid; t < P2 / 2; t += kBigCtaThreads) {
                    const uint32_t i = 2 * t - (t & (j - 1));  // 2 j (t / j) + t % j, j a power of two
                    const uint32_t partner = i + j;
                    const bool up = (i & k) == 0;
                    const unsigned long long a = keys[i], b = keys[partner];
                    if ((a > b) == up) {
                        keys[i] = b;
                        keys[partner] = a;
                    }
                }
                __syncthreads();
            }
        }
        if (warp == 0) {
            const uint32_t ch = replay_keys(keys, S, p, K, set_dist, set_id, set_size, set_maxslot, set_bound, lane);
            if (ch && lane == 0) atomicAdd(changed_count, 1u);
        }
        __syncthreads();  // the keys are read before the next point's gather
    }
}

// Queued points with more than kBigSmemKeys survivors: sorted in a per-warp
// global scratch region of `cap` (a power of two >= the largest list) entries.
__global__ void __launch_bounds__(kRefWarps * kWarp)
    k_apply_big(const uint32_t* __restrict__ big, const uint32_t* __restrict__ big_n, int K,
                const uint32_t* __restrict__ surv_count, uint32_t slots, const unsigned long long* __restrict__ surv,
                const unsigned long long* __restrict__ ovf_off, const unsigned long long* __restrict__ ovf,
                unsigned long long* __restrict__ scratch_keys, uint32_t cap, float* __restrict__ set_dist,
                uint32_t* __restrict__ set_id, uint32_t* __restrict__ set_size, uint32_t* __restrict__ set_maxslot,
                float* __restrict__ set_bound, uint32_t* __restrict__ changed_count) {
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    const uint32_t gw = blockIdx.x * kRefWarps + warp;
    unsigned long long* buf = scratch_keys + static_cast<size_t>(gw) * cap;
    const uint32_t total = *big_n;
    for (uint32_t w = gw; w < total; w += gridDim.x * kRefWarps) {
        const uint32_t p = big[w];
        const uint32_t S = surv_count[p];
        const uint32_t P2 = pow2_at_least(S);
        gather_survivors(buf, S, P2, p, slots, surv, ovf_off, ovf, lane);
        const uint32_t ch = replay_sorted(buf, S, P2, p, K, set_dist, set_id, set_size, set_maxslot, set_bound, lane);
        if (ch && lane == 0) atomicAdd(changed_count, 1u);
    }
}

// One 128 x 128 tile of the join's filter: a(m x D) . b(n x D)^T with both
// operands rounded to FP16 and FP32 accumulation (rows past m / n are zero);
// the diagnostic behind knng_debug_tile_gram.
template <int D>
__global__ void __launch_bounds__(kJoinThreads, 1)
    k_tile_gram(const float* __restrict__ a, uint32_t m, const float* __restrict__ b, uint32_t n,
                float* __restrict__ out, uint32_t* __restrict__ error_flag) {
    using L = JoinLayout<D>;
    extern __shared__ __align__(1024) unsigned char smem[];
    const JoinSmem S = join_smem(D, kTile);
    unsigned char* tile_a = smem + S.tiles;
    unsigned char* tile_b = smem + S.tile_b;
    float* norm_a = reinterpret_cast<float*>(smem + S.norm_a);
    float* norm_b = reinterpret_cast<float*>(smem + S.norm_b);
    float* rt_a = reinterpret_cast<float*>(smem + S.rt_a);
    float* rt_b = reinterpret_cast<float*>(smem + S.rt_b);
    float* zero = reinterpret_cast<float*>(smem + S.centre);
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
    for (int j = tid; j < D; j += kJoinThreads) zero[j] = 0.0f;
    if (warp == 0) tc::tmem_alloc(&tmem_slot, kTile);
    if (tid == 0) {
        tc::mbar_init(&mbar, 1);
        tc::fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    __syncthreads();
    convert_rows<D, false>(a, nullptr, static_cast<size_t>(D), m, kTile, tile_a, zero, norm_a, rt_a, tid);
    convert_rows<D, false>(b, nullptr, static_cast<size_t>(D), n, kTile, tile_b, zero, norm_b, rt_b, tid);
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        tc::fence_after_sync();
        tc::issue_tile_16bit(tmem, tc::smem_u32(tile_a), tc::smem_u32(tile_b), kTile, kTile, L::KP,
                             tc::idesc_f16(kTile, kTile));
        tc::mma_commit(&mbar);
    }
    const bool done = tc::mbar_wait(&mbar, 0);
    if (__syncthreads_or(!done)) {
        if (tid == 0) atomicExch(error_flag, 1u);
        tc::mbar_wait(&mbar, 0);
    } else {
        tc::fence_after_sync();
        const int quarter = warp % 4, group = warp / 4, row = quarter * kWarp + lane;
        for (int hh = 0; hh < kGroupCols / 16; ++hh) {
            const int j0 = group * kGroupCols + 16 * hh;
            float g[16];
            tc::tmem_ld16(tmem + (static_cast<uint32_t>(quarter * kWarp) << 16) + j0, g);
            tc::tmem_wait_ld();
#pragma unroll
            for (int u = 0; u < 16; ++u)
                if (static_cast<uint32_t>(row) < m && static_cast<uint32_t>(j0 + u) < n)
                    out[static_cast<size_t>(row) * n + j0 + u] = g[u];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kTile);
    }
}

void device_scan(Context& c, const uint32_t* in, uint64_t n, unsigned long long* out) {
    const uint32_t tiles = static_cast<uint32_t>((n + kScanTile - 1) / kScanTile);
    auto* tsum = static_cast<unsigned long long*>(scratch(c, "scan_tiles", (tiles + 1) * sizeof(unsigned long long)));
    k_scan_reduce<<<tiles, kScanThreads, 0, c.stream>>>(in, n, tsum);
    k_scan_tiles<<<1, kScanThreads, 0, c.stream>>>(tsum, tiles);
    k_scan_apply<<<tiles, kScanThreads, 0, c.stream>>>(in, n, tsum, out);
    c.launches += 3;
    KNNG_CUDA(cudaGetLastError());
}

// ocount[p] = count[p] - slots for points past their slots with no lost
// record, else 0; points with a lost record are listed (in no particular
// order) in lost_list[0 .. *lost_n); *max_count = the largest count among
// the others.
__global__ void k_excess_counts(const uint32_t* __restrict__ count, const uint8_t* __restrict__ lost, uint32_t n,
                                uint32_t slots, uint32_t* __restrict__ ocount, uint32_t* __restrict__ lost_list,
                                uint32_t* __restrict__ lost_n, uint32_t* __restrict__ max_count) {
    uint32_t m = 0;
    const uint32_t lane = threadIdx.x % kWarp;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t p0 = blockIdx.x * blockDim.x; p0 < n; p0 += stride) {
        const uint32_t p = p0 + threadIdx.x;
        const uint32_t v = p < n ? count[p] : 0u;
        const bool is_lost = p < n && lost[p] != 0;
        if (p < n) ocount[p] = !is_lost && v > slots ? v - slots : 0u;
        if (!is_lost) m = max(m, v);
        const unsigned b = __ballot_sync(kFull, is_lost);
        if (b) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(lost_n, static_cast<uint32_t>(__popc(b)));
            base = __shfl_sync(kFull, base, 0);
            if (is_lost) lost_list[base + __popc(b & ((1u << lane) - 1u))] = p;
        }
    }
    for (int o = kWarp / 2; o > 0; o /= 2) m = max(m, __shfl_xor_sync(kFull, m, o));
    if (lane == 0 && m) atomicMax(max_count, m);
}

// Counting-sort scatter of the pool regions into per-point lists:
// ovf[ovf_off[p] + cursor] = (candidate << 32) | distance bits, for records
// of points without a lost record. One block per region.
__global__ void __launch_bounds__(256) k_pool_scatter(const uint4* __restrict__ pool, uint32_t pool_cap,
                                                      const uint32_t* __restrict__ pool_fill,
                                                      const uint8_t* __restrict__ lost,
                                                      const unsigned long long* __restrict__ ovf_off,
                                                      uint32_t* __restrict__ ovf_fill,
                                                      unsigned long long* __restrict__ ovf) {
    const uint32_t fill = pool_fill[blockIdx.x];
    const uint4* region = pool + static_cast<size_t>(blockIdx.x) * pool_cap;
    for (uint32_t i = threadIdx.x; i < fill; i += blockDim.x) {
        const uint4 r = region[i];
        if (lost[r.x]) continue;
        const uint32_t at = atomicAdd(&ovf_fill[r.x], 1u);
        ovf[ovf_off[r.x] + at] = (static_cast<unsigned long long>(r.y) << 32) | r.z;
    }
}

}  // namespace

void set_refine_wait_limit(uint32_t polls) { KNNG_CUDA(cudaMemcpyToSymbol(tc::g_wait_limit, &polls, sizeof(polls))); }

void run_tile_gram(Context& c, uint32_t d, const float* d_a, uint32_t m, const float* d_b, uint32_t n, float* d_out) {
    auto* err = static_cast<uint32_t*>(scratch(c, "gram_error", sizeof(uint32_t)));
    KNNG_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), c.stream));
    KNNG_DISPATCH_D(d, {
        const size_t smem = join_smem(D, kTile).bytes;
        auto kern = k_tile_gram<D>;
        allow_max_smem(c, kern);
        kern<<<1, kJoinThreads, smem, c.stream>>>(d_a, m, d_b, n, d_out, err);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    uint32_t h = 0;
    download(c, &h, err, 1);
    if (h) fail(KNNG_ERR_CUDA, "tensor-core tile: the MMA completion wait gave up");
}

uint64_t run_refine_pointwise(Context& c, const uint32_t* snap, const uint32_t* d_list, uint32_t count) {
    const int K = static_cast<int>(c.k);
    const uint32_t cap = pow2_at_least(static_cast<uint32_t>(K * K));
    uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((count + kRefWarps - 1) / kRefWarps, 148 * 5));
    // Each block's warps need cap survivor keys; fewer blocks (a longer grid
    // stride) when the budget leaves less room.
    const uint64_t per_block = static_cast<uint64_t>(kRefWarps) * cap * sizeof(unsigned long long);
    const uint64_t held_other = c.held - scratch_bytes(c, "refine_keys");
    const uint64_t room = c.budget > held_other + (16ull << 20) ? c.budget - held_other - (16ull << 20) : 0;
    blocks = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(blocks, room / per_block)));
    auto* keys = static_cast<unsigned long long*>(
        scratch(c, "refine_keys", static_cast<size_t>(blocks) * kRefWarps * cap * sizeof(unsigned long long)));
    auto* changed = static_cast<uint32_t*>(scratch(c, "refine_changed", sizeof(uint32_t)));
    KNNG_CUDA(cudaMemsetAsync(changed, 0, sizeof(uint32_t), c.stream));
    KNNG_DISPATCH_D(c.d, {
        k_refine<D><<<blocks, kRefWarps * kWarp, 0, c.stream>>>(snap, c.points, c.ld, c.set_dist, c.set_id,
                                                               c.set_size, c.set_maxslot, c.set_bound, K, count,
                                                               d_list, keys, cap, changed);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    uint32_t h = 0;
    download(c, &h, changed, 1);
    return h;
}

uint64_t run_refine(Context& c) {
    if (c.n == 0) return 0;
    const int K = static_cast<int>(c.k);
    const uint32_t n = c.n;
    uint32_t* snap = static_cast<uint32_t*>(scratch(c, "refine_snap", static_cast<size_t>(n) * K * sizeof(uint32_t)));
    // The join skips pairs the previous join pass offered (both edges in that
    // pass's lists): with the previous lists kept, the snapshot marks each
    // entry that was already there.  Ids must fit 31 bits (the marks ride in
    // bit 31 of the reverse lists).
    const size_t old_bytes = static_cast<size_t>(n) * kOldWords * 4;
    const bool marks = c.refine_mode == 0 && c.refine_skip_old && c.snap_prev_valid && n < (1u << 31) &&
                       (scratch_bytes(c, "refine_old") >= old_bytes || c.held + old_bytes <= c.budget);
    uint32_t* prev = marks ? static_cast<uint32_t*>(scratch(c, "refine_snap_prev", static_cast<size_t>(n) * K * 4))
                           : nullptr;
    uint32_t* old = marks ? static_cast<uint32_t*>(scratch(c, "refine_old", static_cast<size_t>(n) * kOldWords * 4))
                          : nullptr;
    c.snap_prev_valid = false;  // valid again once this pass completes
    const uint32_t sblocks = std::min<uint32_t>((n + kSnapWarps - 1) / kSnapWarps, 148 * 8);
    k_snapshot<<<sblocks, kSnapWarps * kWarp, 0, c.stream>>>(c.set_id, n, K, snap, prev, old);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    if (c.refine_mode == 1) return run_refine_pointwise(c, snap, nullptr, n);

    Context::RefineRecord rec;
    cudaEvent_t ev[4];
    for (auto& e : ev) KNNG_CUDA(cudaEventCreate(&e));
    KNNG_CUDA(cudaEventRecord(ev[0], c.stream));
    // Reverse lists.
    auto* cnt = static_cast<uint32_t*>(scratch(c, "rev_count", (static_cast<size_t>(n) + 1) * sizeof(uint32_t)));
    auto* cur = static_cast<uint32_t*>(scratch(c, "rev_cursor", (static_cast<size_t>(n) + 1) * sizeof(uint32_t)));
    auto* off = static_cast<unsigned long long*>(
        scratch(c, "rev_offsets", (static_cast<size_t>(n) + 1) * sizeof(unsigned long long)));
    auto* rev = static_cast<uint32_t*>(scratch(c, "rev_ids", static_cast<size_t>(n) * K * sizeof(uint32_t)));
    KNNG_CUDA(cudaMemsetAsync(cnt, 0, static_cast<size_t>(n) * sizeof(uint32_t), c.stream));
    KNNG_CUDA(cudaMemsetAsync(cur, 0, static_cast<size_t>(n) * sizeof(uint32_t), c.stream));
    const uint32_t wblocks = std::min<uint32_t>((n + 7) / 8, 148 * 16);
    k_rev_count<<<wblocks, 256, 0, c.stream>>>(snap, n, K, cnt);
    device_scan(c, cnt, n, off);
    k_rev_fill<<<wblocks, 256, 0, c.stream>>>(snap, n, K, off, cur, rev, old, c.join_order_ids ? nullptr : c.indices);
    c.launches += 2;
    KNNG_CUDA(cudaGetLastError());

    // Join grid: kJoinPerSm persistent CTAs per SM; each owns one pool region.
    const uint32_t join_bytes = join_smem(static_cast<int>(c.d), static_cast<uint32_t>(K)).bytes;
    // CTAs per SM from the SM's shared memory and registers (the kernel's
    // launch bounds ask for two).
    int sms = 0, smem_sm = 0, smem_reserved = 0, regs_sm = 0;
    KNNG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device));
    KNNG_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c.device));
    KNNG_CUDA(cudaDeviceGetAttribute(&smem_reserved, cudaDevAttrReservedSharedMemoryPerBlock, c.device));
    KNNG_CUDA(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, c.device));
    cudaFuncAttributes fa{};
    KNNG_DISPATCH_D(c.d, {
        auto kern = k_join<D>;
        allow_max_smem(c, kern);
        KNNG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       static_cast<int>(cudaSharedmemCarveoutMaxShared)));
        KNNG_CUDA(cudaFuncGetAttributes(&fa, kern));
    });
    const size_t per_cta_smem = join_bytes + fa.sharedSizeBytes + static_cast<size_t>(smem_reserved);
    const int by_smem = static_cast<int>(static_cast<size_t>(smem_sm) / per_cta_smem);
    const int by_regs = fa.numRegs > 0 ? regs_sm / (fa.numRegs * kJoinThreads) : 2;
    const int per_sm = std::min({by_smem, by_regs, kJoinPerSm});
    if (per_sm < 1) fail(KNNG_ERR_UNSUPPORTED, "the join kernel does not fit on an SM");
    const uint32_t kJoinBlocks = static_cast<uint32_t>(sms) * static_cast<uint32_t>(per_sm);
    // Survivor storage: `slots` per point, then per-CTA pool regions for the
    // rest, both sized from the free budget (counting what they already hold).
    const uint64_t held_other = c.held - scratch_bytes(c, "surv_direct") - scratch_bytes(c, "surv_pool");
    const uint64_t reserve = std::min<uint64_t>(1ull << 30, c.budget / 8) + static_cast<uint64_t>(n) * 32;
    const uint64_t avail = c.budget > held_other + reserve ? c.budget - held_other - reserve : 0;
    uint32_t slots = 0;
    if (c.refine_slots >= 0) {
        slots = std::min<uint32_t>(static_cast<uint32_t>(c.refine_slots), kApplyCap);
    } else {
        slots = static_cast<uint32_t>(std::min<uint64_t>(kApplyCap, avail * 2 / 5 / (static_cast<uint64_t>(n) * 8)));
        if (slots < 8) slots = 0;
    }
    uint32_t pool_cap = 0;  // records per CTA region
    if (c.refine_pool >= 0) {
        pool_cap = static_cast<uint32_t>(c.refine_pool);
    } else {
        const uint64_t after = avail > static_cast<uint64_t>(n) * slots * 8 ? avail - static_cast<uint64_t>(n) * slots * 8 : 0;
        // Half of what the slots leave: with fewer slots (a smaller budget)
        // more records go to the pool, and a region that fills sends its
        // points to the slow per-point pass.
        pool_cap = static_cast<uint32_t>(std::min<uint64_t>(after / 2 / (kJoinBlocks * 16ull), 1u << 30));
    }
    auto* scount = static_cast<uint32_t*>(scratch(c, "surv_count", static_cast<size_t>(n) * sizeof(uint32_t)));
    auto* ocount = static_cast<uint32_t*>(scratch(c, "surv_excess", static_cast<size_t>(n) * sizeof(uint32_t)));
    auto* ofill = static_cast<uint32_t*>(scratch(c, "surv_excess_fill", static_cast<size_t>(n) * sizeof(uint32_t)));
    auto* lost = static_cast<uint8_t*>(scratch(c, "surv_lost", n));
    auto* lost_list = static_cast<uint32_t*>(scratch(c, "surv_lost_list", static_cast<size_t>(n) * sizeof(uint32_t)));
    auto* soff = static_cast<unsigned long long*>(
        scratch(c, "surv_offsets", (static_cast<size_t>(n) + 1) * sizeof(unsigned long long)));
    auto* pool_fill = static_cast<uint32_t*>(scratch(c, "surv_pool_fill", kJoinBlocks * sizeof(uint32_t)));
    auto* err = static_cast<uint32_t*>(scratch(c, "join_error", sizeof(uint32_t)));
    auto* jc = static_cast<unsigned long long*>(scratch(c, "join_counters", 24 * sizeof(unsigned long long)));
    auto* counters = static_cast<uint32_t*>(scratch(c, "apply_counters", 4 * sizeof(uint32_t)));
    auto* work = static_cast<uint32_t*>(scratch(c, "join_work", sizeof(uint32_t)));
    auto* big = static_cast<uint32_t*>(scratch(c, "apply_big", static_cast<size_t>(n) * sizeof(uint32_t)));
    unsigned long long* direct =
        slots ? static_cast<unsigned long long*>(
                    scratch(c, "surv_direct", static_cast<size_t>(n) * slots * sizeof(unsigned long long)))
              : nullptr;
    uint4* pool = pool_cap ? static_cast<uint4*>(
                                 scratch(c, "surv_pool", static_cast<size_t>(kJoinBlocks) * pool_cap * sizeof(uint4)))
                           : nullptr;
    KNNG_CUDA(cudaMemsetAsync(scount, 0, static_cast<size_t>(n) * sizeof(uint32_t), c.stream));
    KNNG_CUDA(cudaMemsetAsync(ofill, 0, static_cast<size_t>(n) * sizeof(uint32_t), c.stream));
    KNNG_CUDA(cudaMemsetAsync(lost, 0, n, c.stream));
    KNNG_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), c.stream));
    KNNG_CUDA(cudaMemsetAsync(jc, 0, 24 * sizeof(unsigned long long), c.stream));
    KNNG_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(uint32_t), c.stream));
    KNNG_CUDA(cudaMemsetAsync(work, 0, sizeof(uint32_t), c.stream));
    // Points in the leaf order of the last repetition (c.indices), unless the
    // context was created with KNNG_JOIN_ORDER=id.
    const uint32_t* order = c.join_order_ids ? nullptr : c.indices;
    auto elapsed = [](cudaEvent_t a, cudaEvent_t b) {
        float ms = 0.f;
        KNNG_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms;
    };
    KNNG_CUDA(cudaEventRecord(ev[1], c.stream));
    KNNG_DISPATCH_D(c.d, {
        k_join<D><<<kJoinBlocks, kJoinThreads, join_bytes, c.stream>>>(snap, off, rev, c.points, c.ld, c.set_bound, c.set_size, K,
                                                            n, slots, scount, direct, pool, pool_cap, pool_fill, lost,
                                                            err, jc, order, work, old);
    });
    ++c.launches;
    ++rec.join_launches;
    KNNG_CUDA(cudaGetLastError());
    KNNG_CUDA(cudaEventRecord(ev[2], c.stream));
    // Per-point lists of the pooled records, then one replay over every point.
    const uint32_t oblocks = std::max<uint32_t>(1, std::min<uint32_t>((n + 255) / 256, 148 * 8));
    k_excess_counts<<<oblocks, 256, 0, c.stream>>>(scount, lost, n, slots, ocount, lost_list, counters + 3,
                                                   counters + 2);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    device_scan(c, ocount, n, soff);
    unsigned long long total = 0;
    uint32_t hc32[4] = {0, 0, 0, 0};
    download(c, &total, soff + n, 1);
    download(c, hc32, counters, 4);
    uint32_t herr = 0;
    download(c, &herr, err, 1);
    if (herr) {
        for (auto& e : ev) cudaEventDestroy(e);
        fail(KNNG_ERR_CUDA, "tensor-core join: a copy or MMA completion wait gave up");
    }
    const uint32_t max_count = hc32[2], lost_points = hc32[3];
    auto* ovf = static_cast<unsigned long long*>(
        scratch(c, "surv_lists", (std::max<unsigned long long>(total, 1)) * sizeof(unsigned long long)));
    if (total > 0) {
        k_pool_scatter<<<kJoinBlocks, 256, 0, c.stream>>>(pool, pool_cap, pool_fill, lost, soff, ofill, ovf);
        ++c.launches;
        KNNG_CUDA(cudaGetLastError());
    }
    const uint32_t big_cap = pow2_at_least(std::max<uint32_t>(max_count, 2));
    const uint32_t ablocks = std::max<uint32_t>(1, std::min<uint32_t>((n + kRefWarps - 1) / kRefWarps, 148 * 16));
    k_apply<<<ablocks, kRefWarps * kWarp, 0, c.stream>>>(n, K, scount, slots, direct, soff, ovf, lost, c.set_dist,
                                                         c.set_id, c.set_size, c.set_maxslot, c.set_bound, big,
                                                         counters, counters + 1);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    uint32_t* rest = nullptr;
    if (max_count > static_cast<uint32_t>(kApplyCap)) {
        // Lists of up to kBigSmemKeys: one CTA each, sorted in shared memory.
        // counters[2] (the largest count, already read) becomes the count of
        // the longer lists queued for the per-warp global sort below.
        rest = static_cast<uint32_t*>(scratch(c, "apply_rest", static_cast<size_t>(n) * sizeof(uint32_t)));
        KNNG_CUDA(cudaMemsetAsync(counters + 2, 0, sizeof(uint32_t), c.stream));
        const size_t big_smem = kBigSmemKeys * sizeof(unsigned long long);
        allow_max_smem(c, k_apply_big_cta);
        k_apply_big_cta<<<2 * sms, kBigCtaThreads, big_smem, c.stream>>>(
            big, counters, K, scount, slots, direct, soff, ovf, c.set_dist, c.set_id, c.set_size, c.set_maxslot,
            c.set_bound, counters + 1, rest, counters + 2);
        ++c.launches;
        KNNG_CUDA(cudaGetLastError());
    }
    if (max_count > kBigSmemKeys) {
        // Each block's warps sort in big_cap keys of global scratch, which
        // stays within half of L2 (the sorts make many passes over it): one
        // block per SM at most, fewer (a longer grid stride) for large lists
        // or when the budget leaves less room.
        const uint64_t per_block = static_cast<uint64_t>(kRefWarps) * big_cap * sizeof(unsigned long long);
        const uint64_t held_other = c.held - scratch_bytes(c, "apply_big_keys");
        const uint64_t room = c.budget > held_other + (16ull << 20) ? c.budget - held_other - (16ull << 20) : 0;
        const uint64_t l2_half = 60ull << 20;
        const uint32_t big_blocks = static_cast<uint32_t>(std::max<uint64_t>(
            1, std::min<uint64_t>({static_cast<uint64_t>(sms), room / per_block, l2_half / per_block})));
        auto* big_keys = static_cast<unsigned long long*>(
            scratch(c, "apply_big_keys", static_cast<size_t>(big_blocks) * per_block));
        k_apply_big<<<big_blocks, kRefWarps * kWarp, 0, c.stream>>>(rest, counters + 2, K, scount, slots, direct, soff, ovf,
                                                                    big_keys, big_cap, c.set_dist, c.set_id,
                                                                    c.set_size, c.set_maxslot, c.set_bound,
                                                                    counters + 1);
        ++c.launches;
        KNNG_CUDA(cudaGetLastError());
    }
    KNNG_CUDA(cudaEventRecord(ev[3], c.stream));
    // Points with a lost record (their pool region filled up): the
    // one-warp-per-point pass over their list.
    uint64_t changed_lost = 0;
    float ms_lost = 0.f;
    if (lost_points > 0) {
        cudaEvent_t r1, r2;
        KNNG_CUDA(cudaEventCreate(&r1));
        KNNG_CUDA(cudaEventCreate(&r2));
        KNNG_CUDA(cudaEventRecord(r1, c.stream));
        changed_lost = run_refine_pointwise(c, snap, lost_list, lost_points);
        KNNG_CUDA(cudaEventRecord(r2, c.stream));
        KNNG_CUDA(cudaEventSynchronize(r2));
        ms_lost = elapsed(r1, r2);
        cudaEventDestroy(r1);
        cudaEventDestroy(r2);
    }
    uint32_t h[2] = {0, 0};
    unsigned long long hc[24] = {0};
    download(c, h, counters, 2);
    download(c, hc, jc, 24);
#ifdef KNNG_JOIN_PHASES
    {
        static const char* names[] = {"fetch", "columns", "chunk_setup", "rows_wait", "convert", "mma",
                                      "filter",  "scan1",   "lists_wait",  "member",    "scan2",   "exact"};
        double tot = 0;
        for (int i = 0; i < 12; ++i) tot += static_cast<double>(hc[8 + i]);
        fprintf(stderr, "join phases:");
        for (int i = 0; i < 12; ++i) fprintf(stderr, " %s=%.3f", names[i], hc[8 + i] / std::max(tot, 1.0));
        fprintf(stderr, "\n");
    }
#endif
    uint64_t changed = h[1] + changed_lost;
    KNNG_CUDA(cudaEventSynchronize(ev[3]));
    const float ms_all = elapsed(ev[0], ev[3]);
    rec.ms_join = elapsed(ev[1], ev[2]);
    rec.ms_apply = elapsed(ev[2], ev[3]);
    rec.ms_prep = std::max(0.0, ms_all - rec.ms_join - rec.ms_apply);
    rec.ms_fallback = ms_lost;
    for (auto& e : ev) cudaEventDestroy(e);
    rec.pairs = hc[0];
    rec.filter_pass = hc[1];
    rec.member_skip = hc[2];
    rec.exact = hc[3];
    rec.emits = hc[4];
    rec.overflow = total;
    rec.lost = lost_points;
    c.last_refine = rec;
    // This pass offered every pair of its lists: keep them for the next one
    // (when the budget has room for them; else the next pass skips nothing).
    const size_t snap_bytes = static_cast<size_t>(n) * K * 4;
    if (c.refine_skip_old && n < (1u << 31) &&
        (scratch_bytes(c, "refine_snap_prev") >= snap_bytes || c.held + snap_bytes + old_bytes <= c.budget)) {
        uint32_t* keep = static_cast<uint32_t*>(scratch(c, "refine_snap_prev", static_cast<size_t>(n) * K * 4));
        KNNG_CUDA(cudaMemcpyAsync(keep, snap, static_cast<size_t>(n) * K * 4, cudaMemcpyDeviceToDevice, c.stream));
        c.snap_prev_valid = true;
    }
    return changed;
}

}  // namespace knng

// ------------------------------------------------------------------------
// Allocation-free neighbour-of-neighbour pass.
//
// Some callers cannot allocate device memory while they call into this
// library: code that runs inside another framework's memory pool or under a
// strict memory budget, code that only receives device pointers from a host
// application, and code paths where a cudaMalloc would synchronise the device
// at the wrong moment.  knng_refine_pointwise_noalloc serves them: it runs the
// one-warp-per-point pass on buffers the caller passes in, and keeps its only
// scratch -- each warp's survivor records -- in the fixed device array below,
// which every GPU that loads the library holds until the process exits.
//
// The array is cut into one region per warp of pow2(k*k) records (a point has
// at most k*k candidates), so the launch is as wide as the array allows for
// the caller's k: 256 warps at k = 100, 1024 at k <= 64, up to 2,368 (16 per
// SM) at k <= 32.
namespace {

constexpr uint64_t kNoAllocRecords = 1ull << 22;  // 32 MiB of 8-byte survivor records
constexpr uint32_t kNoAllocMaxWarps = 148 * 16;
static __device__ __align__(256) unsigned long long g_noalloc_survivors[kNoAllocRecords];

// The device address of that array differs per CUDA context, and a context
// handle can be reused after its context is destroyed, so the cache is keyed on
// the context's unique id (cuCtxGetId), resolved through the runtime's driver
// entry points (no link-time dependence on the driver library).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

struct NoAllocEntry {
    unsigned long long ctx_id;
    void* addr;
};

std::mutex g_noalloc_mutex;
std::vector<NoAllocEntry> g_noalloc_cache;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

cudaError_t current_context_id(unsigned long long* id) {
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void* f = nullptr;
        void* g = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q1);
        if (e != cudaSuccess) return e;
        e = cudaGetDriverEntryPoint("cuCtxGetId", &g, cudaEnableDefault, &q2);
        if (e != cudaSuccess) return e;
        if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f || !g)
            return cudaErrorNotSupported;
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(g);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return cudaErrorDeviceUninitialized;
    return g_ctx_get_id(ctx, id) == CUDA_SUCCESS ? cudaSuccess : cudaErrorDeviceUninitialized;
}

// Device address of the scratch array in the current context, looked up with
// cudaGetSymbolAddress the first time a context calls (the array's name in host
// code is a host-side stand-in, not a device address).
cudaError_t noalloc_scratch(unsigned long long** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    unsigned long long id = 0;
    cudaError_t e = current_context_id(&id);
    if (e == cudaErrorDeviceUninitialized) {
        // No context is current yet: the lookup below makes the device's
        // primary context current, then its id is taken.
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_survivors);
        if (e != cudaSuccess) return e;
        e = current_context_id(&id);
    }
    if (e != cudaSuccess) return e;
    for (const NoAllocEntry& c : g_noalloc_cache) {
        if (c.ctx_id == id) {
            *out = static_cast<unsigned long long*>(c.addr);
            return cudaSuccess;
        }
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_survivors);
    if (e != cudaSuccess) return e;
    g_noalloc_cache.push_back({id, p});
    *out = static_cast<unsigned long long*>(p);
    return cudaSuccess;
}

}  // namespace

extern "C" knng_status knng_refine_pointwise_noalloc(const float* d_points, uint32_t n, uint32_t d, uint32_t k,
                                                     uint32_t* d_snapshot, float* d_dist, uint32_t* d_ids,
                                                     uint32_t* d_size, uint32_t* d_maxslot, float* d_bound,
                                                     uint32_t* d_changed, void* stream) {
    using namespace knng;
    // A point has at most k*k candidates; the set capacity is at most 128.
    if (k == 0 || k > static_cast<uint32_t>(kMaxK)) return KNNG_ERR_UNSUPPORTED;
    if (!dim_supported(d)) return KNNG_ERR_UNSUPPORTED;
    if (n == 0) return KNNG_OK;
    if (!d_points || !d_snapshot || !d_dist || !d_ids || !d_size || !d_maxslot || !d_bound || !d_changed)
        return KNNG_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(d_points) % 16 != 0) return KNNG_ERR_INVALID_ARGUMENT;
    unsigned long long* scratch_keys = nullptr;
    if (noalloc_scratch(&scratch_keys) != cudaSuccess) {
        cudaGetLastError();
        return KNNG_ERR_CUDA;
    }
    // One region of pow2(k*k) records per warp; whole blocks of kRefWarps.
    const uint32_t region = pow2_at_least(k * k);
    const uint64_t fit = kNoAllocRecords / region;
    const uint32_t warps = static_cast<uint32_t>(std::min<uint64_t>(fit, kNoAllocMaxWarps)) / kRefWarps * kRefWarps;
    const uint32_t need = (n + kRefWarps - 1) / kRefWarps * kRefWarps;
    const uint32_t blocks = std::max<uint32_t>(1, std::min(warps, need) / kRefWarps);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int K = static_cast<int>(k);
    if (cudaMemsetAsync(d_changed, 0, sizeof(uint32_t), s) != cudaSuccess) {
        cudaGetLastError();
        return KNNG_ERR_CUDA;
    }
    const uint32_t sblocks = std::min<uint32_t>((n + kSnapWarps - 1) / kSnapWarps, 148 * 8);
    k_snapshot<<<sblocks, kSnapWarps * kWarp, 0, s>>>(d_ids, n, K, d_snapshot, nullptr, nullptr);
    try {
        KNNG_DISPATCH_D(d, {
            k_refine<D><<<blocks, kRefWarps * kWarp, 0, s>>>(d_snapshot, d_points, static_cast<int>(d), d_dist,
                                                             d_ids, d_size, d_maxslot, d_bound, K, n, nullptr,
                                                             scratch_keys, region, d_changed);
        });
    } catch (const Error& e) {
        return e.status;
    }
    if (cudaGetLastError() != cudaSuccess) return KNNG_ERR_CUDA;
    return KNNG_OK;
}
