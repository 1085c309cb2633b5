// Neighbour-of-neighbour pass: SolutionKmeans::topUpSingle
// (src/SolutionKmeans.hpp:480-555).
//
// Snapshot: every set's k slot ids, sorted ascending, unfilled slots included
// as id 0 -- the reference reads all 100 current_ids (:494).  Then, per point
// p, the candidates are the union of the snapshot lists of p's snapshot list,
// minus p, each offered with the exact distance when dist < bound.
//
// The reference iterates its candidate set in hash order; this pass offers
// them in ascending id order.  The order can only matter between candidates
// that beat the bound p had when its pass started, so each warp evaluates all
// candidates (one lane per candidate, row gathered from HBM/L2), keeps the
// survivors (dist < starting bound), sorts them by id and replays them in that
// order through the sequential set update.  Survivors are staged in a
// per-warp scratch region of k*k entries (rounded up to a power of two) and
// sorted in shared memory when they fit.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "context.hpp"
#include "dispatch.hpp"

namespace knng {
namespace {

constexpr int kRefWarps = 8;
constexpr int kSurvCap = 512;

__host__ __device__ uint32_t pow2_at_least(uint32_t v) {
    uint32_t p = 2;
    while (p < v) p <<= 1;
    return p;
}

__global__ void __launch_bounds__(kRefWarps * kWarp) k_snapshot(const uint32_t* __restrict__ set_id, uint32_t n, int K,
                                                                uint32_t* __restrict__ snap) {
    __shared__ unsigned long long keys_s[kRefWarps][kMaxK];
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    unsigned long long* keys = keys_s[warp];
    for (uint32_t p = blockIdx.x * kRefWarps + warp; p < n; p += gridDim.x * kRefWarps) {
        const size_t base = static_cast<size_t>(p) * K;
        for (int slot = lane; slot < kMaxK; slot += kWarp) keys[slot] = slot < K ? set_id[base + slot] : ~0ull;
        __syncwarp();
        warp_bitonic_sort(keys, kMaxK, lane);
        for (int i = lane; i < K; i += kWarp) snap[base + i] = static_cast<uint32_t>(keys[i]);
        __syncwarp();
    }
}

template <int D>
__global__ void __launch_bounds__(kRefWarps * kWarp)
    k_refine(const uint32_t* __restrict__ snap, const float* __restrict__ pts, int ld, float* __restrict__ set_dist,
             uint32_t* __restrict__ set_id, uint32_t* __restrict__ set_size, uint32_t* __restrict__ set_maxslot,
             float* __restrict__ set_bound, int K, uint32_t n, unsigned long long* __restrict__ scratch_keys,
             uint32_t warp_capacity, uint32_t* __restrict__ changed_count) {
    constexpr int Q = D / 4;
    __shared__ float4 rowp_s[kRefWarps][Q];
    __shared__ unsigned long long surv_s[kRefWarps][kSurvCap];
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    const uint32_t gw = blockIdx.x * kRefWarps + warp;
    const uint32_t nw = gridDim.x * kRefWarps;
    unsigned long long* gbuf = scratch_keys + static_cast<size_t>(gw) * warp_capacity;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (uint32_t p = gw; p < n; p += nw) {
        for (int q = lane; q < Q; q += kWarp)
            rowp_s[warp][q] = __ldg(reinterpret_cast<const float4*>(pts + static_cast<size_t>(p) * ld) + q);
        WarpSet s;
        set_load(s, set_dist, set_id, set_size, set_maxslot, set_bound, p, K, lane);
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
                const bool valid = c != p;
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

}  // namespace

uint64_t run_refine(Context& c) {
    if (c.n == 0) return 0;
    const int K = static_cast<int>(c.k);
    uint32_t* snap = static_cast<uint32_t*>(scratch(c, "refine_snap", static_cast<size_t>(c.n) * K * sizeof(uint32_t)));
    const uint32_t sblocks = std::min<uint32_t>((c.n + kRefWarps - 1) / kRefWarps, 148 * 8);
    k_snapshot<<<sblocks, kRefWarps * kWarp, 0, c.stream>>>(c.set_id, c.n, K, snap);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    const uint32_t cap = pow2_at_least(static_cast<uint32_t>(K * K));
    const uint32_t blocks = std::min<uint32_t>((c.n + kRefWarps - 1) / kRefWarps, 148 * 2);
    auto* keys = static_cast<unsigned long long*>(
        scratch(c, "refine_keys", static_cast<size_t>(blocks) * kRefWarps * cap * sizeof(unsigned long long)));
    auto* changed = static_cast<uint32_t*>(scratch(c, "refine_changed", sizeof(uint32_t)));
    KNNG_CUDA(cudaMemsetAsync(changed, 0, sizeof(uint32_t), c.stream));
    KNNG_DISPATCH_D(c.d, {
        k_refine<D><<<blocks, kRefWarps * kWarp, 0, c.stream>>>(snap, c.points, c.ld, c.set_dist, c.set_id,
                                                               c.set_size, c.set_maxslot, c.set_bound, K, c.n, keys,
                                                               cap, changed);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    uint32_t h = 0;
    download(c, &h, changed, 1);
    return h;
}

}  // namespace knng
