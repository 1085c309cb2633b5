// Device-side building blocks shared by the k-NN graph kernels.
//
//  * canonical_distance / canonical_dot: the reference's FP32 evaluation order
//    (src/LinearAlgebra.hpp:53-77 and :179-200): eight lanes, lane l an FMA
//    chain over dims l, l+8, ... below the largest multiple of 8 <= D, lanes
//    summed left to right into 0.0f, then each tail dim added as a separately
//    rounded product.  Written with __f*_rn intrinsics so nvcc cannot contract
//    or reorder them.
//  * Warp-resident neighbour sets: lane l holds slots l, l+32, l+64, l+96 of a
//    set of capacity K <= 128; warp_argmax reproduces the slot that
//    KnnSetScannableSimd::getMaxIdx (src/KnnSets.hpp:82-111) selects.
//  * mix64 / counter_position: the counter-based RNG of the device-seeded build.
#pragma once

#include <cfloat>
#include <cstdint>

namespace knng {

constexpr int kWarp = 32;
constexpr int kMaxK = 128;
constexpr int kSlotsPerLane = kMaxK / kWarp;
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr unsigned kFull = 0xFFFFFFFFu;

// ---------------------------------------------------------------- arithmetic

template <int D>
__device__ __forceinline__ float canonical_distance(const float* __restrict__ a, const float* __restrict__ b) {
    constexpr int M = D / 8 * 8;
    float lane[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) lane[l] = 0.0f;
#pragma unroll
    for (int base = 0; base < M; base += 8) {
#pragma unroll
        for (int l = 0; l < 8; ++l) {
            float diff = __fsub_rn(a[base + l], b[base + l]);
            lane[l] = __fmaf_rn(diff, diff, lane[l]);
        }
    }
    float acc = 0.0f;
#pragma unroll
    for (int l = 0; l < 8; ++l) acc = __fadd_rn(acc, lane[l]);
#pragma unroll
    for (int i = M; i < D; ++i) {
        float diff = __fsub_rn(a[i], b[i]);
        acc = __fadd_rn(acc, __fmul_rn(diff, diff));
    }
    return acc;
}

template <int D>
__device__ __forceinline__ float canonical_dot(const float* __restrict__ a, const float* __restrict__ b) {
    constexpr int M = D / 8 * 8;
    float lane[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) lane[l] = 0.0f;
#pragma unroll
    for (int base = 0; base < M; base += 8) {
#pragma unroll
        for (int l = 0; l < 8; ++l) lane[l] = __fmaf_rn(b[base + l], a[base + l], lane[l]);
    }
    float acc = 0.0f;
#pragma unroll
    for (int l = 0; l < 8; ++l) acc = __fadd_rn(acc, lane[l]);
#pragma unroll
    for (int i = M; i < D; ++i) acc = __fadd_rn(acc, __fmul_rn(a[i], b[i]));
    return acc;
}

// Same order, operands read as float4 (both rows 16-byte aligned, D % 4 == 0).
template <int D>
__device__ __forceinline__ float canonical_dot4(const float4* __restrict__ a, const float4* __restrict__ b) {
    static_assert(D % 4 == 0, "float4 path needs D % 4 == 0");
    constexpr int M = D / 8 * 8;
    float lane[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) lane[l] = 0.0f;
#pragma unroll
    for (int q = 0; q < M / 4; ++q) {
        float4 x = a[q];
        float4 y = b[q];
        const int l0 = (q & 1) * 4;
        lane[l0 + 0] = __fmaf_rn(y.x, x.x, lane[l0 + 0]);
        lane[l0 + 1] = __fmaf_rn(y.y, x.y, lane[l0 + 1]);
        lane[l0 + 2] = __fmaf_rn(y.z, x.z, lane[l0 + 2]);
        lane[l0 + 3] = __fmaf_rn(y.w, x.w, lane[l0 + 3]);
    }
    float acc = 0.0f;
#pragma unroll
    for (int l = 0; l < 8; ++l) acc = __fadd_rn(acc, lane[l]);
#pragma unroll
    for (int q = M / 4; q < D / 4; ++q) {
        float4 x = a[q];
        float4 y = b[q];
        acc = __fadd_rn(acc, __fmul_rn(x.x, y.x));
        acc = __fadd_rn(acc, __fmul_rn(x.y, y.y));
        acc = __fadd_rn(acc, __fmul_rn(x.z, y.z));
        acc = __fadd_rn(acc, __fmul_rn(x.w, y.w));
    }
    return acc;
}

template <int D>
__device__ __forceinline__ float canonical_distance4(const float4* __restrict__ a, const float4* __restrict__ b) {
    static_assert(D % 4 == 0, "float4 path needs D % 4 == 0");
    constexpr int M = D / 8 * 8;
    float lane[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) lane[l] = 0.0f;
#pragma unroll
    for (int q = 0; q < M / 4; ++q) {
        float4 x = a[q];
        float4 y = b[q];
        const int l0 = (q & 1) * 4;
        float d0 = __fsub_rn(x.x, y.x), d1 = __fsub_rn(x.y, y.y), d2 = __fsub_rn(x.z, y.z), d3 = __fsub_rn(x.w, y.w);
        lane[l0 + 0] = __fmaf_rn(d0, d0, lane[l0 + 0]);
        lane[l0 + 1] = __fmaf_rn(d1, d1, lane[l0 + 1]);
        lane[l0 + 2] = __fmaf_rn(d2, d2, lane[l0 + 2]);
        lane[l0 + 3] = __fmaf_rn(d3, d3, lane[l0 + 3]);
    }
    float acc = 0.0f;
#pragma unroll
    for (int l = 0; l < 8; ++l) acc = __fadd_rn(acc, lane[l]);
#pragma unroll
    for (int q = M / 4; q < D / 4; ++q) {
        float4 x = a[q];
        float4 y = b[q];
        float d0 = __fsub_rn(x.x, y.x), d1 = __fsub_rn(x.y, y.y), d2 = __fsub_rn(x.z, y.z), d3 = __fsub_rn(x.w, y.w);
        acc = __fadd_rn(acc, __fmul_rn(d0, d0));
        acc = __fadd_rn(acc, __fmul_rn(d1, d1));
        acc = __fadd_rn(acc, __fmul_rn(d2, d2));
        acc = __fadd_rn(acc, __fmul_rn(d3, d3));
    }
    return acc;
}

// The same order as canonical_distance4, one 8-dimension step at a time
// (four float4 loads live per step): for callers with little register room.
template <int D>
__device__ __forceinline__ float canonical_distance4_lean(const float4* __restrict__ a, const float4* __restrict__ b) {
    static_assert(D % 4 == 0, "float4 path needs D % 4 == 0");
    constexpr int M = D / 8 * 8;
    float lane[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) lane[l] = 0.0f;
#pragma unroll 1
    for (int q = 0; q < M / 4; q += 2) {
        const float4 x0 = a[q], x1 = a[q + 1];
        const float4 y0 = b[q], y1 = b[q + 1];
        float d;
        d = __fsub_rn(x0.x, y0.x); lane[0] = __fmaf_rn(d, d, lane[0]);
        d = __fsub_rn(x0.y, y0.y); lane[1] = __fmaf_rn(d, d, lane[1]);
        d = __fsub_rn(x0.z, y0.z); lane[2] = __fmaf_rn(d, d, lane[2]);
        d = __fsub_rn(x0.w, y0.w); lane[3] = __fmaf_rn(d, d, lane[3]);
        d = __fsub_rn(x1.x, y1.x); lane[4] = __fmaf_rn(d, d, lane[4]);
        d = __fsub_rn(x1.y, y1.y); lane[5] = __fmaf_rn(d, d, lane[5]);
        d = __fsub_rn(x1.z, y1.z); lane[6] = __fmaf_rn(d, d, lane[6]);
        d = __fsub_rn(x1.w, y1.w); lane[7] = __fmaf_rn(d, d, lane[7]);
    }
    float acc = 0.0f;
#pragma unroll
    for (int l = 0; l < 8; ++l) acc = __fadd_rn(acc, lane[l]);
#pragma unroll
    for (int q = M / 4; q < D / 4; ++q) {
        const float4 x = a[q];
        const float4 y = b[q];
        float d0 = __fsub_rn(x.x, y.x), d1 = __fsub_rn(x.y, y.y), d2 = __fsub_rn(x.z, y.z), d3 = __fsub_rn(x.w, y.w);
        acc = __fadd_rn(acc, __fmul_rn(d0, d0));
        acc = __fadd_rn(acc, __fmul_rn(d1, d1));
        acc = __fadd_rn(acc, __fmul_rn(d2, d2));
        acc = __fadd_rn(acc, __fmul_rn(d3, d3));
    }
    return acc;
}

// ---------------------------------------------------------- neighbour sets
//
// Tie order of getMaxIdx: among slots holding the maximum distance, the one
// with the smallest (slot % 8), then the smallest (slot / 8).

struct WarpSet {
    float dist[kSlotsPerLane];
    uint32_t id[kSlotsPerLane];
    uint32_t size;     // warp-uniform
    uint32_t maxslot;  // warp-uniform
    float bound;       // warp-uniform
};

// Loads point p's set from the slot arrays (row stride K) into the warp.
__device__ __forceinline__ void set_load(WarpSet& s, const float* __restrict__ dist, const uint32_t* __restrict__ ids,
                                         const uint32_t* __restrict__ sizes, const uint32_t* __restrict__ maxslot,
                                         const float* __restrict__ bounds, uint32_t p, int K, int lane) {
    const size_t base = static_cast<size_t>(p) * K;
#pragma unroll
    for (int r = 0; r < kSlotsPerLane; ++r) {
        const int slot = lane + r * kWarp;
        s.dist[r] = slot < K ? dist[base + slot] : 0.0f;
        s.id[r] = slot < K ? ids[base + slot] : 0u;
    }
    s.size = sizes[p];
    s.maxslot = maxslot[p];
    s.bound = bounds[p];
}

__device__ __forceinline__ void set_store(const WarpSet& s, float* __restrict__ dist, uint32_t* __restrict__ ids,
                                          uint32_t* __restrict__ sizes, uint32_t* __restrict__ maxslot,
                                          float* __restrict__ bounds, uint32_t p, int K, int lane) {
    const size_t base = static_cast<size_t>(p) * K;
#pragma unroll
    for (int r = 0; r < kSlotsPerLane; ++r) {
        const int slot = lane + r * kWarp;
        if (slot < K) {
            dist[base + slot] = s.dist[r];
            ids[base + slot] = s.id[r];
        }
    }
    if (lane == 0) {
        sizes[p] = s.size;
        maxslot[p] = s.maxslot;
        bounds[p] = s.bound;
    }
}

// Slot of the maximum distance over K filled slots, in getMaxIdx's tie order;
// sets s.maxslot and s.bound (warp-uniform).  Distances are sums of squares
// (+0 or positive), so their bit patterns order like their values: one warp
// max reduction finds the largest distance, a second one, over the slots
// holding it, the winner of the tie order (smallest slot % 8, then slot / 8,
// encoded so that the preferred slot has the largest key).
__device__ __forceinline__ void warp_argmax(WarpSet& s, int K, int lane) {
    uint32_t vb = 0;
#pragma unroll
    for (int r = 0; r < kSlotsPerLane; ++r) {
        const uint32_t slot = lane + r * kWarp;
        if (slot < static_cast<uint32_t>(K)) vb = max(vb, __float_as_uint(s.dist[r]));
    }
    const uint32_t top = __reduce_max_sync(kFull, vb);
    uint32_t tk = 0;  // 128 - (slot % 8 * 16 + slot / 8) for slots holding `top`, else 0
#pragma unroll
    for (int r = 0; r < kSlotsPerLane; ++r) {
        const uint32_t slot = lane + r * kWarp;
        if (slot < static_cast<uint32_t>(K) && __float_as_uint(s.dist[r]) == top)
            tk = max(tk, 128u - (((slot & 7u) << 4) | (slot >> 3)));
    }
    const uint32_t t = 128u - __reduce_max_sync(kFull, tk);
    s.maxslot = (t & 15u) * 8u + (t >> 4);
    s.bound = __uint_as_float(top);
}

__device__ __forceinline__ bool set_contains(const WarpSet& s, uint32_t cand, int lane) {
    bool hit = false;
#pragma unroll
    for (int r = 0; r < kSlotsPerLane; ++r) {
        const uint32_t slot = lane + r * kWarp;
        hit |= (slot < s.size) && (s.id[r] == cand);
    }
    return __any_sync(kFull, hit);
}

__device__ __forceinline__ void set_write_slot(WarpSet& s, uint32_t slot, uint32_t cand, float d, int lane) {
#pragma unroll
    for (int r = 0; r < kSlotsPerLane; ++r) {
        if (slot == static_cast<uint32_t>(lane + r * kWarp)) {
            s.dist[r] = d;
            s.id[r] = cand;
        }
    }
}

// addCandidateLessThan (src/KnnSets.hpp:39-57) for a warp-uniform offer that
// already passed d < s.bound.  Returns true if the set changed.
__device__ __forceinline__ bool set_offer(WarpSet& s, uint32_t cand, float d, int K, int lane) {
    if (set_contains(s, cand, lane)) return false;
    if (s.size < static_cast<uint32_t>(K)) {
        set_write_slot(s, s.size, cand, d, lane);
        s.size += 1;
        if (s.size == static_cast<uint32_t>(K)) warp_argmax(s, K, lane);
        return true;
    }
    set_write_slot(s, s.maxslot, cand, d, lane);
    warp_argmax(s, K, lane);
    return true;
}

// Offers the warp's 32 candidates (lane j holds (cand_j, d_j), valid_j) in lane
// order, with the sequential semantics of the reference's inner loop.
__device__ __forceinline__ uint32_t set_offer_batch(WarpSet& s, uint32_t cand, float d, bool valid, int K, int lane) {
    uint32_t changed = 0;
    unsigned pending = __ballot_sync(kFull, valid && d < s.bound);
    while (pending) {
        const int src = __ffs(pending) - 1;
        pending &= pending - 1;
        const float dj = __shfl_sync(kFull, d, src);
        const uint32_t cj = __shfl_sync(kFull, cand, src);
        if (dj < s.bound) changed += set_offer(s, cj, dj, K, lane) ? 1u : 0u;
        // The bound only decreases: drop the candidates it now excludes.
        pending &= __ballot_sync(kFull, valid && d < s.bound);
    }
    return changed;
}

// Ascending bitonic sort of n (power of two, n >= 2) unsigned keys by one
// warp; keys may live in shared or global memory.
template <class Key>
__device__ __forceinline__ void warp_bitonic_sort(Key* keys, uint32_t n, int lane) {
    for (uint32_t k = 2; k <= n; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t t = lane; t < n / 2; t += kWarp) {
                const uint32_t i = 2 * t - (t & (j - 1));  // 2 j (t / j) + t % j, j a power of two
                const uint32_t partner = i + j;
                const bool up = (i & k) == 0;
                const Key a = keys[i], b = keys[partner];
                if ((a > b) == up) {
                    keys[i] = b;
                    keys[partner] = a;
                }
            }
            __syncwarp();
        }
    }
}

// --------------------------------------------------------------- randomness

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    // splitmix64 finaliser (Steele, Lea, Flood 2014).
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// Draw t of node [start, end) at the given attempt: a position in [start, end).
__host__ __device__ __forceinline__ uint32_t counter_position(uint64_t seed, uint32_t rep, uint32_t start, uint32_t end,
                                                              uint32_t attempt, uint32_t t) {
    uint64_t h = mix64(seed + 0x9e3779b97f4a7c15ULL * (static_cast<uint64_t>(rep) + 1));
    h = mix64(h ^ ((static_cast<uint64_t>(start) << 32) | end));
    h = mix64(h ^ ((static_cast<uint64_t>(attempt) << 32) | t));
    const uint64_t n = end - start;
    return start + static_cast<uint32_t>(((h >> 32) * n) >> 32);
}

}  // namespace knng
