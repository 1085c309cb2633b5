// Output stage: KnnSetScannableSimd::finalize (src/KnnSets.hpp:113-126) --
// each set sorted by (distance, id) ascending -- and padResult
// (src/KnnSets.hpp:334-344), which pads short rows with id 1.  One warp per
// point sorts its (at most 128) entries as 64-bit keys (distance bits << 32 |
// id; distances are non-negative, so the bit order is the numeric order) with
// a bitonic network in shared memory.  Batched builds (several independent
// point sets in one build) report ids relative to each point's set.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "common.cuh"
#include "context.hpp"

namespace knng {

namespace {

constexpr int kFinWarps = 8;

__global__ void __launch_bounds__(kFinWarps * kWarp) k_finalize(const float* __restrict__ set_dist,
                                                                const uint32_t* __restrict__ set_id,
                                                                const uint32_t* __restrict__ set_size, uint32_t n,
                                                                int K, uint32_t* __restrict__ out_ids,
                                                                float* __restrict__ out_dist) {
    __shared__ unsigned long long keys_s[kFinWarps][kMaxK];
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    unsigned long long* keys = keys_s[warp];
    for (uint32_t p = blockIdx.x * kFinWarps + warp; p < n; p += gridDim.x * kFinWarps) {
        const uint32_t size = set_size[p];
        const size_t base = static_cast<size_t>(p) * K;
        for (int slot = lane; slot < kMaxK; slot += kWarp) {
            unsigned long long key = ~0ull;
            if (slot < K && static_cast<uint32_t>(slot) < size)
                key = (static_cast<unsigned long long>(__float_as_uint(set_dist[base + slot])) << 32) | set_id[base + slot];
            keys[slot] = key;
        }
        __syncwarp();
        warp_bitonic_sort(keys, kMaxK, lane);
        for (int i = lane; i < K; i += kWarp) {
            const bool real = static_cast<uint32_t>(i) < size;
            out_ids[base + i] = real ? static_cast<uint32_t>(keys[i] & 0xFFFFFFFFu) : 1u;
            if (out_dist) out_dist[base + i] = real ? __uint_as_float(static_cast<uint32_t>(keys[i] >> 32)) : INFINITY;
        }
        __syncwarp();
    }
}

__global__ void k_reset_sets(float* __restrict__ bound, uint32_t* __restrict__ maxslot, uint32_t* __restrict__ size,
                             uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        bound[i] = FLT_MAX;
        maxslot[i] = kNone;
        size[i] = 0;
    }
}

// Set of point p: the last s with offsets[s] <= p.
__device__ __forceinline__ uint32_t set_base(const uint32_t* __restrict__ offsets, uint32_t n_sets, uint32_t p) {
    uint32_t a = 0, b = n_sets - 1;
    while (a < b) {
        const uint32_t mid = (a + b + 1) / 2;
        if (offsets[mid] <= p) a = mid; else b = mid - 1;
    }
    return offsets[a];
}

// Batched builds: every slot id of point p starts as its set's first id (the
// id an empty slot holds in a set built alone is 0, that set's first id).
__global__ void k_reset_ids(uint32_t* __restrict__ ids, uint32_t n, int K, const uint32_t* __restrict__ offsets,
                            uint32_t n_sets) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t b = set_base(offsets, n_sets, p);
        for (int j = 0; j < K; ++j) ids[static_cast<size_t>(p) * K + j] = b;
    }
}

// Batched builds: finalized ids relative to each point's set; padding (id 1
// past the set's size) stays as it is.
__global__ void k_rebase_ids(uint32_t* __restrict__ ids, const uint32_t* __restrict__ set_size, uint32_t n, int K,
                             const uint32_t* __restrict__ offsets, uint32_t n_sets) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t b = set_base(offsets, n_sets, p);
        const uint32_t real = min(set_size[p], static_cast<uint32_t>(K));
        for (uint32_t j = 0; j < real; ++j) ids[static_cast<size_t>(p) * K + j] -= b;
    }
}

}  // namespace

void launch_rebase_ids(Context& c, uint32_t* d_ids) {
    if (c.n == 0 || c.set_offsets.size() <= 2) return;
    const uint32_t n_sets = static_cast<uint32_t>(c.set_offsets.size() - 1);
    k_rebase_ids<<<std::min<uint32_t>((c.n + 255) / 256, 148 * 16), 256, 0, c.stream>>>(
        d_ids, c.set_size, c.n, static_cast<int>(c.k), c.d_set_offsets, n_sets);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

void launch_finalize(Context& c, uint32_t* d_ids, float* d_dists) {
    if (c.n == 0) return;
    const uint32_t blocks = std::min<uint32_t>((c.n + kFinWarps - 1) / kFinWarps, 148 * 8);
    k_finalize<<<blocks, kFinWarps * kWarp, 0, c.stream>>>(c.set_dist, c.set_id, c.set_size, c.n,
                                                           static_cast<int>(c.k), d_ids, d_dists);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

void launch_reset_sets(Context& c) {
    c.snap_prev_valid = false;
    if (c.n == 0) return;
    const size_t nk = static_cast<size_t>(c.n) * c.k;
    KNNG_CUDA(cudaMemsetAsync(c.set_dist, 0, nk * sizeof(float), c.stream));
    if (c.set_offsets.size() > 2) {
        k_reset_ids<<<std::min<uint32_t>((c.n + 255) / 256, 148 * 16), 256, 0, c.stream>>>(
            c.set_id, c.n, static_cast<int>(c.k), c.d_set_offsets, static_cast<uint32_t>(c.set_offsets.size() - 1));
        ++c.launches;
        KNNG_CUDA(cudaGetLastError());
    } else {
        KNNG_CUDA(cudaMemsetAsync(c.set_id, 0, nk * sizeof(uint32_t), c.stream));
    }
    k_reset_sets<<<std::min<uint32_t>((c.n + 255) / 256, 148 * 16), 256, 0, c.stream>>>(c.set_bound, c.set_maxslot,
                                                                                       c.set_size, c.n);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

}  // namespace knng
