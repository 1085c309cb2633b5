// Output stage: KnnSetScannableSimd::finalize (src/KnnSets.hpp:113-126) --
// each set sorted by (distance, id) ascending -- and padResult
// (src/KnnSets.hpp:334-344), which pads short rows with id 1.  One warp per
// point sorts its (at most 128) entries as 64-bit keys (distance bits << 32 |
// id; distances are non-negative, so the bit order is the numeric order) with
// a bitonic network in shared memory.
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

}  // namespace

void launch_finalize(Context& c, uint32_t* d_ids, float* d_dists) {
    if (c.n == 0) return;
    const uint32_t blocks = std::min<uint32_t>((c.n + kFinWarps - 1) / kFinWarps, 148 * 8);
    k_finalize<<<blocks, kFinWarps * kWarp, 0, c.stream>>>(c.set_dist, c.set_id, c.set_size, c.n,
                                                           static_cast<int>(c.k), d_ids, d_dists);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

void launch_reset_sets(Context& c) {
    if (c.n == 0) return;
    const size_t nk = static_cast<size_t>(c.n) * c.k;
    KNNG_CUDA(cudaMemsetAsync(c.set_dist, 0, nk * sizeof(float), c.stream));
    KNNG_CUDA(cudaMemsetAsync(c.set_id, 0, nk * sizeof(uint32_t), c.stream));
    k_reset_sets<<<std::min<uint32_t>((c.n + 255) / 256, 148 * 16), 256, 0, c.stream>>>(c.set_bound, c.set_maxslot,
                                                                                       c.set_size, c.n);
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
}

}  // namespace knng
