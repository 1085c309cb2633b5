// Random-rotation KD splitter: SolutionRandomKD (src/SolutionRandomKD.hpp:45-430),
// the reference's alternative solution (disabled at src/main.cpp:58), as a
// second splitter behind the same side test, stable partition and bucket pass
// as the 2-means tree.
//
// One repetition (rotateRandom :258-275, split :284-375):
//   * new_dims rotation vectors, made on the host as rotateRandom makes them:
//     each of d normal draws (std::normal_distribution<double>(0, 1), a new
//     distribution per vector, on a std::mt19937) rounded to float and divided
//     by its norm (normalizeInPlace, src/LinearAlgebra.hpp:86-91: the norm is
//     the square root of a float sum of float squares), then the reference's
//     Gram-Schmidt (:211-222), whose normalize returns its input (:93-101), so
//     that only the first vector has unit length; projections use the
//     reference's dot (:179-200);
//   * rotated values rot[p][c] = dot(u_c, x_p) on the device (k_kd_rotate),
//     in the reference's dot order;
//   * per node of at least max_leaf points: the mean and the (size - 1)
//     variance of every rotated dimension in double (pickIndexFull :196-224,
//     getMean :92-114, getVariance :116-143), summed in a fixed order -- per
//     chunk of 1,024 positions in index order, then the chunk sums in chunk
//     order (the reference sums per TBB block and combines in thread order,
//     so its order is not fixed); the dimension drawn with probability
//     proportional to its variance (pairs sorted in descending order, a float
//     running total, a uniform draw in [0, total) -- here from the counter
//     RNG, keyed by the node, instead of the reference's generator); split
//     value = that dimension's mean; the points with rot < mean first
//     (:316-358).  Statistics, pick and hyperplane stay on the device
//     (k_kd_chunk_sums, k_kd_node_stats, k_kd_pick); the host reads back only
//     each node's side count.  The partition is the 2-means side test with
//     coefficients -u and offset -F, F the largest float below the mean:
//     dot(-u, x) >= -F is rot < mean bit for bit (negating every operand
//     negates the dot exactly);
//   * nodes below max_leaf points are buckets for the usual bucket pass.
//
// Deliberate differences.  The reference's getMean / getVariance read the
// rows indices[0 .. size) -- the first `size` entries of the whole
// permutation -- instead of the node's range, so its splits depend on the
// final order of every node to its left (and on thread timing under TBB);
// here the statistics are the node's own.  When every point falls on one
// side the reference recurses on the same range; here the node is redrawn
// (next attempt) up to 64 times, then split at its index midpoint.  The
// reference gathers each side per TBB block and concatenates the blocks in
// combine order (:331-351); here each side keeps index order (stable).  Its
// KnnSetScannable (src/KnnSets.hpp:225-282) overwrites the first maximum slot
// in slot order; the bucket pass here uses the 2-means form's set (the same
// offers in the same order and the same accepted candidates; ties at the
// maximum resolved in getMaxIdx's order).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <random>
#include <vector>

#include "common.cuh"
#include "context.hpp"
#include "dispatch.hpp"

namespace knng {

namespace {

constexpr uint32_t kMaxKdDims = 32;  // one lane per rotated dimension

// The reference's dot (src/LinearAlgebra.hpp:179-200) for d values: eight FMA
// chains over the dimensions below the last multiple of 8 (rhs * lhs + sum),
// the lanes added left to right to 0, then each remaining product added.
float host_ref_dot(const float* lhs, const float* rhs, uint32_t d) {
    const uint32_t m = d / 8 * 8;
    float lane[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i = 0; i < m; i += 8)
        for (int l = 0; l < 8; ++l) lane[l] = std::fma(rhs[i + l], lhs[i + l], lane[l]);
    float ans = 0.0f;
    for (int l = 0; l < 8; ++l) ans += lane[l];
    for (uint32_t i = m; i < d; ++i) {
        const float prod = lhs[i] * rhs[i];
        ans += prod;
    }
    return ans;
}

// normalizeInPlace: v / sqrt(float sum of float squares), divided in double.
void host_normalize(std::vector<float>& v) {
    float sum_squares = 0.0f;
    for (float x : v) {
        const float sq = x * x;
        sum_squares += sq;
    }
    const double norm = std::sqrt(static_cast<double>(sum_squares));
    for (float& x : v) x = static_cast<float>(static_cast<double>(x) / norm);
}

}  // namespace

std::vector<float> kd_rotation(uint32_t new_dims, uint32_t d, uint64_t seed) {
    std::mt19937 rng(static_cast<std::mt19937::result_type>(seed));
    std::vector<std::vector<float>> v(new_dims, std::vector<float>(d));
    for (uint32_t h = 0; h < new_dims; ++h) {
        std::normal_distribution<> normal(0, 1);
        for (uint32_t i = 0; i < d; ++i) v[h][i] = static_cast<float>(normal(rng));
        host_normalize(v[h]);
    }
    // gramSchmidt: u_i = v_i - sum_j dot(u_j, v_i) u_j, each subtraction of
    // the float product rounded; no rescaling after the first vector.
    std::vector<std::vector<float>> u(new_dims);
    for (uint32_t i = 0; i < new_dims; ++i) {
        u[i] = v[i];
        for (uint32_t j = 0; j < i; ++j) {
            const float s = host_ref_dot(u[j].data(), v[i].data(), d);
            for (uint32_t k = 0; k < d; ++k) {
                const float prod = s * u[j][k];
                u[i][k] = u[i][k] - prod;
            }
        }
    }
    std::vector<float> out(static_cast<size_t>(new_dims) * d);
    for (uint32_t i = 0; i < new_dims; ++i) std::copy(u[i].begin(), u[i].end(), out.begin() + static_cast<size_t>(i) * d);
    return out;
}

namespace {

// rot[p * nd + c] = dot(u_c, x_p) in the reference's order: one warp per pair
// of points, lane c < nd one rotated dimension.  The vectors sit in shared
// memory with row stride kKdStride<D> (a multiple of 4 that is 4 mod 32, so
// the lanes' 16-byte loads of a quarter-warp hit distinct bank groups); the
// two rows are read as 16-byte broadcasts.  Each step of eight dimensions
// takes two vector loads and two row loads per point for sixteen FMAs; chain
// l (dimensions l, l + 8, ...) and the order of the sums are the reference's.
template <int D>
constexpr int kKdStride = D + (36 - D % 32) % 32;

template <int D>
__global__ void __launch_bounds__(256) k_kd_rotate(const float* __restrict__ pts, int ld, uint32_t n,
                                                   const float* __restrict__ rotation, uint32_t nd,
                                                   float* __restrict__ rot) {
    constexpr int S = kKdStride<D>;
    static_assert(S % 4 == 0 && S % 32 == 4 && S >= D, "vector row stride");
    __shared__ __align__(16) float u_s[kMaxKdDims * S];
    __shared__ __align__(16) float x_s[8][2][D];
    for (uint32_t f = threadIdx.x; f < nd * D; f += blockDim.x) u_s[(f / D) * S + f % D] = rotation[f];
    __syncthreads();
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    constexpr int M = D / 8 * 8;
    constexpr int Q = D / 4;
    const float* u = u_s + lane * S;
    for (uint32_t p0 = (blockIdx.x * 8 + warp) * 2; p0 < n; p0 += gridDim.x * 16) {
        for (int f = lane; f < 2 * Q; f += kWarp) {
            const uint32_t p = p0 + static_cast<uint32_t>(f / Q);
            const float4 v = p < n ? *reinterpret_cast<const float4*>(pts + static_cast<size_t>(p) * ld + 4 * (f % Q))
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
            *reinterpret_cast<float4*>(&x_s[warp][f / Q][4 * (f % Q)]) = v;
        }
        __syncwarp();
        if (static_cast<uint32_t>(lane) < nd) {
            float chain[2][8];
#pragma unroll
            for (int q = 0; q < 2; ++q)
#pragma unroll
                for (int l = 0; l < 8; ++l) chain[q][l] = 0.0f;
#pragma unroll 4
            for (int i = 0; i < M; i += 8) {
                const float4 ua = *reinterpret_cast<const float4*>(u + i);
                const float4 ub = *reinterpret_cast<const float4*>(u + i + 4);
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const float4 xa = *reinterpret_cast<const float4*>(&x_s[warp][q][i]);
                    const float4 xb = *reinterpret_cast<const float4*>(&x_s[warp][q][i + 4]);
                    chain[q][0] = __fmaf_rn(xa.x, ua.x, chain[q][0]);
                    chain[q][1] = __fmaf_rn(xa.y, ua.y, chain[q][1]);
                    chain[q][2] = __fmaf_rn(xa.z, ua.z, chain[q][2]);
                    chain[q][3] = __fmaf_rn(xa.w, ua.w, chain[q][3]);
                    chain[q][4] = __fmaf_rn(xb.x, ub.x, chain[q][4]);
                    chain[q][5] = __fmaf_rn(xb.y, ub.y, chain[q][5]);
                    chain[q][6] = __fmaf_rn(xb.z, ub.z, chain[q][6]);
                    chain[q][7] = __fmaf_rn(xb.w, ub.w, chain[q][7]);
                }
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const uint32_t p = p0 + static_cast<uint32_t>(q);
                float ans = 0.0f;
#pragma unroll
                for (int l = 0; l < 8; ++l) ans = __fadd_rn(ans, chain[q][l]);
#pragma unroll
                for (int i = M; i < D; ++i) ans = __fadd_rn(ans, __fmul_rn(u[i], x_s[warp][q][i]));
                if (p < n) rot[static_cast<size_t>(p) * nd + lane] = ans;
            }
        }
        __syncwarp();
    }
}

// Node statistics in a fixed order that does not depend on the launch: a
// node's positions in chunks of kKdChunk; each chunk's values added one at a
// time in index order to a double starting at 0 (k_kd_chunk_sums, one warp per
// chunk, lane c one rotated dimension), then the chunk sums one at a time in
// chunk order (k_kd_node_stats, one warp per node).  With `mean` null the
// values are rot; otherwise (rot - mean)^2 in double.
constexpr uint32_t kKdChunk = 1024;
constexpr int kKdWarps = 8;

struct KdChunk {
    uint32_t node, begin, end;
};

__global__ void __launch_bounds__(kKdWarps * kWarp) k_kd_chunk_sums(const KdChunk* __restrict__ chunks, uint32_t count,
                                                                    const uint32_t* __restrict__ idx,
                                                                    const float* __restrict__ rot, uint32_t nd,
                                                                    const double* __restrict__ mean,
                                                                    double* __restrict__ partial) {
    const uint32_t item = blockIdx.x * kKdWarps + threadIdx.x / kWarp;
    const uint32_t c = threadIdx.x % kWarp;
    if (item >= count || c >= nd) return;
    const KdChunk ch = chunks[item];
    double s = 0.0;
    if (mean == nullptr) {
#pragma unroll 8
        for (uint32_t i = ch.begin; i < ch.end; ++i)
            s = __dadd_rn(s, static_cast<double>(rot[static_cast<size_t>(idx[i]) * nd + c]));
    } else {
        const double m = mean[static_cast<size_t>(ch.node) * nd + c];
#pragma unroll 8
        for (uint32_t i = ch.begin; i < ch.end; ++i) {
            const double diff = __dsub_rn(static_cast<double>(rot[static_cast<size_t>(idx[i]) * nd + c]), m);
            s = __dadd_rn(s, __dmul_rn(diff, diff));
        }
    }
    partial[static_cast<size_t>(item) * nd + c] = s;
}

// out[node][c] = (sum of the node's chunk sums in chunk order) / divisor,
// divisor = size (means) or size - 1 (variances).
__global__ void __launch_bounds__(kKdWarps * kWarp) k_kd_node_stats(const uint32_t* __restrict__ first_chunk,
                                                                    const uint32_t* __restrict__ sizes, uint32_t m,
                                                                    const double* __restrict__ partial, uint32_t nd,
                                                                    uint32_t minus, double* __restrict__ out) {
    const uint32_t node = blockIdx.x * kKdWarps + threadIdx.x / kWarp;
    const uint32_t c = threadIdx.x % kWarp;
    if (node >= m || c >= nd) return;
    double s = 0.0;
#pragma unroll 8
    for (uint32_t j = first_chunk[node]; j < first_chunk[node + 1]; ++j)
        s = __dadd_rn(s, partial[static_cast<size_t>(j) * nd + c]);
    out[static_cast<size_t>(node) * nd + c] = __ddiv_rn(s, static_cast<double>(sizes[node] - minus));
}

}  // namespace

namespace {

constexpr uint32_t kMaxKdAttempts = 64;

// The uniform draw of a node's dimension pick: a float in [0, 1) from the
// counter RNG keyed by (seed, repetition, node range, attempt).
__device__ __forceinline__ float kd_uniform(uint64_t seed, uint32_t rep, uint32_t start, uint32_t end,
                                            uint32_t attempt) {
    uint64_t h = mix64(seed + 0x9e3779b97f4a7c15ULL * (static_cast<uint64_t>(rep) + 1));
    h = mix64(h ^ ((static_cast<uint64_t>(start) << 32) | end));
    h = mix64(h ^ ((static_cast<uint64_t>(attempt) << 32) | 0x4b44u));
    return __fmul_rn(static_cast<float>(h >> 40), 5.9604644775390625e-08f);  // 2^-24
}

// Per node of a level (one warp): pickIndexFull's choice
// (src/SolutionRandomKD.hpp:200-224) from the node's variances -- the float
// total of the variances in dimension order, the pairs (variance, dimension)
// in descending order (lane c's rank: the pairs above it), a float running
// sum in that order, the first dimension whose running sum reaches u * total
// (the last one if none does) -- then the node's hyperplane: coefficients
// -u_dim and offset -F, F the largest float below the dimension's mean.
__global__ void __launch_bounds__(kKdWarps * kWarp) k_kd_pick(const uint32_t* __restrict__ starts,
                                                              const uint32_t* __restrict__ ends,
                                                              const uint32_t* __restrict__ attempts, uint32_t m,
                                                              const double* __restrict__ mean,
                                                              const double* __restrict__ var, uint32_t nd,
                                                              const float* __restrict__ rotation, uint32_t d, int ld,
                                                              uint64_t seed, uint32_t rep, float* __restrict__ coefs,
                                                              float* __restrict__ offs) {
    const uint32_t node = blockIdx.x * kKdWarps + threadIdx.x / kWarp;
    const uint32_t lane = threadIdx.x % kWarp;
    if (node >= m) return;  // warp-uniform
    const double v = lane < nd ? var[static_cast<size_t>(node) * nd + lane] : 0.0;
    float total = 0.0f;
    uint32_t rank = 0;
    for (uint32_t j = 0; j < nd; ++j) {
        const double vj = __shfl_sync(kFull, v, static_cast<int>(j));
        total = __double2float_rn(__dadd_rn(static_cast<double>(total), vj));
        rank += (vj > v || (vj == v && j > lane)) ? 1u : 0u;
    }
    const float sample = __fmul_rn(kd_uniform(seed, rep, starts[node], ends[node], attempts[node]), total);
    float so_far = 0.0f;
    uint32_t dim = 0;
    for (uint32_t i = 0; i < nd; ++i) {
        const unsigned who = __ballot_sync(kFull, lane < nd && rank == i);
        if (who == 0) break;  // only with NaN variances: keep the last dimension found
        dim = static_cast<uint32_t>(__ffs(who) - 1);
        so_far = __double2float_rn(__dadd_rn(static_cast<double>(so_far), __shfl_sync(kFull, v, static_cast<int>(dim))));
        if (so_far >= sample) break;  // warp-uniform
    }
    const double mu = mean[static_cast<size_t>(node) * nd + dim];
    for (uint32_t k = lane; k < static_cast<uint32_t>(ld); k += kWarp)
        coefs[static_cast<size_t>(node) * ld + k] = k < d ? -rotation[static_cast<size_t>(dim) * d + k] : 0.0f;
    if (lane == 0) {
        float f = __double2float_rn(mu);
        // The nearest float is at most one step above the mean.
        for (int t = 0; t < 4 && static_cast<double>(f) >= mu; ++t) f = nextafterf(f, -INFINITY);
        offs[node] = -f;
    }
}

}  // namespace

void run_rep_kd(Context& c, uint32_t max_leaf, uint32_t new_dims, uint64_t seed, uint32_t rep, KdRepResult& out) {
    if (new_dims < 1 || new_dims > kMaxKdDims) fail(KNNG_ERR_INVALID_ARGUMENT, "new_dims must be in [1, 32]");
    if (max_leaf < 2) fail(KNNG_ERR_INVALID_ARGUMENT, "max_leaf must be >= 2");
    const uint32_t n = c.n, d = c.d, nd = new_dims;
    cudaEvent_t ev[3];
    for (auto& e : ev) KNNG_CUDA(cudaEventCreate(&e));
    KNNG_CUDA(cudaEventRecord(ev[0], c.stream));
    // Rotation (repetition r uses the generator seeded with seed + r) and the
    // rotated values.
    const std::vector<float> rotation = kd_rotation(nd, d, seed + rep);
    float* d_rotation = upload(c, "kd_rotation", rotation.data(), rotation.size());
    auto* rot = static_cast<float*>(scratch(c, "kd_rot", static_cast<size_t>(n) * nd * sizeof(float)));
    KNNG_DISPATCH_D(d, {
        const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((n + 15) / 16, c.sms * 8));
        k_kd_rotate<D><<<blocks, 256, 0, c.stream>>>(c.points, c.ld, n, d_rotation, nd, rot);
    });
    ++c.launches;
    KNNG_CUDA(cudaGetLastError());
    launch_iota(c);
    // Level by level: nodes of at least max_leaf points split, the others are
    // buckets.
    struct KdNode {
        uint32_t start, end, attempt;
    };
    std::vector<KdNode> level;
    std::vector<uint32_t> leaf_start, leaf_end;
    auto place = [&](uint32_t s, uint32_t e, std::vector<KdNode>& next) {
        if (e - s < max_leaf) {
            leaf_start.push_back(s);
            leaf_end.push_back(e);
        } else {
            next.push_back({s, e, 0});
        }
    };
    for (size_t s = 0; s + 1 < c.set_offsets.size(); ++s) {
        std::vector<KdNode> roots;
        place(c.set_offsets[s], c.set_offsets[s + 1], roots);
        level.insert(level.end(), roots.begin(), roots.end());
    }
    const uint32_t ld = c.ld;
    while (!level.empty()) {
        const uint32_t m = static_cast<uint32_t>(level.size());
        out.levels += 1;
        out.nodes += m;
        std::vector<uint32_t> hs(m), he(m);
        for (uint32_t i = 0; i < m; ++i) {
            hs[i] = level[i].start;
            he[i] = level[i].end;
        }
        uint32_t* d_s = upload(c, "kd_starts", hs.data(), m);
        // Chunks of every node of the level, in node order.
        std::vector<KdChunk> chunks;
        std::vector<uint32_t> first(m + 1), sizes(m);
        for (uint32_t i = 0; i < m; ++i) {
            first[i] = static_cast<uint32_t>(chunks.size());
            sizes[i] = he[i] - hs[i];
            for (uint32_t b = hs[i]; b < he[i]; b += std::min(kKdChunk, he[i] - b))
                chunks.push_back({i, b, b + std::min(kKdChunk, he[i] - b)});
        }
        first[m] = static_cast<uint32_t>(chunks.size());
        const uint32_t nc = first[m];
        const KdChunk* d_chunks = upload(c, "kd_chunks", chunks.data(), nc);
        const uint32_t* d_first = upload(c, "kd_first_chunk", first.data(), m + 1);
        const uint32_t* d_sizes = upload(c, "kd_sizes", sizes.data(), m);
        auto* d_partial = static_cast<double*>(scratch(c, "kd_partial", static_cast<size_t>(nc) * nd * sizeof(double)));
        auto* d_mean = static_cast<double*>(scratch(c, "kd_mean", static_cast<size_t>(m) * nd * sizeof(double)));
        auto* d_var = static_cast<double*>(scratch(c, "kd_var", static_cast<size_t>(m) * nd * sizeof(double)));
        const uint32_t cb = (nc + kKdWarps - 1) / kKdWarps, nb = (m + kKdWarps - 1) / kKdWarps;
        k_kd_chunk_sums<<<cb, kKdWarps * kWarp, 0, c.stream>>>(d_chunks, nc, c.indices, rot, nd, nullptr, d_partial);
        k_kd_node_stats<<<nb, kKdWarps * kWarp, 0, c.stream>>>(d_first, d_sizes, m, d_partial, nd, 0, d_mean);
        k_kd_chunk_sums<<<cb, kKdWarps * kWarp, 0, c.stream>>>(d_chunks, nc, c.indices, rot, nd, d_mean, d_partial);
        k_kd_node_stats<<<nb, kKdWarps * kWarp, 0, c.stream>>>(d_first, d_sizes, m, d_partial, nd, 1, d_var);
        c.launches += 4;
        KNNG_CUDA(cudaGetLastError());
        // Dimension picks and hyperplanes on the device.
        std::vector<uint32_t> att(m);
        for (uint32_t i = 0; i < m; ++i) att[i] = level[i].attempt;
        const uint32_t* d_e = upload(c, "kd_ends", he.data(), m);
        const uint32_t* d_att = upload(c, "kd_attempts", att.data(), m);
        auto* d_c = static_cast<float*>(scratch(c, "kd_coefs", static_cast<size_t>(m) * ld * sizeof(float)));
        auto* d_o = static_cast<float*>(scratch(c, "kd_offsets", m * sizeof(float)));
        k_kd_pick<<<nb, kKdWarps * kWarp, 0, c.stream>>>(d_s, d_e, d_att, m, d_mean, d_var, nd, d_rotation, d, ld, seed,
                                                         rep, d_c, d_o);
        ++c.launches;
        KNNG_CUDA(cudaGetLastError());
        auto* d_t = static_cast<uint32_t*>(scratch(c, "kd_true", m * sizeof(uint32_t)));
        launch_partition(c, m, hs.data(), he.data(), d_s, d_c, d_o, d_t);
        std::vector<uint32_t> t(m);
        download(c, t.data(), d_t, m);
        std::vector<KdNode> next;
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t s = hs[i], e = he[i];
            uint32_t mid = s + t[i];
            if (mid == s || mid == e) {  // every point on one side
                if (level[i].attempt + 1 < kMaxKdAttempts) {
                    next.push_back({s, e, level[i].attempt + 1});
                    out.restarts += 1;
                    continue;
                }
                mid = s + (e - s) / 2;  // the partition left the order unchanged
                out.fallbacks += 1;
            }
            place(s, mid, next);
            place(mid, e, next);
        }
        level.swap(next);
    }
    KNNG_CUDA(cudaEventRecord(ev[1], c.stream));
    // The bucket pass over every leaf.
    const uint32_t nl = static_cast<uint32_t>(leaf_start.size());
    uint32_t max_bucket = 0;
    for (uint32_t i = 0; i < nl; ++i) max_bucket = std::max(max_bucket, leaf_end[i] - leaf_start[i]);
    if (nl > 0) {
        uint32_t* d_ls = upload(c, "kd_leaf_start", leaf_start.data(), nl);
        uint32_t* d_le = upload(c, "kd_leaf_end", leaf_end.data(), nl);
        launch_leaves(c, nl, d_ls, d_le, max_bucket, nullptr);
    }
    KNNG_CUDA(cudaEventRecord(ev[2], c.stream));
    KNNG_CUDA(cudaEventSynchronize(ev[2]));
    float ms = 0.f;
    KNNG_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    out.ms_split = ms;
    KNNG_CUDA(cudaEventElapsedTime(&ms, ev[1], ev[2]));
    out.ms_leaf = ms;
    for (auto& e : ev) cudaEventDestroy(e);
    out.leaf_start = std::move(leaf_start);
    out.leaf_end = std::move(leaf_end);
}

}  // namespace knng
