// Driver around the reference's OWN k-NN graph code (TEST INFRASTRUCTURE ONLY).
//
// This file compiles the reference headers unmodified, straight from the
// reference tree (src/ann.hpp, src/SolutionKmeans.hpp, src/KnnSets.hpp,
// src/LinearAlgebra.hpp, src/Constants.hpp), against the stand-in headers in
// oracle/ref_shim/, and exposes a tiny C ABI so that Python tests can drive
//   SolutionKmeans::splitKmeansBinaryProcess   src/SolutionKmeans.hpp:142-311
//   SolutionKmeans::topUpSingle                src/SolutionKmeans.hpp:480-555
//   KnnSetScannableSimd::finalize + padResult  src/KnnSets.hpp:113-126, :334-344
//   SolutionRandomKD::rotateRandom              src/SolutionRandomKD.hpp:258-275
// with fixed parameters instead of the reference's wall-clock loop
// (src/SolutionKmeans.hpp:579-602).  Built by oracle/Makefile into
// oracle/_ref/ (never committed): libref_serial.so pins the oracle,
// libref_threads.so is the timed CPU baseline.
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>

#include <thread>

#include "ann.hpp"  // defines the processTime global the hot path updates
#include "SolutionKmeans.hpp"
#include "SolutionRandomKD.hpp"

namespace {

struct CoutSilencer {
    std::streambuf* saved;
    std::ofstream sink;
    CoutSilencer() : saved(std::cout.rdbuf()), sink("/dev/null") { std::cout.rdbuf(sink.rdbuf()); }
    ~CoutSilencer() { std::cout.rdbuf(saved); }
};

struct RefCtx {
    uint32_t n = 0;
    float (*points)[112] = nullptr;
    float (*pointsCopy)[112] = nullptr;
    std::vector<KnnSetScannableSimd> idToKnn;
    std::vector<uint32_t> indices;
    std::vector<float> bounds;
};

}  // namespace

extern "C" {

// Copies n rows of 100 floats (row stride ld floats) into the reference's
// 112-float, 64-byte aligned row layout (src/io.h:66-95).
void* ref_create(const float* pts, uint32_t n, uint32_t ld) {
    auto* c = new RefCtx();
    c->n = n;
    size_t bytes = static_cast<size_t>(n) * 112 * sizeof(float);
    if (bytes == 0) bytes = 64;
    c->points = static_cast<float(*)[112]>(std::aligned_alloc(64, bytes));
    c->pointsCopy = static_cast<float(*)[112]>(std::aligned_alloc(64, bytes));
    std::memset(c->points, 0, bytes);
    std::memset(c->pointsCopy, 0, bytes);
    for (uint32_t i = 0; i < n; ++i) std::memcpy(c->points[i], pts + static_cast<size_t>(i) * ld, 100 * sizeof(float));
    c->idToKnn.resize(n);
    c->indices.resize(n);
    c->bounds.assign(n, std::numeric_limits<float>::max());
    return c;
}

void ref_destroy(void* ctx) {
    auto* c = static_cast<RefCtx*>(ctx);
    std::free(c->points);
    std::free(c->pointsCopy);
    delete c;
}

// Restarts the calling thread's reference RNG (src/Constants.hpp:22).
void ref_reseed(uint32_t seed) { rd.seed(seed); }

// One repetition, as one iteration of src/SolutionKmeans.hpp:579-602 does:
// iota(indices) then splitKmeansBinaryProcess over [0, n).
void ref_rep(void* ctx, uint32_t knn_iterations, uint32_t max_group_size) {
    auto* c = static_cast<RefCtx*>(ctx);
    CoutSilencer quiet;
    std::iota(c->indices.begin(), c->indices.end(), 0);
    SolutionKmeans::splitKmeansBinaryProcess({0, c->n}, knn_iterations, max_group_size, c->points, c->pointsCopy,
                                             c->indices, c->idToKnn, c->bounds);
}

// The neighbour-of-neighbour pass, with no time bound.
uint64_t ref_topup(void* ctx) {
    auto* c = static_cast<RefCtx*>(ctx);
    CoutSilencer quiet;
    return SolutionKmeans::topUpSingle(c->points, c->idToKnn, c->bounds, LONG_MAX / 4, hclock::now());
}

void ref_get_indices(void* ctx, uint32_t* out) {
    auto* c = static_cast<RefCtx*>(ctx);
    std::memcpy(out, c->indices.data(), c->n * sizeof(uint32_t));
}

// Raw KnnSet state in slot order: dists/ids n*100, size, lowerBoundIdx, bound.
void ref_get_sets(void* ctx, float* dists, uint32_t* ids, uint32_t* sizes, uint32_t* lower_bound_idx, float* bounds) {
    auto* c = static_cast<RefCtx*>(ctx);
    for (uint32_t i = 0; i < c->n; ++i) {
        const auto& s = c->idToKnn[i];
        std::memcpy(dists + static_cast<size_t>(i) * 100, s.dists, 100 * sizeof(float));
        std::memcpy(ids + static_cast<size_t>(i) * 100, s.current_ids, 100 * sizeof(uint32_t));
        sizes[i] = s.size;
        lower_bound_idx[i] = s.lowerBoundIdx;
        bounds[i] = c->bounds[i];
    }
}

// finalize() every set, then padResult (src/SolutionKmeans.hpp:606-610).
void ref_finalize(void* ctx, uint32_t* out) {
    auto* c = static_cast<RefCtx*>(ctx);
    CoutSilencer quiet;
    std::vector<std::vector<uint32_t>> result(c->n);
    for (uint32_t id = 0; id < c->n; ++id) result[id] = c->idToKnn[id].finalize();
    padResult(c->n, result);
    for (uint32_t id = 0; id < c->n; ++id) std::memcpy(out + static_cast<size_t>(id) * 100, result[id].data(), 100 * sizeof(uint32_t));
}

// The reference's squared L2 distance and dot product (src/LinearAlgebra.hpp:53-77,
// :179-200) on two 100-float rows; inputs are copied to aligned storage first.
float ref_distance(const float* a, const float* b) {
    alignas(32) float x[112] = {0};
    alignas(32) float y[112] = {0};
    std::memcpy(x, a, 100 * sizeof(float));
    std::memcpy(y, b, 100 * sizeof(float));
    return distance(x, y);
}

float ref_dot(const float* a, const float* b) {
    alignas(32) float x[112] = {0};
    alignas(32) float y[112] = {0};
    std::memcpy(x, a, 100 * sizeof(float));
    std::memcpy(y, b, 100 * sizeof(float));
    return dot(x, y);
}

// Replays a sequence of offers into one fresh KnnSetScannableSimd, calling
// addCandidateLessThan only when dist < bound, exactly as the leaf loop does
// (src/KnnSets.hpp:152-157); returns the final state.
void ref_knnset_replay(const uint32_t* cand_ids, const float* cand_dists, uint32_t count, float* dists, uint32_t* ids,
                       uint32_t* size, uint32_t* lower_bound_idx, float* bound) {
    KnnSetScannableSimd s;
    float b = std::numeric_limits<float>::max();
    for (uint32_t t = 0; t < count; ++t) {
        if (cand_dists[t] < b) s.addCandidateLessThan(b, cand_ids[t], cand_dists[t]);
    }
    std::memcpy(dists, s.dists, 100 * sizeof(float));
    std::memcpy(ids, s.current_ids, 100 * sizeof(uint32_t));
    *size = s.size;
    *lower_bound_idx = s.lowerBoundIdx;
    *bound = b;
}

// SolutionRandomKD::rotateRandom (src/SolutionRandomKD.hpp:258-275) on the
// context's points, run on a fresh thread so that its thread_local generator
// (src/Constants.hpp:22) starts from its seed: the rotated values, n rows of
// new_dims floats, of the KD solution's first iteration.
void ref_kd_rotate(void* ctx, uint32_t new_dims, float* out) {
    auto* c = static_cast<RefCtx*>(ctx);
    std::thread t([&] { SolutionRandomKD::rotateRandom(new_dims, c->n, c->points, out); });
    t.join();
}

}  // extern "C"
