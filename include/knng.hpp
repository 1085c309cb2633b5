// knng.hpp -- header-only C++ convenience over the C ABI in knng.h.
//
// constructResult() has the signature of the reference's entry point
// SolutionKmeans::constructResult(float points[][112], uint32_t numPoints,
// vector<vector<uint32_t>>& result) (src/SolutionKmeans.hpp:558), so a caller
// of the reference can switch by changing one call.  Errors are reported as
// std::runtime_error (the ABI itself never throws).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "knng.h"

namespace knng_b200 {

class Context {
public:
    explicit Context(int device = 0, uint64_t hbm_budget_bytes = 0) {
        check(knng_create(device, hbm_budget_bytes, &ctx_), nullptr);
    }
    ~Context() {
        if (ctx_) knng_destroy(ctx_);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    knng_context* get() const { return ctx_; }

    static void check(knng_status s, knng_context* ctx) {
        if (s == KNNG_OK) return;
        std::string msg = knng_status_string(s);
        if (ctx) {
            const char* e = knng_last_error(ctx);
            if (e && *e) msg += std::string(": ") + e;
        }
        throw std::runtime_error("knng: " + msg);
    }

private:
    knng_context* ctx_ = nullptr;
};

// Rows of `stride` floats (the reference uses 112), first `dims` used.
template <int Stride>
void constructResult(float points[][Stride], uint32_t numPoints, std::vector<std::vector<uint32_t>>& result,
                     const knng_params* params = nullptr, uint32_t dims = 100, int device = 0) {
    knng_params p;
    knng_default_params(&p);
    if (params) p = *params;
    Context ctx(device);
    std::vector<uint32_t> ids(static_cast<size_t>(numPoints) * p.k);
    Context::check(knng_build(ctx.get(), &points[0][0], numPoints, dims, sizeof(float) * Stride, &p, ids.data(), nullptr,
                              nullptr),
                   ctx.get());
    result.resize(numPoints);
    for (uint32_t i = 0; i < numPoints; ++i)
        result[i].assign(ids.begin() + static_cast<size_t>(i) * p.k, ids.begin() + static_cast<size_t>(i + 1) * p.k);
}

// The reference's alternative solution, SolutionRandomKD::constructResult
// (src/SolutionRandomKD.hpp:377-430): five repetitions of the random-rotation
// KD split (30 rotated dimensions, buckets below 400 points), no
// neighbour-of-neighbour pass, then the sorted, padded lists.
template <int Stride>
void constructResultKD(float points[][Stride], uint32_t numPoints, std::vector<std::vector<uint32_t>>& result,
                       const knng_params* params = nullptr, uint32_t new_dims = 30, uint32_t dims = 100,
                       int device = 0) {
    knng_params p;
    knng_default_params(&p);
    p.reps = 5;
    p.max_leaf = 400;
    p.max_leaf_odd = 0;
    p.refine = 0;
    if (params) p = *params;
    Context ctx(device);
    std::vector<uint32_t> ids(static_cast<size_t>(numPoints) * p.k);
    Context::check(knng_build_kd(ctx.get(), &points[0][0], numPoints, dims, sizeof(float) * Stride, &p, new_dims,
                                 ids.data(), nullptr, nullptr),
                   ctx.get());
    result.resize(numPoints);
    for (uint32_t i = 0; i < numPoints; ++i)
        result[i].assign(ids.begin() + static_cast<size_t>(i) * p.k, ids.begin() + static_cast<size_t>(i + 1) * p.k);
}

// The reference's schedule by wall clock (src/SolutionKmeans.hpp:579-604):
// repetitions while less than build_ms has passed (the reference: 1,210 s, or
// 20 s on its local runs), then refinement passes while less than
// build_ms + refine_ms has (the reference: 500 s / 20 s more).  The default
// parameters are the reference's (buckets < 200 / < 400 alternating, one Lloyd
// iteration, one pass), with no cap on the repetitions.
template <int Stride>
void constructResultTimed(float points[][Stride], uint32_t numPoints, std::vector<std::vector<uint32_t>>& result,
                          uint64_t build_ms, uint64_t refine_ms, const knng_params* params = nullptr,
                          uint32_t dims = 100, int device = 0) {
    knng_params p;
    knng_default_params(&p);
    p.reps = 0;
    if (params) p = *params;
    Context ctx(device);
    std::vector<uint32_t> ids(static_cast<size_t>(numPoints) * p.k);
    Context::check(knng_build_timed(ctx.get(), &points[0][0], numPoints, dims, sizeof(float) * Stride, &p, build_ms,
                                    refine_ms, ids.data(), nullptr, nullptr),
                   ctx.get());
    result.resize(numPoints);
    for (uint32_t i = 0; i < numPoints; ++i)
        result[i].assign(ids.begin() + static_cast<size_t>(i) * p.k, ids.begin() + static_cast<size_t>(i + 1) * p.k);
}

}  // namespace knng_b200
