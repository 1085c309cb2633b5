// knng_build -- the reference's command line (src/main.cpp:39-71) on the GPU:
//
//   knng_build [input.bin] [output.bin] [reps] [refine passes] [max_leaf]
//   knng_build input.bin output.bin --timed build_ms refine_ms
//   knng_build input.bin output.bin --kd [reps] [max_leaf]
//
// The second form is the reference's wall-clock schedule
// (SolutionKmeans::constructResult, src/SolutionKmeans.hpp:579-604):
// repetitions while build_ms has not passed, then passes while
// build_ms + refine_ms has not (the reference: 1,210,000 and 500,000 ms).
// The third is the reference's alternative random-rotation KD solution
// (SolutionRandomKD::constructResult, src/SolutionRandomKD.hpp:377-430):
// `reps` repetitions (default 5) with buckets below max_leaf (default 400),
// 30 rotated dimensions, no neighbour-of-neighbour pass.
//
// input.bin: uint32 N, then N rows of 100 float32 (the contest format read by
// ReadBinArray, src/io.h:66-95).  output.bin: N rows of 100 uint32 neighbour
// ids, sorted by distance, no header (SaveKNNG, src/io.h:21-33).  Defaults:
// dummy-data.bin, output.bin, the reference's parameters (knng_default_params).
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "knng.h"

int main(int argc, char** argv) {
    const std::string in = argc > 1 ? argv[1] : "dummy-data.bin";
    const std::string out = argc > 2 ? argv[2] : "output.bin";
    knng_params p;
    knng_default_params(&p);
    const bool timed = argc > 3 && std::string(argv[3]) == "--timed";
    const bool kd = argc > 3 && std::string(argv[3]) == "--kd";
    uint64_t build_ms = 0, refine_ms = 0;
    if (kd) {
        p.reps = argc > 4 ? static_cast<uint32_t>(std::atoi(argv[4])) : 5u;
        p.max_leaf = argc > 5 ? static_cast<uint32_t>(std::atoi(argv[5])) : 400u;
        p.max_leaf_odd = 0;
        p.refine = 0;
    } else if (timed) {
        if (argc < 6) {
            std::fprintf(stderr, "usage: knng_build input.bin output.bin --timed build_ms refine_ms\n");
            return 2;
        }
        build_ms = std::strtoull(argv[4], nullptr, 10);
        refine_ms = std::strtoull(argv[5], nullptr, 10);
        p.reps = 0;  // no cap: the clock decides
    } else if (argc > 3) {
        p.reps = static_cast<uint32_t>(std::atoi(argv[3]));
    }
    if (!timed && !kd && argc > 4) p.refine = static_cast<uint32_t>(std::atoi(argv[4]));
    if (!timed && !kd && argc > 5) {
        p.max_leaf = static_cast<uint32_t>(std::atoi(argv[5]));
        p.max_leaf_odd = 0;
    }
    const auto t0 = std::chrono::steady_clock::now();
    std::ifstream f(in, std::ios::binary);
    if (!f) {
        std::fprintf(stderr, "cannot open %s\n", in.c_str());
        return 2;
    }
    uint32_t n = 0;
    f.read(reinterpret_cast<char*>(&n), sizeof(n));
    std::vector<float> pts(static_cast<size_t>(n) * 100);
    f.read(reinterpret_cast<char*>(pts.data()), static_cast<std::streamsize>(pts.size() * sizeof(float)));
    if (!f) {
        std::fprintf(stderr, "%s: expected %u rows of 100 float32\n", in.c_str(), n);
        return 2;
    }
    knng_context* ctx = nullptr;
    knng_status s = knng_create(0, 0, &ctx);
    if (s != KNNG_OK) {
        std::fprintf(stderr, "knng_create: %s\n", knng_status_string(s));
        return 3;
    }
    std::vector<uint32_t> ids(static_cast<size_t>(n) * p.k);
    knng_stats st;
    s = kd      ? knng_build_kd(ctx, pts.data(), n, 100, 400, &p, 30, ids.data(), nullptr, &st)
        : timed ? knng_build_timed(ctx, pts.data(), n, 100, 400, &p, build_ms, refine_ms, ids.data(), nullptr, &st)
                : knng_build(ctx, pts.data(), n, 100, 400, &p, ids.data(), nullptr, &st);
    if (s != KNNG_OK) {
        std::fprintf(stderr, "knng_build: %s: %s\n", knng_status_string(s), knng_last_error(ctx));
        knng_destroy(ctx);
        return 3;
    }
    knng_destroy(ctx);
    std::ofstream o(out, std::ios::binary);
    o.write(reinterpret_cast<const char*>(ids.data()), static_cast<std::streamsize>(ids.size() * sizeof(uint32_t)));
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::printf("points %u  reps %llu  refine passes %llu  device ms %.1f  total ms %.1f  -> %s\n", n,
                static_cast<unsigned long long>(st.reps_done),
                static_cast<unsigned long long>(st.refine_passes_done), st.ms_total + st.ms_finalize, ms,
                out.c_str());
    return 0;
}
