// knng_grade -- recall of a k-NN graph file against a ground-truth file, with
// the reference grader's arithmetic (src/grade.cpp:42-98): for every row, the
// number of ground-truth ids present in the tested row; prints the average
// (out of 100) and the recall fraction.
//
//   knng_grade truth.bin test.bin n
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <unordered_set>
#include <vector>

static bool read_rows(const char* path, uint32_t n, std::vector<uint32_t>& rows) {
    std::ifstream f(path, std::ios::binary);
    rows.assign(static_cast<size_t>(n) * 100, 0);
    f.read(reinterpret_cast<char*>(rows.data()), static_cast<std::streamsize>(rows.size() * sizeof(uint32_t)));
    return static_cast<bool>(f);
}

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: knng_grade truth.bin test.bin n\n");
        return 2;
    }
    const uint32_t n = static_cast<uint32_t>(std::strtoul(argv[3], nullptr, 10));
    std::vector<uint32_t> truth, test;
    if (!read_rows(argv[1], n, truth) || !read_rows(argv[2], n, test)) {
        std::fprintf(stderr, "cannot read %u rows of 100 uint32\n", n);
        return 2;
    }
    uint64_t correct = 0;
    for (uint32_t i = 0; i < n; ++i) {
        std::unordered_set<uint32_t> t(test.begin() + static_cast<size_t>(i) * 100,
                                       test.begin() + static_cast<size_t>(i + 1) * 100);
        for (int j = 0; j < 100; ++j) correct += t.count(truth[static_cast<size_t>(i) * 100 + j]);
    }
    const double avg = n ? static_cast<double>(correct) / n : 0.0;
    std::printf("avg percent: %g\nrecall: %.6f\n", avg, avg / 100.0);
    return 0;
}
