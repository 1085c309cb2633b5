"""CPU test of the serving loop's admission rule (csrc/admission.hpp): a job
starts when its reservation fits beside the running jobs' and a slot is free;
jobs start in arrival order.  The header is compiled with g++ into a small
harness that replays a queue against the rule."""
from __future__ import annotations

import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r'''
#include <cstdio>
#include <deque>
#include <vector>
#include "admission.hpp"
using knng::admits;
int main() {
    int bad = 0;
    // truth table
    bad += !admits(0, 10, 10, 0, 1);        // exactly fits
    bad += admits(1, 10, 10, 0, 1);         // one byte over
    bad += admits(0, 1, 10, 1, 1);          // no free slot
    bad += !admits(5, 5, 10, 1, 2);
    // FIFO replay: budget 10, two slots; jobs (need, duration) arrive at t = 0.
    struct Job { unsigned need, dur; int start = -1, end = -1; };
    std::vector<Job> jobs = {{6, 3}, {3, 1}, {8, 2}, {1, 1}, {4, 2}};
    std::deque<int> queue = {0, 1, 2, 3, 4};
    unsigned long long in_use = 0; unsigned running = 0;
    for (int t = 0; t < 100 && (!queue.empty() || running); ++t) {
        for (auto& j : jobs) if (j.start >= 0 && j.end == t) { in_use -= j.need; --running; }
        while (!queue.empty() && admits(in_use, jobs[queue.front()].need, 10, running, 2)) {
            Job& j = jobs[queue.front()]; queue.pop_front();
            j.start = t; j.end = t + (int)j.dur; in_use += j.need; ++running;
        }
    }
    for (auto& j : jobs) std::printf("%d %d\n", j.start, j.end);
    return bad;
}
'''


def test_admission_rule_and_arrival_order(tmp_path):
    src = tmp_path / "harness.cpp"
    src.write_text(HARNESS)
    exe = tmp_path / "harness"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-I", os.path.join(ROOT, "sigmod23ann_b200", "csrc"), str(src),
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, "truth table"
    spans = [tuple(map(int, line.split())) for line in r.stdout.split("\n") if line.strip()]
    # job 0 (6) and job 1 (3) start at once; job 2 (8) waits until both have
    # ended (t = 3), job 3 (1) then fits beside it; job 4 (4) waits until job 2
    # has ended and there is room (t = 5).
    assert spans == [(0, 3), (0, 1), (3, 5), (3, 4), (5, 7)]
    starts = [s for s, _ in spans]
    assert starts == sorted(starts)  # arrival order
