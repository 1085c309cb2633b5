"""CPU tests of the C ABI: the library builds, loads and exports every symbol
include/knng.h declares; host-only entry points behave.  No kernel runs."""
from __future__ import annotations

import ctypes
import os
import re

import pytest

from sigmod23ann_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols() -> list[str]:
    names = []
    for h in ("knng.h",):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(knng_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(api.EXPORTED)


def test_library_exports_every_declared_symbol(knng_lib):
    for name in declared_symbols():
        assert hasattr(knng_lib, name), name


def test_default_params_are_the_references(knng_lib):
    p = api.default_params()
    assert (p.k, p.max_leaf, p.max_leaf_odd, p.lloyd_iters, p.small_threshold, p.seed) == (100, 200, 400, 1, 3000,
                                                                                            12345)
    assert p.refine == 1 and p.precision == api.PRECISION_FP32


def test_kd_params_are_the_kd_forms(knng_lib):
    """kd_params(): the reference's KD form (src/SolutionRandomKD.hpp:390-401):
    five repetitions, buckets below 400 points, no neighbour-of-neighbour pass."""
    p = api.kd_params()
    assert (p.k, p.reps, p.max_leaf, p.max_leaf_odd, p.refine, p.seed) == (100, 5, 400, 0, 0, 12345)
    assert api.kd_params(reps=2, k=10).reps == 2


def test_status_strings(knng_lib):
    for code in range(9):
        assert knng_lib.knng_status_string(code)
    assert knng_lib.knng_status_string(0) == b"ok"


def test_struct_layouts_match_header(tmp_path):
    """Sizes and field offsets of the ctypes mirrors equal the C header's (a C
    program compiled against include/knng.h prints them)."""
    import subprocess

    assert ctypes.sizeof(api.Params) == 40
    assert ctypes.sizeof(api.Stats) == 11 * 8 + 21 * 8
    checks = [("knng_stats", name) for name, _ in api.Stats._fields_] + \
             [("knng_params", name) for name, _ in api.Params._fields_]
    src = tmp_path / "layout.c"
    body = "".join(f'    printf("%zu\\n", offsetof({t}, {f}));\n' for t, f in checks)
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "knng.h"\nint main(void) {\n'
                   '    printf("%zu\\n%zu\\n", sizeof(knng_stats), sizeof(knng_params));\n' + body +
                   "    return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [ctypes.sizeof(api.Stats), ctypes.sizeof(api.Params)] + \
           [getattr(api.Stats if t == "knng_stats" else api.Params, f).offset for t, f in checks]
    assert got == want


def test_create_without_device_reports_no_device(knng_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.KnngError) as e:
        api.KnngContext(0)
    assert e.value.status == 7


def test_cpp_wrapper_compiles_links_and_reports_no_device(knng_lib, tmp_path):
    """A C++ caller of the reference's shape (float[][112] rows) builds against
    include/knng.hpp and libknng.so; without a GPU the wrapper throws with
    KNNG_ERR_NO_DEVICE's message."""
    import subprocess

    import torch

    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include <cstdio>
#include <cstdlib>
#include "knng.hpp"
static float pts[4][112];
int main() {
    std::vector<std::vector<uint32_t>> result;
    try {
        knng_b200::constructResult(pts, 4, result);
        knng_b200::constructResultTimed(pts, 4, result, 50, 50);
        knng_b200::constructResultKD(pts, 4, result);
    } catch (const std::runtime_error& e) {
        std::printf("%s\n", e.what());
        return 3;
    }
    std::printf("rows %zu\n", result.size());
    return result.size() == 4 ? 0 : 1;
}
''')
    exe = tmp_path / "caller"
    libdir = os.path.join(ROOT, "sigmod23ann_b200")
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    f"-L{libdir}", "-lknng", f"-Wl,-rpath,{libdir}"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    if torch.cuda.is_available():
        assert r.returncode == 0, r.stdout + r.stderr
    else:
        assert r.returncode == 3 and "no sm_100" in r.stdout, r.stdout + r.stderr


def test_job_reservation_arithmetic(knng_lib):
    """A served job reserves its points, order, sets, refinement lists and
    survivor storage plus fixed scratch: linear in n, growing with d and k."""
    from sigmod23ann_b200 import job_reservation

    fixed = 256 << 20
    r1 = job_reservation(1_000_000, 100, 100)
    per_point = 100 * 4 + 8 + (100 * 8 + 12) + (100 * 8 + 40) + 100 * 96
    assert r1 == fixed + 1_000_000 * per_point
    assert job_reservation(2_000_000, 100, 100) - fixed == 2 * (r1 - fixed)
    assert job_reservation(1_000_000, 128, 100) > r1 > job_reservation(1_000_000, 64, 100)
    assert job_reservation(1_000_000, 100, 10) < r1


def test_server_without_device_reports_no_device(knng_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.KnngError) as e:
        api.KnngServer(0)
    assert e.value.status == 7


def test_null_handles_are_refused(knng_lib):
    """Entry points given a null context or server answer
    KNNG_ERR_INVALID_ARGUMENT without touching a device."""
    from sigmod23ann_b200.api import JobInfo, Params

    p = Params()
    knng_lib.knng_default_params(ctypes.byref(p))
    job = ctypes.c_uint64()
    info = JobInfo()
    assert knng_lib.knng_server_submit(None, None, 10, 100, 400, ctypes.byref(p), None, None, ctypes.byref(job)) == 1
    assert knng_lib.knng_server_poll(None, 1, ctypes.byref(info)) == 1
    assert knng_lib.knng_server_wait(None, 1, 0, ctypes.byref(info)) == 1
    assert knng_lib.knng_server_release(None, 1) == 1
    assert knng_lib.knng_server_destroy(None) == 1
    assert knng_lib.knng_server_job_error(None, 1) == b"null server"
    assert knng_lib.knng_build_batch(None, None, 10, 100, 400, None, 1, 0, ctypes.byref(p), None, None, None) == 1
    out = ctypes.c_void_p()
    assert knng_lib.knng_server_create(0, 0, 0, ctypes.byref(out)) == 1  # max_running must be >= 1


def test_set_state_entry_points_refuse_null(knng_lib):
    assert knng_lib.knng_save_sets(None, b"/nonexistent") == 1
    assert knng_lib.knng_load_sets(None, b"/nonexistent") == 1


def test_schedule_and_tuning_entry_points_refuse_null(knng_lib):
    """The adaptive schedule, the bucket-pass autotuner and the wait-limit
    diagnostic answer KNNG_ERR_INVALID_ARGUMENT for a null context."""
    ms = (ctypes.c_double * 4)()
    choice = ctypes.c_uint32()
    assert knng_lib.knng_tune_buckets(None, 1025, 2, 3000, 1, ms, ctypes.byref(choice)) == 1
    assert knng_lib.knng_debug_set_wait_limit(None, 0) == 1
    assert knng_lib.knng_build_adaptive(None, None, 10, 100, 400, None, 0.9, 10, None, None, None) == 1


def test_kd_rotation_entry_point_matches_oracle(knng_lib, oracle_lib):
    """knng_kd_rotation (host only) makes the KD solution's rotation vectors
    bit for bit as the oracle's restatement does, for several seeds and sizes;
    out-of-range sizes are refused."""
    import numpy as np

    for nd, d, seed in [(30, 100, 12345), (8, 100, 7), (32, 100, 2**40 + 3), (1, 100, 0), (16, 128, 99)]:
        mine = api.kd_rotation(nd, d, seed)
        want = oracle_lib.kd_vectors(nd, d, seed)
        assert np.array_equal(mine.view(np.uint32), want.view(np.uint32)), (nd, d, seed)
    out = np.zeros(33 * 100, np.float32)
    ptr = out.ctypes.data_as(ctypes.c_void_p)
    assert knng_lib.knng_kd_rotation(33, 100, 1, ptr) == 1
    assert knng_lib.knng_kd_rotation(0, 100, 1, ptr) == 1
    assert knng_lib.knng_kd_rotation(4, 100, 1, None) == 1
    assert knng_lib.knng_run_rep_kd(None, 400, 30, 1, 0, None) == 1
    assert knng_lib.knng_build_kd(None, None, 0, 100, 0, None, 30, None, None, None) == 1
