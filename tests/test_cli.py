"""The command-line tools: contest-format build (src/main.cpp's shape) and
the grader (src/grade.cpp's arithmetic)."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from sigmod23ann_b200 import workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "sigmod23ann_b200", "cli")


def write_contest_file(path, pts: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(np.uint32(len(pts)).tobytes())
        f.write(np.ascontiguousarray(pts, np.float32).tobytes())


def test_grader_known_answer(knng_lib, tmp_path):
    truth = np.arange(300, dtype=np.uint32).reshape(3, 100)
    test = truth.copy()
    test[1, :50] = 999            # row 1: 50 correct
    test[2] = test[2][::-1]       # order does not matter
    (tmp_path / "t.bin").write_bytes(truth.tobytes())
    (tmp_path / "x.bin").write_bytes(test.tobytes())
    r = subprocess.run([os.path.join(CLI, "knng_grade"), str(tmp_path / "t.bin"), str(tmp_path / "x.bin"), "3"],
                       capture_output=True, text=True, check=True)
    assert "avg percent: 83.3333" in r.stdout and "recall: 0.833333" in r.stdout


def test_build_cli_without_device(knng_lib, tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    write_contest_file(tmp_path / "in.bin", np.zeros((10, 100), np.float32))
    r = subprocess.run([os.path.join(CLI, "knng_build"), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")],
                       capture_output=True, text=True)
    assert r.returncode == 3 and "no sm_100" in r.stderr
    r = subprocess.run([os.path.join(CLI, "knng_build"), str(tmp_path / "in.bin"), str(tmp_path / "out.bin"),
                        "--timed", "100", "100"], capture_output=True, text=True)
    assert r.returncode == 3 and "no sm_100" in r.stderr
    r = subprocess.run([os.path.join(CLI, "knng_build"), str(tmp_path / "in.bin"), str(tmp_path / "out.bin"),
                        "--timed", "100"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
def test_build_cli_matches_oracle(oracle_lib, knng_lib, tmp_path):
    """contest file in -> output.bin out, with the reference's default schedule
    (leaf 200/400 alternating, 1 Lloyd iteration, 8 repetitions, 1 top-up)."""
    pts = workloads.gaussian_mixture(n=2500, d=100, clusters=8, sigma=0.15, seed=31)
    write_contest_file(tmp_path / "in.bin", pts)
    subprocess.run([os.path.join(CLI, "knng_build"), str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), "3", "1"],
                   check=True, capture_output=True)
    ids = np.fromfile(tmp_path / "out.bin", dtype=np.uint32).reshape(2500, 100)
    o = oracle_lib.Oracle(pts, k=100, rng_mode=1, seed=12345)
    for r in range(3):
        o.rep(1, 400 if r % 2 else 200, r)
    o.refine()
    np.testing.assert_array_equal(ids, o.finalize()[0])
    o.finalize()[0].tofile(tmp_path / "truth.bin")
    g = subprocess.run([os.path.join(CLI, "knng_grade"), str(tmp_path / "truth.bin"), str(tmp_path / "out.bin"),
                        "2500"], capture_output=True, text=True, check=True)
    assert "recall: 1.000000" in g.stdout


@pytest.mark.gpu
def test_build_cli_kd_form_matches_oracle(oracle_lib, knng_lib, tmp_path):
    """--kd: the reference's KD solution (5 repetitions of the random-rotation
    KD split by default; here 3, buckets below 300), no top-up."""
    pts = workloads.gaussian_mixture(n=2500, d=100, clusters=8, sigma=0.15, seed=32)
    write_contest_file(tmp_path / "in.bin", pts)
    subprocess.run([os.path.join(CLI, "knng_build"), str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), "--kd", "3",
                    "300"], check=True, capture_output=True)
    ids = np.fromfile(tmp_path / "out.bin", dtype=np.uint32).reshape(2500, 100)
    o = oracle_lib.Oracle(pts, k=100, rng_mode=1, seed=12345)
    for r in range(3):
        o.kd_rep(300, 30, 12345, r)
    np.testing.assert_array_equal(ids, o.finalize()[0])
