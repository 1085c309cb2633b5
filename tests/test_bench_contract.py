"""CPU test of bench.py's reference arm: it runs the reference's own CPU code
(compiled from its sources into oracle/_ref) on a small sample and prints one
JSON line with the keys the measurement contract asks for."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    sys.path.insert(0, ROOT)
    from oracle import bindings

    if not bindings.reference_available():
        pytest.skip("the reference was not compiled here")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", KNNG_REF_THREADS="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "20000",
                        "--steps", "1", "--warmup", "0", "--cpu-seconds", "0.5"],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "points/s"
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["config"]["workload"].startswith("20,000 x 100 f32")


def test_kd_cpu_baseline_leg_times_the_oracle_port():
    """The --kd line's CPU baseline: the oracle's KD repetition on a prefix of
    the bench's points, one host thread."""
    sys.path.insert(0, ROOT)
    import bench

    r = bench.oracle_kd_rate(3000, 257, 0.2)
    assert r["kind"] == "port" and r["cores"] == 1
    assert r["sample_points"] == 3000 and r["points_per_s_per_rep"] > 0
