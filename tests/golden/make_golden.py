"""Generates tests/golden/golden.json from the REFERENCE's own code.

Run where the reference tree exists (it is compiled by oracle/Makefile into
oracle/_ref/libref_serial.so, the reference headers plus stand-in TBB /
Boost / robin_set headers, serial scheduler):

    python tests/golden/make_golden.py

The inputs are seeded synthetic point sets regenerated by the tests, plus
the reference's own fixture dummy-data.bin (10,000 x 100, the input its
main() reads by default), which this script stores beside golden.json as
dummy-data.bin.xz so the GPU tests have it on a host without the reference
tree.  Only the reference's outputs are stored for them: SHA-256 digests of
whole arrays plus a few rows verbatim.
"""
from __future__ import annotations

import hashlib
import json
import lzma
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import bindings  # noqa: E402
from sigmod23ann_b200 import workloads  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "golden.json")
FIXTURE = "dummy-data.bin.xz"

# (name, generator kwargs or {"file": fixture}, [(lloyd iterations, maxGroupSize) per repetition], top-up)
CASES = [
    # The reference's schedule on its own fixture: one Lloyd iteration
    # (src/SolutionKmeans.hpp:591), buckets alternating below 200 / 400
    # (:582-587), then the top-up (:604).
    ("dummy_data", {"file": FIXTURE}, [(1, 200), (1, 400), (1, 200), (1, 400)], True),
    ("mix6k", dict(n=6000, d=100, clusters=16, sigma=0.15, seed=7), [(1, 200), (2, 400)], True),
    ("mix3500_leaf64", dict(n=3500, d=100, clusters=8, sigma=0.2, seed=11), [(2, 64)], True),
    ("mix250_one_bucket", dict(n=250, d=100, clusters=4, sigma=0.3, seed=5), [(1, 400)], False),
]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def sets_digest(s: dict) -> str:
    h = hashlib.sha256()
    for key in ("dist", "id", "size", "maxslot", "bound"):
        h.update(np.ascontiguousarray(s[key]).view(np.uint32).tobytes())
    return h.hexdigest()


def case_points(gen: dict) -> np.ndarray:
    if "file" in gen:
        with lzma.open(os.path.join(HERE, gen["file"])) as f:
            raw = f.read()
        n = int(np.frombuffer(raw[:4], np.uint32)[0])
        return np.frombuffer(raw[4:4 + n * 400], np.float32).reshape(n, 100).copy()
    return workloads.gaussian_mixture(**gen)


def main() -> int:
    bindings.build(with_reference=True)
    with open(bindings.REFERENCE_FIXTURE, "rb") as f:
        raw = f.read()
    with lzma.open(os.path.join(HERE, FIXTURE), "wb", preset=9) as f:
        f.write(raw)
    golden = {"cases": {}, "arith": {}, "knnset": {}, "kd_rotation": {}}
    for name, gen, reps, topup in CASES:
        pts = case_points(gen)
        ref = bindings.ReferenceShim(pts)
        ref.reseed(12345)
        entry = {"generator": gen, "reps": reps, "topup": topup, "indices": [], "sets": []}
        for iters, leaf in reps:
            ref.rep(iters, leaf)
            entry["indices"].append(digest(ref.indices()))
            entry["sets"].append(sets_digest(ref.sets()))
        if topup:
            entry["topup_changed"] = ref.topup()
            entry["topup_sets"] = sets_digest(ref.sets())
        final = ref.finalize()
        entry["final"] = digest(final)
        entry["final_rows"] = {str(r): final[r].tolist() for r in (0, 1, len(final) - 1)}
        golden["cases"][name] = entry
        ref.close()
        print(name, "done")
    # The reference's distance() and dot() on seeded vectors (bit patterns).
    rng = np.random.default_rng(3)
    a = rng.standard_normal((64, 100)).astype(np.float32)
    b = rng.standard_normal((64, 100)).astype(np.float32)
    ref = bindings.ReferenceShim(a[:2])
    golden["arith"] = {
        "seed": 3,
        "distance_bits": [int(np.float32(ref.distance(x, y)).view(np.uint32)) for x, y in zip(a, b)],
        "dot_bits": [int(np.float32(ref.dot(x, y)).view(np.uint32)) for x, y in zip(a, b)],
    }
    # KnnSetScannableSimd replays: the reference's known-answer shapes
    # (test/TestKnnSet.cpp:25-71) on the SIMD set, plus ties.
    seqs = {}
    perm = np.random.default_rng(123).permutation(1000)
    seqs["shuffled_1000"] = (perm.astype(np.uint32), (0.01 * perm).astype(np.float32))
    perm100 = np.random.default_rng(123).permutation(100)
    ids = np.concatenate([perm100, [100]]).astype(np.uint32)
    seqs["after_100_plus_small"] = (ids, np.concatenate([0.01 * perm100, [0.0001]]).astype(np.float32))
    tie_ids = np.arange(300, dtype=np.uint32)
    tie_d = np.repeat(np.float32([0.5, 0.25, 0.125]), 100)[np.random.default_rng(9).permutation(300)]
    seqs["ties"] = (tie_ids, tie_d.astype(np.float32))
    dup_ids = np.concatenate([np.arange(150), np.arange(150)]).astype(np.uint32)
    seqs["duplicates"] = (dup_ids, np.concatenate([np.linspace(1, 0, 150), np.linspace(1, 0, 150)]).astype(np.float32))
    for key, (i, d) in seqs.items():
        r = ref.knnset_replay(i, d)
        golden["knnset"][key] = {
            "ids": i.tolist(), "dist_bits": d.view(np.uint32).tolist(),
            "out_ids": r["id"].tolist(), "out_dist_bits": r["dist"].view(np.uint32).tolist(),
            "size": r["size"], "maxslot": r["maxslot"], "bound_bits": int(np.float32(r["bound"]).view(np.uint32)),
        }
    ref.close()
    # SolutionRandomKD::rotateRandom (src/SolutionRandomKD.hpp:258-275) with
    # the solution's 30 new dimensions (:390), its generator at the seed: the
    # rotated values of the reference fixture and of a seeded mixture.
    for name, gen in (("dummy_data", {"file": FIXTURE}),
                      ("mix6k", dict(n=6000, d=100, clusters=16, sigma=0.15, seed=7))):
        pts = case_points(gen)
        ref = bindings.ReferenceShim(pts)
        rot = ref.kd_rotate(30)
        golden["kd_rotation"][name] = {
            "generator": gen, "new_dims": 30, "seed": 12345, "digest": digest(rot),
            "rows_bits": {str(r): rot[r].view(np.uint32).tolist() for r in (0, len(rot) - 1)},
        }
        ref.close()
    with open(OUT, "w") as f:
        json.dump(golden, f, indent=0, sort_keys=True)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())
