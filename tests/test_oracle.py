"""CPU tests: the oracle against the reference's golden outputs, known-answer
set behaviour (test/TestKnnSet.cpp re-expressed), arithmetic order, and
generators.  No GPU needed."""
from __future__ import annotations

import os

import numpy as np
import pytest

from helpers import case_points, digest, sets_digest
from sigmod23ann_b200 import workloads


def test_oracle_matches_reference_golden(oracle_lib, golden):
    """The C++ restatement reproduces the reference's own outputs bit for bit:
    index permutation after every repetition, full set state, top-up, final ids."""
    for name, case in golden["cases"].items():
        pts = case_points(case["generator"])
        o = oracle_lib.Oracle(pts, k=100, rng_mode=0, seed=12345)
        for r, (iters, leaf) in enumerate(case["reps"]):
            o.rep(iters, leaf, r)
            assert digest(o.indices()) == case["indices"][r], f"{name} rep {r} indices"
            assert sets_digest(o.sets()) == case["sets"][r], f"{name} rep {r} sets"
        if case["topup"]:
            assert o.refine() == case["topup_changed"]
            assert sets_digest(o.sets()) == case["topup_sets"], f"{name} top-up"
        final, _ = o.finalize()
        assert digest(final) == case["final"], f"{name} final"
        for row, ids in case["final_rows"].items():
            assert final[int(row)].tolist() == ids


def test_oracle_arithmetic_matches_reference(oracle_lib, golden):
    rng = np.random.default_rng(golden["arith"]["seed"])
    a = rng.standard_normal((64, 100)).astype(np.float32)
    b = rng.standard_normal((64, 100)).astype(np.float32)
    dist = [int(np.float32(oracle_lib.distance(x, y)).view(np.uint32)) for x, y in zip(a, b)]
    dot = [int(np.float32(oracle_lib.dot(x, y)).view(np.uint32)) for x, y in zip(a, b)]
    assert dist == golden["arith"]["distance_bits"]
    assert dot == golden["arith"]["dot_bits"]


def test_distance_is_symmetric_and_order_sensitive(oracle_lib):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(100).astype(np.float32)
    b = rng.standard_normal(100).astype(np.float32)
    assert oracle_lib.distance(a, b) == oracle_lib.distance(b, a)
    # The canonical order differs from a plain left-to-right float32 sum in general.
    plain = np.float32(0)
    for x, y in zip(a, b):
        plain = np.float32(plain + np.float32(x - y) * np.float32(x - y))
    assert abs(oracle_lib.distance(a, b) - float(plain)) < 1e-3 * float(plain)


def test_knnset_replays_match_reference(oracle_lib, golden):
    for key, g in golden["knnset"].items():
        ids = np.array(g["ids"], np.uint32)
        d = np.array(g["dist_bits"], np.uint32).view(np.float32)
        r = oracle_lib.knnset_replay(100, ids, d)
        assert r["id"].tolist() == g["out_ids"], key
        assert r["dist"].view(np.uint32).tolist() == g["out_dist_bits"], key
        assert r["size"] == g["size"] and r["maxslot"] == g["maxslot"], key
        assert int(np.float32(r["bound"]).view(np.uint32)) == g["bound_bits"], key


def test_knnset_known_answers(oracle_lib):
    """test/TestKnnSet.cpp:25-71, on the set the hot path uses."""
    # Bound stays FLT_MAX while filling, then is the maximum (0.99) at 100.
    ids = np.arange(100, dtype=np.uint32)
    d = (0.01 * np.arange(100)).astype(np.float32)
    for i in range(1, 100):
        r = oracle_lib.knnset_replay(100, ids[:i], d[:i])
        assert r["size"] == i and r["bound"] == np.finfo(np.float32).max
    r = oracle_lib.knnset_replay(100, ids, d)
    assert r["bound"] == pytest.approx(0.99) and r["maxslot"] == 99
    # After 100 shuffled inserts a smaller new id evicts the largest: bound 0.98.
    perm = np.random.default_rng(123).permutation(100)
    r = oracle_lib.knnset_replay(100, np.append(perm, 100).astype(np.uint32),
                                 np.append(0.01 * perm, 0.0001).astype(np.float32))
    assert r["bound"] == pytest.approx(0.98)
    # 1000 shuffled candidates: the set ends with ids 0..99.
    perm = np.random.default_rng(123).permutation(1000)
    r = oracle_lib.knnset_replay(100, perm.astype(np.uint32), (0.01 * perm).astype(np.float32))
    assert sorted(r["id"].tolist()) == list(range(100))
    # contains: a repeated id is rejected, full or not.
    r = oracle_lib.knnset_replay(100, np.array([99, 99], np.uint32), np.array([0.1, 0.05], np.float32))
    assert r["size"] == 1 and r["id"][0] == 99 and r["dist"][0] == np.float32(0.1)


def test_knnset_tie_rule(oracle_lib):
    """getMaxIdx picks, among equal maxima, the smallest slot % 8 then slot / 8."""
    d = np.full(100, 0.5, np.float32)
    r = oracle_lib.knnset_replay(100, np.arange(100, dtype=np.uint32), d)
    assert r["maxslot"] == 0
    d[[3, 11, 19]] = 0.9
    r = oracle_lib.knnset_replay(100, np.arange(100, dtype=np.uint32), d)
    assert r["maxslot"] == 3
    d[[3]] = 0.1
    r = oracle_lib.knnset_replay(100, np.arange(100, dtype=np.uint32), d)
    assert r["maxslot"] == 11


def test_sampling_rules(oracle_lib):
    # Values quoted in the reference's comments (src/SolutionKmeans.hpp:52, :70).
    assert oracle_lib.start_count(10_000_000) == 129
    assert oracle_lib.start_count(1220) == 16
    assert 53_000 < oracle_lib.sample_count(10_000_000) < 54_500
    assert oracle_lib.sample_count(3000) == pytest.approx(400, rel=0.05)


def test_counter_rng_range(oracle_lib):
    for (s, e) in [(0, 1), (5, 9), (100, 1_000_000), (0, 2**32 - 1)]:
        vals = [oracle_lib.counter_position(7, 3, s, e, 0, t) for t in range(200)]
        assert all(s <= v < e for v in vals)
    assert oracle_lib.counter_position(7, 3, 0, 1000, 0, 1) != oracle_lib.counter_position(7, 3, 0, 1000, 1, 1) or \
        oracle_lib.counter_position(7, 3, 0, 1000, 0, 2) != oracle_lib.counter_position(7, 3, 0, 1000, 1, 2)


def test_oracle_degenerate_input_terminates(oracle_lib):
    """Identical points make the reference loop forever; the oracle falls back
    to midpoint splits and still fills every set."""
    pts = np.zeros((700, 100), np.float32)
    o = oracle_lib.Oracle(pts, k=10, rng_mode=1, seed=1)
    o.rep(1, 100, 0)
    s = o.sets()
    assert (s["size"] == 10).all()
    assert (s["dist"] == 0).all()


def test_counter_mode_rep_is_deterministic(oracle_lib):
    pts = workloads.gaussian_mixture(n=2500, d=64, clusters=8, seed=2)
    a = oracle_lib.Oracle(pts, k=20, rng_mode=1, seed=99)
    b = oracle_lib.Oracle(pts, k=20, rng_mode=1, seed=99)
    a.rep(2, 128, 0)
    b.rep(2, 128, 0)
    assert np.array_equal(a.indices(), b.indices())
    assert sets_digest(a.sets()) == sets_digest(b.sets())


@pytest.mark.skipif(not os.path.isdir(__import__("oracle.bindings").bindings.REFERENCE_SRC),
                    reason="needs the reference tree")
def test_oracle_equals_reference_on_fresh_input(oracle_lib):
    """Cross-check on an input the fixtures do not cover (only where the
    reference sources exist)."""
    pts = workloads.gaussian_mixture(n=4200, d=100, clusters=12, sigma=0.12, seed=21)
    ref = oracle_lib.ReferenceShim(pts)
    ref.reseed(12345)
    o = oracle_lib.Oracle(pts, k=100, rng_mode=0, seed=12345)
    for r, (iters, leaf) in enumerate([(2, 300), (1, 150)]):
        ref.rep(iters, leaf)
        o.rep(iters, leaf, r)
        assert np.array_equal(ref.indices(), o.indices())
        assert sets_digest(ref.sets()) == sets_digest(o.sets())


def test_kd_rotation_matches_reference_golden(oracle_lib, golden):
    """The restated rotateRandom (vectors from the seeded mt19937, the
    reference's normalisation and Gram-Schmidt, its dot) reproduces the
    reference's rotated values bit for bit."""
    for name, g in golden["kd_rotation"].items():
        pts = case_points(g["generator"])
        o = oracle_lib.Oracle(pts, k=10)
        rot = o.kd_rotate(oracle_lib.kd_vectors(g["new_dims"], pts.shape[1], g["seed"]))
        assert digest(rot) == g["digest"], name
        for row, bits in g["rows_bits"].items():
            assert rot[int(row)].view(np.uint32).tolist() == bits


def test_kd_oracle_buckets_and_degenerate_input(oracle_lib):
    """The KD restatement tiles the points with buckets below max_leaf and
    fills every set from its bucket; identical points (zero variance, every
    split one-sided) end in midpoint splits."""
    pts = workloads.gaussian_mixture(n=3000, d=100, clusters=8, sigma=0.2, seed=4)
    o = oracle_lib.Oracle(pts, k=100, rng_mode=1, seed=5)
    o.kd_rep(300, 30, 5, 0)
    idx = o.indices()
    assert np.array_equal(np.sort(idx), np.arange(3000))
    t = o.trace()
    order = np.argsort(t["leaf_start"])
    s, e = t["leaf_start"][order], t["leaf_end"][order]
    assert s[0] == 0 and e[-1] == 3000 and np.array_equal(s[1:], e[:-1])
    assert (e - s).max() < 300
    size = o.sets()["size"]
    for a, b in zip(s, e):
        assert (size[idx[a:b]] == min(100, b - a - 1)).all()
    same = np.ones((700, 100), np.float32)
    o2 = oracle_lib.Oracle(same, k=10, rng_mode=1, seed=1)
    o2.kd_rep(200, 30, 1, 0)
    t2 = o2.trace()
    assert sorted(zip(t2["leaf_start"].tolist(), t2["leaf_end"].tolist())) == [(0, 175), (175, 350), (350, 525),
                                                                               (525, 700)]


@pytest.mark.skipif(not os.path.isdir(__import__("oracle.bindings").bindings.REFERENCE_SRC),
                    reason="needs the reference tree")
def test_kd_rotation_equals_reference_on_fresh_input(oracle_lib):
    pts = workloads.gaussian_mixture(n=2000, d=100, clusters=5, sigma=0.3, seed=31)
    ref = oracle_lib.ReferenceShim(pts)
    want = ref.kd_rotate(30)
    got = oracle_lib.Oracle(pts, k=10).kd_rotate(oracle_lib.kd_vectors(30, 100, 12345))
    assert np.array_equal(want.view(np.uint32), got.view(np.uint32))


def test_workload_generators():
    a = workloads.gaussian_mixture(1000, 100, 8, 0.15, seed=0)
    b = workloads.gaussian_mixture(1000, 100, 8, 0.15, seed=0)
    assert a.dtype == np.float32 and a.shape == (1000, 100) and np.array_equal(a, b)
    s = workloads.zipf_sizes(10_000_000, 1024, 1.1)
    assert s.sum() == 10_000_000 and s[0] > s[1] > s[-1] > 0
    c = workloads.subspace_mixture(5000, 100, clusters=16, seed=1)
    assert c.shape == (5000, 100) and np.isfinite(c).all()


def test_groundtruth_and_recall():
    from sigmod23ann_b200 import groundtruth

    pts = workloads.gaussian_mixture(600, 64, 4, 0.2, seed=3)
    q = np.arange(0, 600, 7)
    gt = groundtruth.exact_knn_numpy(pts, q, 10)
    d = ((pts[q][:, None, :].astype(np.float64) - pts[None, :, :]) ** 2).sum(-1)
    d[np.arange(len(q)), q] = np.inf
    brute = np.argsort(d, axis=1, kind="stable")[:, :10]
    assert (np.sort(gt, 1) == np.sort(brute, 1)).mean() > 0.99
    full = np.zeros((600, 10), np.int64)
    full[q] = gt
    assert groundtruth.recall(full, gt, q) == 1.0


def test_lloyd_sums_follow_point_order(oracle_lib):
    """The oracle's centroid sums run one point at a time in the Lloyd set's
    order (src/SolutionKmeans.hpp:170-175): on data whose partial sums round,
    the result is the one-at-a-time mean, which 256-point partials miss."""
    from helpers import mean_in_order, rounding_points

    pts = rounding_points()
    a = pts[:512, 0]
    assert mean_in_order(a) == np.float32(0.5)
    assert mean_in_order(a, 256) == np.float32(0.5) + np.float32(2.0 ** -24)
    o = oracle_lib.Oracle(pts, k=10)
    coefs, off, ok = o.lloyd(np.arange(1024, dtype=np.uint32), pts[0], pts[512], 2)
    assert ok
    # c1 = (0.5, 1000, 0, ...), c2 = (0, -1000, 0.5, ...): coefs = (c1 - c2) / 2.
    assert coefs[0] == np.float32(0.25) and coefs[2] == np.float32(-0.25) and coefs[1] == np.float32(1000.0)


def test_kd_oracle_edge_cases(oracle_lib):
    """One bucket when n < max_leaf (every pair offered); one rotated
    dimension; the same seed and repetition give the same permutation, another
    repetition (another rotation and draws) a different one."""
    pts = workloads.gaussian_mixture(n=150, d=100, clusters=3, sigma=0.3, seed=9)
    o = oracle_lib.Oracle(pts, k=10, rng_mode=1, seed=1)
    o.kd_rep(400, 30, 1, 0)
    t = o.trace()
    assert t["leaf_start"].tolist() == [0] and t["leaf_end"].tolist() == [150]
    assert np.array_equal(o.indices(), np.arange(150))
    assert (o.sets()["size"] == 10).all()
    big = workloads.gaussian_mixture(n=2000, d=100, clusters=6, sigma=0.2, seed=10)
    a = oracle_lib.Oracle(big, k=10, rng_mode=1, seed=1)
    a.kd_rep(200, 1, 5, 0)
    ta = a.trace()
    assert (ta["leaf_end"] - ta["leaf_start"]).max() < 200
    b = oracle_lib.Oracle(big, k=10, rng_mode=1, seed=1)
    b.kd_rep(200, 1, 5, 0)
    assert np.array_equal(a.indices(), b.indices())
    b.kd_rep(200, 1, 5, 1)
    assert not np.array_equal(a.indices(), b.indices())
