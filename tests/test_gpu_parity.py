"""GPU parity tests: the CUDA library, called through the C ABI, against the
oracle (and, through the golden fixtures, against the reference's own code).

Bar: bit-exact index permutations, set states (distance bits, ids, sizes,
max slots, bounds) and final ids, given the same hyperplanes and buckets."""
from __future__ import annotations

import os

import numpy as np
import pytest

from helpers import assert_sets_equal, case_points, digest, feed_trace, sets_digest
from sigmod23ann_b200 import KnngContext, KnngError, default_params, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(knng_lib):
    c = KnngContext(0)
    yield c
    c.close()


def oracle_rep_and_feed(oracle_lib, ctx, pts, reps, k=100, check_each=True):
    """Runs the oracle with the reference RNG, then drives the GPU with the
    oracle's hyperplanes and buckets; returns (oracle, per-rep checks)."""
    o = oracle_lib.Oracle(pts, k=k, rng_mode=0, seed=12345)
    ctx.load_points(pts)
    ctx.reset_sets(k)
    for r, (iters, leaf) in enumerate(reps):
        o.rep(iters, leaf, r)
        t = o.trace()
        ctx.begin_rep()
        feed_trace(ctx, t)
        np.testing.assert_array_equal(ctx.indices(), o.indices())
        ctx.process_leaves(t["leaf_start"], t["leaf_end"])
        if check_each:
            assert_sets_equal(ctx.sets(), o.sets(), f"rep {r}")
    return o


def test_golden_cases_through_gpu(oracle_lib, ctx, golden):
    """Reference outputs (fixtures) reproduced by the GPU fed the hyperplanes."""
    for name, case in golden["cases"].items():
        pts = case_points(case["generator"])
        o = oracle_lib.Oracle(pts, k=100, rng_mode=0, seed=12345)
        ctx.load_points(pts)
        ctx.reset_sets(100)
        for r, (iters, leaf) in enumerate(case["reps"]):
            o.rep(iters, leaf, r)
            t = o.trace()
            ctx.begin_rep()
            feed_trace(ctx, t)
            assert digest(ctx.indices()) == case["indices"][r], f"{name} rep {r} indices"
            ctx.process_leaves(t["leaf_start"], t["leaf_end"])
            assert sets_digest(ctx.sets()) == case["sets"][r], f"{name} rep {r} sets"
        if case["topup"]:
            assert ctx.refine() == case["topup_changed"]
            assert sets_digest(ctx.sets()) == case["topup_sets"], f"{name} top-up"
        assert digest(ctx.finalize()) == case["final"], f"{name} final"


def test_split_leaf_parity_config1_shape(oracle_lib, ctx):
    """20k points of the 64-Gaussian config-1 distribution, leaf <= 256, 2 Lloyd
    iterations, 3 repetitions: every permutation and set state bit-exact."""
    pts = workloads.gaussian_mixture(n=20_000, d=100, clusters=64, sigma=0.15, seed=0)
    o = oracle_rep_and_feed(oracle_lib, ctx, pts, [(2, 257)] * 3)
    ids, dist = ctx.finalize(want_dists=True)
    oids, odist = o.finalize()
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(dist.view(np.uint32), odist.view(np.uint32))


def test_refine_parity(oracle_lib, ctx):
    pts = workloads.gaussian_mixture(n=5000, d=100, clusters=16, sigma=0.2, seed=4)
    o = oracle_rep_and_feed(oracle_lib, ctx, pts, [(1, 200), (1, 400)])
    assert ctx.refine() == o.refine()
    assert_sets_equal(ctx.sets(), o.sets(), "refine")


def test_refine_parity_unfilled_sets(oracle_lib, ctx):
    """Sets below k after tiny buckets: unfilled slots read as id 0 (quirk of
    src/SolutionKmeans.hpp:494)."""
    pts = workloads.gaussian_mixture(n=3000, d=100, clusters=8, sigma=0.2, seed=8)
    o = oracle_rep_and_feed(oracle_lib, ctx, pts, [(1, 40)])
    assert (o.sets()["size"] < 100).all()
    assert ctx.refine() == o.refine()
    assert_sets_equal(ctx.sets(), o.sets(), "refine unfilled")


def test_farthest_pair_and_lloyd_parity(oracle_lib, ctx):
    """Device seeding and Lloyd iterations from the oracle's seeds / samples
    give the oracle's starting centres and hyperplanes."""
    pts = workloads.gaussian_mixture(n=12_000, d=100, clusters=32, sigma=0.15, seed=6)
    o = oracle_lib.Oracle(pts, k=100, rng_mode=0, seed=12345)
    o.rep(2, 300, 0)
    t = o.trace()
    # Replay the permutation each node saw: feed level by level, checking per level.
    ctx.load_points(pts)
    ctx.reset_sets(100)
    ctx.begin_rep()
    from helpers import trace_levels

    for sel in trace_levels(t):
        off = np.zeros(len(sel) + 1, np.uint64)
        pos = []
        for j, i in enumerate(sel):
            p = t["start_pos"][int(t["start_off"][i]):int(t["start_off"][i + 1])]
            pos.append(p)
            off[j + 1] = off[j] + len(p)
        first, second, ok = ctx.farthest_pair(off, np.concatenate(pos))
        assert ok.all()
        idx = ctx.indices()
        for j, i in enumerate(sel):
            c1 = pts[idx[pos[j][first[j]]]]
            c2 = pts[idx[pos[j][second[j]]]]
            np.testing.assert_array_equal(c1, t["c1_start"][i])
            np.testing.assert_array_equal(c2, t["c2_start"][i])
        lo = np.zeros(len(sel) + 1, np.uint64)
        lpos = []
        for j, i in enumerate(sel):
            p = t["lloyd_pos"][int(t["lloyd_off"][i]):int(t["lloyd_off"][i + 1])]
            lpos.append(p)
            lo[j + 1] = lo[j] + len(p)
        coefs, offs, ok = ctx.lloyd(t["start"][sel], t["end"][sel], lo,
                                    np.concatenate(lpos) if lpos else np.zeros(0, np.uint32),
                                    t["c1_start"][sel], t["c2_start"][sel], 2)
        assert ok.all()
        np.testing.assert_array_equal(coefs.view(np.uint32), t["coefs"][sel].view(np.uint32))
        np.testing.assert_array_equal(offs.view(np.uint32), t["offset"][sel].view(np.uint32))
        mids = ctx.split_nodes(t["start"][sel], t["end"][sel], coefs, offs)
        np.testing.assert_array_equal(mids, t["mid"][sel])
    np.testing.assert_array_equal(ctx.indices(), o.indices())


def test_lloyd_sums_round_in_point_order(oracle_lib, ctx):
    """Centroid sums whose partial sums round (values from 2^-45 to 2^8): the
    device adds one point at a time in the Lloyd set's order, as the
    reference does, so its hyperplanes equal the oracle's bit for bit; 256-point
    partial sums would move dims 0 and 2 by one float ulp.  Covers a small
    node (the whole range), a large node's position list, and a shuffled list
    with repeats (samples are drawn with replacement)."""
    from helpers import rounding_points

    rng = np.random.default_rng(5)
    shuffled = rng.integers(0, 1024, 3000).astype(np.uint32)
    cases = [(1024, np.zeros(0, np.uint32)), (4096, np.arange(1024, dtype=np.uint32)), (4096, shuffled)]
    for n, plist in cases:
        pts = rounding_points(n)
        ctx.load_points(pts)
        ctx.reset_sets(10)
        ctx.begin_rep()
        off = np.array([0, len(plist)], np.uint64)
        coefs, offs, ok = ctx.lloyd(np.array([0], np.uint32), np.array([n], np.uint32), off, plist,
                                    pts[0:1], pts[512:513], 2)
        o = oracle_lib.Oracle(pts, k=10)
        ids = plist if len(plist) else np.arange(n, dtype=np.uint32)
        oc, oo, ook = o.lloyd(ids, pts[0], pts[512], 2)
        assert ok.all() and ook
        np.testing.assert_array_equal(coefs[0].view(np.uint32), oc.view(np.uint32))
        assert np.float32(offs[0]).view(np.uint32) == np.float32(oo).view(np.uint32)


def test_device_seeded_rep_matches_counter_oracle(oracle_lib, ctx):
    """knng_run_rep (device RNG, device Lloyd, device partition, buckets) equals
    the oracle driven by the same counter RNG."""
    pts = workloads.gaussian_mixture(n=15_000, d=100, clusters=32, sigma=0.15, seed=12)
    o = oracle_lib.Oracle(pts, k=100, rng_mode=1, seed=777)
    ctx.load_points(pts)
    ctx.reset_sets(100)
    for r, leaf in enumerate([257, 400]):
        o.rep(2, leaf, r)
        ctx.run_rep(leaf, 2, 3000, 777, r)
        np.testing.assert_array_equal(ctx.indices(), o.indices())
        s, e = ctx.leaves()
        t = o.trace()
        order = np.argsort(t["leaf_start"])
        np.testing.assert_array_equal(s, t["leaf_start"][order])
        np.testing.assert_array_equal(e, t["leaf_end"][order])
        assert_sets_equal(ctx.sets(), o.sets(), f"device rep {r}")


def test_build_end_to_end_matches_oracle(oracle_lib, ctx):
    pts = workloads.gaussian_mixture(n=8000, d=100, clusters=16, sigma=0.15, seed=13)
    p = default_params(reps=3, max_leaf=200, max_leaf_odd=400, lloyd_iters=2, refine=1, seed=4242)
    ids, dist = ctx.build(pts, p, want_dists=True)
    o = oracle_lib.Oracle(pts, k=100, rng_mode=1, seed=4242)
    for r in range(3):
        o.rep(2, 400 if r % 2 else 200, r)
    o.refine()
    oids, odist = o.finalize()
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(dist.view(np.uint32), odist.view(np.uint32))


def test_config1_full_build_matches_oracle(oracle_lib, ctx):
    """The 100k-point config at full size: 64 Gaussians (sigma 0.15, seed 0),
    k = 100, buckets <= 256, 2 Lloyd iterations, 8 repetitions + 1
    neighbour-of-neighbour pass.  Final ids and distance bits equal the
    oracle's (driven by the same counter RNG)."""
    pts = workloads.gaussian_mixture(n=100_000, d=100, clusters=64, sigma=0.15, seed=0)
    p = default_params(reps=8, max_leaf=257, max_leaf_odd=0, lloyd_iters=2, refine=1, seed=12345)
    ids, dist = ctx.build(pts, p, want_dists=True)
    o = oracle_lib.Oracle(pts, k=100, rng_mode=1, seed=12345)
    for r in range(8):
        o.rep(2, 257, r)
    o.refine()
    oids, odist = o.finalize()
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(dist.view(np.uint32), odist.view(np.uint32))


@pytest.mark.parametrize("d,k", [(64, 10), (128, 50), (100, 1), (64, 128)])
def test_other_shapes(oracle_lib, ctx, d, k):
    pts = workloads.gaussian_mixture(n=3100, d=d, clusters=8, sigma=0.2, seed=d + k)
    p = default_params(k=k, reps=2, max_leaf=150, max_leaf_odd=0, lloyd_iters=1, refine=1, seed=5)
    ids = ctx.build(pts, p)
    o = oracle_lib.Oracle(pts, k=k, rng_mode=1, seed=5)
    for r in range(2):
        o.rep(1, 150, r)
    o.refine()
    np.testing.assert_array_equal(ids, o.finalize()[0])


def test_edge_cases(oracle_lib, ctx):
    # One point: no pairs, row padded with id 1.
    ids = ctx.build(np.ones((1, 100), np.float32), default_params(reps=1, refine=1))
    assert ids.shape == (1, 100) and (ids == 1).all()
    # Fewer points than k: rows hold n-1 neighbours then padding.
    pts = workloads.gaussian_mixture(n=37, d=100, clusters=2, seed=1)
    ids = ctx.build(pts, default_params(reps=2, refine=1))
    for i in range(37):
        assert sorted(ids[i, :36].tolist()) == sorted(set(range(37)) - {i})
        assert (ids[i, 36:] == 1).all()
    # Identical points: the reference loops forever; here every split falls back
    # to the index midpoint and every distance is 0.
    pts = np.zeros((900, 100), np.float32)
    ids, dist = ctx.build(pts, default_params(k=16, reps=1, max_leaf=100, max_leaf_odd=0, refine=0),
                          want_dists=True)
    assert (dist == 0).all()
    o = oracle_lib.Oracle(pts, k=16, rng_mode=1, seed=12345)
    o.rep(1, 100, 0)
    np.testing.assert_array_equal(ids, o.finalize()[0])
    # Buckets of size 1 and 2 through the stepwise API.
    pts = workloads.gaussian_mixture(n=10, d=100, clusters=2, seed=2)
    ctx.load_points(pts)
    ctx.reset_sets(4)
    ctx.process_leaves([0, 1, 3], [1, 3, 10])
    o = oracle_lib.Oracle(pts, k=4)
    o.process_leaves(np.array([0, 1, 3]), np.array([1, 3, 10]))
    assert_sets_equal(ctx.sets(), o.sets(), "tiny buckets")


@pytest.mark.parametrize("d,m,n", [(100, 128, 128), (100, 77, 113), (64, 128, 16), (128, 5, 128)])
def test_tensor_core_tile_against_fp64(ctx, d, m, n):
    """One tcgen05 kind::f16 tile (FP16 operands, FP32 accumulation) against
    an FP64 matmul: the error stays inside the FP16 operand-rounding bound
    (2^-11 relative per operand, so 2^-10 of sum |a_k b_k|) that the
    refinement filter's margin is built on, with room to spare."""
    from sigmod23ann_b200.api import debug_tile_gram

    rng = np.random.default_rng(d + m + n)
    a = rng.standard_normal((m, d)).astype(np.float32)
    b = rng.standard_normal((n, d)).astype(np.float32)
    g = debug_tile_gram(ctx, a, b)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    scale = np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64).T
    err = np.abs(g - ref)
    assert (err <= 2.0 ** -10 * scale + 1e-6).all(), float((err / scale).max())
    # and the operands really were rounded to FP16 (not used in FP32)
    assert float((err / scale).max()) > 2.0 ** -20


@pytest.fixture(scope="module")
def refine_case(knng_lib):
    """Sets after two repetitions of a 20k-point build, and the sets after one
    neighbour-of-neighbour pass of the one-warp-per-point kernel."""
    pts = workloads.gaussian_mixture(n=20_000, d=100, clusters=32, sigma=0.15, seed=3)
    p = default_params(reps=2, max_leaf=257, max_leaf_odd=0, lloyd_iters=2, refine=0, seed=9)
    with KnngContext(0) as a:
        a.build(pts, p)
        s0 = a.sets()
    os.environ["KNNG_REFINE"] = "pointwise"
    try:
        with KnngContext(0) as b:
            b.load_points(pts)
            b.reset_sets(100)
            b.set_sets(s0)
            changed = b.refine()
            s1 = b.sets()
    finally:
        del os.environ["KNNG_REFINE"]
    return pts, s0, changed, s1


@pytest.mark.parametrize("slots,pool,order", [(None, None, None), (None, None, "id"), ("16", "1000000", None),
                                              ("0", "1000000", None), ("16", "64", None), ("0", "0", None)])
def test_refine_join_equals_pointwise(refine_case, monkeypatch, slots, pool, order):
    """The tensor-core local join and the one-warp-per-point pass leave
    identical sets, however the join's survivors are stored: per-point slots
    sized from the budget, small or no slots with the rest pooled, or pool
    regions so small that points lose records and are redone point by point;
    and whichever order the join takes the points in (leaf order or id order)."""
    from sigmod23ann_b200.api import Stats

    pts, s0, changed, s1 = refine_case
    if order is not None:
        monkeypatch.setenv("KNNG_JOIN_ORDER", order)
    if slots is not None:
        monkeypatch.setenv("KNNG_REFINE_SLOTS", slots)
    if pool is not None:
        monkeypatch.setenv("KNNG_REFINE_POOL", pool)
    st = Stats()
    with KnngContext(0) as a:
        a.load_points(pts)
        a.reset_sets(100)
        a.set_sets(s0)
        # The join walks the points in the order the context's index
        # permutation gives (a repetition's leaf order); any permutation must
        # give the same sets.
        a.set_indices(np.random.default_rng(11).permutation(len(pts)).astype(np.uint32))
        ch = a.refine(st)
        sa = a.sets()
    assert ch == changed
    assert_sets_equal(sa, s1, "join vs pointwise")
    if pool is not None and int(pool) >= 1000000:
        assert st.refine_overflow > 0 and st.refine_lost == 0  # records pooled, none lost
    if pool is not None and int(pool) < 1000000:
        assert st.refine_lost > 0  # points redone point by point


def test_invalid_arguments(ctx):
    with pytest.raises(KnngError) as e:
        ctx.build(np.zeros((10, 99), np.float32))
    assert e.value.status == 6
    with pytest.raises(KnngError) as e:
        ctx.build(np.zeros((10, 100), np.float32), default_params(k=0))
    assert e.value.status == 6
    ctx.load_points(np.zeros((10, 100), np.float32))
    ctx.reset_sets(4)
    with pytest.raises(KnngError) as e:
        ctx.process_leaves([0, 5], [6, 10])
    assert e.value.status == 1
    with pytest.raises(KnngError) as e:
        ctx.set_indices(np.zeros(10, np.uint32))
    assert e.value.status == 1


def test_budget_is_enforced(knng_lib):
    c = KnngContext(0, hbm_budget_bytes=1 << 20)
    with pytest.raises(KnngError) as e:
        c.build(np.zeros((100_000, 100), np.float32))
    assert e.value.status == 4
    c.close()


def test_batched_build_equals_builds_alone(knng_lib):
    """Several independent point sets in one batched build give, per set, the
    same ids and distances (bit for bit) as building each set alone -- a set
    smaller than k + 1 (whose neighbour sets never fill) included."""
    sizes = [3000, 1500, 50, 1200, 7000]
    sets = [workloads.gaussian_mixture(n=m, d=100, clusters=6, sigma=0.2, seed=40 + i) for i, m in enumerate(sizes)]
    params = default_params(reps=2, refine=1, max_leaf=257, max_leaf_odd=0, lloyd_iters=2, seed=77)
    with KnngContext(0) as ctx:
        b_ids, b_d = ctx.build_batch(sets, params, want_dists=True)
    for s, pts in enumerate(sets):
        with KnngContext(0) as ctx:
            ids, dist = ctx.build(pts, params, want_dists=True)
        assert np.array_equal(b_ids[s], ids), f"set {s} ids"
        assert np.array_equal(b_d[s].view(np.uint32), dist.view(np.uint32)), f"set {s} distances"


def test_timed_build_equals_fixed_count_build(knng_lib):
    """knng_build_timed (the reference's wall-clock schedule: repetitions with
    alternating bucket bounds while the budget lasts, then passes) builds the
    same graph as knng_build with the repetition and pass counts it reached;
    a budget of 1 ms still runs one repetition."""
    from sigmod23ann_b200.api import Stats

    pts = workloads.gaussian_mixture(n=20_000, d=100, clusters=16, sigma=0.15, seed=4)
    params = default_params(reps=0, refine=1, max_leaf=200, max_leaf_odd=400, lloyd_iters=1, seed=3)
    st = Stats()
    with KnngContext(0) as ctx:
        ids = ctx.build_timed(pts, build_ms=400, refine_ms=2000, params=params, stats=st)
        assert st.reps_done >= 1
        fixed = ctx.build(pts, default_params(reps=int(st.reps_done), refine=int(st.refine_passes_done),
                                              max_leaf=200, max_leaf_odd=400, lloyd_iters=1, seed=3))
        assert np.array_equal(ids, fixed)
        one = Stats()
        ctx.build_timed(pts, build_ms=1, refine_ms=0, params=params, stats=one)
        assert one.reps_done == 1 and one.refine_passes_done == 0


def test_sets_snapshot_and_resume(knng_lib, tmp_path):
    """Two repetitions, the sets saved to a file; a fresh context with the
    same points loads them and runs repetition 2 and a pass: the graph equals
    a straight three-repetition build."""
    pts = workloads.gaussian_mixture(n=20_000, d=100, clusters=16, sigma=0.15, seed=8)
    params = default_params(reps=3, refine=1, max_leaf=257, max_leaf_odd=0, lloyd_iters=2, seed=5)
    with KnngContext(0) as ctx:
        straight = ctx.build(pts, params)
    path = str(tmp_path / "sets.bin")
    with KnngContext(0) as a:
        a.load_points(pts)
        a.reset_sets(100)
        for r in range(2):
            a.run_rep(257, 2, 3000, seed=5, rep_index=r)
        a.save_sets(path)
    with KnngContext(0) as b:
        b.load_points(pts)
        b.load_sets(path)
        b.run_rep(257, 2, 3000, seed=5, rep_index=2)
        b.refine()
        resumed = b.finalize()
    assert np.array_equal(resumed, straight)


@pytest.mark.parametrize("loop", ["device", "host"])
def test_rep_graph_equals_other_level_loops(knng_lib, monkeypatch, loop):
    """A repetition run as one CUDA graph (device-side tree levels under a
    WHILE node, then the persistent bucket pass over the device's leaf list)
    leaves the same index permutation, leaves and sets, bit for bit, as the
    same levels launched one by one and as the host-sequenced levels; over
    several repetitions with alternating bucket bounds, a neighbour-of-
    neighbour pass, and a batch of point sets."""
    pts = workloads.gaussian_mixture(n=30_000, d=100, clusters=32, sigma=0.15, seed=21)

    def run(mode):
        if mode is None:
            monkeypatch.delenv("KNNG_REP_LOOP", raising=False)
        else:
            monkeypatch.setenv("KNNG_REP_LOOP", mode)
        out = []
        with KnngContext(0) as c:
            c.load_points(pts)
            c.reset_sets(100)
            for r, leaf in enumerate([257, 400, 257]):
                c.run_rep(leaf, 2, 3000, seed=9, rep_index=r)
                out.append((c.indices(), c.leaves(), c.sets()))
            c.refine()
            final = c.finalize(want_dists=True)
        return out, final

    graph, gfinal = run(None)
    other, ofinal = run(loop)
    for r, ((gi, gl, gs), (oi, ol, os_)) in enumerate(zip(graph, other)):
        np.testing.assert_array_equal(gi, oi)
        np.testing.assert_array_equal(gl[0], ol[0])
        np.testing.assert_array_equal(gl[1], ol[1])
        assert_sets_equal(gs, os_, f"rep {r}")
    np.testing.assert_array_equal(gfinal[0], ofinal[0])
    np.testing.assert_array_equal(gfinal[1].view(np.uint32), ofinal[1].view(np.uint32))
    # A batch of sets of uneven size (one below the bucket bound).
    sizes = [5000, 200, 12_000, 800]
    sets = [workloads.gaussian_mixture(n=m, d=100, clusters=6, sigma=0.2, seed=60 + i) for i, m in enumerate(sizes)]
    params = default_params(reps=2, refine=1, max_leaf=257, max_leaf_odd=400, lloyd_iters=2, seed=5)
    monkeypatch.delenv("KNNG_REP_LOOP", raising=False)
    with KnngContext(0) as c:
        g_ids, g_d = c.build_batch(sets, params, want_dists=True)
    monkeypatch.setenv("KNNG_REP_LOOP", loop)
    with KnngContext(0) as c:
        o_ids, o_d = c.build_batch(sets, params, want_dists=True)
    for s in range(len(sets)):
        np.testing.assert_array_equal(g_ids[s], o_ids[s])
        np.testing.assert_array_equal(g_d[s].view(np.uint32), o_d[s].view(np.uint32))


@pytest.mark.parametrize("loop", [None, "host"])
def test_filtered_bucket_pass_equals_plain(knng_lib, monkeypatch, loop):
    """The bucket pass that computes distances only for pairs its tensor-core
    filter cannot rule out (KNNG_LEAF=tc) leaves the same sets, bit for bit, as
    the pass that computes every pair's distance (the default): over
    repetitions whose sets start empty, fill, and then reject most offers,
    with buckets up to 1,024 points, in the graph and in the host level loop."""
    pts = workloads.gaussian_mixture(n=40_000, d=100, clusters=24, sigma=0.2, seed=33)
    if loop is None:
        monkeypatch.delenv("KNNG_REP_LOOP", raising=False)
    else:
        monkeypatch.setenv("KNNG_REP_LOOP", loop)

    def run(leaf):
        if leaf is None:
            monkeypatch.delenv("KNNG_LEAF", raising=False)
        else:
            monkeypatch.setenv("KNNG_LEAF", leaf)
        out = []
        with KnngContext(0) as c:
            c.load_points(pts)
            c.reset_sets(100)
            for r, max_leaf in enumerate([1025, 257, 1025]):
                c.run_rep(max_leaf, 2, 3000, seed=13, rep_index=r)
                out.append(c.sets())
        return out

    filtered, plain = run("tc"), run(None)
    for r, (a, b) in enumerate(zip(filtered, plain)):
        assert_sets_equal(a, b, f"rep {r}")


def test_later_passes_skip_old_pairs_and_match_oracle(oracle_lib, monkeypatch):
    """A neighbour-of-neighbour pass after the first leaves out the pairs whose
    two edges were both in the previous pass's lists (offering them again
    changes nothing).  Three passes after two repetitions, a pass between
    repetitions, and sets whose lists change a lot between passes: every
    pass's set state equals the oracle's (which offers every pair) and the
    build with the skip switched off (KNNG_REFINE_SKIP=0), bit for bit."""
    from sigmod23ann_b200.api import Stats

    pts = workloads.gaussian_mixture(n=12_000, d=100, clusters=24, sigma=0.2, seed=44)

    def run(skip):
        if skip:
            monkeypatch.delenv("KNNG_REFINE_SKIP", raising=False)
        else:
            monkeypatch.setenv("KNNG_REFINE_SKIP", "0")
        out, stats = [], []
        with KnngContext(0) as c:
            c.load_points(pts)
            c.reset_sets(100)
            for step in ["rep", "rep", "pass", "rep", "pass", "pass", "pass"]:
                if step == "rep":
                    r = sum(1 for s in out if s[0] == "rep")
                    c.run_rep(257 if r % 2 == 0 else 400, 2, 3000, seed=77, rep_index=r)
                    out.append(("rep", c.sets()))
                else:
                    st = Stats()
                    c.refine(st)
                    out.append(("pass", c.sets()))
                    stats.append(int(st.refine_filter_pass))
        return out, stats

    with_skip, pass_with = run(True)
    without, pass_without = run(False)
    for i, ((kind, a), (_, b)) in enumerate(zip(with_skip, without)):
        assert_sets_equal(a, b, f"step {i} ({kind})")
    # The first pass skips nothing; the later ones leave pairs out.
    assert pass_with[0] == pass_without[0]
    assert all(w < wo for w, wo in zip(pass_with[1:], pass_without[1:])), (pass_with, pass_without)
    # And the oracle (every pair offered, counter RNG) agrees after each pass.
    o = oracle_lib.Oracle(pts, k=100, rng_mode=1, seed=77)
    reps = 0
    for i, (kind, sets) in enumerate(with_skip):
        if kind == "rep":
            o.rep(2, 257 if reps % 2 == 0 else 400, reps)
            reps += 1
        else:
            o.refine()
        assert_sets_equal(sets, o.sets(), f"oracle step {i} ({kind})")


def test_bucket_tuner_restores_sets_and_changes_no_result(knng_lib):
    """knng_tune_buckets times the four bucket-pass variants on a repetition of
    the context's points and sets and keeps the fastest: the sets afterwards
    are the ones before, and the next repetitions and a pass give the same
    sets, bit for bit, as a context that was never tuned."""
    pts = workloads.gaussian_mixture(n=30_000, d=100, clusters=16, sigma=0.2, seed=55)

    def run(tune):
        with KnngContext(0) as c:
            c.load_points(pts)
            c.reset_sets(100)
            c.run_rep(1025, 2, 3000, seed=8, rep_index=0)
            tuned = None
            if tune:
                before = c.sets()
                ms, choice = c.tune_buckets(1025, 2, 3000, seed=8)
                assert all(m > 0 for m in ms) and 0 <= choice < 4
                assert choice == int(np.argmin(ms))
                assert_sets_equal(c.sets(), before, "after tuning")
                tuned = choice
            for r in (1, 2):
                c.run_rep(257 if r == 1 else 1025, 2, 3000, seed=8, rep_index=r)
            c.refine()
            return c.sets(), tuned

    tuned_sets, choice = run(True)
    plain_sets, _ = run(False)
    assert_sets_equal(tuned_sets, plain_sets, f"tuned (variant {choice}) vs untuned")


def test_refine_long_survivor_lists_equal_pointwise(knng_lib, monkeypatch):
    """k = 128 and three repetitions of buckets under 43 points: each set holds
    up to 126 ids (not full, so its bound is still FLT_MAX) from three
    different buckets, and every neighbour brings about 84 candidates of its
    own, so every pair survives: thousands of records per point, many past
    8,192.  The join's replay sorts lists of 1,025-8,192 records in shared
    memory (one CTA each) and longer ones in global scratch; both must leave
    the sets the one-warp-per-point pass leaves."""
    from sigmod23ann_b200.api import Stats

    pts = workloads.gaussian_mixture(n=20_000, d=100, clusters=16, sigma=0.2, seed=71)
    with KnngContext(0) as a:
        a.load_points(pts)
        a.reset_sets(128)
        for r in range(3):
            a.run_rep(43, 2, 3000, seed=3, rep_index=r)
        s0 = a.sets()
        st = Stats()
        a.refine(st)
        joined = a.sets()
    assert (s0["size"] < 128).mean() > 0.9
    # Records per point well past the per-warp sort's 1,024 on average.
    assert st.refine_emits > 2_000 * len(pts), st.refine_emits
    monkeypatch.setenv("KNNG_REFINE", "pointwise")
    with KnngContext(0) as b:
        b.load_points(pts)
        b.reset_sets(128)
        b.set_sets(s0)
        b.refine()
        pointwise = b.sets()
    assert_sets_equal(joined, pointwise, "join vs pointwise, long lists")


def test_kd_rep_matches_oracle(oracle_lib, ctx):
    """knng_run_rep_kd (rotation on the host, rotated values, node statistics,
    side test, stable partition and buckets on the device) equals the oracle's
    KD restatement: permutation, buckets and sets after every repetition, then
    the top-up and the final lists.  The second input has 1,500 copies of one
    point, whose nodes have every point on one side until the midpoint split."""
    mix = workloads.gaussian_mixture(n=12_000, d=100, clusters=24, sigma=0.15, seed=17)
    dup = np.concatenate([np.repeat(mix[:1], 1500, axis=0), mix[:1500]])
    for pts, reps in ((mix, [(400, 0), (257, 1), (400, 2)]), (dup, [(200, 0), (129, 5)])):
        o = oracle_lib.Oracle(pts, k=100, rng_mode=1, seed=12345)
        ctx.load_points(pts)
        ctx.reset_sets(100)
        for leaf, r in reps:
            o.kd_rep(leaf, 30, 12345, r)
            ctx.run_rep_kd(leaf, 30, 12345, r)
            np.testing.assert_array_equal(ctx.indices(), o.indices())
            s, e = ctx.leaves()
            t = o.trace()
            order = np.argsort(t["leaf_start"])
            np.testing.assert_array_equal(s, t["leaf_start"][order])
            np.testing.assert_array_equal(e, t["leaf_end"][order])
            assert_sets_equal(ctx.sets(), o.sets(), f"kd rep {r}")
        assert ctx.refine() == o.refine()
        ids, dist = ctx.finalize(want_dists=True)
        oids, odist = o.finalize()
        np.testing.assert_array_equal(ids, oids)
        np.testing.assert_array_equal(dist.view(np.uint32), odist.view(np.uint32))


def test_build_kd_matches_oracle(oracle_lib, ctx):
    """knng_build_kd (the reference's KD form as one call: 5 repetitions,
    buckets below 400, no pass; then a variant with alternating bounds and one
    pass) gives the oracle's final lists and distances."""
    from sigmod23ann_b200 import kd_params

    pts = workloads.gaussian_mixture(n=9000, d=100, clusters=20, sigma=0.15, seed=23)
    for p, leafs in ((kd_params(seed=12345), [400] * 5),
                     (kd_params(seed=7, reps=3, max_leaf=300, max_leaf_odd=500, refine=1, k=64), [300, 500, 300])):
        ids, dist = ctx.build_kd(pts, p, want_dists=True)
        o = oracle_lib.Oracle(pts, k=p.k, rng_mode=1, seed=p.seed)
        for r, leaf in enumerate(leafs):
            o.kd_rep(leaf, 30, p.seed, r)
        for _ in range(p.refine):
            o.refine()
        oids, odist = o.finalize()
        np.testing.assert_array_equal(ids, oids)
        np.testing.assert_array_equal(dist.view(np.uint32), odist.view(np.uint32))
