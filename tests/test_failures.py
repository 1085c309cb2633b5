"""Failure detection without a GPU fault: every wait a kernel makes on its own
bulk copies or tensor-core operations has a poll limit.  A diagnostic entry
point shortens the limit to 0 so that the waits run out on purpose; the kernel
then records the failure, drains what it has in flight and returns, the call
reports KNNG_ERR_CUDA, and the same context runs the next call normally."""
from __future__ import annotations

import numpy as np
import pytest

from sigmod23ann_b200 import KnngContext, KnngError, default_params, workloads
from sigmod23ann_b200.api import debug_set_wait_limit

pytestmark = pytest.mark.gpu

DEFAULT_LIMIT = 1 << 26


def _same_sets(a: dict, b: dict) -> bool:
    return all(np.array_equal(np.asarray(a[k]).view(np.uint32), np.asarray(b[k]).view(np.uint32)) for k in a)


def test_split_wait_runs_out_and_context_recovers(knng_lib):
    """The Lloyd sums' bulk-copy waits (tree construction) give up at once."""
    pts = workloads.gaussian_mixture(n=6000, d=100, clusters=8, sigma=0.2, seed=31)
    params = default_params(reps=2, refine=1, max_leaf=257, max_leaf_odd=0, lloyd_iters=2, seed=3)
    with KnngContext(0) as ref:
        want = ref.build(pts, params)
    with KnngContext(0) as ctx:
        try:
            debug_set_wait_limit(ctx, 0)
            with pytest.raises(KnngError) as e:
                ctx.build(pts, params)
            assert e.value.status == 2 and "gave up" in str(e.value)
        finally:
            debug_set_wait_limit(ctx, DEFAULT_LIMIT)
        assert np.array_equal(ctx.build(pts, params), want)


def test_join_wait_runs_out_and_context_recovers(knng_lib):
    """The neighbour-of-neighbour join's copy / MMA waits give up at once; the
    sets are left as they were, and the pass then runs normally."""
    pts = workloads.gaussian_mixture(n=6000, d=100, clusters=8, sigma=0.2, seed=32)
    with KnngContext(0) as ref:
        ref.load_points(pts)
        ref.reset_sets(100)
        for r in range(2):
            ref.run_rep(257, 2, 3000, seed=4, rep_index=r)
        ref.refine()
        want = ref.sets()
    with KnngContext(0) as ctx:
        ctx.load_points(pts)
        ctx.reset_sets(100)
        for r in range(2):
            ctx.run_rep(257, 2, 3000, seed=4, rep_index=r)
        before = ctx.sets()
        try:
            debug_set_wait_limit(ctx, 0)
            with pytest.raises(KnngError) as e:
                ctx.refine()
            assert e.value.status == 2 and "gave up" in str(e.value)
        finally:
            debug_set_wait_limit(ctx, DEFAULT_LIMIT)
        assert _same_sets(before, ctx.sets())
        ctx.refine()
        assert _same_sets(want, ctx.sets())
