"""The adaptive schedule (knng_build_adaptive): repetitions and
neighbour-of-neighbour passes are added until the recall estimated on a
sample of points reaches a target.  The estimate is checked against FP64
ground truth on the same sample, and the schedule against its rule."""
from __future__ import annotations

import numpy as np
import pytest

from sigmod23ann_b200 import KnngContext, Stats, default_params, groundtruth, workloads

pytestmark = pytest.mark.gpu


def _sample(n: int, q: int) -> np.ndarray:
    return (np.arange(q, dtype=np.int64) * n) // q


@pytest.mark.parametrize("target", [0.9, 0.99])
def test_adaptive_build_reaches_target(knng_lib, target):
    import torch

    pts = workloads.gaussian_mixture(n=40_000, d=100, clusters=32, sigma=0.15, seed=17)
    params = default_params(reps=8, refine=4, max_leaf=257, max_leaf_odd=0, lloyd_iters=2, seed=3)
    st = Stats()
    with KnngContext(0) as ctx:
        ids = ctx.build_adaptive(pts, target, sample=1000, params=params, stats=st)
        again = ctx.build_adaptive(pts, target, sample=1000, params=params)
    assert np.array_equal(ids, again), "the adaptive schedule is not deterministic"
    assert st.estimate_queries == 1000
    exhausted = st.reps_done == 8 and st.refine_passes_done == 4
    assert st.recall_estimate >= target or exhausted
    # The rule: at least two repetitions; never more than two passes in a row
    # unless the repetitions are used up; the maxima hold.
    assert 2 <= st.reps_done <= 8 and st.refine_passes_done <= 4
    assert st.refine_passes_done <= 2 * st.reps_done
    # The estimate is the recall of the sample's sets against their exact
    # nearest neighbours (FP32 distances there, FP64 here: only exact ties at
    # the k-th place can differ).
    q = _sample(len(pts), 1000)
    gt = groundtruth.exact_knn_torch(torch.from_numpy(pts).cuda(), q, 100)
    rec = groundtruth.recall(ids.astype(np.int64), gt, q)
    assert abs(rec - st.recall_estimate) < 0.003, (rec, st.recall_estimate)


def test_adaptive_stops_at_once_when_reached(knng_lib):
    """A target the first two repetitions already reach adds nothing more."""
    pts = workloads.gaussian_mixture(n=5_000, d=100, clusters=4, sigma=0.3, seed=2)
    params = default_params(reps=6, refine=3, max_leaf=1025, max_leaf_odd=0, lloyd_iters=1, seed=1)
    st = Stats()
    with KnngContext(0) as ctx:
        ctx.build_adaptive(pts, 0.5, sample=200, params=params, stats=st)
    assert st.reps_done == 2 and st.refine_passes_done == 0 and st.recall_estimate >= 0.5
