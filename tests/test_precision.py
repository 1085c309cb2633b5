"""GPU tests of the precision form (KNNG_PRECISION_BF16_RERANK): BF16
tensor-core bucket estimates, the 128 best candidates per point re-ranked with
exact FP32 distances.  Its results are not the FP32 form's; the tests bound the
recall change, check that every returned distance is the exact FP32 distance
in the reference's order, and that the form is deterministic."""
from __future__ import annotations

import numpy as np
import pytest

from sigmod23ann_b200 import KnngContext, default_params, groundtruth, workloads
from sigmod23ann_b200.api import PRECISION_BF16_RERANK, PRECISION_FP32

pytestmark = pytest.mark.gpu


def _recall(pts, ids, k, queries):
    import torch

    x = torch.from_numpy(pts).cuda()
    gt = groundtruth.exact_knn_torch(x, queries, k)
    return groundtruth.recall(ids.astype(np.int64), gt, queries)


@pytest.mark.parametrize("max_leaf", [257, 513, 1025])
def test_bf16_rerank_recall_and_exact_distances(oracle_lib, max_leaf):
    """Buckets of up to 256, 512 and 1024 points (the last one reads eight
    128-column tiles per row block through the heap selection)."""
    pts = workloads.gaussian_mixture(n=20_000, d=100, clusters=64, sigma=0.15, seed=0)
    common = dict(reps=4, refine=1, max_leaf=max_leaf, max_leaf_odd=0, lloyd_iters=2, seed=11)
    with KnngContext(0) as ctx:
        ids32 = ctx.build(pts, default_params(precision=PRECISION_FP32, **common))
        ids16, d16 = ctx.build(pts, default_params(precision=PRECISION_BF16_RERANK, **common), want_dists=True)
        again, _ = ctx.build(pts, default_params(precision=PRECISION_BF16_RERANK, **common), want_dists=True)
    assert np.array_equal(ids16, again), "the BF16 form is not deterministic"
    q = np.random.default_rng(5).choice(len(pts), 1000, replace=False)
    r32 = _recall(pts, ids32, 100, q)
    r16 = _recall(pts, ids16, 100, q)
    assert r16 >= 0.9 and r16 >= r32 - 0.01, (r16, r32)
    # Returned distances are exact FP32 in the reference's order.
    for row in np.random.default_rng(6).choice(len(pts), 50, replace=False):
        for j in range(0, 100, 7):
            ref = oracle_lib.distance(pts[row], pts[ids16[row, j]])
            assert np.float32(ref).view(np.uint32) == d16[row, j].view(np.uint32)


def test_bf16_rerank_rejects_large_buckets():
    """Buckets above 1024 points (max_leaf above 1025) are refused."""
    from sigmod23ann_b200 import KnngError

    pts = workloads.gaussian_mixture(n=2_000, d=100, clusters=4, seed=1)
    with KnngContext(0) as ctx:
        with pytest.raises(KnngError) as e:
            ctx.build(pts, default_params(precision=PRECISION_BF16_RERANK, max_leaf=1026, max_leaf_odd=0))
    assert e.value.status == 6


@pytest.mark.parametrize("d,m,n", [(100, 128, 128), (64, 77, 113), (128, 5, 128)])
def test_bf16_tile_against_fp64(knng_lib, d, m, n):
    """One tcgen05 kind::f16 BF16 tile against an FP64 matmul: within the
    BF16 operand-rounding bound (2^-8 relative per operand), and not coarser
    than BF16."""
    from sigmod23ann_b200.api import debug_tile_gram_bf16

    rng = np.random.default_rng(d + m + n)
    a = rng.standard_normal((m, d)).astype(np.float32)
    b = rng.standard_normal((n, d)).astype(np.float32)
    with KnngContext(0) as ctx:
        g = debug_tile_gram_bf16(ctx, a, b)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    scale = np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64).T
    err = np.abs(g - ref)
    assert (err <= 2.0 ** -7 * scale + 1e-6).all(), float((err / scale).max())
    assert float((err / scale).max()) > 2.0 ** -14  # BF16 operands, not FP32
