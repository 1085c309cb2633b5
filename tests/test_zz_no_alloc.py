"""The allocation-free neighbour-of-neighbour pass (knng_refine_pointwise_noalloc).

Callers that cannot allocate device memory during the call -- code inside
another framework's memory pool or under a hard memory cap, or holding only
device pointers a host application handed over -- pass every buffer in; the
only scratch is a fixed device array inside the library.  This file runs last
so that a failure here never hides the rest of the GPU suite."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import assert_sets_equal
from sigmod23ann_b200 import KnngContext, default_params, load_library, workloads
from sigmod23ann_b200.api import STATUS_NAMES

pytestmark = pytest.mark.gpu


def _run_noalloc(lib, pts: np.ndarray, sets: dict, k: int):
    import torch

    dev = torch.device("cuda")
    n, d = pts.shape
    P = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    dist = torch.from_numpy(np.ascontiguousarray(sets["dist"])).to(dev)
    ids = torch.from_numpy(np.ascontiguousarray(sets["id"]).view(np.int32)).to(dev)
    size = torch.from_numpy(np.ascontiguousarray(sets["size"]).view(np.int32)).to(dev)
    maxslot = torch.from_numpy(np.ascontiguousarray(sets["maxslot"]).view(np.int32)).to(dev)
    bound = torch.from_numpy(np.ascontiguousarray(sets["bound"])).to(dev)
    snap = torch.empty(n * k, dtype=torch.int32, device=dev)
    changed = torch.full((1,), 12345, dtype=torch.int32, device=dev)  # the call must clear it
    stream = torch.cuda.current_stream()
    status = lib.knng_refine_pointwise_noalloc(P.data_ptr(), n, d, k, snap.data_ptr(), dist.data_ptr(),
                                               ids.data_ptr(), size.data_ptr(), maxslot.data_ptr(), bound.data_ptr(),
                                               changed.data_ptr(), stream.cuda_stream)
    assert status == 0, STATUS_NAMES.get(status, status)
    torch.cuda.synchronize()
    out = {
        "dist": dist.cpu().numpy(), "id": ids.cpu().numpy().view(np.uint32),
        "size": size.cpu().numpy().view(np.uint32), "maxslot": maxslot.cpu().numpy().view(np.uint32),
        "bound": bound.cpu().numpy(),
    }
    return out, int(changed.cpu().numpy()[0])


def test_noalloc_pass_matches_knng_refine_on_two_calls_in_a_row(oracle_lib):
    lib = load_library()
    # Two calls in a row on different inputs: the shared scratch array keeps the
    # first call's records, which must not leak into the second.
    for seed, (n, k) in ((1, (6000, 100)), (2, (4500, 64))):
        pts = workloads.gaussian_mixture(n=n, d=100, clusters=16, sigma=0.15, seed=seed)
        with KnngContext(0) as ctx:
            ctx.build(pts, default_params(k=k, reps=2, max_leaf=257, max_leaf_odd=0, lloyd_iters=2, refine=0,
                                          seed=seed))
            before = ctx.sets()
            changed_ref = ctx.refine()
            after_ref = ctx.sets()
        after, changed = _run_noalloc(lib, pts, before, k)
        assert changed == changed_ref
        # Bit-exact, the tolerance of every set comparison in this suite.
        assert_sets_equal(after, after_ref, f"allocation-free pass, seed {seed}")
        # and the oracle's neighbour-of-neighbour pass from the same sets.
        o = oracle_lib.Oracle(pts, k=k)
        o.set_sets(before)
        assert o.refine() == changed
        assert_sets_equal(after, o.sets(), f"allocation-free pass vs oracle, seed {seed}")


def test_noalloc_rejects_k_beyond_its_scratch():
    lib = load_library()
    # Sets hold at most 128 neighbours: k = 129 is refused before anything
    # runs (null buffers are never touched).
    status = lib.knng_refine_pointwise_noalloc(None, 10, 100, 129, None, None, None, None, None, None, None, None)
    assert STATUS_NAMES[status] == "KNNG_ERR_UNSUPPORTED"
