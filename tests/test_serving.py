"""GPU tests of the serving form (knng_server_*): each job's result is the
same alone and in a mix of concurrent jobs; admission follows the HBM budget
and arrival order; oversized jobs are refused."""
from __future__ import annotations

import numpy as np
import pytest

from sigmod23ann_b200 import KnngContext, KnngError, KnngServer, default_params, job_reservation, workloads
from sigmod23ann_b200.api import JOB_DONE

pytestmark = pytest.mark.gpu


def _jobs():
    """Jobs of different sizes, dimensions and k (seeded data)."""
    specs = [(12_000, 100, 100, 1), (5_000, 64, 10, 2), (20_000, 128, 50, 3), (3_000, 100, 100, 4),
             (9_000, 64, 50, 5)]
    out = []
    for n, d, k, seed in specs:
        pts = workloads.gaussian_mixture(n=n, d=d, clusters=12, sigma=0.2, seed=seed)
        params = default_params(k=k, reps=2, refine=1, max_leaf=257, max_leaf_odd=0, lloyd_iters=2, seed=seed)
        out.append((pts, params))
    return out


def _alone(pts, params):
    with KnngContext(0) as ctx:
        return ctx.build(pts, params, want_dists=True)


def test_jobs_same_alone_and_in_the_mix(knng_lib):
    """Five jobs submitted at once to a server running three at a time give
    bit-identical ids and distances to the same builds run alone."""
    jobs = _jobs()
    alone = [_alone(p, q) for p, q in jobs]
    with KnngServer(0, max_running=3) as srv:
        ids = [srv.submit(p, q, want_dists=True) for p, q in jobs]
        infos = [srv.wait(j) for j in ids]
        results = [srv.result(j) for j in ids]
    for (a_ids, a_d), (m_ids, m_d), info in zip(alone, results, infos):
        assert info.state == JOB_DONE and info.status == 0
        assert np.array_equal(a_ids, m_ids)
        assert np.array_equal(a_d.view(np.uint32), m_d.view(np.uint32))


def test_admission_by_budget_and_overlap(knng_lib):
    """With room for one job at a time the jobs run one after another in
    arrival order; with room for all, several run at once."""
    jobs = _jobs()[:3]
    need = max(job_reservation(p.shape[0], p.shape[1], q.k) for p, q in jobs)
    with KnngServer(0, hbm_budget_bytes=need + need // 2, max_running=3) as srv:
        ids = [srv.submit(p, q) for p, q in jobs]
        infos = [srv.wait(j) for j in ids]
    spans = [(i.ms_queued, i.ms_queued + i.ms_run) for i in infos]
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0 - 5.0  # the next job started after the previous ended
    with KnngServer(0, max_running=3) as srv:
        ids = [srv.submit(p, q) for p, q in jobs]
        infos = [srv.wait(j) for j in ids]
    starts = [i.ms_queued for i in infos]
    ends = [i.ms_queued + i.ms_run for i in infos]
    assert min(ends) > max(starts)  # every job started before the first one ended


def test_oversized_job_refused(knng_lib):
    pts = workloads.gaussian_mixture(n=4_000, d=100, clusters=4, seed=1)
    with KnngServer(0, hbm_budget_bytes=1 << 20, max_running=1) as srv:
        with pytest.raises(KnngError) as e:
            srv.submit(pts, default_params(reps=1, refine=0))
    assert e.value.status == 4
