"""CPU test of the multi-process path of bench.py (one process per GPU under
torchrun): two gloo ranks on 127.0.0.1 run bench.py's own process-group
set-up, max-over-ranks timing reduction and barrier.  The build has no
exchange step, so these are the only collectives (replicas only)."""
from __future__ import annotations

import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world), "CUDA_VISIBLE_DEVICES": ""})
    sys.path.insert(0, ROOT)
    import bench

    args = bench.parse_args(["--gpus", str(world)])
    w, r, local = bench.dist_setup(args)
    assert (w, r, local) == (world, rank, rank)
    # Each rank's step time differs; the reported time is the maximum.
    t = bench.dist_max(10.0 + rank, w)
    bench.dist_barrier(w)
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{t}\n")
    bench.dist_done(w)


def test_two_gloo_ranks_reduce_step_time_to_the_maximum(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    got = [float((tmp_path / f"rank{r}.txt").read_text()) for r in range(world)]
    assert got == [11.0, 11.0]


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    for key in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        if key in os.environ:
            pytest.skip("running under a launcher")
    w, r, local = bench.dist_setup(bench.parse_args([]))
    assert (w, r, local) == (1, 0, 0)
    assert bench.dist_max(3.5, w) == 3.5
