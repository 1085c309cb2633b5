#!/usr/bin/env python
"""k-NN graph build throughput on B200: points/s for the 10M x 100, k=100
build at recall >= 0.94 against an FP64 exact oracle.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one whole graph build (every repetition of split + bucket pass,
then finalize) of the 10,000,000-point, 100-d, 1,024-cluster Zipf(1.1)
24-d-subspace mixture (seed 1), leaf buckets <= 1024, through the library's C
ABI.  `value` is measured with the points already in HBM (knng_build_device),
timed by CUDA events on the library's launching stream; `e2e` is the same
build through knng_build with pinned host buffers, host<->device copies inside
the timed region.  The input (4 GB) is larger than L2, so no flush is needed
between steps.  With N > 1 (torchrun), every rank builds its own replica: the
path has no exchange step, so scaling is weak and there is no collective on
the data path; the step time is the maximum over ranks.

--impl reference times the reference's own CPU code (oracle/_ref, the
reference headers compiled against a std::thread-pool stand-in for TBB) on the
host cores: each step runs the same schedule -- every repetition of
splitKmeansBinaryProcess, then every topUpSingle pass -- over a bounded prefix
of the same point set (value = prefix points / step seconds).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "points/sec k-NN graph build at recall>=0.94 (10M x 100, k=100); p50/p99 latency"
N_POINTS = 10_000_000
DIM = 100
K = 100
MAX_LEAF = 1025        # buckets of at most 1024 points (leaf iff size < max_leaf)
LLOYD_ITERS = 2
REPS = 4
REFINE = 2
SEED = 1
QUERIES = 10_000
# DRAM read + write bytes of one k_join launch at 500k points (ncu capture,
# profiles/k_join_500k.md); the bench scales it by the points processed.
JOIN_DRAM_BYTES_500K = 55.56e9


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_POINTS)
    ap.add_argument("--reps", type=int, default=REPS)
    ap.add_argument("--refine", type=int, default=REFINE)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU work per reference sample")
    ap.add_argument("--serving-requests", type=int, default=200,
                    help="requests of the serving stream measured beside the build")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="skip the bucket-pass autotuner before the timed builds")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="skip the precision, batched and serving figures of the default line")
    ap.add_argument("--serving", action="store_true", help="measure only the serving stream")
    ap.add_argument("--batched", action="store_true", help="measure only the batched form (4,096 sets, 5 waves)")
    ap.add_argument("--bf16", action="store_true",
                    help="time the precision form (BF16 estimates + FP32 re-rank) instead")
    ap.add_argument("--max-leaf", type=int, default=0, help="leaf test bound (0: 1025, buckets of at most 1024)")
    ap.add_argument("--precision", action="store_true",
                    help="measure only the precision form against the FP32 form (100k-point config)")
    ap.add_argument("--kd", action="store_true",
                    help="measure only the KD splitter beside the 2-means splitter")
    ap.add_argument("--batched-waves", type=int, default=5, help="waves of the batched form to run (of 5)")
    return ap.parse_args(argv)


# ----------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ distributed

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def dist_max(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def dist_done(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def workload_config(n: int, reps: int, refine: int, max_leaf: int, bf16: bool, world: int) -> dict:
    """The `config` object of the build line, the same for both arms."""
    return {"workload": f"{n:,} x {DIM} f32 1024-cluster Zipf(1.1) 24-d subspace mixture (seed {SEED}), "
                        f"k={K}, leaf<={max_leaf - 1}, {reps} reps x {LLOYD_ITERS} Lloyd iters, {refine} top-up passes"
                        + (", BF16 estimates + FP32 re-rank" if bf16 else ", FP32"),
            "parallelism": f"replicas x{world}", "l2": "4 GB input > L2, no flush"}


# ------------------------------------------------------------ reference arm

def reference_prefix(n: int, m: int) -> np.ndarray:
    """The first m points of the benchmark point set (generated on the GPU when
    one is present, as the GPU arm does; the set is randomly permuted, so a
    prefix is a uniform sample)."""
    from sigmod23ann_b200 import workloads

    try:
        import torch

        if torch.cuda.is_available():
            x = workloads.subspace_mixture_torch(n, seed=SEED)
            out = x[:m].cpu().numpy().copy()
            del x
            torch.cuda.empty_cache()
            return out
    except Exception:
        pass
    return workloads.subspace_mixture(max(m, min(n, 1_000_000)), seed=SEED)[:m]


def host_cpu_model() -> str:
    """The host CPU's model name (first processor in /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_sample_rate(n: int, reps: int, passes: int, target_s: float, steps: int, warmup: int):
    """Times the reference's own code (all host threads) on a prefix of the
    point set: each step = `reps` repetitions of splitKmeansBinaryProcess
    (leaf <= 1024, 2 Lloyd iterations) then `passes` topUpSingle passes, from
    empty sets.  The prefix is sized so one step takes about target_s."""
    from oracle import bindings

    cores = os.cpu_count() or 1
    os.environ.setdefault("KNNG_REF_THREADS", str(cores))
    cores = int(os.environ["KNNG_REF_THREADS"])
    if not bindings.reference_available():
        return None

    def one_step(pts):
        ref = bindings.ReferenceShim(pts, threaded=True)
        t = time.perf_counter()
        for _ in range(reps):
            ref.rep(LLOYD_ITERS, MAX_LEAF)
        for _ in range(passes):
            ref.topup()
        dt = time.perf_counter() - t
        ref.close()
        return dt

    m = min(n, 20_000)
    pool = reference_prefix(n, min(n, 2_000_000))
    while True:
        dt = one_step(pool[:m])
        if dt >= target_s / 2 or m >= len(pool):
            break
        m = min(len(pool), int(m * min(8.0, max(1.5, target_s / max(dt, 1e-3)))))
    sample = pool[:m]
    for _ in range(warmup):
        one_step(sample)
    secs = [one_step(sample) for _ in range(steps)]
    return {"rates": [m / t for t in secs], "seconds": secs, "sample_points": m, "cores": cores}


def run_reference(args):
    world, rank, _ = dist_setup(args)
    try:
        if rank != 0:
            return 0
        res = reference_sample_rate(args.n, args.reps, args.refine, args.cpu_seconds, args.steps, args.warmup)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (needs the reference sources)"}))
            return 0
        value = statistics.mean(res["rates"])
        sample = (f"the reference's splitKmeansBinaryProcess x{args.reps} (leaf<=1024, {LLOYD_ITERS} Lloyd "
                  f"iterations) then topUpSingle x{args.refine}, from empty sets, on the first "
                  f"{res['sample_points']:,} points of the 10M seed-1 subspace mixture; points/s = sample / step time")
        # ms_per_step is the measured step (the bounded sample); a whole
        # 10M-point build at the same rate would take n / value seconds, a
        # linear extrapolation reported beside it.
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.mean(res["seconds"]),
            "sample_points": res["sample_points"],
            "ms_per_build_extrapolated": {"value": args.n / value * 1000.0, "points": args.n,
                                          "how": "linear in points from the measured sample rate"},
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.n, args.reps, args.refine, MAX_LEAF, False, args.gpus),
            "cpu_baseline": {"value": value, "unit": "points/s", "cores": res["cores"], "kind": "reference",
                             "cpu": host_cpu_model(), "sample": sample},
            "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return 0
    finally:
        dist_done(world)


# ------------------------------------------------------------ serving arm

SERVING_RATE = 50.0  # requests per second (Poisson), the serving config's arrival rate
SERVING_MAX_RUNNING = 8  # worker threads of the server: concurrent jobs on the device at most


def serving_stream(requests: int, seed: int = 3):
    """The serving config's requests: sizes log-uniform in [1e4, 2e6] points, d
    in {64, 100, 128}, k in {10, 50, 100}, Poisson gaps at 50 req/s (seed 3)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(1e4), np.log(2e6), size=requests)).astype(np.int64)
    dims = rng.choice([64, 100, 128], size=requests)
    ks = rng.choice([10, 50, 100], size=requests)
    gaps = rng.exponential(1.0, size=requests)  # unit-rate gaps, scaled by the stream's rate
    return sizes, dims, ks, gaps


def run_serving(requests: int, rate: float = SERVING_RATE, device: int = 0, capacity: float | None = None,
                per_job: bool = False) -> dict:
    """Serving form: build requests arrive as a Poisson stream at `rate`
    req/s; each request's points are a slice of a 64-cluster 24-d-subspace
    mixture held in pinned host memory.  A server with an 80% HBM budget
    admits them in arrival order as memory and worker slots free up (its
    worker count is derived from the budget: the median request's
    reservation, at most SERVING_MAX_RUNNING).  Latency = arrival to result
    (host ids written); p50/p99 over the requests; aggregate points/s = all
    points / (last result - first arrival).  offered_points_per_s = rate x
    mean request size; with `capacity` (points/s the device sustains) the
    offered load is stated as a fraction of it.  Recall of every job is
    checked afterwards on 1k sampled points against FP64 brute force.  Every
    job is built with the reference's k = 100 and answered with the first k of
    each (distance-sorted) row: with shorter lists the neighbour-of-neighbour
    pass sees too few candidates to reach the recall target (k = 10 lists
    reach 0.77-0.89; k = 50 lists fall to 0.92 on the largest jobs)."""
    import torch

    from sigmod23ann_b200 import KnngServer, default_params, groundtruth, workloads
    from sigmod23ann_b200.api import job_reservation

    sizes, dims, ks, gaps = serving_stream(requests)
    gaps = gaps / rate
    pool_n = int(sizes.max())
    pool = workloads.subspace_mixture_torch(pool_n, d=128, clusters=64, seed=3, device=f"cuda:{device}")
    host = torch.empty((pool_n, 128), dtype=torch.float32, pin_memory=True)
    host.copy_(pool.cpu())
    hp = host.numpy()
    rng = np.random.default_rng(4)
    offs = [int(rng.integers(0, pool_n - n + 1)) for n in sizes]
    views = [hp[o:o + int(n), :int(d)] for o, n, d in zip(offs, sizes, dims)]
    build_k = [max(int(k), K) for k in ks]
    params = [default_params(k=bk, max_leaf=MAX_LEAF, max_leaf_odd=0, lloyd_iters=LLOYD_ITERS, reps=REPS,
                             refine=REFINE, seed=SEED) for bk in build_k]
    budget = int(0.8 * torch.cuda.get_device_properties(device).total_memory)
    median = int(np.median(sizes))
    max_running = int(max(1, min(SERVING_MAX_RUNNING, budget // job_reservation(median, 128, 100))))
    srv = KnngServer(device, 0, max_running)
    arrivals = np.cumsum(gaps)
    t0 = time.perf_counter()
    jobs = []
    for i in range(requests):
        delay = t0 + arrivals[i] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        jobs.append(srv.submit(views[i], params[i]))
    infos = [srv.wait(j) for j in jobs]
    lat = np.array([info.ms_latency for info in infos])
    queued = np.array([info.ms_queued for info in infos])
    end = max(arrivals[i] + lat[i] / 1000.0 for i in range(requests))
    failed = [int(info.status) for info in infos if info.state != 2]
    recalls = []
    for i, j in enumerate(jobs):
        ids, _ = srv.result(j)
        ids = ids[:, :int(ks[i])]
        n = int(sizes[i])
        q = np.random.default_rng(i).choice(n, min(1000, n), replace=False)
        x = pool[offs[i]:offs[i] + n, :int(dims[i])]
        gt = groundtruth.exact_knn_torch(x, q, int(ks[i]))
        recalls.append(groundtruth.recall(ids.astype(np.int64), gt, q))
        srv.release(j)
    srv.close()
    del pool
    torch.cuda.empty_cache()
    offered = rate * float(sizes.mean())
    out = {
        "rate_per_s": rate, "requests": requests, "max_running": max_running,
        "offered_points_per_s": offered,
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "mean_queued_ms": float(queued.mean()),
        "points_per_s": float(sizes.sum()) / end, "failed": len(failed),
        "min_recall": float(min(recalls)), "all_recall_ok": bool(min(recalls) >= 0.94),
    }
    if capacity:
        out["offered_over_capacity"] = offered / capacity
    if per_job:
        out["jobs"] = [{"n": int(sizes[i]), "d": int(dims[i]), "k": int(ks[i]), "latency_ms": round(float(lat[i]), 1),
                        "recall": round(float(recalls[i]), 4)} for i in range(requests)]
    return out


def run_serving_pair(requests: int, device: int = 0) -> dict:
    """The serving config's stream (50 req/s), which offers several times what
    one B200 builds, so its latencies grow with the queue; then the same kind
    of stream at 70% of the capacity the first one measured, whose latencies
    describe the system rather than the backlog."""
    over = run_serving(requests, SERVING_RATE, device)
    capacity = over["points_per_s"]
    over["offered_over_capacity"] = over["offered_points_per_s"] / capacity
    mean_size = float(serving_stream(requests)[0].mean())
    rate = 0.7 * capacity / mean_size
    under = run_serving(max(20, requests // 2), rate, device, capacity=capacity)
    return {"stream_50_per_s": over, "at_70pct_capacity": under,
            "workload": "Poisson arrivals (seed 3), sizes log-uniform [1e4, 2e6], d in {64,100,128}, "
                        "k in {10,50,100} (built with k = 100), 64-cluster 24-d subspace mixture; "
                        f"{REPS} repetitions + {REFINE} passes per job; 80% HBM budget"}


# ------------------------------------------------------------ precision arm

def run_precision(device: int = 0, steps: int = 3, cpu_reference: bool = True) -> dict:
    """Precision form on the 100k-point config (64 Gaussians, sigma 0.15, seed
    0; k=100, buckets <= 256, 2 Lloyd iterations, 8 repetitions + 1 pass):
    BF16 tensor-core bucket estimates + FP32 re-rank of each point's 128 best
    candidates, against the plain FP32 form at the same repetition count.
    Recall over all points against FP64 brute force; the error of the returned
    distances and of the BF16 estimates (on 16 groups of 128 nearest
    neighbours, centred on the group's first point as a bucket is) against
    FP64; device time per build (CUDA events on the library's stream)."""
    import torch

    from sigmod23ann_b200 import KnngContext, Stats, default_params, groundtruth, workloads
    from sigmod23ann_b200.api import PRECISION_BF16_RERANK, PRECISION_FP32, debug_tile_gram_bf16

    pts = workloads.gaussian_mixture(n=100_000, d=100, clusters=64, sigma=0.15, seed=0)
    n = len(pts)
    x = torch.from_numpy(pts).to(f"cuda:{device}")
    gt = np.concatenate([groundtruth.exact_knn_torch(x, np.arange(a, min(n, a + 8192)), K)
                         for a in range(0, n, 8192)])
    out = {}
    with KnngContext(device) as ctx:
        for name, prec in (("fp32", PRECISION_FP32), ("bf16_rerank", PRECISION_BF16_RERANK)):
            params = default_params(k=K, max_leaf=257, max_leaf_odd=0, lloyd_iters=2, reps=8, refine=1, seed=SEED,
                                    precision=prec)
            ids = torch.empty((n, K), dtype=torch.int32, device=x.device)
            dist = torch.empty((n, K), dtype=torch.float32, device=x.device)
            ctx.build_device(x.data_ptr(), n, DIM, ids.data_ptr(), dist.data_ptr(), params)
            times = []
            for _ in range(steps):
                st = Stats()
                ctx.build_device(x.data_ptr(), n, DIM, ids.data_ptr(), dist.data_ptr(), params, stats=st)
                times.append(st.ms_total + st.ms_finalize)
            ids_np = ids.cpu().numpy().view(np.uint32).astype(np.int64)
            rec = groundtruth.recall(ids_np, gt, np.arange(n))
            # returned distances against FP64 (sampled rows, every neighbour)
            rows = np.random.default_rng(1).choice(n, 2000, replace=False)
            xr = x[torch.as_tensor(rows, device=x.device)].double()
            xn = x[torch.as_tensor(ids_np[rows].reshape(-1), device=x.device)].double().reshape(len(rows), K, DIM)
            exact = ((xn - xr[:, None, :]) ** 2).sum(-1)
            got = dist[torch.as_tensor(rows, device=x.device)].double()
            rel = ((got - exact).abs() / exact.clamp_min(1e-30)).cpu().numpy()
            out[name] = {"recall": rec, "ms_per_build": float(np.mean(times)),
                         "points_per_s": n / (np.mean(times) / 1000.0),
                         "dist_rel_err_max": float(rel.max()), "dist_rel_err_mean": float(rel.mean())}
        # BF16 estimates on bucket-like groups (a point and its 127 nearest)
        errs = []
        for g in np.random.default_rng(2).choice(n, 16, replace=False):
            grp = np.concatenate([[g], gt[g][:127]])
            rows32 = pts[grp].astype(np.float32)
            cen = (rows32 - rows32[0]).astype(np.float32)
            gram = debug_tile_gram_bf16(ctx, cen, cen).astype(np.float64)
            nrm = (cen.astype(np.float64) ** 2).sum(1)
            est = nrm[:, None] + nrm[None, :] - 2.0 * gram
            ex = ((rows32[:, None, :].astype(np.float64) - rows32[None, :, :]) ** 2).sum(-1)
            mask = ~np.eye(len(grp), dtype=bool)
            errs.append(np.abs(est - ex)[mask] / ex[mask])
        e = np.concatenate(errs)
        out["bf16_estimate_rel_err_max"] = float(e.max())
        out["bf16_estimate_rel_err_mean"] = float(e.mean())
    # The reference's own CPU code on the same config, in full (all host threads).
    try:
        if not cpu_reference:
            raise StopIteration
        from oracle import bindings

        os.environ.setdefault("KNNG_REF_THREADS", str(os.cpu_count() or 1))
        if bindings.reference_available():
            ref = bindings.ReferenceShim(pts, threaded=True)
            t = time.perf_counter()
            for _ in range(8):
                ref.rep(2, 257)
            ref.topup()
            dt = time.perf_counter() - t
            ref.close()
            out["cpu_reference"] = {"seconds": dt, "points_per_s": n / dt, "cores": int(os.environ["KNNG_REF_THREADS"]),
                                    "kind": "reference"}
    except StopIteration:
        pass
    except Exception as e:  # the baseline must not hide the GPU figures
        out["cpu_reference"] = {"error": str(e)}
    out["recall_change"] = out["bf16_rerank"]["recall"] - out["fp32"]["recall"]
    out["speedup"] = out["fp32"]["ms_per_build"] / out["bf16_rerank"]["ms_per_build"]
    out["workload"] = ("100,000 x 100 f32, 64 Gaussians (sigma 0.15, seed 0), k=100, buckets <= 256, 2 Lloyd "
                       "iterations, 8 repetitions + 1 neighbour-of-neighbour pass; recall over all points vs FP64")
    return out


# ------------------------------------------------------------ KD splitter

def refine_breakdown(st) -> dict:
    """One neighbour-of-neighbour pass's device time by stage (ms) and its
    survivor records that went past the pool to the per-point pass."""
    return {"ms": sig(st.ms_refine), "prep": sig(st.ms_refine_prep), "join": sig(st.ms_refine_join),
            "replay": sig(st.ms_refine_apply), "per_point": sig(st.ms_refine_fallback),
            "overflow": int(st.refine_overflow), "changed": int(st.refine_changed),
            "pairs": int(st.refine_pairs), "filter_kept": int(st.refine_filter_pass),
            "exact": int(st.refine_exact), "survivors": int(st.refine_emits)}


def oracle_kd_rate(n: int, max_leaf: int, target_s: float) -> dict:
    """The oracle's KD repetition (the C++ restatement, one host thread) on a
    prefix of the bench's points, grown until one repetition takes about
    target_s / 2: rotation, node statistics, partition, buckets."""
    from oracle import bindings

    pool = reference_prefix(n, min(n, 2_000_000))
    m = min(len(pool), 20_000)
    while True:
        o = bindings.Oracle(pool[:m], k=K, rng_mode=1, seed=SEED)
        t = time.perf_counter()
        o.kd_rep(max_leaf, 30, SEED, 0)
        dt = time.perf_counter() - t
        o.close()
        if dt >= target_s / 2 or m >= len(pool):
            break
        m = min(len(pool), int(m * min(8.0, max(1.5, target_s / max(dt, 1e-3)))))
    return {"points_per_s_per_rep": sig(m / dt), "seconds": sig(dt), "sample_points": m, "cores": 1, "kind": "port",
            "sample": f"oracle KD repetition (30 dims, buckets < {max_leaf}) from empty sets, first {m:,} points"}


def run_kd_compare(n: int, device: int = 0, reps: int = REPS, max_leaf: int = MAX_LEAF) -> dict:
    """The random-rotation KD splitter (30 rotated dimensions) beside the
    2-means splitter on the bench's points: `reps` repetitions of each from
    empty sets, buckets below max_leaf, then one neighbour-of-neighbour pass;
    device time of the split stage and of the bucket pass (CUDA events on the
    library's stream), recall on sampled points against FP64 brute force after
    every repetition and after the pass."""
    import torch

    from sigmod23ann_b200 import KnngContext, Stats, groundtruth, workloads

    x = workloads.subspace_mixture_torch(n, seed=SEED, device=f"cuda:{device}")
    q = np.random.default_rng(SEED).choice(n, min(2000, n), replace=False)
    gt = groundtruth.exact_knn_torch(x, q, K)
    host = x.cpu().numpy()
    x = None
    torch.cuda.empty_cache()
    out = {"workload": f"{n:,} x {DIM} f32 subspace mixture (seed {SEED}), k={K}, buckets < {max_leaf}, "
                       f"{reps} repetitions + 1 pass, recall on {len(q):,} points"}
    with KnngContext(device) as ctx:
        ctx.load_points(host)
        # One untimed repetition and pass first: the context's first pass
        # allocates its scratch and loads the kernels.
        ctx.reset_sets(K)
        ctx.run_rep(max_leaf, LLOYD_ITERS, 3000, SEED, 0)
        st = Stats()
        ctx.refine(st)
        out["first_pass"] = refine_breakdown(st)
        for name in ("two_means", "kd"):
            ctx.reset_sets(K)
            split = leaf = 0.0
            buckets = 0
            per_rep = []
            for r in range(reps):
                st = Stats()
                if name == "kd":
                    ctx.run_rep_kd(max_leaf, 30, SEED, r, st)
                else:
                    ctx.run_rep(max_leaf, LLOYD_ITERS, 3000, SEED, r, st)
                split += st.ms_split
                leaf += st.ms_leaf
                buckets += st.buckets
                per_rep.append(sig(groundtruth.recall(ctx.finalize().astype(np.int64), gt, q)))
            st = Stats()
            ctx.refine(st)
            ids = ctx.finalize()
            out[name] = {"recall_after_each_rep": per_rep,
                         "split_ms_per_rep": sig(split / reps), "bucket_ms_per_rep": sig(leaf / reps),
                         "buckets_per_rep": buckets // reps, "pass": refine_breakdown(st),
                         "recall": sig(groundtruth.recall(ids.astype(np.int64), gt, q))}
    return out


# ------------------------------------------------------------ batched arm

def batched_sets(seed: int = 2, count: int = 4096):
    """Sizes of the batched form: log-uniform in [1e3, 2e5] (seed 2)."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(1e3), np.log(2e5), size=count)).astype(np.int64)


def batched_wave_points(sizes, wave_seed: int, device: str):
    """One wave's sets, concatenated: each set a mixture of 16 Gaussians
    (sigma 0.2, centres uniform in [-1,1]^100, equal weights)."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(wave_seed)
    s = len(sizes)
    centres = torch.rand((s, 16, DIM), generator=g, device=device) * 2.0 - 1.0
    set_of = torch.repeat_interleave(torch.arange(s, device=device), torch.as_tensor(sizes, device=device))
    label = torch.randint(0, 16, (int(sizes.sum()),), generator=g, device=device)
    x = centres[set_of, label] + 0.2 * torch.randn((int(sizes.sum()), DIM), generator=g, device=device)
    return x.contiguous()


def sig(x, digits: int = 4):
    """x rounded to `digits` significant digits (keeps the bench line short)."""
    if isinstance(x, float) and x != 0.0 and np.isfinite(x):
        return float(f"{x:.{digits}g}")
    return x


def precision_summary(res: dict) -> dict:
    """The precision object of the default line (the 100k-point config)."""
    f, b = res["fp32"], res["bf16_rerank"]
    return {"fp32_ms": sig(f["ms_per_build"]), "bf16_ms": sig(b["ms_per_build"]), "speedup": sig(res["speedup"]),
            "fp32_recall": sig(f["recall"]), "bf16_recall": sig(b["recall"]),
            "dist_err_max": sig(b["dist_rel_err_max"], 2), "est_err_max": sig(res["bf16_estimate_rel_err_max"], 2),
            "est_err_mean": sig(res["bf16_estimate_rel_err_mean"], 2)}


def batched_summary(res: dict) -> dict:
    """The batched object of the default line: wave 1 of the batched config."""
    return {"sets": res["sets"], "points": res["points"], "points_per_s": sig(res["points_per_s"]),
            "min_recall": sig(res["min_recall"])}


def serving_summary(res: dict) -> dict:
    """The serving object of the default line."""
    o, u = res["stream_50_per_s"], res["at_70pct_capacity"]
    return {"at_50_per_s": {"p50_ms": sig(o["p50_ms"]), "p99_ms": sig(o["p99_ms"]), "pts_per_s": sig(o["points_per_s"]),
                            "offered_over_capacity": sig(o["offered_over_capacity"], 3), "n": o["requests"]},
            "at_70pct": {"rate": sig(u["rate_per_s"], 3), "p50_ms": sig(u["p50_ms"]), "p99_ms": sig(u["p99_ms"]),
                         "pts_per_s": sig(u["points_per_s"]), "n": u["requests"]},
            "recall_ok": bool(o["all_recall_ok"] and u["all_recall_ok"]),
            "min_recall": sig(min(o["min_recall"], u["min_recall"]), 4)}


def run_batched(waves: int, device: int = 0) -> dict:
    """Batched form: 4,096 independent sets (about 160M points) in 5 waves of
    about 820 sets; each wave is one knng_build_batch on device-resident
    points (every tree level, bucket pass and join shared by the wave's sets).
    points/s = points built / device time (CUDA events on the library's
    stream).  Recall on 1k sampled points of 16 sampled sets per wave."""
    import torch

    from sigmod23ann_b200 import KnngContext, Stats, default_params, groundtruth
    from sigmod23ann_b200.api import _ptr

    sizes = batched_sets()
    per_wave = np.array_split(np.arange(len(sizes)), 5)
    params = default_params(k=K, max_leaf=MAX_LEAF, max_leaf_odd=0, lloyd_iters=LLOYD_ITERS, reps=REPS,
                            refine=REFINE, seed=SEED)
    dev = f"cuda:{device}"
    total_points, total_ms, recalls, waves_out = 0, 0.0, [], []
    import ctypes

    torch.cuda.empty_cache()  # blocks the caller's earlier work left in torch's cache

    for w in range(min(waves, 5)):
        ws = sizes[per_wave[w]]
        x = batched_wave_points(ws, 100 + w, dev)
        offs = np.zeros(len(ws) + 1, np.uint32)
        offs[1:] = np.cumsum(ws)
        n = int(offs[-1])
        ids = torch.empty((n, K), dtype=torch.int32, device=dev)
        # The context is created once the wave's tensors exist, so that its
        # default budget (bounded by the memory free at creation) leaves them
        # out.
        ctx = KnngContext(device)
        st = Stats()
        try:
            ctx._check(ctx._lib.knng_build_batch(ctx._h, _ptr(x), n, DIM, DIM * 4, _ptr(offs), len(ws), 1,
                                                 ctypes.byref(params), _ptr(ids), None, ctypes.byref(st)))
        finally:
            ctx.close()
        ms = st.ms_total + st.ms_finalize
        total_points += n
        total_ms += ms
        rng = np.random.default_rng(w)
        for s in rng.choice(len(ws), 16, replace=False):
            a, b = int(offs[s]), int(offs[s + 1])
            q = rng.choice(b - a, min(1000, b - a), replace=False)
            gt = groundtruth.exact_knn_torch(x[a:b], q, K)
            recalls.append(groundtruth.recall(ids[a:b].cpu().numpy().view(np.uint32).astype(np.int64), gt, q))
        waves_out.append({"sets": len(ws), "points": n, "ms": ms})
        del x, ids
        torch.cuda.empty_cache()
    return {"sets": int(sum(w["sets"] for w in waves_out)), "points": total_points, "ms": total_ms,
            "points_per_s": total_points / (total_ms / 1000.0), "waves": waves_out,
            "min_recall": float(min(recalls)), "mean_recall": float(np.mean(recalls)),
            "workload": "4,096 sets (seed 2), sizes log-uniform [1e3, 2e5], 16-Gaussian mixtures (sigma 0.2), "
                        "d=100, k=100, 5 waves; FP32 distances, 4 repetitions + 2 passes per set"}


# ------------------------------------------------------------ our arm

def run_ours(args):
    import torch

    from sigmod23ann_b200 import KnngContext, Stats, default_params, groundtruth, workloads

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    n = args.n
    from sigmod23ann_b200.api import PRECISION_BF16_RERANK, PRECISION_FP32

    max_leaf = args.max_leaf or MAX_LEAF
    params = default_params(k=K, max_leaf=max_leaf, max_leaf_odd=0, lloyd_iters=LLOYD_ITERS, reps=args.reps,
                            refine=args.refine, seed=SEED,
                            precision=PRECISION_BF16_RERANK if args.bf16 else PRECISION_FP32)
    x = workloads.subspace_mixture_torch(n, seed=SEED, device=f"cuda:{local}")
    ids = torch.empty((n, K), dtype=torch.int32, device=f"cuda:{local}")
    ctx = KnngContext(local)
    for _ in range(args.warmup):
        ctx.build_device(x.data_ptr(), n, DIM, ids.data_ptr(), None, params)
    # The bucket-pass autotuner, on the warm-up build's points and sets (they
    # are restored): the timed builds use the variant it keeps.
    tuning = None
    if args.tune and not args.bf16 and args.warmup > 0:
        tms, choice = ctx.tune_buckets(max_leaf, LLOYD_ITERS, 3000, SEED)
        names = ["every pair x2", "every pair x1", "tc filter x2", "tc filter x1"]
        tuning = {"ms": [round(v, 1) for v in tms], "kept": names[choice]}
    torch.cuda.synchronize()
    dist_barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    device_ms, leaf_ms, launches, leaf_launches, pairs, stats_list = 0.0, 0.0, 0, 0, 0, []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = Stats()
        ctx.build_device(x.data_ptr(), n, DIM, ids.data_ptr(), None, params, stats=st)
        device_ms += st.ms_total + st.ms_finalize
        leaf_ms += st.ms_leaf_kernel
        launches += st.kernel_launches
        leaf_launches += st.leaf_launches
        pairs += st.bucket_pairs
        stats_list.append(st.as_dict())
    ev1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clock = clocks.stop()
    dist_barrier(world)
    stream_ms = ev0.elapsed_time(ev1)
    ms_step = dist_max(device_ms / args.steps, world)
    value = world * n / (ms_step / 1000.0)

    # Recall of the last build against the FP64 oracle on sampled points.
    q = np.random.default_rng(SEED).choice(n, min(QUERIES, n), replace=False)
    gt = groundtruth.exact_knn_torch(x, q, K)
    rec = groundtruth.recall(ids.cpu().numpy().view(np.uint32), gt, q)

    # End to end through the host-pointer ABI, pinned buffers.
    e2e = None
    if not args.no_e2e:
        host_in = torch.empty((n, DIM), dtype=torch.float32, pin_memory=True)
        host_in.copy_(x.cpu())
        host_out = torch.empty((n, K), dtype=torch.int32, pin_memory=True)
        x = ids = None
        torch.cuda.empty_cache()
        hin, hout = host_in.numpy(), host_out.numpy().view(np.uint32)
        lib = ctx._lib
        import ctypes

        from sigmod23ann_b200.api import _ptr

        def one():
            st = Stats()
            ctx._check(lib.knng_build(ctx._h, _ptr(hin), n, DIM, DIM * 4, ctypes.byref(params), _ptr(hout), None,
                                      ctypes.byref(st)))

        one()
        torch.cuda.synchronize()
        dist_barrier(world)
        times = []
        for _ in range(args.steps):
            t = time.perf_counter()
            one()
            times.append(time.perf_counter() - t)
        e_ms = dist_max(1000.0 * statistics.mean(times), world)
        e2e = {"value": sig(world * n / (e_ms / 1000.0)), "unit": "points/s", "h2d_bytes_per_step": n * DIM * 4,
               "d2h_bytes_per_step": n * K * 4, "ms_per_step": sig(e_ms)}

    # Adaptive schedule on the same points: repetitions and passes until the
    # recall estimated on 1,000 sampled points reaches 0.94 (at most 8 + 4);
    # its recall is checked on the line's own 10k-point FP64 sample.
    adaptive = None
    if args.extras and not args.no_e2e and world == 1 and not args.bf16:
        try:
            ap = default_params(k=K, max_leaf=max_leaf, max_leaf_odd=0, lloyd_iters=LLOYD_ITERS, reps=8, refine=4,
                                seed=SEED)
            ast = Stats()
            aids = ctx.build_adaptive(hin, 0.94, sample=1000, params=ap, stats=ast)
            adaptive = {"target": 0.94, "reps": int(ast.reps_done), "passes": int(ast.refine_passes_done),
                        "ms": sig(ast.ms_total + ast.ms_finalize), "recall_est": sig(ast.recall_estimate),
                        "recall": sig(groundtruth.recall(aids.astype(np.int64), gt, q))}
        except Exception as e:  # the adaptive figure must not hide the build number
            adaptive = {"error": str(e)[:200]}

    line = None
    if rank == 0:
        peaks = {}
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peaks = json.load(f)
        except OSError:
            pass
        hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
        # Dominant kernel: the tensor-core join of the neighbour-of-neighbour
        # pass.  Algorithmic bytes per launch: for every point q, the rows of
        # R(q) and S(q) (4d bytes each) and the lists S(p) of R(q) (4k bytes
        # each); sum_q |R(q)| = sum_q |S(q)| = n*k.
        join_ms = sum(st["ms_refine_join"] for st in stats_list)
        join_launches = sum(st["refine_join_launches"] for st in stats_list)
        per_launch_ms = join_ms / max(1, join_launches)
        bytes_per_launch = (2.0 * n * K * DIM * 4) + (1.0 * n * K * K * 4)
        achieved = bytes_per_launch / (per_launch_ms / 1000.0) / 1e9
        # DRAM bytes of one launch from the committed ncu capture at 500k
        # points, scaled by the points processed.
        traffic = JOIN_DRAM_BYTES_500K * n / 500_000
        roofline = {"bound": "hbm", "achieved": sig(achieved), "peak": hbm_peak, "unit": "GB/s",
                    "frac": sig(achieved / hbm_peak), "traffic": sig(traffic),
                    "kernel": "k_join", "peak_source": "measured" if peaks else "fallback",
                    "ms_per_launch": sig(per_launch_ms), "share_of_step": sig(join_ms / max(device_ms, 1e-9), 3)}
        last = stats_list[-1]
        stages = {k: round(last[v]) for k, v in (
            ("split", "ms_split"), ("buckets", "ms_leaf"), ("join", "ms_refine_join"), ("replay", "ms_refine_apply"),
            ("refine_prep", "ms_refine_prep"), ("finalize", "ms_finalize"))}
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(n, args.reps, args.refine, max_leaf, args.bf16, world),
            "clocks": {k: clock[k] for k in ("sm_mhz", "sm_max_mhz", "reasons") if k in clock},
            "gpu_launches": launches, "roofline": roofline, "e2e": e2e, "bucket_tuning": tuning,
            "stages_ms_last_step": stages,
            # The joins' pair funnel in the last step (both passes): pairs
            # evaluated, pairs the tensor-core bound kept, of those already in
            # the point's list, exact distances, survivor records.
            "join_pairs_last_step": {k: int(last[v]) for k, v in (
                ("pairs", "refine_pairs"), ("filter_kept", "refine_filter_pass"),
                ("members", "refine_member_skip"), ("exact", "refine_exact"), ("survivors", "refine_emits"))},
        }
        if adaptive is not None:
            line["adaptive"] = adaptive
    ctx.close()
    x = ids = None
    torch.cuda.empty_cache()
    extras = rank == 0 and world == 1 and not args.bf16
    if extras and args.extras:
        for key, fn in (("precision", lambda: precision_summary(run_precision(local, 3, cpu_reference=False))),
                        ("batched", lambda: batched_summary(run_batched(1, local))),
                        ("serving", lambda: serving_summary(run_serving_pair(args.serving_requests, local))),
                        ("kd_splitter", lambda: run_kd_compare(n, local, args.reps, max_leaf))):
            try:
                line[key] = fn()
            except Exception as e:  # an extra figure must not hide the build number
                line[key] = {"error": str(e)[:200]}
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        try:
            res = reference_sample_rate(n, args.reps, args.refine, args.cpu_seconds, 1, 0)
            if res:
                line["cpu_baseline"] = {
                    "value": sig(res["rates"][0]), "unit": "points/s", "cores": res["cores"], "kind": "reference",
                    "cpu": host_cpu_model()[:48], "sample": f"reference splitKmeansBinaryProcess x{args.reps} + topUpSingle x{args.refine}, all host "
                              f"threads, first {res['sample_points']:,} points of the same set"}
        except Exception as e:  # the baseline must not hide the GPU number
            line["cpu_baseline"] = {"error": str(e)[:200]}
    if rank == 0:
        # The recall of the measured build goes last, so the tail of the output
        # always holds it.
        line["recall"] = rec
        line["recall_queries"] = len(q)
        line["meets_recall_target"] = bool(rec >= 0.94)
        print(json.dumps(line))
    dist_done(world)
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.precision:
        res = run_precision()
        print(json.dumps({"metric": "precision form: recall change and speed vs the FP32 form (100k config)",
                          "value": res["bf16_rerank"]["points_per_s"], "unit": "points/s", "higher_is_better": True,
                          "n_gpus": 1, "dtype": "bf16 estimates + f32 re-rank", "precision": res}))
        return 0
    if args.batched:
        res = run_batched(args.batched_waves)
        print(json.dumps({"metric": "points/sec, batched k-NN graph builds (4,096 sets)", "value": res["points_per_s"],
                          "unit": "points/s", "higher_is_better": True, "n_gpus": 1, "dtype": "f32",
                          "batched": res}))
        return 0
    if args.kd:
        res = run_kd_compare(args.n, 0, args.reps, args.max_leaf or MAX_LEAF)
        if not args.no_cpu_baseline:
            cpu = oracle_kd_rate(args.n, args.max_leaf or MAX_LEAF, args.cpu_seconds)
            kd = res["kd"]
            cpu["gpu_points_per_s_per_rep"] = sig(args.n / ((kd["split_ms_per_rep"] + kd["bucket_ms_per_rep"]) / 1e3))
            res["cpu_baseline"] = cpu
        print(json.dumps({"metric": "KD splitter beside the 2-means splitter: ms per repetition, recall",
                          "value": res["kd"]["split_ms_per_rep"] + res["kd"]["bucket_ms_per_rep"], "unit": "ms",
                          "higher_is_better": False, "n_gpus": 1, "dtype": "f32", "kd_splitter": res}))
        return 0
    if args.serving:
        res = run_serving_pair(max(1, args.serving_requests))
        print(json.dumps({"metric": "p50/p99 latency of k-NN graph build jobs (serving stream)",
                          "value": res["at_70pct_capacity"]["p99_ms"], "unit": "ms", "higher_is_better": False,
                          "n_gpus": 1, "serving": res}))
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
