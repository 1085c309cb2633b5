"""Python host mirror of the C ABI in include/knng.h (ctypes over libknng.so).

The reference's entry point is ``SolutionKmeans::constructResult(points,
numPoints, result)`` (src/SolutionKmeans.hpp:558); :func:`construct_result`
mirrors it.  :class:`KnngContext` exposes every stage separately so tests can
feed the reference's intermediate state (hyperplanes, buckets, sets) and
compare.  There is no CPU fallback: if libknng.so is missing or no sm_100
device is present, the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, Structure, c_char_p, c_double, c_float, c_int, c_int32, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libknng.so")

KNNG_OK = 0
STATUS_NAMES = {
    0: "KNNG_OK", 1: "KNNG_ERR_INVALID_ARGUMENT", 2: "KNNG_ERR_CUDA", 3: "KNNG_ERR_OUT_OF_MEMORY",
    4: "KNNG_ERR_BUDGET", 5: "KNNG_ERR_STATE", 6: "KNNG_ERR_UNSUPPORTED", 7: "KNNG_ERR_NO_DEVICE",
    8: "KNNG_ERR_PENDING",
}
KNNG_ERR_PENDING = 8
JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3
PRECISION_FP32 = 0
PRECISION_BF16_RERANK = 1

# Every symbol include/knng.h declares (checked by the CPU test suite).
EXPORTED = [
    "knng_default_params", "knng_status_string", "knng_create", "knng_destroy", "knng_last_error", "knng_build",
    "knng_build_device", "knng_load_points", "knng_reset_sets", "knng_begin_rep", "knng_split_nodes",
    "knng_farthest_pair", "knng_lloyd", "knng_process_leaves", "knng_run_rep", "knng_run_rep_kd", "knng_build_kd", "knng_kd_rotation", "knng_tune_buckets", "knng_get_leaves", "knng_refine",
    "knng_get_indices", "knng_set_indices", "knng_get_sets", "knng_set_sets", "knng_finalize",
    "knng_debug_tile_gram", "knng_debug_tile_gram_bf16", "knng_debug_set_wait_limit", "knng_refine_pointwise_noalloc",
    "knng_build_batch",
    "knng_build_timed", "knng_build_adaptive", "knng_save_sets", "knng_load_sets", "knng_job_reservation", "knng_server_create", "knng_server_submit", "knng_server_poll", "knng_server_wait",
    "knng_server_job_error", "knng_server_release", "knng_server_destroy",
]


class Params(Structure):
    _fields_ = [
        ("k", c_uint32), ("max_leaf", c_uint32), ("max_leaf_odd", c_uint32), ("lloyd_iters", c_uint32),
        ("reps", c_uint32), ("refine", c_uint32), ("small_threshold", c_uint32), ("precision", c_uint32),
        ("seed", c_uint64),
    ]


class Stats(Structure):
    _fields_ = [
        ("ms_total", c_double), ("ms_split", c_double), ("ms_leaf", c_double), ("ms_leaf_kernel", c_double),
        ("ms_refine", c_double), ("ms_finalize", c_double),
        ("reps_done", c_uint64), ("split_levels", c_uint64), ("split_nodes", c_uint64), ("restarts", c_uint64),
        ("fallback_splits", c_uint64), ("buckets", c_uint64), ("bucket_pairs", c_uint64),
        ("bucket_pair_evals", c_uint64), ("leaf_launches", c_uint64), ("kernel_launches", c_uint64),
        ("refine_changed", c_uint64),
        ("ms_refine_join", c_double), ("ms_refine_apply", c_double), ("ms_refine_fallback", c_double),
        ("refine_pairs", c_uint64), ("refine_filter_pass", c_uint64), ("refine_member_skip", c_uint64),
        ("refine_exact", c_uint64), ("refine_emits", c_uint64), ("refine_overflow", c_uint64),
        ("ms_refine_prep", c_double), ("refine_join_launches", c_uint64), ("refine_lost", c_uint64),
        ("refine_passes_done", c_uint64), ("recall_estimate", c_double), ("estimate_queries", c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class JobInfo(Structure):
    _fields_ = [
        ("state", c_uint32), ("status", c_int32), ("n", c_uint32), ("d", c_uint32), ("k", c_uint32),
        ("reserved0", c_uint32), ("reserved_bytes", c_uint64), ("ms_queued", c_double), ("ms_run", c_double),
        ("ms_latency", c_double), ("stats", Stats),
    ]


class KnngError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


_lib = None


def load_library(path: str = LIB_PATH):
    """Loads libknng.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: run `python -m sigmod23ann_b200.build`")
    lib = ctypes.CDLL(path)
    P = c_void_p
    sigs = {
        "knng_default_params": (None, [POINTER(Params)]),
        "knng_status_string": (c_char_p, [c_int]),
        "knng_create": (c_int, [c_int, c_uint64, POINTER(c_void_p)]),
        "knng_destroy": (c_int, [P]),
        "knng_last_error": (c_char_p, [P]),
        "knng_build": (c_int, [P, P, c_uint32, c_uint32, c_uint64, POINTER(Params), P, P, POINTER(Stats)]),
        "knng_build_device": (c_int, [P, P, c_uint32, c_uint32, c_uint64, POINTER(Params), P, P, POINTER(Stats)]),
        "knng_load_points": (c_int, [P, P, c_uint32, c_uint32, c_uint64, c_int]),
        "knng_reset_sets": (c_int, [P, c_uint32]),
        "knng_begin_rep": (c_int, [P]),
        "knng_split_nodes": (c_int, [P, c_uint32, P, P, P, P, P]),
        "knng_farthest_pair": (c_int, [P, c_uint32, P, P, P, P, P]),
        "knng_lloyd": (c_int, [P, c_uint32, P, P, P, P, P, P, c_uint32, P, P, P]),
        "knng_process_leaves": (c_int, [P, c_uint32, P, P]),
        "knng_run_rep": (c_int, [P, c_uint32, c_uint32, c_uint32, c_uint64, c_uint32, POINTER(Stats)]),
        "knng_run_rep_kd": (c_int, [P, c_uint32, c_uint32, c_uint64, c_uint32, POINTER(Stats)]),
        "knng_build_kd": (c_int, [P, P, c_uint32, c_uint32, c_uint64, POINTER(Params), c_uint32, P, P,
                                  POINTER(Stats)]),
        "knng_kd_rotation": (c_int, [c_uint32, c_uint32, c_uint64, P]),
        "knng_tune_buckets": (c_int, [P, c_uint32, c_uint32, c_uint32, c_uint64, POINTER(ctypes.c_double),
                                      POINTER(c_uint32)]),
        "knng_get_leaves": (c_int, [P, c_uint32, P, P, P]),
        "knng_refine": (c_int, [P, P, POINTER(Stats)]),
        "knng_get_indices": (c_int, [P, P]),
        "knng_set_indices": (c_int, [P, P]),
        "knng_get_sets": (c_int, [P, P, P, P, P, P]),
        "knng_set_sets": (c_int, [P, P, P, P, P, P]),
        "knng_finalize": (c_int, [P, P, P]),
        "knng_debug_tile_gram": (c_int, [P, P, c_uint32, P, c_uint32, c_uint32, P]),
        "knng_debug_set_wait_limit": (c_int, [P, c_uint32]),
        "knng_debug_tile_gram_bf16": (c_int, [P, P, c_uint32, P, c_uint32, c_uint32, P]),
        "knng_refine_pointwise_noalloc": (c_int, [P, c_uint32, c_uint32, c_uint32, P, P, P, P, P, P, P, P]),
        "knng_save_sets": (c_int, [P, c_char_p]),
        "knng_load_sets": (c_int, [P, c_char_p]),
        "knng_build_timed": (c_int, [P, P, c_uint32, c_uint32, c_uint64, POINTER(Params), c_uint64, c_uint64, P, P,
                                     POINTER(Stats)]),
        "knng_build_adaptive": (c_int, [P, P, c_uint32, c_uint32, c_uint64, POINTER(Params), c_double, c_uint32, P, P,
                                        POINTER(Stats)]),
        "knng_build_batch": (c_int, [P, P, c_uint32, c_uint32, c_uint64, P, c_uint32, c_int, POINTER(Params), P, P,
                                     POINTER(Stats)]),
        "knng_job_reservation": (c_uint64, [c_uint32, c_uint32, c_uint32]),
        "knng_server_create": (c_int, [c_int, c_uint64, c_uint32, POINTER(c_void_p)]),
        "knng_server_submit": (c_int, [P, P, c_uint32, c_uint32, c_uint64, POINTER(Params), P, P,
                                       POINTER(c_uint64)]),
        "knng_server_poll": (c_int, [P, c_uint64, POINTER(JobInfo)]),
        "knng_server_wait": (c_int, [P, c_uint64, ctypes.c_int64, POINTER(JobInfo)]),
        "knng_server_job_error": (c_char_p, [P, c_uint64]),
        "knng_server_release": (c_int, [P, c_uint64]),
        "knng_server_destroy": (c_int, [P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def default_params(**overrides) -> Params:
    p = Params()
    load_library().knng_default_params(ctypes.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def kd_params(**overrides) -> Params:
    """The reference's KD form (src/SolutionRandomKD.hpp:377-430): 5
    repetitions, buckets below 400 points, no neighbour-of-neighbour pass."""
    base = dict(reps=5, max_leaf=400, max_leaf_odd=0, refine=0)
    base.update(overrides)
    return default_params(**base)


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(c_void_p)
    if isinstance(a, int):
        return c_void_p(a)
    return c_void_p(a.data_ptr())  # torch tensor


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class KnngContext:
    """One device context (not re-entrant)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self._lib = load_library()
        h = c_void_p()
        self._check(self._lib.knng_create(device, hbm_budget_bytes, ctypes.byref(h)), ctx=None)
        self._h = h
        self.n = 0
        self.d = 0
        self.k = 0

    # ------------------------------------------------------------- plumbing
    def _check(self, status: int, ctx="self"):
        if status != KNNG_OK:
            msg = ""
            if ctx is not None and getattr(self, "_h", None):
                raw = self._lib.knng_last_error(self._h)
                msg = raw.decode() if raw else ""
            if not msg:
                msg = self._lib.knng_status_string(status).decode()
            raise KnngError(status, msg)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.knng_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------- one call
    def build(self, points: np.ndarray, params: Params | None = None, want_dists: bool = False,
              stats: Stats | None = None):
        pts = _f32(points)
        n, d = pts.shape
        p = params or default_params()
        ids = np.empty((n, p.k), np.uint32)
        dists = np.empty((n, p.k), np.float32) if want_dists else None
        st = stats if stats is not None else Stats()
        self._check(self._lib.knng_build(self._h, _ptr(pts), n, d, pts.strides[0], ctypes.byref(p), _ptr(ids),
                                         _ptr(dists), ctypes.byref(st)))
        self.n, self.d, self.k = n, d, p.k
        return (ids, dists) if want_dists else ids

    def build_kd(self, points: np.ndarray, params: Params | None = None, new_dims: int = 30,
                 want_dists: bool = False, stats: Stats | None = None):
        """knng_build_kd: a whole build with the random-rotation KD splitter
        (default: the reference's KD form, kd_params())."""
        pts = _f32(points)
        n, d = pts.shape
        p = params or kd_params()
        ids = np.empty((n, p.k), np.uint32)
        dists = np.empty((n, p.k), np.float32) if want_dists else None
        st = stats if stats is not None else Stats()
        self._check(self._lib.knng_build_kd(self._h, _ptr(pts), n, d, pts.strides[0], ctypes.byref(p), new_dims,
                                            _ptr(ids), _ptr(dists), ctypes.byref(st)))
        self.n, self.d, self.k = n, d, p.k
        return (ids, dists) if want_dists else ids

    def build_timed(self, points: np.ndarray, build_ms: int, refine_ms: int, params: Params | None = None,
                    want_dists: bool = False, stats: Stats | None = None):
        """knng_build_timed: repetitions while build_ms has not passed, then
        refinement passes while build_ms + refine_ms has not."""
        pts = _f32(points)
        n, d = pts.shape
        p = params or default_params()
        ids = np.empty((n, p.k), np.uint32)
        dists = np.empty((n, p.k), np.float32) if want_dists else None
        st = stats if stats is not None else Stats()
        self._check(self._lib.knng_build_timed(self._h, _ptr(pts), n, d, pts.strides[0], ctypes.byref(p), build_ms,
                                               refine_ms, _ptr(ids), _ptr(dists), ctypes.byref(st)))
        self.n, self.d, self.k = n, d, p.k
        return (ids, dists) if want_dists else ids

    def build_adaptive(self, points: np.ndarray, target_recall: float, sample: int = 1000,
                       params: Params | None = None, want_dists: bool = False, stats: Stats | None = None):
        """knng_build_adaptive: repetitions and passes until the recall estimated
        on `sample` points reaches target_recall (params.reps / params.refine
        are the maxima)."""
        pts = _f32(points)
        n, d = pts.shape
        p = params or default_params()
        ids = np.empty((n, p.k), np.uint32)
        dists = np.empty((n, p.k), np.float32) if want_dists else None
        st = stats if stats is not None else Stats()
        self._check(self._lib.knng_build_adaptive(self._h, _ptr(pts), n, d, pts.strides[0], ctypes.byref(p),
                                                  target_recall, sample, _ptr(ids), _ptr(dists), ctypes.byref(st)))
        self.n, self.d, self.k = n, d, p.k
        return (ids, dists) if want_dists else ids

    def build_batch(self, sets, params: Params | None = None, want_dists: bool = False,
                    stats: Stats | None = None):
        """Builds every point set of `sets` (a list of n_s x d float32 arrays)
        in one batched build; returns per-set id arrays (ids relative to the
        set), and distance arrays when asked."""
        arrays = [_f32(a) for a in sets]
        offsets = np.zeros(len(arrays) + 1, np.uint32)
        offsets[1:] = np.cumsum([a.shape[0] for a in arrays])
        pts = np.ascontiguousarray(np.concatenate(arrays, axis=0))
        n, d = pts.shape
        p = params or default_params()
        ids = np.empty((n, p.k), np.uint32)
        dists = np.empty((n, p.k), np.float32) if want_dists else None
        st = stats if stats is not None else Stats()
        self._check(self._lib.knng_build_batch(self._h, _ptr(pts), n, d, pts.strides[0], _ptr(offsets),
                                               len(arrays), 0, ctypes.byref(p), _ptr(ids), _ptr(dists),
                                               ctypes.byref(st)))
        self.n, self.d, self.k = n, d, p.k
        out_ids = [ids[offsets[s]:offsets[s + 1]] for s in range(len(arrays))]
        if not want_dists:
            return out_ids
        return out_ids, [dists[offsets[s]:offsets[s + 1]] for s in range(len(arrays))]

    def build_device(self, points_ptr: int, n: int, d: int, out_ids_ptr: int, out_dists_ptr: int | None = None,
                     params: Params | None = None, stats: Stats | None = None, ld_bytes: int = 0) -> Stats:
        """Device-resident build: pointers are device addresses (e.g. torch data_ptr())."""
        p = params or default_params()
        st = stats if stats is not None else Stats()
        self._check(self._lib.knng_build_device(self._h, c_void_p(points_ptr), n, d, ld_bytes or 4 * d,
                                                ctypes.byref(p), c_void_p(out_ids_ptr),
                                                c_void_p(out_dists_ptr) if out_dists_ptr else None,
                                                ctypes.byref(st)))
        self.n, self.d, self.k = n, d, p.k
        return st

    # ------------------------------------------------------------- stepwise
    def load_points(self, points: np.ndarray) -> None:
        pts = _f32(points)
        self.n, self.d = pts.shape
        self._check(self._lib.knng_load_points(self._h, _ptr(pts), self.n, self.d, pts.strides[0], 0))

    def reset_sets(self, k: int) -> None:
        self._check(self._lib.knng_reset_sets(self._h, k))
        self.k = k

    def begin_rep(self) -> None:
        self._check(self._lib.knng_begin_rep(self._h))

    def split_nodes(self, starts, ends, coefs, offsets) -> np.ndarray:
        s, e, c, o = _u32(starts), _u32(ends), _f32(coefs), _f32(offsets)
        mids = np.zeros(len(s), np.uint32)
        self._check(self._lib.knng_split_nodes(self._h, len(s), _ptr(s), _ptr(e), _ptr(c), _ptr(o), _ptr(mids)))
        return mids

    def farthest_pair(self, offsets, positions):
        off = np.ascontiguousarray(offsets, np.uint64)
        pos = _u32(positions)
        m = len(off) - 1
        f = np.zeros(m, np.uint32)
        s = np.zeros(m, np.uint32)
        ok = np.zeros(m, np.int32)
        self._check(self._lib.knng_farthest_pair(self._h, m, _ptr(off), _ptr(pos), _ptr(f), _ptr(s), _ptr(ok)))
        return f, s, ok

    def lloyd(self, starts, ends, lloyd_offsets, lloyd_positions, c1, c2, iters: int):
        s, e = _u32(starts), _u32(ends)
        off = np.ascontiguousarray(lloyd_offsets, np.uint64)
        pos = _u32(lloyd_positions)
        a, b = _f32(c1), _f32(c2)
        m = len(s)
        coefs = np.zeros((m, self.d), np.float32)
        offs = np.zeros(m, np.float32)
        ok = np.zeros(m, np.int32)
        self._check(self._lib.knng_lloyd(self._h, m, _ptr(s), _ptr(e), _ptr(off), _ptr(pos), _ptr(a), _ptr(b),
                                         iters, _ptr(coefs), _ptr(offs), _ptr(ok)))
        return coefs, offs, ok

    def process_leaves(self, starts, ends) -> None:
        s, e = _u32(starts), _u32(ends)
        self._check(self._lib.knng_process_leaves(self._h, len(s), _ptr(s), _ptr(e)))

    def run_rep(self, max_leaf: int, lloyd_iters: int, small_threshold: int = 3000, seed: int = 12345,
                rep_index: int = 0, stats: Stats | None = None) -> Stats:
        st = stats if stats is not None else Stats()
        self._check(self._lib.knng_run_rep(self._h, max_leaf, lloyd_iters, small_threshold, seed, rep_index,
                                           ctypes.byref(st)))
        return st

    def run_rep_kd(self, max_leaf: int, new_dims: int = 30, seed: int = 12345, rep_index: int = 0,
                   stats: Stats | None = None) -> Stats:
        """knng_run_rep_kd: one repetition with the random-rotation KD splitter."""
        st = stats if stats is not None else Stats()
        self._check(self._lib.knng_run_rep_kd(self._h, max_leaf, new_dims, seed, rep_index, ctypes.byref(st)))
        return st

    def tune_buckets(self, max_leaf: int, lloyd_iters: int, small_threshold: int = 3000,
                     seed: int = 12345) -> tuple[list[float], int]:
        """knng_tune_buckets: bucket-pass ms of the four variants (every pair /
        tensor-core filtered, x 2 / 1 CTAs per SM) on one repetition of the
        current points and sets (restored afterwards), and the variant kept."""
        ms = (ctypes.c_double * 4)()
        choice = c_uint32()
        self._check(self._lib.knng_tune_buckets(self._h, max_leaf, lloyd_iters, small_threshold, seed, ms,
                                                ctypes.byref(choice)))
        return [float(v) for v in ms], int(choice.value)

    def leaves(self):
        cnt = c_uint32()
        self._check(self._lib.knng_get_leaves(self._h, 0, None, None, ctypes.byref(cnt)))
        s = np.zeros(cnt.value, np.uint32)
        e = np.zeros(cnt.value, np.uint32)
        self._check(self._lib.knng_get_leaves(self._h, cnt.value, _ptr(s), _ptr(e), ctypes.byref(cnt)))
        return s, e

    def refine(self, stats: Stats | None = None) -> int:
        out = np.zeros(1, np.uint64)
        self._check(self._lib.knng_refine(self._h, _ptr(out), ctypes.byref(stats) if stats is not None else None))
        return int(out[0])

    def indices(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint32)
        self._check(self._lib.knng_get_indices(self._h, _ptr(out)))
        return out

    def set_indices(self, idx) -> None:
        a = _u32(idx)
        self._check(self._lib.knng_set_indices(self._h, _ptr(a)))

    def sets(self) -> dict:
        n, k = self.n, self.k
        out = {
            "dist": np.zeros((n, k), np.float32), "id": np.zeros((n, k), np.uint32),
            "size": np.zeros(n, np.uint32), "maxslot": np.zeros(n, np.uint32), "bound": np.zeros(n, np.float32),
        }
        self._check(self._lib.knng_get_sets(self._h, *(_ptr(out[x]) for x in ("dist", "id", "size", "maxslot",
                                                                              "bound"))))
        return out

    def set_sets(self, s: dict) -> None:
        arrs = [_f32(s["dist"]), _u32(s["id"]), _u32(s["size"]), _u32(s["maxslot"]), _f32(s["bound"])]
        self._check(self._lib.knng_set_sets(self._h, *(_ptr(a) for a in arrs)))

    def save_sets(self, path: str) -> None:
        """Writes the neighbour sets to a file (knng_save_sets)."""
        self._check(self._lib.knng_save_sets(self._h, os.fsencode(path)))

    def load_sets(self, path: str) -> None:
        """Reads neighbour sets saved for the same points (knng_load_sets)."""
        self._check(self._lib.knng_load_sets(self._h, os.fsencode(path)))
        with open(path, "rb") as f:
            f.seek(16)
            self.k = int(np.frombuffer(f.read(4), np.uint32)[0])

    def finalize(self, want_dists: bool = False):
        ids = np.zeros((self.n, self.k), np.uint32)
        dists = np.zeros((self.n, self.k), np.float32) if want_dists else None
        self._check(self._lib.knng_finalize(self._h, _ptr(ids), _ptr(dists)))
        return (ids, dists) if want_dists else ids


def debug_set_wait_limit(ctx: "KnngContext", polls: int) -> None:
    """Poll limit of the kernels' bounded waits on the context's device (diagnostic; default 2**26)."""
    ctx._check(ctx._lib.knng_debug_set_wait_limit(ctx._h, polls))


def debug_tile_gram(ctx: "KnngContext", a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """a . b^T through one tcgen05 tile, FP16 operands, FP32 accumulation (diagnostic)."""
    a = _f32(a)
    b = _f32(b)
    out = np.zeros((a.shape[0], b.shape[0]), np.float32)
    ctx._check(ctx._lib.knng_debug_tile_gram(ctx._h, _ptr(a), a.shape[0], _ptr(b), b.shape[0], a.shape[1], _ptr(out)))
    return out


def debug_tile_gram_bf16(ctx: "KnngContext", a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """a . b^T through one tcgen05 BF16 tile, FP32 accumulation (diagnostic)."""
    a = _f32(a)
    b = _f32(b)
    out = np.zeros((a.shape[0], b.shape[0]), np.float32)
    ctx._check(ctx._lib.knng_debug_tile_gram_bf16(ctx._h, _ptr(a), a.shape[0], _ptr(b), b.shape[0], a.shape[1],
                                                  _ptr(out)))
    return out


def construct_result(points: np.ndarray, params: Params | None = None, device: int = 0) -> np.ndarray:
    """SolutionKmeans::constructResult (src/SolutionKmeans.hpp:558-616) on the GPU:
    returns the n x k neighbour ids, sorted by (distance, id), short rows padded with id 1."""
    with KnngContext(device) as ctx:
        return ctx.build(points, params)


class KnngServer:
    """Serving form (knng_server_*): build jobs queued as they arrive, admitted
    in arrival order within an HBM budget, up to `max_running` at once, each on
    its own device context and stream.  A job's host buffers are held by this
    object until the job is released."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, max_running: int = 4):
        self._lib = load_library()
        h = c_void_p()
        st = self._lib.knng_server_create(device, hbm_budget_bytes, max_running, ctypes.byref(h))
        if st != KNNG_OK:
            raise KnngError(st, self._lib.knng_status_string(st).decode())
        self._h = h
        self._buffers: dict[int, tuple] = {}

    def submit(self, points: np.ndarray, params: Params | None = None, want_dists: bool = False) -> int:
        """Queues a build of `points` (n x d float32, rows may be strided);
        returns the job id."""
        pts = points if points.dtype == np.float32 and points.strides[1] == 4 else _f32(points)
        n, d = pts.shape
        p = params or default_params()
        ids = np.empty((n, p.k), np.uint32)
        dists = np.empty((n, p.k), np.float32) if want_dists else None
        job = c_uint64()
        st = self._lib.knng_server_submit(self._h, _ptr(pts), n, d, pts.strides[0], ctypes.byref(p), _ptr(ids),
                                          _ptr(dists), ctypes.byref(job))
        if st != KNNG_OK:
            raise KnngError(st, self._lib.knng_status_string(st).decode())
        self._buffers[job.value] = (pts, p, ids, dists)
        return job.value

    def poll(self, job: int) -> JobInfo:
        info = JobInfo()
        st = self._lib.knng_server_poll(self._h, job, ctypes.byref(info))
        if st != KNNG_OK:
            raise KnngError(st, self._lib.knng_status_string(st).decode())
        return info

    def wait(self, job: int, timeout_ms: int = -1) -> JobInfo | None:
        """The job's info once it has ended, or None after timeout_ms."""
        info = JobInfo()
        st = self._lib.knng_server_wait(self._h, job, timeout_ms, ctypes.byref(info))
        if st == KNNG_ERR_PENDING:
            return None
        if st != KNNG_OK:
            raise KnngError(st, self._lib.knng_status_string(st).decode())
        return info

    def result(self, job: int):
        """(ids, dists or None) of an ended job; raises if it failed."""
        info = self.wait(job)
        if info.state != JOB_DONE:
            msg = self._lib.knng_server_job_error(self._h, job)
            raise KnngError(info.status, msg.decode() if msg else "")
        _, _, ids, dists = self._buffers[job]
        return ids, dists

    def release(self, job: int) -> None:
        st = self._lib.knng_server_release(self._h, job)
        if st != KNNG_OK:
            raise KnngError(st, self._lib.knng_status_string(st).decode())
        self._buffers.pop(job, None)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.knng_server_destroy(self._h)
            self._h = None
            self._buffers.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def job_reservation(n: int, d: int, k: int) -> int:
    """HBM bytes a served job of n points, d dims, k neighbours reserves."""
    return int(load_library().knng_job_reservation(n, d, k))


def kd_rotation(new_dims: int, d: int, seed: int) -> np.ndarray:
    """knng_kd_rotation: the KD splitter's rotation vectors (new_dims x d), host only."""
    out = np.zeros((new_dims, d), np.float32)
    status = load_library().knng_kd_rotation(new_dims, d, seed, out.ctypes.data_as(c_void_p))
    if status != 0:
        raise KnngError(status, "knng_kd_rotation refused its arguments")
    return out
