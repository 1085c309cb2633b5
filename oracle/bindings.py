"""ctypes bindings for the CPU checkers (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
bench.py may import this module.  It wraps

* ``oracle/_build/libknng_oracle.so`` -- the C++ restatement in cpu_ref.cpp;
* ``oracle/_ref/libref_{serial,threads}.so`` -- the reference's own headers
  compiled against the stand-ins in oracle/ref_shim (built only where the
  reference tree exists; the prebuilt files travel with the repository).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_float, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libknng_oracle.so")
REF_SERIAL_SO = os.path.join(HERE, "_ref", "libref_serial.so")
REF_THREADS_SO = os.path.join(HERE, "_ref", "libref_threads.so")
# The reference's source tree: KNNG_REFERENCE_SRC, else beside this
# repository (../reference/src from its root).
REFERENCE_SRC = os.environ.get("KNNG_REFERENCE_SRC",
                               os.path.normpath(os.path.join(HERE, "..", "..", "reference", "src")))
# The reference's own test fixture (u32 N, then N x 100 float32), beside its sources.
REFERENCE_FIXTURE = os.path.join(os.path.dirname(REFERENCE_SRC), "dummy-data.bin")


def build(with_reference: bool | None = None) -> None:
    """Compile the oracle (and, where the reference tree exists, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if with_reference is None:
        with_reference = os.path.isdir(REFERENCE_SRC)
    if with_reference:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_SRC={REFERENCE_SRC}"], check=True)


def reference_available() -> bool:
    return os.path.exists(REF_SERIAL_SO) and os.path.exists(REF_THREADS_SO)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(c_void_p)


_oracle_lib = None


def _olib():
    global _oracle_lib
    if _oracle_lib is None:
        if not os.path.exists(ORACLE_SO):
            build(with_reference=False)
        lib = ctypes.CDLL(ORACLE_SO)
        lib.ko_create.restype = c_void_p
        lib.ko_create.argtypes = [c_void_p, c_uint32, c_uint32, c_uint32, c_uint32, c_uint32, c_uint64]
        lib.ko_destroy.argtypes = [c_void_p]
        lib.ko_set_small_threshold.argtypes = [c_void_p, c_uint32]
        lib.ko_rep.argtypes = [c_void_p, c_uint32, c_uint32, c_uint32]
        lib.ko_refine.argtypes = [c_void_p]
        lib.ko_refine.restype = c_uint64
        lib.ko_process_leaves.argtypes = [c_void_p, c_uint32, c_void_p, c_void_p]
        lib.ko_get_indices.argtypes = [c_void_p, c_void_p]
        lib.ko_set_indices.argtypes = [c_void_p, c_void_p]
        lib.ko_get_sets.argtypes = [c_void_p] + [c_void_p] * 5
        lib.ko_set_sets.argtypes = [c_void_p] + [c_void_p] * 5
        lib.ko_finalize.argtypes = [c_void_p, c_void_p, c_void_p]
        lib.ko_trace_count.argtypes = [c_void_p]
        lib.ko_trace_count.restype = c_uint32
        lib.ko_trace_get.argtypes = [c_void_p] + [c_void_p] * 10
        lib.ko_trace_lloyd_total.argtypes = [c_void_p]
        lib.ko_trace_lloyd_total.restype = c_uint64
        lib.ko_trace_lloyd.argtypes = [c_void_p, c_void_p, c_void_p]
        lib.ko_trace_start_total.argtypes = [c_void_p]
        lib.ko_trace_start_total.restype = c_uint64
        lib.ko_trace_start.argtypes = [c_void_p, c_void_p, c_void_p]
        lib.ko_leaf_count.argtypes = [c_void_p]
        lib.ko_leaf_count.restype = c_uint32
        lib.ko_leaves.argtypes = [c_void_p, c_void_p, c_void_p]
        lib.ko_lloyd.argtypes = [c_void_p, c_void_p, c_uint64, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p]
        lib.ko_lloyd.restype = ctypes.c_int
        lib.ko_distance.argtypes = [c_void_p, c_void_p, c_uint32]
        lib.ko_distance.restype = c_float
        lib.ko_dot.argtypes = [c_void_p, c_void_p, c_uint32]
        lib.ko_dot.restype = c_float
        lib.ko_sample_count.argtypes = [c_uint32]
        lib.ko_sample_count.restype = c_uint32
        lib.ko_start_count.argtypes = [c_uint32]
        lib.ko_start_count.restype = c_uint32
        lib.ko_counter_position.argtypes = [c_uint64, c_uint32, c_uint32, c_uint32, c_uint32, c_uint32]
        lib.ko_counter_position.restype = c_uint32
        lib.ko_knnset_replay.argtypes = [c_uint32, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
        lib.ko_kd_vectors.argtypes = [c_uint32, c_uint32, c_uint64, c_void_p]
        lib.ko_kd_rotate.argtypes = [c_void_p, c_void_p, c_uint32, c_void_p]
        lib.ko_kd_rep.argtypes = [c_void_p, c_uint32, c_uint32, c_uint64, c_uint32]
        _oracle_lib = lib
    return _oracle_lib


def distance(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(_olib().ko_distance(_ptr(a), _ptr(b), a.shape[0]))


def dot(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(_olib().ko_dot(_ptr(a), _ptr(b), a.shape[0]))


def kd_vectors(new_dims: int, d: int, seed: int) -> np.ndarray:
    """The KD solution's rotation vectors (new_dims x d) from a mt19937 seeded with seed."""
    out = np.zeros((new_dims, d), np.float32)
    _olib().ko_kd_vectors(new_dims, d, seed, _ptr(out))
    return out


def sample_count(n: int) -> int:
    return int(_olib().ko_sample_count(n))


def start_count(n: int) -> int:
    return int(_olib().ko_start_count(n))


def counter_position(seed: int, rep: int, start: int, end: int, attempt: int, t: int) -> int:
    return int(_olib().ko_counter_position(seed, rep, start, end, attempt, t))


def knnset_replay(k: int, ids: np.ndarray, dists: np.ndarray):
    """Offers (ids[t], dists[t]) in order to one empty set; returns its state."""
    ids = np.ascontiguousarray(ids, np.uint32)
    dists = np.ascontiguousarray(dists, np.float32)
    od = np.zeros(k, np.float32)
    oi = np.zeros(k, np.uint32)
    sz = np.zeros(1, np.uint32)
    ms = np.zeros(1, np.uint32)
    bd = np.zeros(1, np.float32)
    _olib().ko_knnset_replay(k, _ptr(ids), _ptr(dists), len(ids), _ptr(od), _ptr(oi), _ptr(sz), _ptr(ms), _ptr(bd))
    return {"dist": od, "id": oi, "size": int(sz[0]), "maxslot": int(ms[0]), "bound": float(bd[0])}


class Oracle:
    """The C++ restatement; one instance per point set."""

    def __init__(self, points: np.ndarray, k: int = 100, rng_mode: int = 0, seed: int = 12345,
                 small_threshold: int = 3000):
        pts = np.ascontiguousarray(points, np.float32)
        self.n, self.d = pts.shape
        self.k = k
        self._lib = _olib()
        self._h = self._lib.ko_create(_ptr(pts), self.n, self.d, self.d, k, rng_mode, seed)
        self._lib.ko_set_small_threshold(self._h, small_threshold)

    def close(self):
        if self._h:
            self._lib.ko_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rep(self, iters: int, max_group: int, rep_index: int = 0) -> None:
        self._lib.ko_rep(self._h, iters, max_group, rep_index)

    def refine(self) -> int:
        return int(self._lib.ko_refine(self._h))

    def kd_rep(self, max_leaf: int, new_dims: int = 30, seed: int = 12345, rep_index: int = 0) -> None:
        """One repetition with the random-rotation KD splitter."""
        self._lib.ko_kd_rep(self._h, max_leaf, new_dims, seed, rep_index)

    def kd_rotate(self, vectors: np.ndarray) -> np.ndarray:
        """rot[p, c] = dot(vectors[c], x_p) with the reference's dot."""
        v = np.ascontiguousarray(vectors, np.float32)
        out = np.zeros((self.n, v.shape[0]), np.float32)
        self._lib.ko_kd_rotate(self._h, _ptr(v), v.shape[0], _ptr(out))
        return out

    def lloyd(self, ids: np.ndarray, c1: np.ndarray, c2: np.ndarray, iters: int):
        """Lloyd steps over the point ids in the given order from centres c1, c2;
        returns (coefs, offset, ok)."""
        a = np.ascontiguousarray(ids, np.uint32)
        x = np.ascontiguousarray(c1, np.float32)
        y = np.ascontiguousarray(c2, np.float32)
        coefs = np.zeros(self.d, np.float32)
        off = np.zeros(1, np.float32)
        ok = self._lib.ko_lloyd(self._h, _ptr(a), len(a), _ptr(x), _ptr(y), iters, _ptr(coefs), _ptr(off))
        return coefs, off[0], bool(ok)

    def process_leaves(self, starts: np.ndarray, ends: np.ndarray) -> None:
        s = np.ascontiguousarray(starts, np.uint32)
        e = np.ascontiguousarray(ends, np.uint32)
        self._lib.ko_process_leaves(self._h, len(s), _ptr(s), _ptr(e))

    def indices(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint32)
        self._lib.ko_get_indices(self._h, _ptr(out))
        return out

    def set_indices(self, idx: np.ndarray) -> None:
        a = np.ascontiguousarray(idx, np.uint32)
        self._lib.ko_set_indices(self._h, _ptr(a))

    def sets(self) -> dict:
        n, k = self.n, self.k
        out = {
            "dist": np.zeros((n, k), np.float32),
            "id": np.zeros((n, k), np.uint32),
            "size": np.zeros(n, np.uint32),
            "maxslot": np.zeros(n, np.uint32),
            "bound": np.zeros(n, np.float32),
        }
        self._lib.ko_get_sets(self._h, *(_ptr(out[x]) for x in ("dist", "id", "size", "maxslot", "bound")))
        return out

    def set_sets(self, s: dict) -> None:
        arrs = [np.ascontiguousarray(s["dist"], np.float32), np.ascontiguousarray(s["id"], np.uint32),
                np.ascontiguousarray(s["size"], np.uint32), np.ascontiguousarray(s["maxslot"], np.uint32),
                np.ascontiguousarray(s["bound"], np.float32)]
        self._lib.ko_set_sets(self._h, *(_ptr(a) for a in arrs))

    def finalize(self):
        ids = np.zeros((self.n, self.k), np.uint32)
        dist = np.zeros((self.n, self.k), np.float32)
        self._lib.ko_finalize(self._h, _ptr(ids), _ptr(dist))
        return ids, dist

    def trace(self) -> dict:
        m = int(self._lib.ko_trace_count(self._h))
        d = self.d
        t = {
            "start": np.zeros(m, np.uint32), "end": np.zeros(m, np.uint32), "depth": np.zeros(m, np.uint32),
            "mid": np.zeros(m, np.uint32), "large": np.zeros(m, np.uint32), "attempts": np.zeros(m, np.uint32),
            "coefs": np.zeros((m, d), np.float32), "offset": np.zeros(m, np.float32),
            "c1_start": np.zeros((m, d), np.float32), "c2_start": np.zeros((m, d), np.float32),
        }
        self._lib.ko_trace_get(self._h, *(_ptr(t[x]) for x in ("start", "end", "depth", "mid", "large", "attempts",
                                                                "coefs", "offset", "c1_start", "c2_start")))
        tot = int(self._lib.ko_trace_lloyd_total(self._h))
        t["lloyd_off"] = np.zeros(m + 1, np.uint64)
        t["lloyd_pos"] = np.zeros(max(tot, 1), np.uint32)
        self._lib.ko_trace_lloyd(self._h, _ptr(t["lloyd_off"]), _ptr(t["lloyd_pos"]))
        tot = int(self._lib.ko_trace_start_total(self._h))
        t["start_off"] = np.zeros(m + 1, np.uint64)
        t["start_pos"] = np.zeros(max(tot, 1), np.uint32)
        self._lib.ko_trace_start(self._h, _ptr(t["start_off"]), _ptr(t["start_pos"]))
        nl = int(self._lib.ko_leaf_count(self._h))
        t["leaf_start"] = np.zeros(nl, np.uint32)
        t["leaf_end"] = np.zeros(nl, np.uint32)
        self._lib.ko_leaves(self._h, _ptr(t["leaf_start"]), _ptr(t["leaf_end"]))
        return t


class ReferenceShim:
    """The reference's own SolutionKmeans code (d = k = 100 only)."""

    def __init__(self, points: np.ndarray, threaded: bool = False):
        path = REF_THREADS_SO if threaded else REF_SERIAL_SO
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (needs the reference sources)")
        lib = ctypes.CDLL(path)
        lib.ref_create.restype = c_void_p
        lib.ref_create.argtypes = [c_void_p, c_uint32, c_uint32]
        lib.ref_destroy.argtypes = [c_void_p]
        lib.ref_reseed.argtypes = [c_uint32]
        lib.ref_rep.argtypes = [c_void_p, c_uint32, c_uint32]
        lib.ref_topup.argtypes = [c_void_p]
        lib.ref_topup.restype = c_uint64
        lib.ref_get_indices.argtypes = [c_void_p, c_void_p]
        lib.ref_get_sets.argtypes = [c_void_p] + [c_void_p] * 5
        lib.ref_finalize.argtypes = [c_void_p, c_void_p]
        lib.ref_distance.argtypes = [c_void_p, c_void_p]
        lib.ref_distance.restype = c_float
        lib.ref_dot.argtypes = [c_void_p, c_void_p]
        lib.ref_dot.restype = c_float
        lib.ref_kd_rotate.argtypes = [c_void_p, c_uint32, c_void_p]
        lib.ref_knnset_replay.argtypes = [c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
        self._lib = lib
        pts = np.ascontiguousarray(points, np.float32)
        assert pts.shape[1] == 100, "the reference is compiled for 100 dimensions"
        self.n = pts.shape[0]
        self._h = lib.ref_create(_ptr(pts), self.n, 100)

    def close(self):
        if self._h:
            self._lib.ref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reseed(self, seed: int = 12345) -> None:
        self._lib.ref_reseed(seed)

    def rep(self, iters: int, max_group: int) -> None:
        self._lib.ref_rep(self._h, iters, max_group)

    def topup(self) -> int:
        return int(self._lib.ref_topup(self._h))

    def kd_rotate(self, new_dims: int = 30) -> np.ndarray:
        """SolutionRandomKD::rotateRandom on a fresh thread (generator at its seed)."""
        out = np.zeros((self.n, new_dims), np.float32)
        self._lib.ref_kd_rotate(self._h, new_dims, _ptr(out))
        return out

    def indices(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint32)
        self._lib.ref_get_indices(self._h, _ptr(out))
        return out

    def sets(self) -> dict:
        n = self.n
        out = {
            "dist": np.zeros((n, 100), np.float32),
            "id": np.zeros((n, 100), np.uint32),
            "size": np.zeros(n, np.uint32),
            "maxslot": np.zeros(n, np.uint32),
            "bound": np.zeros(n, np.float32),
        }
        self._lib.ref_get_sets(self._h, *(_ptr(out[x]) for x in ("dist", "id", "size", "maxslot", "bound")))
        return out

    def finalize(self) -> np.ndarray:
        out = np.zeros((self.n, 100), np.uint32)
        self._lib.ref_finalize(self._h, _ptr(out))
        return out

    def distance(self, a, b) -> float:
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        return float(self._lib.ref_distance(_ptr(a), _ptr(b)))

    def dot(self, a, b) -> float:
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        return float(self._lib.ref_dot(_ptr(a), _ptr(b)))

    def knnset_replay(self, ids: np.ndarray, dists: np.ndarray) -> dict:
        ids = np.ascontiguousarray(ids, np.uint32)
        dists = np.ascontiguousarray(dists, np.float32)
        od = np.zeros(100, np.float32)
        oi = np.zeros(100, np.uint32)
        sz = np.zeros(1, np.uint32)
        ms = np.zeros(1, np.uint32)
        bd = np.zeros(1, np.float32)
        self._lib.ref_knnset_replay(_ptr(ids), _ptr(dists), len(ids), _ptr(od), _ptr(oi), _ptr(sz), _ptr(ms), _ptr(bd))
        return {"dist": od, "id": oi, "size": int(sz[0]), "maxslot": int(ms[0]), "bound": float(bd[0])}
