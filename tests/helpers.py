"""Shared helpers for the parity tests."""
from __future__ import annotations

import hashlib
import lzma
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

SET_FIELDS = ("dist", "id", "size", "maxslot", "bound")


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def sets_digest(s: dict) -> str:
    h = hashlib.sha256()
    for key in SET_FIELDS:
        h.update(np.ascontiguousarray(s[key]).view(np.uint32).tobytes())
    return h.hexdigest()


def assert_sets_equal(a: dict, b: dict, what: str = "") -> None:
    """Bit-exact comparison of two raw neighbour-set states."""
    for key in SET_FIELDS:
        x = np.ascontiguousarray(a[key]).view(np.uint32)
        y = np.ascontiguousarray(b[key]).view(np.uint32)
        if not np.array_equal(x, y):
            bad = np.argwhere(x != y)
            raise AssertionError(f"{what} field {key}: {len(bad)} entries differ, first at {bad[0].tolist()}: "
                                 f"{x[tuple(bad[0])]} vs {y[tuple(bad[0])]}")


def trace_levels(trace: dict):
    """Groups an oracle split trace by depth: yields index arrays per level."""
    depth = trace["depth"]
    for lvl in range(int(depth.max()) + 1 if len(depth) else 0):
        yield np.nonzero(depth == lvl)[0]


def feed_trace(ctx, trace: dict) -> None:
    """Replays the oracle's hyperplanes level by level through knng_split_nodes
    and checks every node's midpoint."""
    for sel in trace_levels(trace):
        real = sel[trace["attempts"][sel] > 0]
        real = real[np.any(trace["coefs"][real] != 0, axis=1) | (trace["offset"][real] != 0)]
        if len(real) == 0:
            continue
        mids = ctx.split_nodes(trace["start"][real], trace["end"][real], trace["coefs"][real], trace["offset"][real])
        np.testing.assert_array_equal(mids, trace["mid"][real])


def rounding_points(n: int = 1024, d: int = 100) -> np.ndarray:
    """Two clusters (dim 1 at +1000 / -1000, halves of the ids) whose
    per-cluster double sums round: in cluster A, dim 0 holds 256, then 2^-16,
    zeros, and 2^-45 for the second 256 points; cluster B repeats it in dim 2.
    Added one point at a time the 2^-45 terms are lost (each is half an ulp of
    256 + 2^-16 and rounds to even), so the mean is 0.5 + 2^-25 and rounds to
    0.5f; summed as two 256-point partials they survive as 2^-37 and the mean
    rounds up to 0.5f + 2^-24."""
    assert n >= 1024 and d >= 3
    pts = np.zeros((n, d), np.float32)
    pts[:512, 1] = 1000.0
    pts[512:1024, 1] = -1000.0
    for first, dim in ((0, 0), (512, 2)):
        pts[first, dim] = 256.0
        pts[first + 1, dim] = 2.0 ** -16
        pts[first + 256:first + 512, dim] = 2.0 ** -45
    return pts


def mean_in_order(values: np.ndarray, item: int = 0) -> np.float32:
    """Mean of float32 values as float32: a double sum one value at a time
    (item == 0), or of item-sized partials each summed in order."""
    vals = [float(v) for v in values]
    if item == 0:
        s = 0.0
        for v in vals:
            s += v
    else:
        s = 0.0
        for b in range(0, len(vals), item):
            part = 0.0
            for v in vals[b:b + item]:
                part += v
            s += part
    return np.float32(s / len(vals))


def read_points_file(raw: bytes) -> np.ndarray:
    """The contest input format (ReadBin, src/io.h:39-64): u32 N, then N rows
    of 100 float32."""
    n = int(np.frombuffer(raw[:4], np.uint32)[0])
    return np.frombuffer(raw[4:4 + n * 400], np.float32).reshape(n, 100).copy()


def case_points(gen: dict) -> np.ndarray:
    """Points of a golden case: a committed fixture file or a seeded mixture."""
    if "file" in gen:
        with lzma.open(os.path.join(GOLDEN_DIR, gen["file"])) as f:
            return read_points_file(f.read())
    from sigmod23ann_b200 import workloads

    return workloads.gaussian_mixture(**gen)
