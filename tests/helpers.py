"""Shared helpers for the parity tests."""
from __future__ import annotations

import hashlib

import numpy as np

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
