"""Exact FP64 k-nearest neighbours of sampled query points, and recall.

Recall follows the reference's grader (src/grade.cpp:61-95): for each query
row, the number of ground-truth ids present in the tested row, averaged and
divided by k.  The ground truth excludes the query point itself, as the
neighbour sets never contain it.
"""
from __future__ import annotations

import numpy as np


def exact_knn_numpy(points: np.ndarray, queries: np.ndarray, k: int) -> np.ndarray:
    """FP64 brute force on the CPU (small inputs)."""
    x = points.astype(np.float64)
    sq = np.einsum("ij,ij->i", x, x)
    out = np.empty((len(queries), k), np.int64)
    step = max(1, int(2e8 // max(1, len(x))))
    for b in range(0, len(queries), step):
        q = queries[b:b + step]
        d = sq[q][:, None] + sq[None, :] - 2.0 * (x[q] @ x.T)
        d[np.arange(len(q)), q] = np.inf
        part = np.argpartition(d, k, axis=1)[:, :k]
        dd = np.take_along_axis(d, part, axis=1)
        order = np.lexsort((part, dd), axis=1)
        out[b:b + step] = np.take_along_axis(part, order, axis=1)
    return out


def exact_knn_torch(points, queries: np.ndarray, k: int, chunk: int = 1 << 17):
    """FP64 brute force on the GPU.  `points` is a torch tensor (any float
    dtype, on the GPU); returns an int64 numpy array of ids per query."""
    import torch

    dev = points.device
    q_idx = torch.as_tensor(queries, device=dev, dtype=torch.long)
    n = points.shape[0]
    best_d = torch.full((len(queries), k), float("inf"), dtype=torch.float64, device=dev)
    best_i = torch.zeros((len(queries), k), dtype=torch.long, device=dev)
    qx = points[q_idx].to(torch.float64)
    qsq = (qx * qx).sum(1)
    for b in range(0, n, chunk):
        e = min(n, b + chunk)
        x = points[b:e].to(torch.float64)
        d = qsq[:, None] + (x * x).sum(1)[None, :] - 2.0 * (qx @ x.T)
        self_mask = (q_idx >= b) & (q_idx < e)
        rows = torch.nonzero(self_mask).flatten()
        d[rows, q_idx[rows] - b] = float("inf")
        kk = min(k, e - b)
        vd, vi = torch.topk(d, kk, dim=1, largest=False)
        cat_d = torch.cat([best_d, vd], 1)
        cat_i = torch.cat([best_i, vi + b], 1)
        sel_d, sel = torch.topk(cat_d, k, dim=1, largest=False)
        best_d = sel_d
        best_i = torch.gather(cat_i, 1, sel)
    return best_i.cpu().numpy()


def recall(result_ids: np.ndarray, truth_ids: np.ndarray, queries: np.ndarray) -> float:
    """Mean fraction of ground-truth ids found in the result rows of `queries`."""
    k = truth_ids.shape[1]
    rows = np.asarray(result_ids)[queries]
    hits = 0
    for r, t in zip(rows, truth_ids):
        hits += len(np.intersect1d(r, t, assume_unique=False))
    return hits / (len(queries) * k)
