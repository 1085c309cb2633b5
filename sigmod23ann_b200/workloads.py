"""Seeded synthetic point sets with the shapes of the benchmark configurations.

The contest dataset is not available; these generators stand in for it with
the distributions the configurations name:

* :func:`gaussian_mixture` -- isotropic Gaussian clusters with uniform
  [-1, 1]^d centres and equal weights (100k x 100, 64 clusters, sigma 0.15,
  seed 0; and the 16-cluster sets of the batched form).
* :func:`subspace_mixture` -- clusters with Zipf(s) sizes; each point is
  centre + B_c z * scale + noise, B_c a random d x r orthonormal basis,
  z ~ N(0, I_r) (10M x 100, 1,024 clusters, r = 24, scale 0.3, noise 0.05,
  Zipf 1.1, seed 1).
"""
from __future__ import annotations

import numpy as np


def gaussian_mixture(n: int, d: int = 100, clusters: int = 64, sigma: float = 0.15, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-1.0, 1.0, size=(clusters, d)).astype(np.float32)
    labels = rng.integers(0, clusters, size=n)
    out = np.empty((n, d), np.float32)
    chunk = 1 << 20
    for b in range(0, n, chunk):
        e = min(n, b + chunk)
        noise = rng.standard_normal((e - b, d), dtype=np.float32)
        noise *= np.float32(sigma)
        noise += centres[labels[b:e]]
        out[b:e] = noise
    return out


def zipf_sizes(n: int, clusters: int, s: float) -> np.ndarray:
    w = 1.0 / np.arange(1, clusters + 1, dtype=np.float64) ** s
    w /= w.sum()
    sizes = np.floor(w * n).astype(np.int64)
    rem = n - int(sizes.sum())
    sizes[:rem] += 1
    return sizes


def subspace_mixture(n: int, d: int = 100, clusters: int = 1024, rank: int = 24, scale: float = 0.3,
                     noise: float = 0.05, zipf_s: float = 1.1, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    sizes = zipf_sizes(n, clusters, zipf_s)
    out = np.empty((n, d), np.float32)
    row = 0
    for c in range(clusters):
        m = int(sizes[c])
        centre = rng.uniform(-1.0, 1.0, size=d).astype(np.float32)
        basis, _ = np.linalg.qr(rng.standard_normal((d, rank)))
        basis = basis.astype(np.float32) * np.float32(scale)
        done = 0
        while done < m:
            e = min(m, done + (1 << 20))
            z = rng.standard_normal((e - done, rank), dtype=np.float32)
            block = z @ basis.T
            block += rng.standard_normal((e - done, d), dtype=np.float32) * np.float32(noise)
            block += centre
            out[row + done:row + e] = block
            done = e
        row += m
    # Interleave clusters so that point ids carry no cluster order.
    perm = rng.permutation(n)
    return out[perm]


def subspace_mixture_torch(n: int, d: int = 100, clusters: int = 1024, rank: int = 24, scale: float = 0.3,
                           noise: float = 0.05, zipf_s: float = 1.1, seed: int = 1, device: str = "cuda"):
    """The same distribution as :func:`subspace_mixture`, generated with torch
    on `device` (the 10M-point set takes seconds on a GPU instead of minutes on
    a host core).  Returns a float32 tensor on `device`."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    sizes = zipf_sizes(n, clusters, zipf_s)
    out = torch.empty((n, d), dtype=torch.float32, device=device)
    row = 0
    for c in range(clusters):
        m = int(sizes[c])
        centre = torch.rand(d, generator=g, device=device) * 2.0 - 1.0
        basis, _ = torch.linalg.qr(torch.randn(d, rank, generator=g, device=device, dtype=torch.float64))
        basis = basis.to(torch.float32) * scale
        z = torch.randn(m, rank, generator=g, device=device)
        block = z @ basis.T
        block += torch.randn(m, d, generator=g, device=device) * noise
        block += centre
        out[row:row + m] = block
        row += m
    perm = torch.randperm(n, generator=g, device=device)
    return out[perm].contiguous()


def request_sizes(count: int, lo: float, hi: float, seed: int) -> np.ndarray:
    """Log-uniform sizes in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).astype(np.int64)
