"""Seeded synthetic datasets with the shapes of the reference's benchmarks.

The reference measures on SIFT/DEEP-style data (scripts/quick_start.sh:21-30,
readme.md); those datasets are not available here, so seeded Gaussian mixtures
of the same shapes stand in for them:

* uint8 ("sift-like", dim 128): centres uniform in [0, 255], per-dimension
  sigma 20, rounded and clipped to uint8.
* float32 ("deep-like", dim 96): centres N(0, 1), sigma 0.1, rows then scaled to
  unit L2 norm.

Each purpose draws from its own stream: seed 1 = mixture centres, 2 = base
points, 3 = queries, 4 = per-query L/k/arrival draws. ``backend="numpy"`` uses
PCG64 streams (bit-reproducible anywhere; used for test fixtures);
``backend="torch"`` uses torch generators on the given device (fast at 10^7+
points; reproducible on the same GPU/torch build).
"""
from __future__ import annotations

import numpy as np

SEED_CENTRES, SEED_BASE, SEED_QUERIES, SEED_DRAWS = 1, 2, 3, 4

PRESETS = {
    # name: (kind, n, dim, clusters)
    "c0": ("u8", 1_000_000, 128, 1_000),
    "c1": ("f32", 10_000_000, 96, 4_096),
    "c2": ("u8", 100_000_000, 128, 10_000),
    "c4": ("u8", 200_000_000, 128, 20_000),
}


def centres(kind: str, dim: int, clusters: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(SEED_CENTRES))
    if kind == "u8":
        return rng.uniform(0.0, 255.0, size=(clusters, dim)).astype(np.float32)
    return rng.standard_normal(size=(clusters, dim)).astype(np.float32)


def sample_numpy(kind: str, n: int, dim: int, clusters: int, seed: int, chunk: int = 1 << 18) -> np.ndarray:
    """n points of the mixture from the PCG64 stream ``seed`` (numpy backend)."""
    c = centres(kind, dim, clusters)
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.empty((n, dim), dtype=np.uint8 if kind == "u8" else np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        lab = rng.integers(0, clusters, size=e - s)
        noise = rng.standard_normal(size=(e - s, dim)).astype(np.float32)
        if kind == "u8":
            x = c[lab] + np.float32(20.0) * noise
            out[s:e] = np.clip(np.rint(x), 0, 255).astype(np.uint8)
        else:
            x = c[lab] + np.float32(0.1) * noise
            x /= np.linalg.norm(x, axis=1, keepdims=True).astype(np.float32)
            out[s:e] = x
    return out


def sample_torch(kind: str, n: int, dim: int, clusters: int, seed: int, device, chunk: int = 1 << 22):
    """n points of the mixture drawn with a torch generator on ``device``."""
    import torch

    c = torch.from_numpy(centres(kind, dim, clusters)).to(device)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty((n, dim), dtype=torch.uint8 if kind == "u8" else torch.float32, device=device)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        lab = torch.randint(0, clusters, (e - s,), generator=g, device=device)
        noise = torch.randn((e - s, dim), generator=g, device=device, dtype=torch.float32)
        if kind == "u8":
            x = c[lab] + 20.0 * noise
            out[s:e] = torch.clamp(torch.round(x), 0, 255).to(torch.uint8)
        else:
            x = c[lab] + 0.1 * noise
            out[s:e] = x / torch.linalg.vector_norm(x, dim=1, keepdim=True)
    return out


def make(kind: str, n: int, dim: int, clusters: int, n_queries: int, backend: str = "numpy", device=None):
    """Base points (seed 2) and queries (seed 3) of one mixture."""
    if backend == "numpy":
        return (sample_numpy(kind, n, dim, clusters, SEED_BASE),
                sample_numpy(kind, n_queries, dim, clusters, SEED_QUERIES))
    return (sample_torch(kind, n, dim, clusters, SEED_BASE, device),
            sample_torch(kind, n_queries, dim, clusters, SEED_QUERIES, device))


def draws(n_queries: int, L_choices, k_choices) -> tuple[np.ndarray, np.ndarray]:
    """Per-query (L, k) from the seed-4 stream; L is raised to k where it is smaller."""
    rng = np.random.Generator(np.random.PCG64(SEED_DRAWS))
    L = rng.choice(np.asarray(L_choices), size=n_queries).astype(np.int32)
    k = rng.choice(np.asarray(k_choices), size=n_queries).astype(np.int32)
    return np.maximum(L, k), k
