"""Product-quantisation trainer and encoder writing DiskANN's PQ layout.

The layout follows what the reference reads (PQSearch::read_data,
src/pq_search.cu:56-121) and what its table build assumes (pq.cuh:22-43): the
training-set mean goes to ``centroid``; each chunk is a contiguous range of
dimensions (the first ``dim % M`` chunks one dimension longer); each chunk has
256 k-means centres of the centred vectors; a code byte is the nearest centre
of its chunk.
"""
from __future__ import annotations

import numpy as np
import torch

from .builder import _f32, sqdist


def chunk_offsets(dim: int, M: int) -> np.ndarray:
    low, extra = divmod(dim, M)
    sizes = [low + 1] * extra + [low] * (M - extra)
    return np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint32)


def train(x: torch.Tensor, M: int, n_train: int = 1 << 18, iters: int = 15, seed: int = 11):
    """Returns (pivots 256 x dim float32, centroid dim float32, chunk offsets M+1 uint32)."""
    dev = x.device
    n, dim = x.shape
    g = torch.Generator(device="cpu")
    g.manual_seed(seed)
    idx = torch.randperm(n, generator=g)[: min(n, n_train)].to(dev)
    t = _f32(x[idx])
    centroid = t.mean(0)
    t = t - centroid
    offs = chunk_offsets(dim, M)
    pivots = torch.zeros(256, dim, dtype=torch.float32, device=dev)
    for c in range(M):
        b, e = int(offs[c]), int(offs[c + 1])
        s = t[:, b:e].contiguous()
        k = 256
        init = torch.randperm(s.shape[0], generator=g)[:k].to(dev)
        cent = s[init].clone()
        if cent.shape[0] < k:  # fewer training points than centres
            cent = torch.cat([cent, cent[: k - cent.shape[0]]])
        for _ in range(iters):
            lab = sqdist(s, cent).argmin(1)
            sums = torch.zeros_like(cent).index_add_(0, lab, s)
            cnt = torch.bincount(lab, minlength=k).float()
            cent = torch.where((cnt == 0)[:, None], cent, sums / cnt.clamp_min(1)[:, None])
        pivots[:, b:e] = cent
    return pivots.cpu().numpy(), centroid.cpu().numpy().astype(np.float32), offs


def encode(x: torch.Tensor, pivots: np.ndarray, centroid: np.ndarray, offs: np.ndarray,
           chunk: int = 1 << 18) -> np.ndarray:
    dev = x.device
    P = torch.from_numpy(pivots).to(dev)
    mu = torch.from_numpy(centroid).to(dev)
    M = len(offs) - 1
    out = torch.empty((x.shape[0], M), dtype=torch.uint8, device=dev)
    for s in range(0, x.shape[0], chunk):
        r = _f32(x[s:s + chunk]) - mu
        for c in range(M):
            b, e = int(offs[c]), int(offs[c + 1])
            out[s:s + chunk, c] = sqdist(r[:, b:e], P[:, b:e]).argmin(1).to(torch.uint8)
    return out.cpu().numpy()
