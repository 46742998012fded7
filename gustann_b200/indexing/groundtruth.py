"""Brute-force ground truth and the reference's recall measure.

``knn`` returns the exact k nearest base points of each query by squared L2,
ties broken by id: FP32 GEMM distances pick candidates (exact for uint8 data up
to dim 128), then FP64 distances re-rank them. ``recall`` restates
``calc_recall`` (bin/utils.hpp:105-117), which counts every returned id that is
in the first k ground-truth ids (duplicates count again); ``recall_unique``
counts each id once.
"""
from __future__ import annotations

import numpy as np
import torch

from .builder import _f32, sqdist


def knn(base: torch.Tensor, queries: torch.Tensor, k: int, extra: int = 32, block_q: int = 1024,
        block_b: int = 1 << 21) -> np.ndarray:
    dev = base.device
    n = base.shape[0]
    kk = min(n, k + extra)
    out = np.empty((queries.shape[0], k), dtype=np.int32)
    bn = torch.empty(n, dtype=torch.float32, device=dev)
    for s in range(0, n, block_b):
        b = _f32(base[s:s + block_b])
        bn[s:s + block_b] = (b * b).sum(1)
    for qs in range(0, queries.shape[0], block_q):
        q = _f32(queries[qs:qs + block_q])
        best_v = torch.full((q.shape[0], kk), float("inf"), device=dev)
        best_i = torch.full((q.shape[0], kk), -1, dtype=torch.long, device=dev)
        for s in range(0, n, block_b):
            d = sqdist(q, base[s:s + block_b], bn=bn[s:s + block_b])
            v, i = torch.topk(d, min(kk, d.shape[1]), dim=1, largest=False)
            cv = torch.cat([best_v, v], 1)
            ci = torch.cat([best_i, i + s], 1)
            v2, o = torch.topk(cv, kk, dim=1, largest=False)
            best_v, best_i = v2, torch.gather(ci, 1, o)
        # exact FP64 re-rank of the candidates, ties by id
        cand = best_i.clamp_min(0)
        vec = base[cand].double()
        d64 = ((vec - q.double()[:, None, :]) ** 2).sum(-1)
        d64[best_i < 0] = float("inf")
        d_np = d64.cpu().numpy()
        i_np = best_i.cpu().numpy()
        for r in range(q.shape[0]):
            o = np.lexsort((i_np[r], d_np[r]))[:k]
            out[qs + r] = i_np[r][o]
    return out


def recall(result: np.ndarray, gt: np.ndarray, k: int) -> float:
    """calc_recall, bin/utils.hpp:105-117."""
    hits = 0
    for r, g in zip(result[:, :k], gt[:, :k]):
        s = set(g.tolist())
        hits += sum(1 for x in r.tolist() if x in s)
    return hits / (result.shape[0] * k)


def recall_unique(result: np.ndarray, gt: np.ndarray, k: int) -> float:
    hits = 0
    for r, g in zip(result[:, :k], gt[:, :k]):
        hits += len(set(r.tolist()) & set(g.tolist()))
    return hits / (result.shape[0] * k)
