"""Vamana-style graph builder (torch, CPU or GPU).

The reference builds its graphs with DiskANN (``build_disk_index -R -L``,
scripts/build_diskann_index.sh:7; ``build_memory_index -R 32 -L 50`` for the
pivot graph, scripts/gen_pivot_graph.sh:7-14). DiskANN is an empty submodule
here, so this module produces graphs of the same kind for the reference's file
formats. Search parity is defined on a given index file, so the builder only has
to produce valid, navigable graphs; it is not meant to match DiskANN edge for
edge.

Algorithm (a batched, GPU-friendly restatement of Vamana):
1. initial graph: k-nearest-neighbour candidates (exact for small n; for large n
   points are grouped by a coarse k-means and each group searches the members of
   its ``nprobe`` nearest groups) pruned with RobustPrune, plus a few random
   neighbours per node (Vamana starts from a random graph);
2. Vamana passes (alpha 1, then ``alpha``): in batches of points, each point
   runs a greedy beam search (list size ``L_build``) from the medoid on the
   current graph; its expanded nodes plus its neighbours are pruned with
   RobustPrune (a candidate c is dropped when an already kept neighbour j has
   alpha * d(j, c) < d(p, c), squared L2) and every kept edge p->q offers q->p,
   rows over R being pruned again. The graph is updated after every batch.
The medoid is the point nearest to the mean (DiskANN's entry point). The
searches create the long edges that make the graph navigable across the
well-separated clusters of the synthetic mixtures.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def _f32(x: torch.Tensor) -> torch.Tensor:
    return x if x.dtype == torch.float32 else x.float()


def sqdist(a: torch.Tensor, b: torch.Tensor, an: torch.Tensor | None = None, bn: torch.Tensor | None = None):
    """Squared L2 between rows of a (m x d) and b (n x d), FP32 (exact for uint8 data, d <= 128)."""
    a = _f32(a)
    b = _f32(b)
    if an is None:
        an = (a * a).sum(1)
    if bn is None:
        bn = (b * b).sum(1)
    d = an[:, None] + bn[None, :] - 2.0 * (a @ b.T)
    return d.clamp_min_(0.0)


def medoid(x: torch.Tensor, chunk: int = 1 << 20) -> int:
    mean = torch.zeros(x.shape[1], dtype=torch.float64, device=x.device)
    for s in range(0, x.shape[0], chunk):
        mean += _f32(x[s:s + chunk]).double().sum(0)
    mean = (mean / x.shape[0]).float()
    best, best_d = 0, math.inf
    for s in range(0, x.shape[0], chunk):
        d = ((_f32(x[s:s + chunk]) - mean) ** 2).sum(1)
        v, i = torch.min(d, 0)
        if float(v) < best_d:
            best_d, best = float(v), s + int(i)
    return best


def kmeans(x: torch.Tensor, k: int, iters: int, seed: int, sample: int = 1 << 18) -> torch.Tensor:
    """Plain Lloyd k-means on a seeded sample; returns k x d FP32 centres."""
    g = torch.Generator(device="cpu")
    g.manual_seed(seed)
    n = x.shape[0]
    idx = torch.randperm(n, generator=g)[: min(n, sample)].to(x.device)
    s = _f32(x[idx])
    cent = s[torch.randperm(s.shape[0], generator=g)[:k].to(x.device)].clone()
    for _ in range(iters):
        lab = assign(s, cent)
        sums = torch.zeros_like(cent).index_add_(0, lab, s)
        cnt = torch.bincount(lab, minlength=k).float()
        empty = cnt == 0
        cent = torch.where(empty[:, None], cent, sums / cnt.clamp_min(1)[:, None])
    return cent


def assign(x: torch.Tensor, cent: torch.Tensor, chunk: int = 1 << 16) -> torch.Tensor:
    cn = (cent * cent).sum(1)
    out = torch.empty(x.shape[0], dtype=torch.long, device=x.device)
    for s in range(0, x.shape[0], chunk):
        out[s:s + chunk] = sqdist(x[s:s + chunk], cent, bn=cn).argmin(1)
    return out


def knn_candidates(x: torch.Tensor, K: int, n_coarse: int | None = None, nprobe: int = 4, seed: int = 7,
                   block: int = 4096) -> tuple[torch.Tensor, torch.Tensor]:
    """K nearest (approximate for large n) neighbours of every point, self excluded.
    Returns (ids n x K int64, squared distances n x K), rows sorted by distance; -1 pads."""
    n = x.shape[0]
    dev = x.device
    K = min(K, n - 1)
    xn = (_f32(x) ** 2).sum(1) if n <= (1 << 22) else None
    ids = torch.full((n, K), -1, dtype=torch.long, device=dev)
    dis = torch.full((n, K), float("inf"), dtype=torch.float32, device=dev)
    if n_coarse is None:
        n_coarse = 1 if n <= 50_000 else max(1, n // 1000)
    if n_coarse == 1:
        for s in range(0, n, block):
            e = min(n, s + block)
            d = sqdist(x[s:e], x, an=None if xn is None else xn[s:e], bn=xn)
            d[torch.arange(e - s, device=dev), torch.arange(s, e, device=dev)] = float("inf")
            v, i = torch.topk(d, K, dim=1, largest=False)
            ids[s:e], dis[s:e] = i, v
        return ids, dis
    cent = kmeans(x, n_coarse, iters=8, seed=seed)
    lab = assign(x, cent)
    order = torch.argsort(lab)
    counts = torch.bincount(lab, minlength=n_coarse)
    starts = torch.cumsum(counts, 0) - counts
    near = torch.topk(sqdist(cent, cent), min(nprobe, n_coarse), dim=1, largest=False).indices
    counts_h, starts_h, near_h = counts.cpu().numpy(), starts.cpu().numpy(), near.cpu().numpy()
    for c in range(n_coarse):
        if counts_h[c] == 0:
            continue
        mem = order[starts_h[c]: starts_h[c] + counts_h[c]]
        pool = torch.cat([order[starts_h[o]: starts_h[o] + counts_h[o]] for o in near_h[c]])
        kk = min(K, pool.numel() - 1)
        for s in range(0, mem.numel(), block):
            m = mem[s:s + block]
            d = sqdist(x[m], x[pool])
            d[m[:, None] == pool[None, :]] = float("inf")
            v, i = torch.topk(d, kk, dim=1, largest=False)
            ids[m, :kk] = pool[i]
            dis[m, :kk] = v
    return ids, dis


def robust_prune(x: torch.Tensor, cand: torch.Tensor, cand_d: torch.Tensor, R: int, alpha: float,
                 batch: int = 8192, rows: torch.Tensor | None = None) -> torch.Tensor:
    """RobustPrune over rows of candidates sorted by distance (-1 = none).
    Returns n x R int64 neighbour ids (-1 padded), kept in candidate order.
    On the GPU, given the rows' point ids, the same rule runs in the
    gann_build_prune kernel (which re-scores the candidates exactly and orders
    ties by id, as the sorted rows here are)."""
    if x.is_cuda and rows is not None and cand.shape[1] <= 128:
        from .ivf import prune

        return prune(x, cand, R, alpha, rows).long()
    n, K = cand.shape
    batch = max(64, min(batch, int(1.5e9 // (K * K * 4 + K * x.shape[1] * 4))))
    out = torch.full((n, R), -1, dtype=torch.long, device=x.device)
    for s in range(0, n, batch):
        e = min(n, s + batch)
        c = cand[s:e]
        cd = cand_d[s:e]
        valid = c >= 0
        V = _f32(x[c.clamp_min(0)])
        vn = (V * V).sum(-1)
        D = (vn[:, :, None] + vn[:, None, :] - 2.0 * torch.bmm(V, V.transpose(1, 2))).clamp_min_(0.0)
        alive = valid.clone()
        keep = torch.zeros_like(valid)
        count = torch.zeros(e - s, dtype=torch.long, device=x.device)
        col = torch.arange(K, device=x.device)
        for j in range(K):
            sel = alive[:, j] & (count < R)
            if not bool(sel.any()):
                if not bool(alive[:, j:].any()):
                    break
                continue
            keep[:, j] = sel
            count += sel.long()
            kill = sel[:, None] & (alpha * D[:, j, :] < cd) & (col[None, :] > j)
            alive &= ~kill
        pos = torch.cumsum(keep.long(), 1) - 1
        rows = torch.arange(e - s, device=x.device)[:, None].expand(-1, K)
        m = keep & (pos < R)
        out[s:e][rows[m], pos[m]] = c[m]
    return out


def _dedupe_sorted(ids: torch.Tensor, d: torch.Tensor):
    """Sort rows by (distance, id) and blank out repeated ids (-1, inf)."""
    ids = ids.clone()
    d = d.clone()
    d[ids < 0] = float("inf")
    o = torch.argsort(ids, dim=1, stable=True)
    ids = torch.gather(ids, 1, o)
    d = torch.gather(d, 1, o)
    dup = torch.zeros_like(ids, dtype=torch.bool)
    dup[:, 1:] = (ids[:, 1:] == ids[:, :-1]) & (ids[:, 1:] >= 0)
    ids[dup] = -1
    d[dup | (ids < 0)] = float("inf")
    o = torch.argsort(d, dim=1, stable=True)
    return torch.gather(ids, 1, o), torch.gather(d, 1, o)


def beam_search(x: torch.Tensor, g: torch.Tensor, start: int, qidx: torch.Tensor, L: int,
                max_iters: int | None = None) -> torch.Tensor:
    """Batched greedy beam search (Vamana's GreedySearch) from ``start`` for the
    base points ``qidx``, exact distances, list size L. Returns the expanded
    nodes of every query, in expansion order (B x iters, -1 padded)."""
    dev = x.device
    B = qidx.numel()
    R = g.shape[1]
    q = _f32(x[qidx])
    ids = torch.full((B, L), -1, dtype=torch.long, device=dev)
    ds = torch.full((B, L), float("inf"), device=dev)
    ex = torch.zeros((B, L), dtype=torch.bool, device=dev)
    ids[:, 0] = start
    ds[:, 0] = ((q - _f32(x[start])[None, :]) ** 2).sum(1)
    rows = torch.arange(B, device=dev)
    visited = []
    max_iters = max_iters or 2 * L
    for _ in range(max_iters):
        cand = (~ex) & (ids >= 0)
        has = cand.any(1)
        if not bool(has.any()):
            break
        pos = torch.argmax(cand.to(torch.int8), 1)
        u = torch.where(has, ids[rows, pos], torch.full_like(pos, -1))
        ex[rows[has], pos[has]] = True
        visited.append(u)
        nb = g[u.clamp_min(0)]
        nb = torch.where(has[:, None], nb, torch.full_like(nb, -1))
        nd = ((_f32(x[nb.clamp_min(0)]) - q[:, None, :]) ** 2).sum(-1)
        nd[nb < 0] = float("inf")
        a_id = torch.cat([ids, nb], 1)
        a_d = torch.cat([ds, nd], 1)
        a_ex = torch.cat([ex, torch.zeros((B, R), dtype=torch.bool, device=dev)], 1)
        # drop ids already present (keep the copy that is expanded, else the first)
        o = torch.argsort(a_id * 2 + (~a_ex).long(), dim=1)
        s_id = torch.gather(a_id, 1, o)
        dup = torch.zeros_like(s_id, dtype=torch.bool)
        dup[:, 1:] = (s_id[:, 1:] == s_id[:, :-1]) & (s_id[:, 1:] >= 0)
        a_d = a_d.scatter(1, o, torch.where(dup, torch.full_like(a_d, float("inf")), torch.gather(a_d, 1, o)))
        a_d[a_id < 0] = float("inf")
        v, sel = torch.topk(a_d, L, dim=1, largest=False)
        ids = torch.gather(a_id, 1, sel)
        ex = torch.gather(a_ex, 1, sel)
        ids[torch.isinf(v)] = -1
        ds = v
    return torch.stack(visited, 1) if visited else torch.full((B, 1), -1, dtype=torch.long, device=dev)


def vamana_pass(x: torch.Tensor, g: torch.Tensor, start: int, R: int, L: int, alpha: float, rounds: int,
                seed: int, batch_cap: int = 65536) -> torch.Tensor:
    """One Vamana pass in ``rounds`` batches: each point searches the current
    graph from ``start``; its expanded nodes plus its neighbours are pruned
    with alpha; then reverse edges are offered. The graph is updated after every
    batch (Vamana updates after every point)."""
    n = x.shape[0]
    dev = x.device
    gen = torch.Generator(device="cpu")
    gen.manual_seed(seed)
    order = torch.randperm(n, generator=gen).to(dev)
    step = min(batch_cap, max(1, (n + rounds - 1) // rounds))
    for s in range(0, n, step):
        p = order[s:s + step]
        vis = beam_search(x, g, start, p, L)
        cand = torch.cat([vis, g[p]], 1)
        cand = torch.where(cand == p[:, None], torch.full_like(cand, -1), cand)
        V = _f32(x[cand.clamp_min(0)])
        d = ((V - _f32(x[p])[:, None, :]) ** 2).sum(-1)
        cand, d = _dedupe_sorted(cand, d)
        g[p] = robust_prune(x, cand, d, R, alpha, rows=p)
        g = _offer_reverse(x, g, p, R, alpha)
    return g


def _offer_reverse(x: torch.Tensor, g: torch.Tensor, p: torch.Tensor, R: int, alpha: float,
                   in_cap: int | None = None) -> torch.Tensor:
    """For the out-edges p->q of the points p, add q->p; rows over R are pruned.
    Each q considers at most ``in_cap`` (default 2R) of its new in-edges, the
    nearest ones."""
    dev = x.device
    in_cap = in_cap or 2 * R
    src = p[:, None].expand(-1, g.shape[1])
    nb = g[p]
    m = nb >= 0
    tgt, back = nb[m], src[m]
    if tgt.numel() == 0:
        return g
    ed = torch.empty(tgt.numel(), dtype=torch.float32, device=dev)
    for s in range(0, tgt.numel(), 1 << 20):
        ed[s:s + (1 << 20)] = ((_f32(x[tgt[s:s + (1 << 20)]]) - _f32(x[back[s:s + (1 << 20)]])) ** 2).sum(1)
    o = torch.argsort(ed, stable=True)
    tgt, back = tgt[o], back[o]
    o = torch.argsort(tgt, stable=True)  # by target, nearest first within a target
    tgt, back = tgt[o], back[o]
    uniq, cnt = torch.unique_consecutive(tgt, return_counts=True)
    start = torch.cumsum(cnt, 0) - cnt
    rank = torch.arange(tgt.numel(), device=dev) - torch.repeat_interleave(start, cnt)
    keep = rank < in_cap
    cap = int(min(int(cnt.max()), in_cap))
    inc = torch.full((uniq.numel(), cap), -1, dtype=torch.long, device=dev)
    rowi = torch.repeat_interleave(torch.arange(uniq.numel(), device=dev), cnt)
    inc[rowi[keep], rank[keep]] = back[keep]
    for s in range(0, uniq.numel(), 16384):
        u = uniq[s:s + 16384]
        cand = torch.cat([g[u], inc[s:s + 16384]], 1)
        V = _f32(x[cand.clamp_min(0)])
        d = ((V - _f32(x[u])[:, None, :]) ** 2).sum(-1)
        cand, d = _dedupe_sorted(cand, d)
        nuniq = (cand >= 0).sum(1)
        rows = torch.full((u.numel(), R), -1, dtype=torch.long, device=dev)
        small = nuniq <= R
        rows[small] = cand[small, :R]
        if bool((~small).any()):
            big = torch.nonzero(~small).squeeze(1)
            rows[big] = robust_prune(x, cand[big], d[big], R, alpha, rows=u[big])
        g[u] = rows
    return g


def build(x: torch.Tensor, R: int, alpha: float = 1.2, K: int | None = None, n_coarse: int | None = None,
          nprobe: int = 4, seed: int = 7, L_build: int = 100, passes: int = 2, rounds: int = 8,
          random_edges: int = 8) -> tuple[np.ndarray, np.ndarray, int]:
    """Build a graph over the rows of ``x`` (uint8 or float32 tensor).
    Returns (adjacency n x R int32 padded with -1, degrees n int32, medoid).

    Initial graph: pruned k-NN candidates plus ``random_edges`` random
    neighbours per node (Vamana starts from a random graph); then ``passes``
    Vamana passes (alpha 1, then ``alpha``) searching from the medoid with list
    size ``L_build``."""
    K = K or 2 * R
    n = x.shape[0]
    med = medoid(x)
    cand, cand_d = knn_candidates(x, K, n_coarse=n_coarse, nprobe=nprobe, seed=seed)
    r_loc = max(1, R - random_edges) if n > R + 1 else R
    g = robust_prune(x, cand, cand_d, r_loc, alpha, rows=torch.arange(n, device=x.device))
    if r_loc < R:
        gen = torch.Generator(device="cpu")
        gen.manual_seed(seed + 101)
        rnd = torch.randint(0, n, (n, R - r_loc), generator=gen).to(x.device)
        self_ = rnd == torch.arange(n, device=x.device)[:, None]
        rnd = torch.where(self_, (rnd + 1) % n, rnd)
        g = torch.cat([g, rnd], 1)
        # remove duplicate targets within each row
        gd = torch.zeros_like(g, dtype=torch.float32)
        gs, _ = _dedupe_sorted(g, gd)
        g = gs[:, :R]
    for i in range(passes):
        a = 1.0 if (passes > 1 and i == 0) else alpha
        g = vamana_pass(x, g, med, R, L_build, a, rounds, seed + 17 * (i + 1))
    deg = (g >= 0).sum(1)
    # neighbours first, -1 padding last
    o = torch.argsort((g < 0).to(torch.int8), dim=1, stable=True)
    g = torch.gather(g, 1, o)
    return (g.to(torch.int32).cpu().numpy(), deg.to(torch.int32).cpu().numpy(), med)


def reachable_from(graph: np.ndarray, degrees: np.ndarray, start: int) -> np.ndarray:
    """Boolean mask of nodes reachable from ``start`` by breadth-first search."""
    n = graph.shape[0]
    seen = np.zeros(n, dtype=bool)
    seen[start] = True
    frontier = np.array([start])
    mask = np.arange(graph.shape[1])[None, :]
    while frontier.size:
        rows = graph[frontier]
        nb = rows[mask < degrees[frontier][:, None]]
        nb = np.unique(nb[nb >= 0])
        nb = nb[~seen[nb]]
        seen[nb] = True
        frontier = nb
    return seen
