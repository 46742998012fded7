"""Partitioned graph builder for large indexes (10^7 to 10^8 points).

The reference builds its indexes with DiskANN (``build_disk_index -R -L``,
scripts/build_diskann_index.sh:7), an empty submodule here. DiskANN's Vamana
runs one greedy search per point, which is what makes ``builder.build`` take
about two minutes per million points. At 100M points this module instead
builds the graph from exact local neighbourhoods, on the GPU:

1. leaves: k-means over a sample with about ``leaf`` points per centre; every
   point goes to its nearest centre (its leaf) and its second nearest;
2. candidates: each point's ``K`` nearest neighbours among the points of its
   leaf plus the points whose second-nearest centre is that leaf, found by one
   batched GEMM per group of leaves and a top-K;
3. RobustPrune (alpha) of the candidates to R (``gann_build_prune``, one warp
   per point);
4. reverse edges: every kept edge p -> q offers q -> p (at most ``in_cap`` per
   q), and each row is pruned again over its neighbours plus its offers;
5. long edges: the pivot graph (a uniform sample of the points, built with
   Vamana's searches by ``builder.build``) is embedded in the main graph -- the
   last ``nav_slots`` slots of each sampled point's row hold its pivot-graph
   neighbours, so a walk that meets any sampled point can cross between
   distant regions the way the pivot graph does.

Search parity is defined on a given index file, so the builder only has to
produce a valid, navigable graph in the reference's format.
"""
from __future__ import annotations

import contextlib
import ctypes
import math
import time

import numpy as np
import torch

from . import builder
from .builder import _f32


@contextlib.contextmanager
def _tf32():
    """TF32 GEMMs for the candidate search: uint8 vectors are exact in TF32, and
    the kept neighbours are re-scored exactly by the prune kernel anyway."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    try:
        yield
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


def prune(x: torch.Tensor, cand: torch.Tensor, R: int, alpha: float, rows: torch.Tensor | None = None,
          chunk: int = 1 << 24) -> torch.Tensor:
    """RobustPrune of every row's candidate ids (n_rows x K, -1 = none) for the
    points ``rows`` (default: row r is point r). Returns n_rows x R int32, kept
    neighbours in distance order, -1 padded. On the GPU through
    gann_build_prune; on the CPU through builder.robust_prune."""
    n_rows, K = cand.shape
    if not x.is_cuda:
        pts = torch.arange(n_rows, device=x.device) if rows is None else rows.long()
        c = cand.long().clone()
        c[c == pts[:, None]] = -1
        V = _f32(x[c.clamp_min(0)])
        d = ((V - _f32(x[pts])[:, None, :]) ** 2).sum(-1)
        c, d = builder._dedupe_sorted(c, d)
        return builder.robust_prune(x, c, d, R, alpha).to(torch.int32)
    import gustann_b200 as gb

    out = torch.empty((n_rows, R), dtype=torch.int32, device=x.device)
    dtype = 0 if x.dtype == torch.uint8 else 1
    xs = x.contiguous()
    s = torch.cuda.current_stream().cuda_stream
    for a in range(0, n_rows, chunk):
        b = min(n_rows, a + chunk)
        cc = cand[a:b].to(torch.int32).contiguous()
        rr = None if rows is None else rows[a:b].to(torch.int32).contiguous()
        if rr is None and a:
            rr = torch.arange(a, b, dtype=torch.int32, device=x.device)
        gb._check(gb.lib().gann_build_prune(xs.data_ptr(), dtype, xs.shape[0], xs.shape[1],
                                            0 if rr is None else rr.data_ptr(), cc.data_ptr(), b - a, K, R,
                                            ctypes.c_float(alpha), out[a:b].data_ptr(), ctypes.c_void_p(s)))
    return out


def assign2(x: torch.Tensor, cent: torch.Tensor, budget: int = 1 << 28) -> tuple[torch.Tensor, torch.Tensor]:
    """Nearest and second-nearest centre of every row (int64 each)."""
    n = x.shape[0]
    k = cent.shape[0]
    cn = (cent * cent).sum(1)
    a1 = torch.empty(n, dtype=torch.long, device=x.device)
    a2 = torch.empty(n, dtype=torch.long, device=x.device)
    step = max(1024, budget // max(1, k))
    for s in range(0, n, step):
        e = min(n, s + step)
        d = torch.addmm(cn[None, :], _f32(x[s:e]), cent.T, beta=1.0, alpha=-2.0)
        if k == 1:
            a1[s:e] = 0
            a2[s:e] = 0
            continue
        _, i = torch.topk(d, 2, dim=1, largest=False)
        a1[s:e], a2[s:e] = i[:, 0], i[:, 1]
    return a1, a2


def kmeans(x: torch.Tensor, k: int, iters: int, seed: int, sample: int) -> torch.Tensor:
    """Lloyd k-means on a seeded sample of the rows; empty centres keep their place."""
    g = torch.Generator(device="cpu")
    g.manual_seed(seed)
    n = x.shape[0]
    idx = torch.randperm(n, generator=g)[: min(n, sample)].to(x.device)
    s = _f32(x[idx])
    cent = s[torch.randperm(s.shape[0], generator=g)[:k].to(x.device)].clone()
    for _ in range(iters):
        lab, _ = assign2(s, cent)
        sums = torch.zeros_like(cent).index_add_(0, lab, s)
        cnt = torch.bincount(lab, minlength=k).float()
        cent = torch.where((cnt == 0)[:, None], cent, sums / cnt.clamp_min(1)[:, None])
    return cent


def leaf_batches(q_counts: np.ndarray, pool_sizes: np.ndarray, budget: int) -> list[tuple[int, int]]:
    """Groups of consecutive leaves (given in order of falling pool size) for
    one batched GEMM each: (first, count). The first leaf of a group sets the
    pool width, and leaves are added while the distance block count x
    (largest query count so far) x (pool width) stays within the budget; a
    single leaf always forms a group."""
    out = []
    i, n = 0, len(q_counts)
    while i < n:
        sp = max(1, int(pool_sizes[i]))
        G, sq = 0, 0
        while i + G < n:
            mq = max(sq, int(q_counts[i + G]))
            if G and (G + 1) * mq * sp > budget:
                break
            sq, G = mq, G + 1
        out.append((i, G))
        i += G
    return out


def leaf_candidates(x: torch.Tensor, K: int, leaf: int, seed: int, log=None,
                    budget: int = 1 << 29) -> torch.Tensor:
    """K nearest neighbours of every point inside its leaf's pool (n x K int32,
    -1 padded, self excluded, rows sorted by distance)."""
    n, dim = x.shape
    dev = x.device
    k = max(1, n // leaf)
    t0 = time.time()
    cent = kmeans(x, k, iters=8, seed=seed, sample=min(n, 48 * k))
    a1, a2 = assign2(x, cent)
    if k == 1:
        a2 = torch.full_like(a1, -1)
    o1 = torch.argsort(a1)
    c1 = torch.bincount(a1, minlength=k)
    s1 = torch.cumsum(c1, 0) - c1
    m2 = a2 >= 0
    o2 = torch.argsort(torch.where(m2, a2, torch.full_like(a2, k)))
    c2 = torch.bincount(a2[m2], minlength=k)
    s2 = torch.cumsum(c2, 0) - c2
    del a1, a2, m2
    if log:
        log(f"leaves: {k} centres, sizes {int(c1.min())}..{int(c1.max())}, {time.time() - t0:.1f} s")
    cand = torch.full((n, K), -1, dtype=torch.int32, device=dev)
    pool = c1 + c2
    order = torch.argsort(pool, descending=True)
    order = order[c1[order] > 0]
    c1h, poolh, orderh = c1.cpu().numpy(), pool.cpu().numpy(), order.cpu().numpy()
    inf = float("inf")
    groups = []
    for i, G in leaf_batches(c1h[orderh], poolh[orderh], budget):
        sp = max(1, int(poolh[orderh[i]]))
        if G == 1 and int(c1h[orderh[i]]) * sp > budget:  # one leaf too large for one block: split its queries
            step = max(1, budget // sp)
            groups += [(i, 1, a, min(int(c1h[orderh[i]]), a + step)) for a in range(0, int(c1h[orderh[i]]), step)]
        else:
            groups.append((i, G, 0, None))
    for i, G, qa, qb in groups:
        Lb = order[i:i + G]
        q_cnt, p_cnt, c1b = c1[Lb], pool[Lb], c1[Lb]
        q_off = torch.zeros_like(q_cnt)
        if qb is not None:  # a slice [qa, qb) of one large leaf's queries
            q_off = torch.full_like(q_cnt, qa)
            q_cnt = torch.full_like(q_cnt, qb - qa)
        Sq, Sp = int(q_cnt.max()), int(p_cnt.max())
        ar_q = torch.arange(Sq, device=dev)
        ar_p = torch.arange(Sp, device=dev)
        qmask = ar_q[None, :] < q_cnt[:, None]
        qi = o1[(s1[Lb][:, None] + q_off[:, None] + ar_q[None, :]).clamp(max=n - 1)]
        from1 = ar_p[None, :] < c1b[:, None]
        idx1 = (s1[Lb][:, None] + ar_p[None, :]).clamp(max=n - 1)
        idx2 = (s2[Lb][:, None] + ar_p[None, :] - c1b[:, None]).clamp(0, n - 1)
        pi = torch.where(from1, o1[idx1], o2[idx2])
        pmask = ar_p[None, :] < p_cnt[:, None]
        Q = _f32(x[qi.reshape(-1)]).view(G, Sq, dim)
        P = _f32(x[pi.reshape(-1)]).view(G, Sp, dim)
        pn = (P * P).sum(-1)
        D = torch.baddbmm(pn[:, None, :], Q, P.transpose(1, 2), beta=1.0, alpha=-2.0)
        del Q, P
        D.masked_fill_(~pmask[:, None, :], inf)
        D.masked_fill_(pi[:, None, :] == qi[:, :, None], inf)
        kk = min(K, Sp)
        v, j = torch.topk(D, kk, dim=2, largest=False)
        del D
        nb = torch.gather(pi[:, None, :].expand(G, Sq, Sp), 2, j)
        nb = torch.where(torch.isinf(v), torch.full_like(nb, -1), nb).to(torch.int32)
        rows = qi[qmask]
        cand[rows, :kk] = nb[qmask]
    if log:
        log(f"candidates: K={K}, {time.time() - t0:.1f} s")
    return cand


def add_reverse(x: torch.Tensor, g: torch.Tensor, R: int, alpha: float, in_cap: int | None = None,
                parts: int | None = None) -> torch.Tensor:
    """Offer q -> p for every edge p -> q of g (at most in_cap offers per q, by
    source id) and prune each row over its neighbours plus its offers."""
    n = g.shape[0]
    dev = g.device
    in_cap = min(in_cap or 2 * R, 128 - R)
    parts = parts or max(1, math.ceil(n * R / (1 << 29)))
    step = math.ceil(n / parts)
    g0 = g.clone()
    out = g
    for t0 in range(0, n, step):
        t1 = min(n, t0 + step)
        flat = torch.nonzero(((g0 >= t0) & (g0 < t1)).view(-1)).squeeze(1)
        tgt = g0.view(-1)[flat].long() - t0
        src = (flat // g0.shape[1]).to(torch.int32)
        del flat
        o = torch.argsort(tgt, stable=True)
        tgt, src = tgt[o], src[o]
        del o
        cnt = torch.bincount(tgt, minlength=t1 - t0)
        start = torch.cumsum(cnt, 0) - cnt
        rank = torch.arange(tgt.numel(), device=dev) - start[tgt]
        keep = rank < in_cap
        inc = torch.full((t1 - t0, in_cap), -1, dtype=torch.int32, device=dev)
        inc[tgt[keep], rank[keep]] = src[keep]
        del tgt, src, rank, keep
        cand = torch.cat([g0[t0:t1], inc], 1)
        del inc
        rows = torch.arange(t0, t1, dtype=torch.int32, device=dev)
        out[t0:t1] = prune(x, cand, R, alpha, rows)
    return out


def repair_orphans(g: torch.Tensor, passes: int = 3, log=None) -> torch.Tensor:
    """Give every node an in-edge: a node that no row lists is written into
    the row of its own nearest neighbour (the first entry of its row), in the
    last slots, displacing that row's farthest neighbours; rows are compacted
    again. A displaced node left without in-edges is repaired in the next pass."""
    n, R = g.shape
    dev = g.device
    for _ in range(passes):
        indeg = torch.bincount(g[g >= 0].long(), minlength=n)
        orph = torch.nonzero(indeg == 0).squeeze(1)
        orph = orph[g[orph, 0] >= 0]
        if orph.numel() == 0:
            break
        tgt = g[orph, 0].long()
        o = torch.argsort(tgt, stable=True)
        tgt, orph = tgt[o], orph[o]
        uniq, cnt = torch.unique_consecutive(tgt, return_counts=True)
        start = torch.cumsum(cnt, 0) - cnt
        rank = torch.arange(tgt.numel(), device=dev) - torch.repeat_interleave(start, cnt)
        keep = rank < R // 4
        tgt, orph, rank = tgt[keep], orph[keep], rank[keep]
        g[tgt, R - 1 - rank] = orph.to(g.dtype)
        rows = torch.unique(tgt)
        sub = g[rows]
        g[rows] = torch.gather(sub, 1, torch.argsort((sub < 0).to(torch.int8), dim=1, stable=True))
        if log:
            log(f"orphan repair: {int(indeg.eq(0).sum())} nodes without in-edges, {tgt.numel()} linked")
    return g


def embed_pivots(g: torch.Tensor, piv: torch.Tensor, nav_graph: torch.Tensor, nav_slots: int) -> torch.Tensor:
    """Put up to nav_slots pivot-graph neighbours (mapped to global ids) at the
    end of every sampled point's row, after its nearest R - nav_slots
    neighbours; ids already in the row are not repeated. The pivot graph's
    rows are in distance order, so they are read from the far end: the long
    edges that the pivot graph's searches created, which cross between
    clusters, are the ones a walk in the main graph lacks."""
    if nav_slots <= 0 or piv.numel() == 0:
        return g
    R = g.shape[1]
    keep = R - nav_slots
    rows = g[piv].long()  # P x R, kept neighbours first
    ng = nav_graph.long()
    ndeg = (ng >= 0).sum(1)
    back = ndeg[:, None] - 1 - torch.arange(ng.shape[1], device=ng.device)[None, :]
    ng = torch.where(back >= 0, torch.gather(ng, 1, back.clamp_min(0)), torch.full_like(ng, -1))  # farthest first
    glob = torch.where(ng >= 0, piv[ng.clamp_min(0)], torch.full_like(ng, -1))
    dup = (glob[:, :, None] == rows[:, None, :keep]).any(-1) | (glob < 0) | (glob == piv[:, None])
    # first nav_slots non-duplicate entries, in pivot-graph order
    ok = ~dup
    pos = torch.cumsum(ok.long(), 1) - 1
    take = ok & (pos < nav_slots)
    add = torch.full((rows.shape[0], nav_slots), -1, dtype=torch.long, device=g.device)
    r_i, c_i = torch.nonzero(take, as_tuple=True)
    add[r_i, pos[r_i, c_i]] = glob[r_i, c_i]
    new = torch.cat([rows[:, :keep], add], 1)
    new = torch.gather(new, 1, torch.argsort((new < 0).to(torch.int8), dim=1, stable=True))
    g[piv] = new.to(g.dtype)
    return g


def build(x: torch.Tensor, R: int, alpha: float = 1.2, K: int | None = None, leaf: int = 4096, seed: int = 7,
          pivots: np.ndarray | None = None, nav_graph: np.ndarray | None = None, nav_slots: int = 16,
          log=None) -> tuple[torch.Tensor, torch.Tensor, int, dict]:
    """Graph over the rows of x (uint8 or float32, on the GPU for large n).
    Returns (adjacency n x R int32 on x's device, -1 padded; degrees; medoid;
    timings)."""
    K = K or 2 * R
    timings = {}
    t = time.time()
    med = builder.medoid(x)
    with _tf32():
        cand = leaf_candidates(x, K, leaf, seed, log=log)
    timings["candidates_s"] = time.time() - t
    t = time.time()
    g = prune(x, cand, R, alpha)
    del cand
    if x.is_cuda:
        torch.cuda.synchronize()
    timings["prune_s"] = time.time() - t
    t = time.time()
    g = add_reverse(x, g, R, alpha)
    if x.is_cuda:
        torch.cuda.synchronize()
    timings["reverse_s"] = time.time() - t
    if pivots is not None and nav_graph is not None:
        piv = torch.from_numpy(np.asarray(pivots, dtype=np.int64)).to(x.device)
        ng = torch.from_numpy(np.asarray(nav_graph, dtype=np.int64)).to(x.device)
        g = embed_pivots(g, piv, ng, min(nav_slots, R // 2))
    g = repair_orphans(g, log=log)
    deg = (g >= 0).sum(1).to(torch.int32)
    indeg = torch.bincount(g[g >= 0].long(), minlength=x.shape[0])
    timings["no_in_edges"] = int((indeg == 0).sum())
    timings["mean_degree"] = float(deg.float().mean())
    if log:
        log(f"graph: mean degree {timings['mean_degree']:.1f}, {timings['no_in_edges']} nodes without in-edges")
    return g, deg, med, timings
