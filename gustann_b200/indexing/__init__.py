"""Index preparation: synthetic data, graph + PQ + pivot-graph build, file writers.

``build_index`` produces the reference's input files (the ones
``GustANN::init_pure_mem`` reads, src/ssd_search.cu:55-79) from a base matrix:

    <out>/index_disk.index
    <out>/index_pq_pivots.bin, <out>/index_pq_compressed.bin
    <out>/nav/{nav_index, nav_index.data, map.txt}

The pivot graph follows scripts/gen_pivot_graph.sh:7-14: a uniform sample of
the base (bin/gen_small_file.cpp's shuffle), indexed with R=32.
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import builder, formats, pq, synth  # noqa: F401


@dataclass
class IndexFiles:
    index_file: str
    pq_prefix: str
    nav_dir: str | None
    n: int
    dim: int
    dtype: str
    R: int
    M: int
    medoid: int
    timings: dict = field(default_factory=dict)


def _np(x):
    return x.cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


def build_index(base, out_dir: str, R: int, M: int = 32, alpha: float = 1.2, nav_samples: int | None = None,
                nav_R: int = 32, device=None, n_coarse: int | None = None, nprobe: int = 4,
                pq_train: int = 1 << 18, seed: int = 7, legacy_pq: bool = False, method: str = "auto",
                leaf: int = 4096, nav_L_build: int = 100, embed_samples: int | None = None,
                log=None) -> IndexFiles:
    """Build and write every file of one index. ``base`` is an n x dim uint8 or
    float32 array/tensor. ``nav_samples`` = 0 writes no pivot graph.

    ``embed_samples`` (partitioned builder only): the sample whose pivot graph
    supplies the main graph's long edges, when it should differ from the entry
    file's. A sparser entry file routes the entry walk (a beam of 4,
    src/impl/nav.cuh:11-12) better across many clusters, while a denser
    embedded sample gives more nodes long edges; both samples are prefixes of
    the same shuffle, so the entry file's points are embedded points too.

    ``method``: "vamana" (builder.build: Vamana searches from the medoid),
    "ivf" (ivf.build: exact leaf neighbourhoods, pruned, reverse edges, the
    pivot graph embedded as long edges) or "auto" (ivf from 4M points on)."""
    from .. import sample_pivots

    t0 = time.time()
    timings = {}
    os.makedirs(out_dir, exist_ok=True)
    x = base if isinstance(base, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(base))
    if device is not None:
        x = x.to(device)
    n, dim = x.shape
    kind = "u8" if x.dtype == torch.uint8 else "f32"
    large = method == "ivf" or (method == "auto" and n >= 4_000_000)
    if nav_samples is None:
        nav_samples = max(64, n // 100)
    nav = None
    if nav_samples:
        t3 = time.time()
        ids = sample_pivots(n, min(nav_samples, n))
        sub = x[torch.from_numpy(ids.astype(np.int64)).to(x.device)]
        ng, ndeg, nmed = builder.build(sub, nav_R, alpha, seed=seed + 1, L_build=nav_L_build)
        if int(ndeg.min()) < 3:
            raise RuntimeError("pivot graph has a node with fewer than 3 neighbours")
        nav = (ids, sub, ng, ndeg, nmed)
        timings["nav_s"] = time.time() - t3
        if log:
            log(f"pivot graph: {len(ids)} points, {timings['nav_s']:.1f} s")
    embed = (nav[0], nav[2]) if nav else None
    if large and embed_samples and nav and embed_samples != len(nav[0]):
        t3 = time.time()
        eids = sample_pivots(n, min(embed_samples, n))
        esub = x[torch.from_numpy(eids.astype(np.int64)).to(x.device)]
        eg, _, _ = builder.build(esub, nav_R, alpha, seed=seed + 1, L_build=nav_L_build)
        embed = (eids, eg)
        del esub
        timings["embed_pivots_s"] = time.time() - t3
        if log:
            log(f"embedded pivot graph: {len(eids)} points, {timings['embed_pivots_s']:.1f} s")
    t1 = time.time()
    index_file = os.path.join(out_dir, "index_disk.index")
    if large:
        from . import ivf

        g, deg, med, gt = ivf.build(x, R, alpha, seed=seed, leaf=leaf,
                                    pivots=embed[0] if embed else None, nav_graph=embed[1] if embed else None,
                                    log=log)
        timings.update({f"graph_{k}": v for k, v in gt.items()})
        timings["graph_s"] = time.time() - t1
        t2 = time.time()
        formats.write_disk_index_torch(index_file, x, g, deg, med, R)
        del g, deg
        timings["write_index_s"] = time.time() - t2
    else:
        g, deg, med = builder.build(x, R, alpha, n_coarse=n_coarse, nprobe=nprobe, seed=seed)
        timings["graph_s"] = time.time() - t1
        t2 = time.time()
        formats.write_disk_index(index_file, _np(x), g, deg, med, R)
        timings["write_index_s"] = time.time() - t2
    if log:
        log(f"graph + index file: {time.time() - t1:.1f} s")
    t1 = time.time()
    pivots, centroid, offs = pq.train(x, M, n_train=pq_train, seed=seed + 4)
    codes = pq.encode(x, pivots, centroid, offs)
    pq_prefix = os.path.join(out_dir, "index_pq")
    formats.write_pq(pq_prefix, pivots, centroid, offs, codes, legacy=legacy_pq)
    del codes
    timings["pq_s"] = time.time() - t1
    nav_dir = None
    if nav:
        ids, sub, ng, ndeg, nmed = nav
        nav_dir = os.path.join(out_dir, "nav")
        formats.write_nav(nav_dir, _np(sub), ng, ndeg, nmed, ids)
    timings["total_s"] = time.time() - t0
    if log:
        log(f"index built in {timings['total_s']:.1f} s: {timings}")
    return IndexFiles(index_file, pq_prefix, nav_dir, n, dim, kind, R, M, med, timings)
