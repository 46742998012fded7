"""CPU checks of the index tooling (gustann_b200/indexing): PQ chunking and
encoding, RobustPrune's rule, brute-force ground truth, and a small end-to-end
build whose files the oracle searches with high recall."""
import numpy as np
import pytest
import torch

from gustann_b200.indexing import build_index, builder, formats, groundtruth, pq, synth


@pytest.mark.parametrize("dim,M", [(128, 32), (96, 32), (100, 25), (20, 7), (64, 16)])
def test_chunk_offsets_tile_the_dimensions(dim, M):
    o = pq.chunk_offsets(dim, M).astype(np.int64)
    sizes = np.diff(o)
    assert o[0] == 0 and o[-1] == dim and len(o) == M + 1
    assert sizes.min() >= 1 and sizes.max() - sizes.min() <= 1
    assert np.all(np.diff(sizes) <= 0)  # the wider chunks come first


def test_pq_encode_picks_the_nearest_centroid():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((600, 16)).astype(np.float32)
    pivots, mu, offs = pq.train(torch.from_numpy(x), 4, iters=5)
    codes = pq.encode(torch.from_numpy(x), pivots, mu, offs)
    r = x.astype(np.float64) - mu
    for c in range(4):
        b, e = int(offs[c]), int(offs[c + 1])
        d = ((r[:, None, b:e] - pivots[None, :, b:e].astype(np.float64)) ** 2).sum(-1)
        chosen = d[np.arange(len(x)), codes[:, c]]
        assert np.all(chosen <= d.min(1) * (1 + 1e-4) + 1e-6)


def test_robust_prune_rule():
    """Kept neighbours are candidates in distance order; a candidate is dropped
    only if an earlier kept neighbour p satisfies alpha * d(p, c) < d(u, c)."""
    rng = np.random.default_rng(1)
    x = torch.from_numpy(rng.standard_normal((300, 8)).astype(np.float32))
    n, K, R, alpha = 300, 24, 6, 1.2
    d = builder.sqdist(x, x)
    d.fill_diagonal_(float("inf"))
    cd, cand = torch.sort(d, 1)
    cand, cd = cand[:, :K], cd[:, :K]
    out = builder.robust_prune(x, cand, cd, R, alpha).numpy()
    X = x.numpy().astype(np.float64)
    for u in range(0, n, 7):
        kept = [v for v in out[u] if v >= 0]
        assert 1 <= len(kept) <= R
        row = cand[u].tolist()
        assert kept[0] == row[0] and kept == sorted(kept, key=row.index)
        for c in row[: row.index(kept[-1]) + 1]:
            if c in kept:
                continue
            dc = ((X[u] - X[c]) ** 2).sum()
            assert any(alpha * ((X[p] - X[c]) ** 2).sum() < dc * (1 + 1e-4) for p in kept if row.index(p) < row.index(c))


def test_groundtruth_matches_brute_force():
    rng = np.random.default_rng(2)
    base = rng.standard_normal((2000, 12)).astype(np.float32)
    q = rng.standard_normal((30, 12)).astype(np.float32)
    gt = groundtruth.knn(torch.from_numpy(base), torch.from_numpy(q), 10)
    d = ((q[:, None, :].astype(np.float64) - base[None].astype(np.float64)) ** 2).sum(-1)
    np.testing.assert_array_equal(np.asarray(gt)[:, :10], np.argsort(d, 1, kind="stable")[:, :10])
    assert groundtruth.recall(np.asarray(gt)[:, :10], gt, 10) == 1.0


def test_small_build_is_valid_and_searchable(tmp_path, oracle_mod):
    base, qs = synth.make("u8", 3000, 32, 8, 60, backend="numpy")
    f = build_index(base, str(tmp_path), R=16, M=8, nav_samples=200)
    di = formats.read_disk_index(f.index_file, np.uint8)
    np.testing.assert_array_equal(di.data, base)
    assert di.R == 16 and 0 <= di.medoid < 3000
    assert di.degrees.min() >= 1 and di.degrees.max() <= 16
    for u in range(0, 3000, 11):
        nb = di.graph[u, :di.degrees[u]]
        assert np.all((nb >= 0) & (nb < 3000)) and u not in nb and len(set(nb.tolist())) == len(nb)
    reach = builder.reachable_from(di.graph, di.degrees, di.medoid)
    assert reach.mean() > 0.99
    gt = groundtruth.knn(torch.from_numpy(base), torch.from_numpy(qs), 10)
    o = oracle_mod.Oracle(f.index_file, f.pq_prefix, f.nav_dir, 0)
    ids, dis, fnd, hops, flags, ent = o.search(qs.astype(np.float32), 10, 64)
    assert not flags.any()
    assert groundtruth.recall(ids, gt, 10) > 0.9


def test_partitioned_build_is_valid_and_searchable(tmp_path, oracle_mod):
    """The large-index builder (ivf: leaf k-NN, RobustPrune, reverse edges,
    the pivot graph embedded as long edges) on a small mixture, on the CPU:
    valid rows, pivot-graph edges present in the sampled points' rows, and the
    oracle reaches high recall over its files."""
    from gustann_b200 import sample_pivots
    from gustann_b200.indexing import ivf

    base, qs = synth.make("u8", 6000, 32, 12, 60, backend="numpy")
    f = build_index(base, str(tmp_path), R=16, M=8, nav_samples=300, method="ivf", leaf=512)
    di = formats.read_disk_index(f.index_file, np.uint8)
    np.testing.assert_array_equal(di.data, base)
    assert di.degrees.min() >= 1 and di.degrees.max() <= 16
    for u in range(0, 6000, 7):
        nb = di.graph[u, :di.degrees[u]]
        assert np.all((nb >= 0) & (nb < 6000)) and u not in nb and len(set(nb.tolist())) == len(nb)
    piv = sample_pivots(6000, 300)
    nav = formats.read_nav(f.nav_dir) if hasattr(formats, "read_nav") else None
    # every sampled point keeps some of its pivot-graph neighbours as long edges
    pset = set(piv.tolist())
    frac = np.mean([any(int(v) in pset for v in di.graph[u, :di.degrees[u]]) for u in piv])
    assert frac > 0.9
    assert builder.reachable_from(di.graph, di.degrees, di.medoid).mean() > 0.99
    gt = groundtruth.knn(torch.from_numpy(base), torch.from_numpy(qs), 10)
    o = oracle_mod.Oracle(f.index_file, f.pq_prefix, f.nav_dir, 0)
    ids, dis, fnd, hops, flags, ent = o.search(qs.astype(np.float32), 10, 64)
    assert not flags.any()
    assert groundtruth.recall(ids, gt, 10) > 0.9
    del nav, ivf


def test_leaf_candidates_are_the_exact_neighbours_inside_well_separated_leaves():
    from gustann_b200.indexing import ivf

    base, _ = synth.make("u8", 5000, 32, 5, 1, backend="numpy")
    x = torch.from_numpy(base)
    cand = ivf.leaf_candidates(x, 16, 1000, 3)
    d = builder.sqdist(x[:300], x)
    d[torch.arange(300), torch.arange(300)] = float("inf")
    exact = torch.topk(d, 16, largest=False).indices
    hit = np.mean([len(set(cand[i].tolist()) & set(exact[i].tolist())) / 16 for i in range(300)])
    assert hit > 0.97
    assert (cand[torch.arange(5000), 0] != torch.arange(5000)).all()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["u8", "f32"])
def test_prune_kernel_follows_the_rule(kind):
    """gann_build_prune (one warp per point) against builder.robust_prune on
    the same candidate rows (sorted by distance then id, repeats and the point
    itself dropped): identical rows for uint8 (exact int32 distances), nearly
    identical for float (FP32 sums in another order)."""
    from gustann_b200.indexing import ivf

    rng = np.random.default_rng(4)
    n, dim, K, R, alpha = 3000, 128 if kind == "u8" else 96, 96, 24, 1.2
    if kind == "u8":
        x = torch.from_numpy(rng.integers(0, 256, size=(n, dim), dtype=np.uint8))
    else:
        x = torch.from_numpy(rng.standard_normal((n, dim)).astype(np.float32))
    cand = torch.from_numpy(rng.integers(-1, n, size=(n, K)).astype(np.int32))
    cand[:50, 5] = torch.arange(50, dtype=torch.int32)  # the point itself
    cand[:50, 7] = cand[:50, 6]                          # a repeated id
    got = ivf.prune(x.cuda(), cand.cuda(), R, alpha).cpu()
    want = ivf.prune(x, cand, R, alpha)
    if kind == "u8":
        assert torch.equal(got, want)
    else:
        same = (got == want).all(1).float().mean().item()
        assert same > 0.98, same


@pytest.mark.parametrize("name", ["u8_nav", "f32_nav"])
def test_page_readers_match_the_full_parse(tmp_path, name):
    """read_index_vectors (memory-mapped, per node) and read_pq_pivots give the
    same values as the full-file parse and the writer's inputs."""
    from make_fixtures import unpack

    m = unpack(name, tmp_path)
    dt = np.uint8 if m["dtype"] == 0 else np.float32
    di = formats.read_disk_index(m["index_file"], dt)
    ids = np.array([0, 5, di.n - 1, 17, 5])
    np.testing.assert_array_equal(formats.read_index_vectors(m["index_file"], dt, ids), di.data[ids])
    piv, mu, co = formats.read_pq_pivots(m["pq_prefix"])
    assert piv.shape == (256, di.dim) and mu.shape == (di.dim,)
    assert co[0] == 0 and co[-1] == di.dim and np.all(np.diff(co.astype(np.int64)) >= 1)


def test_leaf_batches_respect_the_distance_budget():
    """Every group's block (leaves x largest query count x pool width) stays
    within the budget unless the group is a single leaf, and the groups cover
    every leaf once, in order -- including a small first leaf followed by
    leaves with many more queries."""
    from gustann_b200.indexing import ivf

    rng = np.random.default_rng(3)
    pool = np.sort(rng.integers(1, 30000, size=500))[::-1]
    q = np.minimum(pool, rng.integers(0, 30000, size=500))
    q[0] = 1  # a pool made almost only of second-nearest members
    budget = 1 << 26
    groups = ivf.leaf_batches(q, pool, budget)
    assert [i for i, _ in groups] == list(np.cumsum([0] + [g for _, g in groups[:-1]]))
    assert sum(g for _, g in groups) == 500
    for i, g in groups:
        block = g * max(1, int(q[i:i + g].max())) * max(1, int(pool[i]))
        assert g == 1 or block <= budget


def test_orphans_are_repaired():
    """repair_orphans leaves no node without an in-edge and rows compact."""
    from gustann_b200.indexing import ivf

    g = torch.full((50, 4), -1, dtype=torch.long)
    for i in range(50):
        g[i, 0] = (i + 1) % 50
        if i % 2 == 0:
            g[i, 1] = (i + 2) % 50
    g[:, 0] = torch.where(torch.arange(50) % 5 == 0, torch.full((50,), 1), g[:, 0])
    assert (torch.bincount(g[g >= 0], minlength=50) == 0).any()
    g = ivf.repair_orphans(g)
    indeg = torch.bincount(g[g >= 0], minlength=50)
    assert (indeg > 0).all()
    assert ((g >= 0).int().diff(dim=1) <= 0).all()  # rows stay compact


def test_embedded_pivot_edges_are_the_far_end_of_the_pivot_rows():
    from gustann_b200.indexing import ivf

    g = torch.arange(40).reshape(10, 4).long() + 100  # 10 nodes, R 4, neighbours 100+
    piv = torch.tensor([2, 5])
    nav = torch.tensor([[1, 0, -1], [0, -1, -1]])  # pivot-graph rows (local ids), nearest first
    out = ivf.embed_pivots(g.clone(), piv, nav, 2)
    assert out[2].tolist() == [108, 109, 5, -1]  # kept 2 nearest, then pivot 1 (= node 5); its own id is dropped
    assert out[5].tolist() == [120, 121, 2, -1]


def test_sparser_entry_file_than_embedded_pivots(tmp_path, oracle_mod):
    """embed_samples: the entry file holds the first 150 points of the pivot
    shuffle while the main graph embeds the 600-point pivot graph's long
    edges; the files stay valid and searchable."""
    from gustann_b200 import sample_pivots

    base, qs = synth.make("u8", 6000, 32, 12, 60, backend="numpy")
    f = build_index(base, str(tmp_path), R=16, M=8, nav_samples=150, embed_samples=600, method="ivf", leaf=512)
    assert "embed_pivots_s" in f.timings
    mapping = np.loadtxt(f"{f.nav_dir}/map.txt", dtype=np.int64)
    np.testing.assert_array_equal(mapping, sample_pivots(6000, 150))
    assert set(mapping.tolist()) <= set(sample_pivots(6000, 600).tolist())  # nested samples
    gt = groundtruth.knn(torch.from_numpy(base), torch.from_numpy(qs), 10)
    o = oracle_mod.Oracle(f.index_file, f.pq_prefix, f.nav_dir, 0)
    ids, *_, flags, _ = o.search(qs.astype(np.float32), 10, 64)
    assert not flags.any()
    assert groundtruth.recall(ids, gt, 10) > 0.9
