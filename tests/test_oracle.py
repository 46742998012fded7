"""CPU oracle: regression against the committed fixtures, pinning against the
reference's own outputs (ref.npz, produced on a B200 by make_ref_golden.py),
and unit checks of the restated primitives."""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _cases(meta):
    return [tuple(c) for c in meta["cases"]]


@pytest.mark.parametrize("name", ["u8_nav", "f32_nav", "u8_medoid"])
def test_oracle_reproduces_fixture(golden, oracle_mod, name):
    meta = golden[name]
    exp = np.load(GOLDEN / name / "oracle.npz")
    o = oracle_mod.Oracle(meta["index_file"], meta["pq_prefix"], meta["nav_dir"], meta["dtype"])
    for k, L in _cases(meta):
        ids, dis, fnd, hops, flags, ent = o.search(meta["queries"], k, L, threads=4)
        assert not flags.any()
        np.testing.assert_array_equal(ids, exp[f"ids_k{k}_L{L}"])
        np.testing.assert_array_equal(dis.view(np.uint32), exp[f"dists_k{k}_L{L}"].view(np.uint32))
        np.testing.assert_array_equal(fnd, exp[f"found_k{k}_L{L}"])
        np.testing.assert_array_equal(ent, exp[f"entries_k{k}_L{L}"])


@pytest.mark.parametrize("name", ["u8_nav", "f32_nav", "u8_medoid"])
def test_oracle_matches_reference_outputs(golden, oracle_mod, name):
    """ref.npz holds the reference kernel's own ids/distances on the same files,
    recorded on a B200 (tests/golden/make_ref_golden.py)."""
    ref_path = GOLDEN / name / "ref.npz"
    if not ref_path.exists():
        pytest.skip("reference outputs not recorded yet")
    ref = np.load(ref_path)
    meta = golden[name]
    o = oracle_mod.Oracle(meta["index_file"], meta["pq_prefix"], meta["nav_dir"], meta["dtype"],
                          fma_table=bool(ref["fma_table"]), fma_exact=bool(ref["fma_exact"]))
    for k, L in _cases(meta):
        ids, dis, fnd, *_ = o.search(meta["queries"], k, L, threads=4)
        np.testing.assert_array_equal(ids, ref[f"ids_k{k}_L{L}"])
        np.testing.assert_array_equal(fnd, ref[f"found_k{k}_L{L}"])
        np.testing.assert_array_equal(dis.view(np.uint32), ref[f"dists_k{k}_L{L}"].view(np.uint32))


def test_exact_dist_tree_order(oracle_mod):
    """square_sum_32 (util.cuh:26-46): per-lane strided partial sums, then the
    shfl_down tree; checked against a direct restatement."""
    rng = np.random.default_rng(0)
    for dim in (1, 31, 32, 96, 100, 128, 200):
        q = rng.standard_normal(dim).astype(np.float32)
        v = rng.standard_normal(dim).astype(np.float32)
        for fma in (0, 1):
            lanes = np.zeros(32, np.float32)
            for l in range(32):
                acc = np.float32(0)
                for i in range(l, dim, 32):
                    d = np.float32(q[i] - v[i])
                    if fma:
                        acc = np.float32(np.float64(d) * np.float64(d) + np.float64(acc))
                    else:
                        acc = np.float32(acc + np.float32(d * d))
                lanes[l] = acc
            for off in (16, 8, 4, 2, 1):
                for l in range(32 - off):
                    lanes[l] = np.float32(lanes[l] + lanes[l + off])
            assert oracle_mod.exact_dist(q, v, fma=bool(fma)) == lanes[0]


def test_exact_dist_uint8_is_exact(oracle_mod):
    rng = np.random.default_rng(1)
    for _ in range(20):
        v = rng.integers(0, 256, 128).astype(np.uint8)
        q = rng.integers(0, 256, 128).astype(np.float32)
        exact = float(((q.astype(np.int64) - v.astype(np.int64)) ** 2).sum())
        assert oracle_mod.exact_dist(q, v, True) == exact
        assert oracle_mod.exact_dist(q, v, False) == exact


def test_pq_table_order_and_restore(golden, oracle_mod):
    """pq.cuh:8-59: table accumulated in dimension order; query restored as
    fl(fl(q - mu) + mu)."""
    meta = golden["f32_nav"]
    o = oracle_mod.Oracle(meta["index_file"], meta["pq_prefix"], meta["nav_dir"], meta["dtype"])
    import struct

    piv = open(meta["pq_prefix"] + "_pivots.bin", "rb").read()
    offs = np.frombuffer(piv, np.uint64, count=5, offset=8)
    P = np.frombuffer(piv, np.float32, count=256 * 96, offset=int(offs[0]) + 8).reshape(256, 96)
    mu = np.frombuffer(piv, np.float32, count=96, offset=int(offs[1]) + 8)
    legacy = struct.unpack_from("<i", piv, 0)[0] == 5
    co = np.frombuffer(piv, np.uint32, count=o.M + 1, offset=int(offs[3 if legacy else 2]) + 8)
    q = meta["queries"][3]
    table, qr = o.pq_table(q)
    qc = (q - mu).astype(np.float32)
    for c in range(o.M):
        acc = np.zeros(256, np.float32)
        for i in range(co[c], co[c + 1]):
            d = (qc[i] - P[:, i]).astype(np.float32)
            acc = (d.astype(np.float64) * d + acc).astype(np.float32)
        np.testing.assert_array_equal(table[c], acc)
    np.testing.assert_array_equal(qr, (qc + mu).astype(np.float32))


def test_walk_reaches_recall(golden, oracle_mod):
    import torch

    from gustann_b200.indexing import formats, groundtruth

    meta = golden["u8_nav"]
    di = formats.read_disk_index(meta["index_file"], np.uint8)
    gt = groundtruth.knn(torch.from_numpy(di.data), torch.from_numpy(meta["queries"]), 10)
    o = oracle_mod.Oracle(meta["index_file"], meta["pq_prefix"], meta["nav_dir"], meta["dtype"])
    r = [groundtruth.recall(o.search(meta["queries"], 10, L)[0], gt, 10) for L in (10, 20, 40, 64)]
    assert r == sorted(r) and r[-1] > 0.9


def test_topk_semantics_ties_go_after(golden, oracle_mod):
    """retset_push_32 (util.cuh:116-163): k smallest exact distances over every
    expanded node, equal distances keep insertion order, duplicates allowed."""
    meta = golden["u8_nav"]
    o = oracle_mod.Oracle(meta["index_file"], meta["pq_prefix"], meta["nav_dir"], meta["dtype"])
    from gustann_b200.indexing import formats

    di = formats.read_disk_index(meta["index_file"], np.uint8)
    for qi in range(20):
        q = meta["queries"][qi]
        ids, dis, fnd, trace, flags, ent = o.search_one(q, 10, 32)
        assert flags == 0 and trace[0] == ent
        exact = [oracle_mod.exact_dist(q, di.data[u]) for u in trace]
        order = sorted(range(len(trace)), key=lambda i: (exact[i], i))[:10]
        assert list(ids[:fnd]) == [int(trace[i]) for i in order]
        assert list(dis[:fnd]) == [exact[i] for i in order]


def test_batch_model_is_sane(golden, oracle_mod):
    """The CPU model of the batched walk (tests/batch_model.py): k results in
    ascending order, and close to the reference walk's recall on the fixture."""
    import torch

    from batch_model import BatchModel
    from gustann_b200.indexing import formats, groundtruth

    meta = golden["u8_nav"]
    q = meta["queries"][:40]
    model = BatchModel(oracle_mod, meta)
    di = formats.read_disk_index(meta["index_file"], np.uint8)
    gt = groundtruth.knn(torch.from_numpy(di.data), torch.from_numpy(q), 10)
    o = oracle_mod.Oracle(meta["index_file"], meta["pq_prefix"], meta["nav_dir"], meta["dtype"])
    plain = groundtruth.recall(o.search(q, 10, 40)[0], gt, 10)
    for W in (1, 4):
        ids, dis, fnd = model.search(q, 10, 40, W)
        assert (fnd == 10).all()
        assert np.all(np.diff(dis, axis=1) >= 0)
        assert groundtruth.recall(ids, gt, 10) >= plain - 0.05
