"""GPU checks of the batched (optimised) form: PQ-table error of each
precision against an FP64 oracle, recall against the plain form, uneven L/k,
and that a query's result is the same alone and inside a mixed batch."""
from pathlib import Path

import numpy as np
import pytest

import gustann_b200 as gb
from gustann_b200.indexing import build_index, groundtruth, synth

GOLDEN = Path(__file__).resolve().parent / "golden"


def open_meta(meta):
    g = gb.GustANN(gb.DataType(meta["dtype"]))
    g.init_pure_mem(gb.GustANNConfig(meta["index_file"], meta["pq_prefix"], meta["nav_dir"] or ""))
    return g


def fp64_tables(meta, q):
    import struct

    piv = open(meta["pq_prefix"] + "_pivots.bin", "rb").read()
    nr = struct.unpack_from("<i", piv, 0)[0]
    offs = np.frombuffer(piv, np.uint64, count=nr, offset=8)
    dim = q.shape[1]
    P = np.frombuffer(piv, np.float32, count=256 * dim, offset=int(offs[0]) + 8).reshape(256, dim).astype(np.float64)
    mu = np.frombuffer(piv, np.float32, count=dim, offset=int(offs[1]) + 8).astype(np.float64)
    M = meta["M"]
    co = np.frombuffer(piv, np.uint32, count=M + 1, offset=int(offs[3 if nr == 5 else 2]) + 8)
    r = q.astype(np.float64) - mu
    out = np.zeros((q.shape[0], M, 256))
    for c in range(M):
        b, e = int(co[c]), int(co[c + 1])
        out[:, c, :] = ((r[:, None, b:e] - P[None, :, b:e]) ** 2).sum(-1)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["u8_nav", "f32_nav"])
def test_table_precision_against_fp64(golden, oracle_mod, name):
    """FP32 tables equal the reference's (the oracle's) bit for bit; BF16 forms
    stay within their stated bounds of the FP64 table."""
    meta = golden[name]
    g = open_meta(meta)
    q = meta["queries"][:64]
    ref = fp64_tables(meta, q)
    o = oracle_mod.Oracle(meta["index_file"], meta["pq_prefix"], meta["nav_dir"], meta["dtype"])
    t32 = g.pq_tables(q, gb.PREC_FP32)
    for i in range(4):
        np.testing.assert_array_equal(t32[i], o.pq_table(q[i])[0])
    scale = ref.max(axis=2, keepdims=True)  # per (query, chunk) range of the table
    err = {}
    for prec in (gb.PREC_BF16_CC, gb.PREC_BF16X3, gb.PREC_BF16):
        t = g.pq_tables(q, prec).astype(np.float64)
        err[prec] = float((np.abs(t - ref) / np.maximum(scale, 1e-30)).max())
    # BF16 storage: half an ulp of 2^-8 relative; the split product adds ~2^-16
    assert err[gb.PREC_BF16_CC] <= 2.0 ** -8
    assert err[gb.PREC_BF16X3] <= 2.0 ** -8 + 2.0 ** -12
    # single-pass BF16 operands: cancellation in |r|^2 - 2 r.P + |P|^2
    assert err[gb.PREC_BF16] <= 2.0 ** -5, err


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["u8_nav", "f32_nav"])
def test_rerank_distance_against_fp64(golden, name):
    """Exact-rerank distances of the returned ids against FP64: the batched
    form's int32 path is exact for uint8 vectors with integral queries; FP32
    reranks (batched on float data, and the plain form) stay within
    dim * 2^-24 of the FP64 distance, relative."""
    from gustann_b200.indexing import formats

    meta = golden[name]
    g = open_meta(meta)
    q = meta["queries"]
    vecs = formats.read_disk_index(meta["index_file"], np.uint8 if meta["dtype"] == 0 else np.float32).data
    dim = q.shape[1]
    forms = {"batched": g.search_batch(q, 10, 40, precision=gb.PREC_BF16)[:3], "plain": g.query(q, 10, 40)[:3]}
    for form, (ids, dis, fnd) in forms.items():
        worst = 0.0
        for i in range(len(q)):
            v = vecs[ids[i, :fnd[i]]].astype(np.float64)
            d64 = ((v - q[i].astype(np.float64)) ** 2).sum(1)
            rel = np.abs(dis[i, :fnd[i]].astype(np.float64) - d64) / np.maximum(d64, 1e-30)
            worst = max(worst, float(rel.max()) if len(rel) else 0.0)
        if form == "batched" and meta["dtype"] == 0:
            assert worst == 0.0, (form, worst)
        assert worst <= dim * 2.0 ** -24, (form, worst)


@pytest.fixture(scope="module")
def scale(tmp_path_factory):
    d = tmp_path_factory.mktemp("bscale")
    base, qs = synth.make("u8", 200_000, 128, 200, 2000, backend="torch", device="cuda")
    f = build_index(base, str(d), R=32, M=32, nav_samples=2000, device="cuda")
    gt = groundtruth.knn(base, qs, 10)
    g = gb.GustANN(gb.DataType.UINT8)
    g.init_pure_mem(gb.GustANNConfig(f.index_file, f.pq_prefix, f.nav_dir))
    return g, qs.float().cpu().numpy(), gt


@pytest.mark.gpu
def test_batch_recall_tracks_plain(scale):
    g, q, gt = scale
    for L in (64, 128):
        plain = groundtruth.recall(g.query(q, 10, L)[0], gt, 10)
        for prec in (gb.PREC_FP32, gb.PREC_BF16_CC, gb.PREC_BF16X3, gb.PREC_BF16):
            for W in (1, 4):
                ids, dis, fnd, t = g.search_batch(q, 10, L, precision=prec, beam_width=W)
                assert (fnd == 10).all()
                r = groundtruth.recall(ids, gt, 10)
                assert r >= plain - 0.03, (L, prec, W, r, plain)
                assert np.all(np.diff(dis, axis=1) >= 0)


@pytest.mark.gpu
def test_batch_fp32_w1_matches_plain_mostly(scale):
    """With FP32 tables and one node per step the batched walk differs from the
    reference walk only by its visited filter; most queries return the same ids."""
    g, q, gt = scale
    a = g.query(q, 10, 64)[0]
    b = g.search_batch(q, 10, 64, precision=gb.PREC_FP32, beam_width=1)[0]
    same = (a == b).all(1).mean()
    assert same > 0.8, same


@pytest.mark.gpu
def test_uneven_L_k_and_alone_vs_mixed(scale):
    g, q, gt = scale
    q = q[:300]
    L, k = synth.draws(len(q), [32, 64, 128, 256], [1, 10, 100])
    for prec, W in ((gb.PREC_BF16, 4), (gb.PREC_FP32, 2)):
        ids, dis, fnd, _ = g.search_batch(q, k, L, precision=prec, beam_width=W, hash_bits=11)
        assert ids.shape == (len(q), 100)
        assert (fnd <= k).all() and (fnd == k).mean() > 0.99
        for i in range(0, len(q), 37):  # the same query alone, with its own L and k
            a_ids, a_dis, a_fnd, _ = g.search_batch(q[i:i + 1], int(k[i]), int(L[i]), precision=prec, beam_width=W,
                                                    hash_bits=11)
            assert a_fnd[0] == fnd[i]
            np.testing.assert_array_equal(a_ids[0, :k[i]], ids[i, :k[i]])
            np.testing.assert_array_equal(a_dis[0, :k[i]], dis[i, :k[i]])
            assert (ids[i, k[i]:] == 0).all()


@pytest.mark.gpu
def test_batch_device_form_and_counters(scale):
    import torch

    g, q, gt = scale
    nq = 500
    ids, dis, fnd, _ = g.search_batch(q[:nq], 10, 96, precision=gb.PREC_BF16, beam_width=4, hash_bits=10)
    dq = torch.from_numpy(q[:nq]).cuda()
    di = torch.zeros((nq, 10), dtype=torch.int32, device="cuda")
    dd = torch.zeros((nq, 10), dtype=torch.float32, device="cuda")
    df = torch.zeros(nq, dtype=torch.int32, device="cuda")
    dh = torch.zeros(nq, dtype=torch.int32, device="cuda")
    db = torch.zeros(nq, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    g.search_batch_device(dq.data_ptr(), nq, 0, 0, 10, 96, di.data_ptr(), dd.data_ptr(), df.data_ptr(),
                          dh.data_ptr(), db.data_ptr(), precision=gb.PREC_BF16, beam_width=4, hash_bits=10, stream=s)
    g.check(s)
    np.testing.assert_array_equal(di.cpu().numpy(), ids)
    np.testing.assert_array_equal(dd.cpu().numpy(), dis)
    h = dh.cpu().numpy()
    assert (h >= 96).mean() > 0.9 and (db.cpu().numpy() > 0).all()


@pytest.mark.gpu
def test_batch_argument_errors(scale):
    g, q, gt = scale
    with pytest.raises(gb.GustANNError):
        g.search_batch(q[:4], 10, 64, beam_width=3)
    with pytest.raises(gb.GustANNError):
        g.search_batch(q[:4], 10, 64, hash_bits=20)
    e = g.search_batch(np.zeros((0, 128), np.float32), 10, 64)
    assert e[0].shape == (0, 10)


@pytest.mark.gpu
def test_batch_is_deterministic(scale):
    """Two runs of the same batch give bit-identical ids and distances (the
    visited cache's state does not depend on warp timing)."""
    g, q, gt = scale
    for prec, L, hb in ((gb.PREC_FP32, 48, 6), (gb.PREC_BF16, 64, 7), (gb.PREC_BF16, 256, 0)):
        a = g.search_batch(q, 10, L, precision=prec, beam_width=4, hash_bits=hb)
        for _ in range(2):
            b = g.search_batch(q, 10, L, precision=prec, beam_width=4, hash_bits=hb)
            np.testing.assert_array_equal(a[0], b[0])
            np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


@pytest.mark.gpu
def test_autotune_sets_the_defaults(scale):
    import torch

    g, q, gt = scale
    dq = torch.from_numpy(q).cuda()
    W, hb, secs = g.autotune(dq.data_ptr(), len(q), 10, 128, gb.PREC_BF16)
    assert W in (2, 4, 8) and 4 <= hb <= 16 and secs > 0
    tuned = g.search_batch(q, 10, 128, precision=gb.PREC_BF16)
    explicit = g.search_batch(q, 10, 128, precision=gb.PREC_BF16, beam_width=W, hash_bits=hb)
    np.testing.assert_array_equal(tuned[0], explicit[0])
    np.testing.assert_array_equal(tuned[1].view(np.uint32), explicit[1].view(np.uint32))


@pytest.mark.gpu
def test_graph_replays_match_batch(scale):
    """gann_batch_graph_*: one capture, replayed with run-time counts 300, 0,
    500 and 37 read from device memory; each replay's rows equal
    gann_search_batch on the same queries, rows past the count stay untouched."""
    import torch

    g, q, gt = scale
    q = np.ascontiguousarray(q[:500])
    L, k = synth.draws(len(q), [32, 64, 128, 256], [1, 10, 100])
    L, k = L.astype(np.int32), k.astype(np.int32)
    for prec in (gb.PREC_BF16, gb.PREC_FP32):
        ids, dis, fnd, _ = g.search_batch(q, k, L, precision=prec, beam_width=4, hash_bits=11)
        dq, dk, dl = (torch.from_numpy(x).cuda() for x in (q, k, L))
        dn = torch.zeros(1, dtype=torch.int32, device="cuda")
        nns = torch.empty((500, 100), dtype=torch.int32, device="cuda")
        dd = torch.empty((500, 100), dtype=torch.float32, device="cuda")
        df = torch.empty(500, dtype=torch.int32, device="cuda")
        bg = gb.BatchGraph(g, 500, 100, 256, dq.data_ptr(), dn.data_ptr(), nns.data_ptr(), dd.data_ptr(),
                           df.data_ptr(), d_topk=dk.data_ptr(), d_ef=dl.data_ptr(), precision=prec, beam_width=4,
                           hash_bits=11)
        for n in (300, 0, 500, 37):
            nns.fill_(-7)
            df.fill_(-7)
            dn.fill_(n)
            torch.cuda.synchronize()
            bg.launch()
            torch.cuda.synchronize()
            gi, gd, gf = nns.cpu().numpy(), dd.cpu().numpy(), df.cpu().numpy()
            np.testing.assert_array_equal(gf[:n], fnd[:n])
            for i in range(n):
                np.testing.assert_array_equal(gi[i, :k[i]], ids[i, :k[i]])
                np.testing.assert_array_equal(gd[i, :k[i]].view(np.uint32), dis[i, :k[i]].view(np.uint32))
            assert (gi[n:] == -7).all() and (gf[n:] == -7).all()
        bg.destroy()
    g.check()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["u8_nav", "f32_nav", "u8_medoid"])
def test_batched_fp32_matches_cpu_model(golden, oracle_mod, name):
    """With FP32 tables the batched form is deterministic: ids, distances and
    counts equal the cache-free CPU model (tests/batch_model.py) bit for bit,
    for every W and with visited caches far smaller than L (16 or 32 slots), so
    the cache's evictions and the duplicate removal never change a result."""
    from batch_model import BatchModel

    meta = golden[name]
    model = BatchModel(oracle_mod, meta)
    g = open_meta(meta)
    q = meta["queries"][:100]
    for k, L, W, hb in ((10, 40, 4, 4), (10, 24, 1, 4), (5, 32, 2, 5), (10, 64, 8, 4), (10, 96, 16, 5)):
        ids, dis, fnd, _ = g.search_batch(q, k, L, precision=gb.PREC_FP32, beam_width=W, hash_bits=hb)
        mi, md, mf = model.search(q, k, L, W)
        what = f"{name} k={k} L={L} W={W} hash_bits={hb}"
        np.testing.assert_array_equal(fnd, mf, err_msg=what)
        bad = np.nonzero((ids != mi).any(1))[0]
        assert bad.size == 0, f"{what}: {bad.size} queries differ, first {bad[:5]}"
        np.testing.assert_array_equal(dis.view(np.uint32), md.view(np.uint32), err_msg=what)
    g.check()


def read_pivots(meta):
    """(pivot vectors nav_n x dim, node id of each) from the fixture's pivot graph."""
    import struct

    d = Path(meta["nav_dir"])
    raw = (d / "nav_index.data").read_bytes()
    n, dim = struct.unpack_from("<ii", raw, 0)
    data = np.frombuffer(raw, np.uint8 if meta["dtype"] == 0 else np.float32, count=n * dim, offset=8)
    return data.reshape(n, dim), np.loadtxt(d / "map.txt", dtype=np.int64).reshape(-1)


def nearest_pivots(g, q):
    import torch

    dq = torch.from_numpy(np.ascontiguousarray(q, dtype=np.float32)).cuda()
    piv = torch.full((len(q),), -7, dtype=torch.int32, device="cuda")
    node = torch.full((len(q),), -7, dtype=torch.int32, device="cuda")
    g.nearest_pivots(dq.data_ptr(), len(q), piv.data_ptr(), node.data_ptr())
    torch.cuda.synchronize()
    g.check()
    return piv.cpu().numpy(), node.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["u8_nav", "f32_nav"])
def test_nearest_pivot_entry_is_the_nearest_pivot(golden, name):
    """gann_nearest_pivots (the tensor-core product of queries by pivots with an
    argmin epilogue) against brute force in FP64: for uint8 vectors and
    integral queries the same row, ties to the lowest; for float vectors a
    pivot within the BF16 rounding of the operands. Batches of 1, 100 and all
    queries (one and several CTAs per pivot range)."""
    meta = golden[name]
    g = open_meta(meta)
    data, node_of = read_pivots(meta)
    q = meta["queries"]
    d = ((q.astype(np.float64)[:, None, :] - data.astype(np.float64)[None, :, :]) ** 2).sum(-1)
    best = d.argmin(1)  # first index of the minimum
    for nq in (1, 100, len(q)):
        piv, node = nearest_pivots(g, q[:nq])
        assert (piv >= 0).all() and (piv < len(data)).all()
        np.testing.assert_array_equal(node, node_of[piv])
        rows = np.arange(nq)
        if meta["dtype"] == 0:
            np.testing.assert_array_equal(piv, best[:nq])
        else:
            # BF16 operands: each product q_i x_i is off by at most 2^-8 |q_i x_i|
            # (both roundings), each |x|^2 term by 2^-8 |x|^2
            qx = np.abs(q[:nq].astype(np.float64)) @ np.abs(data.astype(np.float64)).T
            tol = 2.0 ** -7 * (2.0 * qx[rows, piv] + 2.0 * qx[rows, best[:nq]]) + 2.0 ** -7 * (
                (data.astype(np.float64) ** 2).sum(1)[piv] + (data.astype(np.float64) ** 2).sum(1)[best[:nq]])
            assert (d[rows, piv] - d[rows, best[:nq]] <= tol).all()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["u8_nav", "f32_nav"])
def test_nearest_pivot_entry_walk_matches_cpu_model(golden, oracle_mod, name):
    """With GANN_ENTRY_NEAREST_PIVOT and FP32 tables the batched form equals the
    cache-free CPU model started from the same entry nodes, bit for bit; the
    recall at L 40 is at least the pivot-graph walk's minus 0.02."""
    from batch_model import BatchModel

    meta = golden[name]
    model = BatchModel(oracle_mod, meta)
    g = open_meta(meta)
    q = meta["queries"][:100]
    _, node = nearest_pivots(g, q)
    for k, L, W, hb in ((10, 40, 4, 4), (10, 64, 8, 5), (5, 32, 16, 4)):
        ids, dis, fnd, _ = g.search_batch(q, k, L, precision=gb.PREC_FP32, beam_width=W, hash_bits=hb,
                                          entry=gb.ENTRY_NEAREST_PIVOT)
        mi, md, mf = model.search(q, k, L, W, entries=node)
        what = f"{name} k={k} L={L} W={W} hash_bits={hb}"
        np.testing.assert_array_equal(fnd, mf, err_msg=what)
        bad = np.nonzero((ids != mi).any(1))[0]
        assert bad.size == 0, f"{what}: {bad.size} queries differ, first {bad[:5]}"
        np.testing.assert_array_equal(dis.view(np.uint32), md.view(np.uint32), err_msg=what)
    qa = meta["queries"]
    import torch

    from gustann_b200.indexing import formats

    di = formats.read_disk_index(meta["index_file"], np.uint8 if meta["dtype"] == 0 else np.float32)

    gt = groundtruth.knn(torch.from_numpy(np.ascontiguousarray(di.data)), torch.from_numpy(qa), 10)
    rec = {}
    for entry in (gb.ENTRY_NAV_WALK, gb.ENTRY_NEAREST_PIVOT):
        ids, *_ = g.search_batch(qa, 10, 40, precision=gb.PREC_BF16X3, entry=entry)
        rec[entry] = groundtruth.recall(ids, gt, 10)
    assert rec[gb.ENTRY_NEAREST_PIVOT] >= rec[gb.ENTRY_NAV_WALK] - 0.02, rec
    g.check()


@pytest.mark.gpu
def test_nearest_pivot_entry_in_graphs_and_server(golden):
    """The captured graph and the server take the entry option: a graph replay
    equals the direct call, the server's results equal the direct call's, and
    the server charges the entry key in its admission bytes; the no-alloc form
    and an index without a pivot graph refuse the option."""
    import torch

    meta = golden["u8_nav"]
    g = open_meta(meta)
    q = np.ascontiguousarray(meta["queries"][:64], dtype=np.float32)
    k, L = 10, 48
    ids0, dis0, fnd0, _ = g.search_batch(q, k, L, precision=gb.PREC_BF16X3, beam_width=4,
                                         entry=gb.ENTRY_NEAREST_PIVOT)
    dq = torch.from_numpy(q).cuda()
    nq_dev = torch.tensor([len(q)], dtype=torch.int32, device="cuda")
    ids = torch.zeros((len(q), k), dtype=torch.int32, device="cuda")
    dis = torch.zeros((len(q), k), dtype=torch.float32, device="cuda")
    fnd = torch.zeros(len(q), dtype=torch.int32, device="cuda")
    o = gb.GustANN._opts(gb.PREC_BF16X3, 4, 0, gb.ENTRY_NEAREST_PIVOT)
    import ctypes

    gr = ctypes.c_void_p()
    gb._check(gb.lib().gann_batch_graph_create(g.handle, len(q), k, L, ctypes.byref(o), dq.data_ptr(), None, None,
                                               nq_dev.data_ptr(), ids.data_ptr(), dis.data_ptr(), fnd.data_ptr(),
                                               ctypes.byref(gr)))
    try:
        gb._check(gb.lib().gann_batch_graph_launch(gr, None))
        torch.cuda.synchronize()
    finally:
        gb.lib().gann_batch_graph_destroy(gr)
    np.testing.assert_array_equal(ids.cpu().numpy(), ids0)
    np.testing.assert_array_equal(dis.cpu().numpy().view(np.uint32), dis0.view(np.uint32))
    srv_walk = gb.Server(g, max_batch=32, streams=2, topk_max=k, ef_max=L, precision=gb.PREC_BF16X3,
                         beam_width=4)
    srv = gb.Server(g, max_batch=32, streams=2, topk_max=k, ef_max=L, precision=gb.PREC_BF16X3, beam_width=4,
                    entry=gb.ENTRY_NEAREST_PIVOT)
    try:
        assert srv.request_bytes(k, L) == srv_walk.request_bytes(k, L) + 8
        got = {}
        for i in range(len(q)):
            assert srv.submit(q[i], k, L, i)
        import time

        t0 = time.time()
        while len(got) < len(q) and time.time() - t0 < 60:
            tags, ids_r, dis_r, fnd_r, _ = srv.poll(64)
            for j, tag in enumerate(tags):
                got[int(tag)] = (ids_r[j], dis_r[j], fnd_r[j])
        assert len(got) == len(q)
        for i in range(len(q)):
            np.testing.assert_array_equal(got[i][0][:fnd0[i]], ids0[i, :fnd0[i]])
    finally:
        srv.stop()
        srv_walk.stop()
    o2 = gb.GustANN._opts(gb.PREC_BF16X3, 4, 0, gb.ENTRY_NEAREST_PIVOT)
    rc = gb.lib().gann_search_batch_noalloc(g.handle, dq.data_ptr(), len(q), k, L, ctypes.byref(o2), ids.data_ptr(),
                                            dis.data_ptr(), fnd.data_ptr(), None)
    assert rc == gb.GANN_EINVAL
    gm = open_meta(golden["u8_medoid"])
    with pytest.raises(gb.GustANNError):
        gm.search_batch(q, k, L, precision=gb.PREC_BF16X3, entry=gb.ENTRY_NEAREST_PIVOT)
    g.check()


@pytest.mark.gpu
def test_nearest_pivots_many_tiles_per_cta(golden, tmp_path):
    """A pivot file of all 4,000 base points (16 tiles of 256 pivots) and
    enough queries (149 CTA rows of 128, more than the 148 SMs) that each CTA
    walks every tile, so
    the B-stage, norm-slot and TMEM reuse of the tile pipeline all run: the rows
    equal brute force (uint8, exact), twice in a row."""
    import torch

    from gustann_b200.indexing import formats

    meta = golden["u8_nav"]
    data = np.ascontiguousarray(formats.read_disk_index(meta["index_file"], np.uint8).data)
    n = data.shape[0]
    deg = np.full(n, 8, dtype=np.int64)
    graph = ((np.arange(n)[:, None] + np.arange(1, 9)[None, :]) % n).astype(np.int32)
    nav = tmp_path / "nav_all"
    formats.write_nav(str(nav), data, graph, deg, 0, np.arange(n))
    g = gb.GustANN(gb.DataType.UINT8)
    g.init_pure_mem(gb.GustANNConfig(meta["index_file"], meta["pq_prefix"], str(nav)))
    rng = np.random.default_rng(5)
    nq = 149 * 128
    q = np.clip(data[rng.integers(0, n, nq)].astype(np.int64) + rng.integers(-12, 13, (nq, data.shape[1])), 0, 255)
    xf = data.astype(np.float64)
    qf = q.astype(np.float64)
    d = (qf * qf).sum(1)[:, None] - 2.0 * (qf @ xf.T) + (xf * xf).sum(1)[None, :]  # exact: integers < 2^53
    want = d.argmin(1)
    for _ in range(2):
        piv, node = nearest_pivots(g, q.astype(np.float32))
        bad = np.nonzero(piv != want)[0]
        assert bad.size == 0, f"{bad.size} of {nq} queries differ, first {bad[:5]}"
        np.testing.assert_array_equal(node, want)
    g.check()
