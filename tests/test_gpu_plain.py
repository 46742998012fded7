"""GPU parity of the plain (drop-in) form: the CUDA path through the C ABI
against the CPU oracle (bit-exact ids, distances and counts) and against the
reference's own outputs, on the committed fixtures and on larger indexes built
on the device."""
import ctypes
import shutil
import struct
from pathlib import Path

import numpy as np
import pytest

import gustann_b200 as gb
from gustann_b200.indexing import build_index, formats, groundtruth, synth

GOLDEN = Path(__file__).resolve().parent / "golden"
REF_LIB = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libgustann_ref.so"
NAMES = ["u8_nav", "f32_nav", "u8_medoid"]


def fma_flags(name):
    p = GOLDEN / name / "ref.npz"
    if p.exists():
        r = np.load(p)
        return bool(r["fma_table"]), bool(r["fma_exact"])
    return True, True


def open_index(meta, fma=(True, True)):
    g = gb.GustANN(gb.DataType(meta["dtype"]))
    g.init_pure_mem(gb.GustANNConfig(meta["index_file"], meta["pq_prefix"], meta["nav_dir"] or ""))
    g.set_fma(*fma)
    return g


def assert_same(ids, dis, fnd, eids, edis, efnd, what):
    bad = np.nonzero((ids != eids).any(1))[0]
    assert bad.size == 0, f"{what}: {bad.size} queries differ, first {bad[:5]}"
    np.testing.assert_array_equal(dis.view(np.uint32), edis.view(np.uint32), err_msg=what)
    np.testing.assert_array_equal(fnd, efnd, err_msg=what)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_plain_matches_oracle_fixture(golden, name):
    meta = golden[name]
    exp = np.load(GOLDEN / name / "oracle.npz")
    g = open_index(meta)
    for k, L in meta["cases"]:
        ids, dis, fnd, t = g.query(meta["queries"], k, L)
        assert t > 0
        assert_same(ids, dis, fnd, exp[f"ids_k{k}_L{L}"], exp[f"dists_k{k}_L{L}"], exp[f"found_k{k}_L{L}"],
                    f"{name} k={k} L={L}")
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_plain_matches_recorded_reference(golden, name):
    p = GOLDEN / name / "ref.npz"
    if not p.exists():
        pytest.skip("reference outputs not recorded")
    ref = np.load(p)
    meta = golden[name]
    g = open_index(meta, fma_flags(name))
    for k, L in meta["cases"]:
        ids, dis, fnd, _ = g.query(meta["queries"], k, L)
        assert_same(ids, dis, fnd, ref[f"ids_k{k}_L{L}"], ref[f"dists_k{k}_L{L}"], ref[f"found_k{k}_L{L}"],
                    f"{name} k={k} L={L}")


@pytest.fixture(scope="module")
def scale_index(tmp_path_factory):
    """200k uint8 points (C0 generator, 200 clusters of ~1000), R=32, built on the GPU."""
    import torch

    d = tmp_path_factory.mktemp("scale")
    base, qs = synth.make("u8", 200_000, 128, 200, 2000, backend="torch", device="cuda")
    f = build_index(base, str(d), R=32, M=32, nav_samples=2000, device="cuda")
    gt = groundtruth.knn(base, qs, 10)
    return f, qs.float().cpu().numpy(), gt


@pytest.mark.gpu
def test_plain_matches_oracle_at_scale(scale_index, oracle_mod):
    f, q, gt = scale_index
    o = oracle_mod.Oracle(f.index_file, f.pq_prefix, f.nav_dir, 0)
    g = gb.GustANN(gb.DataType.UINT8)
    g.init_pure_mem(gb.GustANNConfig(f.index_file, f.pq_prefix, f.nav_dir))
    for k, L in ((10, 32), (10, 64), (100, 128)):
        ids, dis, fnd, hops, flags, _ = o.search(q, k, L)
        ok = flags == 0
        assert ok.mean() > 0.99
        gi, gd, gf, _ = g.query(q, k, L)
        assert_same(gi[ok], gd[ok], gf[ok], ids[ok], dis[ok], fnd[ok], f"scale k={k} L={L}")
    # recall grows with L and is high once the walk covers the query's cluster
    r = [groundtruth.recall(g.query(q, 10, L)[0], gt, 10) for L in (32, 128, 512)]
    assert r[0] < r[1] < r[2] and r[2] > 0.9, r


@pytest.mark.gpu
def test_plain_matches_reference_live(scale_index, oracle_mod):
    if not REF_LIB.exists():
        pytest.skip("reference library not built")
    f, q, gt = scale_index
    ref = oracle_mod.Reference(f.index_file, f.pq_prefix, f.nav_dir, 0)
    g = gb.GustANN(gb.DataType.UINT8)
    g.init_pure_mem(gb.GustANNConfig(f.index_file, f.pq_prefix, f.nav_dir))
    g.set_fma(*fma_flags("u8_nav"))
    for k, L in ((10, 32), (10, 64)):
        rows, rid, rd, rf, _ = ref.search(q, k, L)  # only the queries the oracle screen passes
        print(f"live reference k={k} L={L}: {rows.size} queries compared, {ref.last_skipped} skipped by the screen")
        assert rows.size > 0.95 * q.shape[0]
        gi, gd, gf, _ = g.query(q, k, L)
        assert_same(gi[rows], gd[rows], gf[rows], rid, rd, rf, f"live reference k={k} L={L}")
    ref.close()


@pytest.mark.gpu
def test_device_entry_point_matches_host(golden):
    import torch

    meta = golden["u8_nav"]
    g = open_index(meta)
    q = meta["queries"]
    ids, dis, fnd, _ = g.query(q, 10, 40)
    dq = torch.from_numpy(q).cuda()
    di = torch.zeros((q.shape[0], 10), dtype=torch.int32, device="cuda")
    dd = torch.zeros((q.shape[0], 10), dtype=torch.float32, device="cuda")
    df = torch.zeros(q.shape[0], dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    g.search_device(dq.data_ptr(), q.shape[0], 10, 40, di.data_ptr(), dd.data_ptr(), df.data_ptr(), s)
    g.check(s)
    assert_same(di.cpu().numpy(), dd.cpu().numpy(), df.cpu().numpy(), ids, dis, fnd, "device form")


@pytest.mark.gpu
def test_edge_shapes_match_oracle(tmp_path, oracle_mod):
    """dim not a multiple of 32, odd R, M not a multiple of 16 (byte-wise code
    loads), k > L, L = 1, k = 1, and an empty batch."""
    base, qs = synth.make("u8", 3000, 100, 3, 100, backend="numpy")
    f = build_index(base, str(tmp_path), R=17, M=25, nav_samples=120)
    o = oracle_mod.Oracle(f.index_file, f.pq_prefix, f.nav_dir, 0)
    g = gb.GustANN(gb.DataType.UINT8)
    g.init_pure_mem(gb.GustANNConfig(f.index_file, f.pq_prefix, f.nav_dir))
    q = qs.astype(np.float32)
    for k, L in ((10, 33), (40, 20), (1, 1), (1, 8), (5, 5)):
        ids, dis, fnd, hops, flags, _ = o.search(q, k, L)
        ok = flags == 0
        gi, gd, gf, _ = g.query(q, k, L)
        assert_same(gi[ok], gd[ok], gf[ok], ids[ok], dis[ok], fnd[ok], f"edge k={k} L={L}")
    e = g.query(np.zeros((0, 100), np.float32), 10, 10)
    assert e[0].shape == (0, 10)


@pytest.mark.gpu
def test_corrupt_record_is_reported_not_read(golden, tmp_path):
    """A neighbour id outside the index: refused at open by the validator; with
    validation off, the kernel checks the id before using it and the call
    returns GANN_EKERNEL."""
    meta = golden["u8_medoid"]
    d = tmp_path / "bad"
    shutil.copytree(Path(meta["index_file"]).parent, d)
    idx = d / "index_disk.index"
    raw = bytearray(idx.read_bytes())
    di = formats.read_disk_index(str(idx), np.uint8)
    med = di.medoid
    off = 4096 + (med // di.npp) * 4096 + (med % di.npp) * di.node_len + di.dim
    struct.pack_into("<i", raw, off + 4, di.n + 5)  # first neighbour of the medoid
    idx.write_bytes(bytes(raw))
    g = gb.GustANN(gb.DataType.UINT8)
    with pytest.raises(gb.GustANNError) as e:
        g.init_pure_mem(gb.GustANNConfig(str(idx), str(d / "index_pq"), ""))
    assert e.value.code == gb.GANN_EFORMAT
    g.init_pure_mem(gb.GustANNConfig(str(idx), str(d / "index_pq"), ""), validate=False)
    with pytest.raises(gb.GustANNError) as e:
        g.query(meta["queries"][:4], 10, 16)
    assert e.value.code == gb.GANN_EKERNEL
    # the handle stays usable after the reported error
    with pytest.raises(gb.GustANNError):
        g.query(meta["queries"][:4], 10, 16)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_host_pages_match_oracle_fixture(golden, name):
    """use_gpu_mem=False (records in pinned host memory, src/pure_mem.cu:51-66):
    the same ids, distances and counts as the oracle."""
    meta = golden[name]
    exp = np.load(GOLDEN / name / "oracle.npz")
    g = gb.GustANN(gb.DataType(meta["dtype"]))
    g.init_pure_mem(gb.GustANNConfig(meta["index_file"], meta["pq_prefix"], meta["nav_dir"] or ""),
                    use_gpu_mem=False)
    inf = g.info()
    assert inf["host_pages"] == 1 and inf["host_bytes"] == inf["num_pages"] * 4096
    for k, L in meta["cases"]:
        ids, dis, fnd, _ = g.query(meta["queries"], k, L)
        assert_same(ids, dis, fnd, exp[f"ids_k{k}_L{L}"], exp[f"dists_k{k}_L{L}"], exp[f"found_k{k}_L{L}"],
                    f"host pages {name} k={k} L={L}")
    g.close()


@pytest.mark.gpu
def test_host_pages_match_hbm_at_scale(scale_index):
    """Both record placements give identical plain and batched results on the
    200k index; the batched form is deterministic, so its ids match exactly too."""
    f, q, gt = scale_index
    cfg = gb.GustANNConfig(f.index_file, f.pq_prefix, f.nav_dir)
    hbm = gb.GustANN(gb.DataType.UINT8)
    hbm.init_pure_mem(cfg)
    host = gb.GustANN(gb.DataType.UINT8)
    host.init_pure_mem(cfg, use_gpu_mem=False)
    hi = host.info()
    assert hi["device_bytes"] + hi["host_bytes"] == hbm.info()["device_bytes"]
    for k, L in ((10, 64), (100, 128)):
        a = hbm.query(q, k, L)
        b = host.query(q, k, L)
        assert_same(b[0], b[1], b[2], a[0], a[1], a[2], f"host vs hbm plain k={k} L={L}")
    for prec in (gb.PREC_BF16, gb.PREC_FP32):
        a = hbm.search_batch(q, 10, 128, precision=prec)
        b = host.search_batch(q, 10, 128, precision=prec)
        assert_same(b[0], b[1], b[2], a[0], a[1], a[2], f"host vs hbm batched precision={prec}")
    hbm.close()
    host.close()


@pytest.mark.gpu
def test_record_cache_keeps_results(scale_index):
    """gann_cache_hot_records on a host-memory handle: the hottest records of a
    sample batch move to HBM and every search returns the same ids, distances
    and counts; a smaller cache replaces it, a zero budget drops it; an HBM
    handle refuses it."""
    import torch

    f, q, gt = scale_index
    cfg = gb.GustANNConfig(f.index_file, f.pq_prefix, f.nav_dir)
    host = gb.GustANN(gb.DataType.UINT8)
    host.init_pure_mem(cfg, use_gpu_mem=False)
    before = (host.query(q, 10, 64), host.search_batch(q, 10, 128))
    dq = torch.from_numpy(np.ascontiguousarray(q[:500])).cuda()
    inf = host.info()
    stride = (inf["node_len"] + 15) // 16 * 16
    budget = inf["num_points"] * stride // 5
    dev0 = inf["device_bytes"]
    for b in (budget, budget // 4, 0):
        n = host.cache_hot_records(dq.data_ptr(), 500, 128, b)
        assert 0 <= n <= b // stride and (n > 0) == (b > 0)
        assert host.info()["device_bytes"] == dev0 + (n * stride + 4 * inf["num_points"] if n else 0)
        after = (host.query(q, 10, 64), host.search_batch(q, 10, 128))
        for (ai, ad, af, _), (bi, bd, bf, _) in zip(before, after):
            assert_same(bi, bd, bf, ai, ad, af, f"record cache {b} bytes")
    host.close()
    hbm = gb.GustANN(gb.DataType.UINT8)
    hbm.init_pure_mem(cfg)
    with pytest.raises(gb.GustANNError) as e:
        hbm.cache_hot_records(dq.data_ptr(), 500, 128, budget)
    assert e.value.code == gb.GANN_EINVAL
    hbm.close()
