"""CPU checks of the C ABI library (exports, argument and file errors that are
raised before any device work) and of the file-format writers/readers."""
import ctypes
import re
import shutil
import struct
from pathlib import Path

import numpy as np
import pytest

import gustann_b200 as gb
from gustann_b200.indexing import formats

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "gann.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(gann_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = gb.lib()
    names = declared_functions()
    assert "gann_open" in names and "gann_search" in names
    for name in names:
        assert hasattr(L, name), name
    assert sorted(gb.exported_symbols()) == names


def _open(index, pq, nav, dtype=0):
    h = ctypes.c_void_p()
    rc = gb.lib().gann_open(index.encode(), pq.encode(), nav.encode() if nav else None, dtype, 0,
                            ctypes.byref(h))
    return rc, gb.lib().gann_last_error().decode()


def test_open_argument_errors():
    h = ctypes.c_void_p()
    assert gb.lib().gann_open(None, b"x", None, 0, 0, ctypes.byref(h)) == gb.GANN_EINVAL
    assert gb.lib().gann_open(b"x", b"x", None, 7, 0, ctypes.byref(h)) == gb.GANN_EINVAL
    assert gb.lib().gann_search(None, None, 1, 1, 1, None, None, None, None) == gb.GANN_EINVAL
    rc, msg = _open("/nonexistent/index", "/nonexistent/pq", None)
    assert rc == gb.GANN_EIO and "cannot open" in msg


def _copy(golden, name, tmp_path):
    meta = golden[name]
    src = Path(meta["index_file"]).parent
    dst = tmp_path / name
    shutil.copytree(src, dst)
    return dst, meta


def test_open_rejects_corrupt_index_header(golden, tmp_path):
    d, meta = _copy(golden, "u8_nav", tmp_path)
    idx = d / "index_disk.index"
    raw = bytearray(idx.read_bytes())
    bad = bytearray(raw)
    struct.pack_into("<Q", bad, 8 + 3 * 8, 5000)  # max_node_len larger than a page
    idx.write_bytes(bytes(bad))
    rc, msg = _open(str(idx), str(d / "index_pq"), str(d / "nav"))
    assert rc == gb.GANN_EFORMAT, msg
    idx.write_bytes(bytes(raw[: 4096 * 3]))  # truncated body
    rc, msg = _open(str(idx), str(d / "index_pq"), str(d / "nav"))
    assert rc == gb.GANN_EIO, msg


def test_open_rejects_bad_pq_and_nav(golden, tmp_path):
    d, meta = _copy(golden, "u8_nav", tmp_path)
    piv = d / "index_pq_pivots.bin"
    raw = bytearray(piv.read_bytes())
    bad = bytearray(raw)
    struct.pack_into("<i", bad, 0, 3)  # offsets table must be 4 or 5 rows (pq_search.cu:77-79)
    piv.write_bytes(bytes(bad))
    rc, msg = _open(str(d / "index_disk.index"), str(d / "index_pq"), str(d / "nav"))
    assert rc == gb.GANN_EFORMAT and "offsets" in msg
    piv.write_bytes(bytes(raw))
    nav = d / "nav" / "nav_index"
    nraw = bytearray(nav.read_bytes())
    bad = bytearray(nraw)
    struct.pack_into("<i", bad, 8, 33)  # max degree > 32 (nav_graph.cu:84)
    nav.write_bytes(bytes(bad))
    rc, msg = _open(str(d / "index_disk.index"), str(d / "index_pq"), str(d / "nav"))
    assert rc == gb.GANN_EFORMAT and "max degree" in msg
    nav.write_bytes(bytes(nraw))
    (d / "nav" / "map.txt").write_text("1\n2\n")
    rc, msg = _open(str(d / "index_disk.index"), str(d / "index_pq"), str(d / "nav"))
    assert rc == gb.GANN_EFORMAT and "map.txt" in msg


def test_open_rejects_mismatched_codes(golden, tmp_path):
    d, meta = _copy(golden, "u8_medoid", tmp_path)
    cmp = d / "index_pq_compressed.bin"
    raw = bytearray(cmp.read_bytes())
    struct.pack_into("<i", raw, 0, meta["n"] - 1)
    cmp.write_bytes(bytes(raw[: 8 + (meta["n"] - 1) * meta["M"]]))
    rc, msg = _open(str(d / "index_disk.index"), str(d / "index_pq"), None)
    assert rc == gb.GANN_EFORMAT and "code count" in msg


def test_host_memory_mode_reports_file_errors():
    """use_gpu_mem=False reads the same files; a missing one is GANN_EIO before any device work."""
    g = gb.GustANN(gb.DataType.UINT8)
    with pytest.raises(gb.GustANNError) as e:
        g.init_pure_mem(gb.GustANNConfig("/nonexistent/index", "/nonexistent/pq", ""), use_gpu_mem=False)
    assert e.value.code == gb.GANN_EIO


def test_info_struct_matches_header():
    """gann_info_t's layout in the ctypes mirror: field order and the trailing host fields."""
    import re as _re

    text = (ROOT / "include" / "gann.h").read_text()
    body = _re.search(r"typedef struct \{([^}]*)\} gann_info_t;", text).group(1)
    names = _re.findall(r"int(?:32|64)_t\s+(\w+);", body)
    assert names == [f for f, _ in gb.GannInfo._fields_]
    assert ctypes.sizeof(gb.GannInfo) == 8 * 7 + 4 * 6 + 8 + 4 * 2 + 8


def test_sample_pivots_properties():
    a = gb.sample_pivots(100000, 1000)
    b = gb.sample_pivots(100000, 1000)
    assert np.array_equal(a, b)
    assert np.all(np.diff(a) > 0) and a[0] >= 0 and a[-1] < 100000
    assert not np.array_equal(a, gb.sample_pivots(100000, 1000, seed=1))
    assert len(gb.sample_pivots(50, 50)) == 50


def test_disk_index_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    for dt, dim, R in ((np.uint8, 128, 64), (np.float32, 96, 32), (np.uint8, 20, 7)):
        n = 1000
        data = (rng.integers(0, 256, (n, dim)) if dt == np.uint8 else rng.standard_normal((n, dim))).astype(dt)
        deg = rng.integers(0, R + 1, n).astype(np.int32)
        g = rng.integers(0, n, (n, R)).astype(np.int32)
        p = tmp_path / f"i_{dim}.index"
        info = formats.write_disk_index(str(p), data, g, deg, 17, R, chunk_nodes=300)
        di = formats.read_disk_index(str(p), dt)
        assert (di.n, di.dim, di.medoid, di.R) == (n, dim, 17, R)
        assert di.npp == 4096 // (dim * np.dtype(dt).itemsize + (R + 1) * 4) == info["npp"]
        np.testing.assert_array_equal(di.data, data)
        np.testing.assert_array_equal(di.degrees, deg)
        mask = np.arange(R)[None, :] < deg[:, None]
        np.testing.assert_array_equal(np.where(mask, di.graph, 0), np.where(mask, g, 0))
        assert p.stat().st_size == 4096 * (info["num_pages"] + 1)


def test_vecs_round_trip(tmp_path):
    a = np.arange(30, dtype=np.float32).reshape(5, 6)
    formats.write_vecs(str(tmp_path / "a.fvecs"), a)
    np.testing.assert_array_equal(formats.read_vecs(str(tmp_path / "a.fvecs"), np.float32), a)
    b = np.arange(30, dtype=np.uint8).reshape(3, 10)
    formats.write_vecs(str(tmp_path / "b.bvecs"), b)
    np.testing.assert_array_equal(formats.read_vecs(str(tmp_path / "b.bvecs"), np.uint8), b)


def test_pq_legacy_and_new_tables_agree(golden, tmp_path, oracle_mod):
    """nr == 5 keeps the chunk offsets in entry 3, nr == 4 in entry 2 (pq_search.cu:100-103)."""
    from gustann_b200.indexing import pq as pqmod

    meta = golden["u8_nav"]
    o = oracle_mod.Oracle(meta["index_file"], meta["pq_prefix"], meta["nav_dir"], 0)
    q = meta["queries"][:5]
    t_new = [o.pq_table(x)[0] for x in q]
    piv = open(meta["pq_prefix"] + "_pivots.bin", "rb").read()
    offs = np.frombuffer(piv, np.uint64, count=4, offset=8)
    P = np.frombuffer(piv, np.float32, count=256 * 128, offset=int(offs[0]) + 8).reshape(256, 128)
    mu = np.frombuffer(piv, np.float32, count=128, offset=int(offs[1]) + 8)
    codes = np.fromfile(meta["pq_prefix"] + "_compressed.bin", np.uint8)[8:].reshape(meta["n"], meta["M"])
    d = tmp_path / "leg"
    shutil.copytree(Path(meta["index_file"]).parent, d)
    formats.write_pq(str(d / "index_pq"), P, mu, pqmod.chunk_offsets(128, 32), codes, legacy=True)
    o2 = oracle_mod.Oracle(str(d / "index_disk.index"), str(d / "index_pq"), str(d / "nav"), 0)
    for x, t in zip(q, t_new):
        np.testing.assert_array_equal(o2.pq_table(x)[0], t)


def test_record_division_is_exact(tmp_path):
    """gann::FastDiv (multiply-shift division by nodes-per-page, used to address
    records in the batched walk) equals integer division for ids below 2^31."""
    import subprocess

    exe = tmp_path / "fastdiv_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", "/usr/local/cuda/include", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "fastdiv_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr


def test_null_handles_are_rejected_before_device_work():
    L = gb.lib()
    out = ctypes.c_void_p()
    assert L.gann_batch_graph_create(None, 1, 1, 1, None, None, None, None, None, None, None, None,
                                     ctypes.byref(out)) == gb.GANN_EINVAL
    assert L.gann_batch_graph_launch(None, None) == gb.GANN_EINVAL
    assert L.gann_batch_graph_destroy(None) == gb.GANN_OK
    n = ctypes.c_int64(0)
    assert L.gann_cache_hot_records(None, None, 1, 10, 0, ctypes.byref(n)) == gb.GANN_EINVAL
    assert L.gann_server_start(None, None, ctypes.byref(out)) == gb.GANN_EINVAL
    assert L.gann_server_stop(None) == gb.GANN_OK
    assert "null" in L.gann_last_error().decode()


@pytest.mark.parametrize("cname,pycls", [("gann_batch_opts_t", "BatchOpts"), ("gann_server_opts_t", "ServerOpts"),
                                         ("gann_load_stats_t", "LoadStats"), ("gann_info_t", "GannInfo")])
def test_ctypes_structs_match_the_header(tmp_path, cname, pycls):
    """Every field offset and the size of each ctypes mirror equal what a C
    compiler lays out from include/gann.h."""
    import subprocess

    cls = getattr(gb, pycls)
    fields = [f for f, _ in cls._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stddef.h>\n#include <stdio.h>\n#include \"gann.h\"\nint main(void) {\n"
                   + f'  printf("%zu\\n", sizeof({cname}));\n'
                   + "".join(f'  printf("%zu\\n", offsetof({cname}, {f}));\n' for f in fields)
                   + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got[0] == ctypes.sizeof(cls)
    assert got[1:] == [getattr(cls, f).offset for f in fields]
