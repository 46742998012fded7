"""search_mem, the reference's search_disk driver (bin/search_disk.cpp) over
libgann: argument and file errors on the CPU; on a GPU, its printed recall for
one and several L equals the recall of the oracle's ids (the drop-in form
returns the oracle's ids), with queries replicated by -R."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "gustann_b200" / "search_mem"


def cli():
    from gustann_b200 import build

    build.build_lib()
    return str(build.build_cli())


def run(args):
    return subprocess.run([cli()] + [str(x) for x in args], capture_output=True, text=True, timeout=300)


def test_cli_argument_errors(tmp_path):
    from gustann_b200.indexing import formats

    assert run([]).returncode == 1
    r = run(["--query", "q", "--index", "i", "--pq_data", "p", "--data_type", "int4"])
    assert r.returncode == 1 and "unrecognized data type" in r.stderr
    r = run(["--query", "q", "--index", "i", "--pq_data", "p", "--data_type", "uint8", "--topk", "50",
             "--ef_search", "20"])
    assert r.returncode == 1 and "below topk" in r.stderr
    r = run(["--query", "/nonexistent/q.bvecs", "--index", "i", "--pq_data", "p", "--data_type", "uint8",
             "--topk", "10", "--ef_search", "20"])
    assert r.returncode == 1 and "cannot open" in r.stderr
    bad = tmp_path / "bad.fvecs"
    formats.write_vecs(str(bad), np.zeros((3, 4), np.float32))
    bad.write_bytes(bad.read_bytes()[:-3])
    r = run(["--query", bad, "--index", "i", "--pq_data", "p", "--data_type", "float", "--topk", "10",
             "--ef_search", "20"])
    assert r.returncode == 1 and "whole number of vectors" in r.stderr
    r = run(["--bogus"])
    assert r.returncode == 1 and "unknown argument" in r.stderr
    r = run(["--query", "q", "--index", "i", "--pq_data", "p", "--data_type", "uint8", "--batched", "--entry", "x"])
    assert r.returncode == 1 and "unrecognized entry" in r.stderr
    r = run(["--query", "q", "--index", "i", "--pq_data", "p", "--data_type", "uint8", "--entry", "nearest"])
    assert r.returncode == 1 and "applies to --batched only" in r.stderr


@pytest.mark.gpu
def test_cli_recall_matches_oracle(golden, oracle_mod, tmp_path):
    import torch

    from gustann_b200.indexing import formats, groundtruth

    meta = golden["u8_nav"]
    q = meta["queries"]
    qf = tmp_path / "q.bvecs"
    formats.write_vecs(str(qf), q.astype(np.uint8))
    di = formats.read_disk_index(meta["index_file"], np.uint8)
    gt = groundtruth.knn(torch.from_numpy(di.data), torch.from_numpy(q), 10)
    gf = tmp_path / "gt.ivecs"
    formats.write_vecs(str(gf), np.asarray(gt, dtype=np.int32))
    o = oracle_mod.Oracle(meta["index_file"], meta["pq_prefix"], meta["nav_dir"], 0)
    want = {L: groundtruth.recall(o.search(q, 10, L)[0], gt, 10) for L in (20, 40)}
    base = ["--query", qf, "--index", meta["index_file"], "--pq_data", meta["pq_prefix"], "--nav_graph",
            meta["nav_dir"], "--data_type", "uint8", "--ground_truth", gf, "--topk", "10", "-R", "2"]
    r = run(base + ["--ef_search", "40", "-G"])
    assert r.returncode == 0, r.stderr
    got = float(re.search(r"Recall @ 10: ([0-9.]+)", r.stdout).group(1))
    assert abs(got - want[40]) < 1e-6, (got, want)
    r = run(base + ["--ef_search", "20", "40"])  # records in host memory, two L
    assert r.returncode == 0, r.stderr
    rows = re.findall(r"^(\d+)\s+([0-9.]+)\s+([0-9.]+)\s+([0-9.]+)\s*$", r.stdout, flags=re.M)
    assert [int(x[0]) for x in rows] == [20, 40]
    for L, _, qps, rec in rows:
        assert float(qps) > 0 and abs(float(rec) - want[int(L)]) < 1e-6, (L, rec, want)
    r = run(base + ["--ef_search", "40", "-G", "--batched"])
    assert r.returncode == 0, r.stderr
    assert float(re.search(r"Recall @ 10: ([0-9.]+)", r.stdout).group(1)) > want[40] - 0.05
    r = run(base + ["--ef_search", "40", "-G", "--batched", "--entry", "nearest"])
    assert r.returncode == 0, r.stderr
    assert float(re.search(r"Recall @ 10: ([0-9.]+)", r.stdout).group(1)) > want[40] - 0.1
