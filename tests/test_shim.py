"""The C++ shim (include/gustann.hpp) lets reference-style host code compile and
link against libgann.so; on a GPU the shim's driver reproduces the oracle."""
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def build_driver(tmp_path: Path) -> Path:
    exe = tmp_path / "shim_driver"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(ROOT / "tests" / "shim_driver.cpp"),
                    "-o", str(exe), "-L", str(ROOT / "gustann_b200"), "-lgann",
                    f"-Wl,-rpath,{ROOT / 'gustann_b200'}"], check=True)
    return exe


def test_shim_compiles_and_links(tmp_path):
    exe = build_driver(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def test_shim_reports_open_errors(tmp_path):
    exe = build_driver(tmp_path)
    q = tmp_path / "q.bin"
    q.write_bytes(struct.pack("<ii", 1, 4) + np.zeros(4, np.float32).tobytes())
    r = subprocess.run([str(exe), "uint8", "/nonexistent", "/nonexistent", "-", str(q), "10", "10",
                        str(tmp_path / "o")], capture_output=True, text=True)
    assert r.returncode == 1 and "cannot open" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("mem", ["gpu", "dram"])
def test_shim_driver_matches_oracle(golden, tmp_path, oracle_mod, mem):
    exe = build_driver(tmp_path)
    meta = golden["u8_nav"]
    q = meta["queries"]
    qf = tmp_path / "q.bin"
    qf.write_bytes(struct.pack("<ii", *q.shape) + q.tobytes())
    out = tmp_path / "out.bin"
    r = subprocess.run([str(exe), "uint8", meta["index_file"], meta["pq_prefix"], meta["nav_dir"], str(qf), "10", "40",
                        str(out), mem], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = out.read_bytes()
    nq = q.shape[0]
    ids = np.frombuffer(raw, np.int32, count=nq * 10).reshape(nq, 10)
    dis = np.frombuffer(raw, np.float32, count=nq * 10, offset=nq * 40).reshape(nq, 10)
    exp = np.load(ROOT / "tests" / "golden" / "u8_nav" / "oracle.npz")
    np.testing.assert_array_equal(ids, exp["ids_k10_L40"])
    np.testing.assert_array_equal(dis.view(np.uint32), exp["dists_k10_L40"].view(np.uint32))
