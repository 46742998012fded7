"""Generate the committed parity fixtures under tests/golden/.

Each fixture is a small index in the reference's file formats, a query set, and
the oracle's outputs for a few (k, L) pairs:

    tests/golden/<name>/index_disk.index.gz, index_pq_pivots.bin.gz, index_pq_compressed.bin.gz,
                        nav/{nav_index,nav_index.data,map.txt}.gz (when present)
    tests/golden/<name>/queries.npy
    tests/golden/<name>/oracle.npz      ids/dists/found/entries/hops per (k, L)

The reference's own outputs on the same files (``ref.npz``) are produced on a
B200 by tests/golden/make_ref_golden.py. Run from the repository root:

    python tests/golden/make_fixtures.py
"""
from __future__ import annotations

import gzip
import json
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from gustann_b200.indexing import build_index, synth  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

HERE = Path(__file__).resolve().parent

# name: kind, n, dim, mixture clusters, R, M, nav samples, legacy PQ table, queries, (k, L) cases
FIXTURES = {
    "u8_nav": ("u8", 4000, 128, 8, 32, 32, 160, False, 200, [(10, 10), (10, 20), (10, 40), (10, 64), (1, 16), (32, 48)]),
    "f32_nav": ("f32", 3000, 96, 6, 32, 32, 120, True, 200, [(10, 10), (10, 32), (10, 64), (5, 24)]),
    "u8_medoid": ("u8", 3000, 64, 1, 24, 16, 0, False, 150, [(10, 16), (10, 40), (20, 64)]),
}


def gz(src: Path, dst: Path) -> None:
    with open(src, "rb") as f, open(dst, "wb") as raw, \
            gzip.GzipFile(fileobj=raw, mode="wb", compresslevel=9, mtime=0) as g:
        shutil.copyfileobj(f, g)


def unpack(name: str, dst: Path) -> dict:
    """Decompress fixture ``name`` into ``dst``; returns its paths and metadata."""
    src = HERE / name
    meta = json.loads((src / "meta.json").read_text())
    for p in src.rglob("*.gz"):
        rel = p.relative_to(src).with_suffix("")
        out = dst / rel
        out.parent.mkdir(parents=True, exist_ok=True)
        with gzip.open(p, "rb") as f, open(out, "wb") as g:
            shutil.copyfileobj(f, g)
    meta["index_file"] = str(dst / "index_disk.index")
    meta["pq_prefix"] = str(dst / "index_pq")
    meta["nav_dir"] = str(dst / "nav") if meta["has_nav"] else None
    meta["queries"] = np.load(src / "queries.npy")
    return meta


def main() -> None:
    for name, (kind, n, dim, clusters, R, M, nav, legacy, nq, cases) in FIXTURES.items():
        base, queries = synth.make(kind, n, dim, clusters, nq, backend="numpy")
        qf = queries.astype(np.float32)
        with tempfile.TemporaryDirectory() as tmp:
            f = build_index(base, tmp, R=R, M=M, nav_samples=nav, legacy_pq=legacy)
            out = HERE / name
            if out.exists():
                shutil.rmtree(out)
            (out / "nav").mkdir(parents=True)
            for p in Path(tmp).rglob("*"):
                if p.is_file():
                    gz(p, out / (str(p.relative_to(tmp)) + ".gz"))
            np.save(out / "queries.npy", qf)
            dtype = 0 if kind == "u8" else 1
            o = Oracle(f.index_file, f.pq_prefix, f.nav_dir, dtype)
            res = {}
            for k, L in cases:
                ids, dis, fnd, hops, flags, ent = o.search(qf, k, L)
                if flags.any():
                    raise SystemExit(f"{name} k={k} L={L}: oracle flags {np.unique(flags)}; pick other sizes")
                for key, arr in (("ids", ids), ("dists", dis), ("found", fnd), ("hops", hops), ("entries", ent)):
                    res[f"{key}_k{k}_L{L}"] = arr
            o.close()
            np.savez_compressed(out / "oracle.npz", **res)
            meta = {"kind": kind, "dtype": dtype, "n": n, "dim": dim, "clusters": clusters, "R": R, "M": M,
                    "has_nav": bool(nav), "legacy_pq": legacy, "cases": cases, "fma_table": 1, "fma_exact": 1}
            (out / "meta.json").write_text(json.dumps(meta, indent=1) + "\n")
            print(name, "ok", {k: v for k, v in f.timings.items()})


if __name__ == "__main__":
    main()
