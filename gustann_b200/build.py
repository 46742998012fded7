"""Build recipe for libgann.so (the product) and the checker libraries.

``build_lib()`` compiles every CUDA/C++ source under ``csrc/`` for sm_100a with
nvcc and links ``gustann_b200/libgann.so`` in-tree, so that the shared object
travels with the source tree. ``build_oracle()`` builds the CPU oracle and, when
the reference sources are available, the reference's own path (both checker
only, under ``oracle/``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgann.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr", "-I", str(ROOT / "include"),
]
EXPORTS = [
    "gann_open", "gann_close", "gann_get_info", "gann_search", "gann_search_device", "gann_search_device_ex", "gann_search_batch", "gann_search_batch_device", "gann_search_batch_noalloc", "gann_pq_tables", "gann_autotune", "gann_server_start", "gann_server_submit", "gann_server_request_bytes", "gann_server_poll", "gann_server_stop", "gann_server_open_loop", "gann_check",
    "gann_set_fma", "gann_last_error", "gann_sample_pivots", "gann_batch_graph_create",
    "gann_batch_graph_launch", "gann_batch_graph_destroy", "gann_cache_hot_records", "gann_build_prune", "gann_nearest_pivots",
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


CLI = PKG / "search_mem"


def build_cli(verbose: bool = False, force: bool = False) -> Path:
    """Compile the search_mem driver (cli/search_mem.cpp) against libgann.so."""
    src = PKG / "cli" / "search_mem.cpp"
    deps = [src, LIB, ROOT / "include" / "gann.h", ROOT / "include" / "gustann.hpp"]
    if force or _stale(CLI, deps):
        cmd = ["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(src), "-o", str(CLI), "-L", str(PKG),
               "-lgann", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return CLI


def build_lib(verbose: bool = False, force: bool = False) -> Path:
    """Compile csrc/ into gustann_b200/libgann.so (incremental)."""
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    headers = _headers()
    objs = []
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
            if src.suffix == ".cpp":
                cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-x", "cu", "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    vscript = BUILD / "exports.map"
    vscript.write_text("{ global: " + " ".join(f"{s};" for s in EXPORTS) + " local: *; };\n")
    if force or _stale(LIB, objs + [vscript]):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
               "-Xlinker", f"--version-script={vscript}", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def build_oracle(verbose: bool = False, ref_dir: str | None = None) -> None:
    """Build the CPU oracle, and the reference's own path when its sources exist
    (checker only). The reference checkout is ``ref_dir`` or $GANN_REF_DIR;
    without either only the oracle is built."""
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    ref_dir = ref_dir or os.environ.get("GANN_REF_DIR")
    if not ref_dir:
        return
    ref = Path(ref_dir)
    out = ROOT / "oracle" / "_ref" / "libgustann_ref.so"
    script = ROOT / "oracle" / "build_ref.sh"
    if (ref / "src" / "pure_mem.cu").exists():
        deps = [script, ROOT / "oracle" / "ref_driver.cu"] + list((ROOT / "oracle" / "ref_shim").rglob("*.h"))
        if _stale(out, deps):
            subprocess.run(["bash", str(script), str(ref)], check=True,
                           stdout=None if verbose else subprocess.DEVNULL,
                           stderr=None if verbose else subprocess.DEVNULL)


if __name__ == "__main__":
    build_lib(verbose="-v" in sys.argv, force="-f" in sys.argv)
    build_cli(verbose="-v" in sys.argv, force="-f" in sys.argv)
    build_oracle(verbose="-v" in sys.argv, ref_dir=next((a for a in sys.argv[1:] if not a.startswith("-")), None))
    print(LIB)
