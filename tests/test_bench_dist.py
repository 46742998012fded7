"""bench.py's multi-rank plumbing on CPU: world size 2 over gloo. Each rank
times its own replica; the reported time is the max over ranks; ranks that do
not build the index wait for the builder's ready file; the reference arm runs
on rank 0 only."""
import json
import os
import socket
import sys
import tempfile
import time
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, tmp, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    dist = bench.init_dist(world, "gloo")
    ready = Path(tmp) / "ready.json"
    if rank == 0:
        time.sleep(0.5)
        ready.write_text("{}")
    else:
        bench.wait_for(ready, 30)
    bench.barrier(world)
    t = bench.max_over_ranks(10.0 * (rank + 1), world)
    results[rank] = t
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_and_ready_file_gloo():
    world = 2
    with tempfile.TemporaryDirectory() as tmp:
        mgr = mp.Manager()
        results = mgr.dict()
        mp.start_processes(_worker, args=(world, _free_port(), tmp, results), nprocs=world, start_method="spawn")
        assert dict(results) == {0: 20.0, 1: 20.0}


def test_single_rank_helpers_are_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5
    bench.barrier(1)
    assert bench.dist_env()[1] >= 1


def test_wait_for_times_out(tmp_path):
    sys.path.insert(0, str(ROOT))
    import bench

    with pytest.raises(TimeoutError):
        bench.wait_for(tmp_path / "never", 0.1)


def test_calibrate_finds_smallest_L():
    """calibrate_L(): walk the L ladder, then bisect to a step of 8, returning
    the smallest L whose recall reaches the target (host logic; both arms use
    it, so bit-exact forms land on the same L)."""
    sys.path.insert(0, str(ROOT))
    import bench

    for threshold in (37, 200, 384, 393, 1000):
        calls = []

        def recall_for(L):
            calls.append(L)
            return 0.96 if L >= threshold else 0.5

        L, rec = bench.calibrate_L(recall_for, 10, 0.95)
        assert rec >= 0.95 and L >= threshold and L - threshold < 8, (threshold, L, calls)
        assert L % 8 == 0 or L in bench.L_LADDER


def test_recall_measures_match_the_tooling():
    """bench.py's vectorised calc_recall / recall_unique equal the indexing
    package's loops (bin/utils.hpp:105-117 and its unique-id variant)."""
    import numpy as np

    sys.path.insert(0, str(ROOT))
    import bench
    from gustann_b200.indexing import groundtruth

    rng = np.random.default_rng(5)
    gt = rng.integers(0, 50, size=(40, 100)).astype(np.int32)
    ids = rng.integers(0, 50, size=(40, 10)).astype(np.int32)
    ids[:, 3] = ids[:, 2]  # repeated ids count twice in calc_recall, once in recall_unique
    for k in (1, 5, 10):
        assert bench.calc_recall(ids, gt, k) == groundtruth.recall(ids, gt, k)
        assert bench.recall_unique(ids, gt, k) == groundtruth.recall_unique(ids, gt, k)


def test_both_arms_state_the_same_config():
    sys.path.insert(0, str(ROOT))
    import bench

    meta = {"workload": "c2", "n": 100_000_000, "dim": 128, "kind": "u8", "R": 32, "M": 32, "nav": 1_000_000}
    a = bench.config_of(meta, 10_000, 10)
    b = bench.config_of(dict(meta), 10_000, 10)
    assert a == b and a["workload"] == "c2" and "l2" in a and a["queries_per_step"] == 10_000
