"""Continuous-batching server: results equal the batched entry point's and are
the same for a request alone and inside a stream of others; admission refuses
work beyond the budget; an open-loop Poisson run reports latencies."""
import time

import numpy as np
import pytest

import gustann_b200 as gb
from gustann_b200.indexing import build_index, groundtruth, synth


@pytest.fixture(scope="module")
def index(tmp_path_factory):
    d = tmp_path_factory.mktemp("srv")
    base, qs = synth.make("u8", 100_000, 128, 100, 1000, backend="torch", device="cuda")
    f = build_index(base, str(d), R=32, M=32, nav_samples=1000, device="cuda")
    g = gb.GustANN(gb.DataType.UINT8)
    g.init_pure_mem(gb.GustANNConfig(f.index_file, f.pq_prefix, f.nav_dir))
    return g, qs.float().cpu().numpy()


def collect(srv, n, timeout=30.0):
    out = {}
    t0 = time.time()
    while len(out) < n and time.time() - t0 < timeout:
        tags, ids, dis, fnd, lat = srv.poll()
        for t, i, d, f, l in zip(tags, ids, dis, fnd, lat):
            out[int(t)] = (i.copy(), d.copy(), int(f), float(l))
        if len(out) < n:
            time.sleep(0.001)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [gb.PREC_BF16, gb.PREC_FP32])
def test_server_same_alone_and_in_the_mix(index, precision):
    g, q = index
    L, k = synth.draws(len(q), [32, 64, 128, 256], [1, 10, 100])
    opts = dict(max_batch=64, streams=3, topk_max=100, ef_max=256, precision=precision, beam_width=4, hash_bits=10)
    srv = gb.Server(g, **opts)
    probe = 17
    assert srv.submit(q[probe], int(k[probe]), int(L[probe]), tag=10**6)
    alone = collect(srv, 1)[10**6]
    n = 600
    res = {}

    def drain():
        tags, ids, dis, fnd, lat = srv.poll()
        for t, i_, d, f, l_ in zip(tags, ids, dis, fnd, lat):
            res[int(t)] = (i_.copy(), d.copy(), int(f), float(l_))

    t0 = time.time()
    for i in range(n):  # the probe again, in the middle of a stream of other requests
        # finished results count against the budget until polled, so poll while waiting
        while not srv.submit(q[i], int(k[i]), int(L[i]), tag=i):
            drain()
            assert time.time() - t0 < 60, "server made no progress"
            time.sleep(0.0005)
    while len(res) < n and time.time() - t0 < 60:
        drain()
        time.sleep(0.001)
    srv.stop()
    assert len(res) == n
    mixed = res[probe]
    np.testing.assert_array_equal(mixed[0], alone[0])
    np.testing.assert_array_equal(mixed[1].view(np.uint32), alone[1].view(np.uint32))
    # every request equals the batched entry point with the same limits and options
    ids, dis, fnd, _ = g.search_batch(q[:n], k[:n], L[:n], precision=precision, beam_width=4, hash_bits=10)
    for i in range(n):
        kk = int(k[i])
        assert res[i][2] == fnd[i]
        np.testing.assert_array_equal(res[i][0][:kk], ids[i, :kk])
        np.testing.assert_array_equal(res[i][1][:kk].view(np.uint32), dis[i, :kk].view(np.uint32))


@pytest.mark.gpu
def test_server_admission_refuses_beyond_budget(index):
    g, q = index
    srv = gb.Server(g, max_batch=4, streams=1, topk_max=10, ef_max=256, max_wait_us=100000, min_batch=4)
    accepted = sum(srv.submit(q[i], 10, 256, tag=i) for i in range(64))
    assert 0 < accepted <= 8  # budget = max_batch * (streams + 1)
    got = collect(srv, accepted)
    assert len(got) == accepted
    assert srv.submit(q[0], 10, 256, tag=99)  # room again once results are polled
    srv.stop()
    with pytest.raises(gb.GustANNError):
        gb.Server(g, max_batch=0, streams=-1)


@pytest.mark.gpu
def test_server_open_loop_reports_latency(index):
    g, q = index
    srv = gb.Server(g, max_batch=256, streams=4, topk_max=10, ef_max=128, precision=gb.PREC_BF16)
    st = srv.open_loop(q, rate_qps=20000, seconds=0.5, topk=np.full(len(q), 10, np.int32),
                       ef_search=np.full(len(q), 64, np.int32))
    srv.stop()
    assert st["submitted"] > 5000 and st["rejected"] == 0
    assert st["completed"] == st["submitted"]
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["p999_ms"] < 1000


@pytest.mark.gpu
def test_admission_by_bytes_refuses_long_lists_before_short_ones(index):
    """With the byte budget nearly full, a request with a long list (large
    ef_search, large topk) is refused while a short one still enters; every
    admitted request is charged gann_server_request_bytes. Nothing is launched
    during the test (a batch waits for max_batch requests or a minute)."""
    g, q = index
    opts = dict(max_batch=64, streams=2, topk_max=100, ef_max=512, precision=gb.PREC_BF16X3,
                max_wait_us=60_000_000, min_batch=64)
    srv = gb.Server(g, **opts)
    big, small = srv.request_bytes(100, 512), srv.request_bytes(1, 32)
    srv.stop()
    assert big - small > 2048 and small > 0
    cap = (2 * big + small + (big - small) // 2) // 1024 * 1024  # two long requests, then room for short ones only
    srv = gb.Server(g, mem_budget_kib=cap // 1024, **opts)
    assert [srv.submit(q[i], 100, 512, i) for i in range(4)] == [True, True, False, False]
    n_small = (cap - 2 * big) // small
    assert n_small >= 1
    took = [srv.submit(q[10 + i], 1, 32, 10 + i) for i in range(n_small + 2)]
    assert took == [True] * n_small + [False, False]
    assert not srv.submit(q[50], 100, 512, 50)
    srv.stop()
