"""gann_search_batch_noalloc: the batched search for callers that cannot
allocate device memory while they search -- a serving loop that must not stall
on cudaMalloc (it can synchronise the device and takes the driver's allocation
lock) or a host program whose memory manager owns all device memory after
start-up. Its scratch lives in a fixed array inside the library.

Checked through the C ABI against gann_search_batch_device (which allocates its
table buffer itself) on the same inputs, on two calls in a row with different
batches, so the second call runs on the scratch the first one left behind.
Collected last so that a stop at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

import gustann_b200 as gb


def _two_calls(g, meta, precision, opts, beam_width, hash_bits):
    """Two no-alloc calls in a row, the second on the first call's leftovers,
    each compared with gann_search_batch_device on the same batch."""
    import torch

    k, L = 10, 48
    stream = torch.cuda.current_stream().cuda_stream
    batches = [meta["queries"], np.ascontiguousarray(meta["queries"][:150][::-1])]
    for q in batches:
        nq = q.shape[0]
        dq = torch.from_numpy(q).cuda()

        def outs():
            return (torch.zeros((nq, k), dtype=torch.int32, device="cuda"),
                    torch.zeros((nq, k), dtype=torch.float32, device="cuda"),
                    torch.zeros(nq, dtype=torch.int32, device="cuda"))

        ref, got = outs(), outs()
        g.search_batch_device(dq.data_ptr(), nq, 0, 0, k, L, ref[0].data_ptr(), ref[1].data_ptr(),
                              ref[2].data_ptr(), precision=precision, beam_width=beam_width, hash_bits=hash_bits,
                              stream=stream)
        rc = gb.lib().gann_search_batch_noalloc(g.handle, dq.data_ptr(), nq, k, L,
                                                None if opts is None else ctypes.byref(opts),
                                                got[0].data_ptr(), got[1].data_ptr(), got[2].data_ptr(),
                                                gb._stream(stream))
        assert rc == gb.GANN_OK, gb.lib().gann_last_error()
        g.check(stream)
        np.testing.assert_array_equal(got[0].cpu().numpy(), ref[0].cpu().numpy())
        np.testing.assert_allclose(got[1].cpu().numpy(), ref[1].cpu().numpy(), rtol=0, atol=0)
        np.testing.assert_array_equal(got[2].cpu().numpy(), ref[2].cpu().numpy())
        assert (got[2].cpu().numpy() == k).all()


def _open(meta):
    g = gb.GustANN(gb.DataType.UINT8)
    g.init_pure_mem(gb.GustANNConfig(meta["index_file"], meta["pq_prefix"], meta["nav_dir"]))
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [gb.PREC_BF16, gb.PREC_BF16X3, gb.PREC_BF16_CC, gb.PREC_FP32])
def test_noalloc_matches_batch_device_on_two_calls(golden, precision):
    meta = golden["u8_nav"]
    g = _open(meta)
    _two_calls(g, meta, precision, gb.GustANN._opts(precision, 4, 10), 4, 10)
    g.close()


@pytest.mark.gpu
def test_noalloc_defaults_follow_the_autotuned_handle(golden):
    """opts NULL (and zeroed beam width / cache size) take the handle's tuned
    defaults, as gann_search_batch_device does."""
    import torch

    meta = golden["u8_nav"]
    g = _open(meta)
    dq = torch.from_numpy(meta["queries"]).cuda()
    g.autotune(dq.data_ptr(), dq.shape[0], 10, 48, gb.PREC_BF16)
    _two_calls(g, meta, gb.PREC_BF16X3, None, 0, 0)  # opts NULL: split-BF16 tensor-core tables
    _two_calls(g, meta, gb.PREC_BF16, gb.GustANN._opts(gb.PREC_BF16, 0, 0), 0, 0)
    g.close()


@pytest.mark.gpu
def test_noalloc_rejects_more_than_its_scratch_holds(golden):
    import torch

    meta = golden["u8_nav"]
    g = gb.GustANN(gb.DataType.UINT8)
    g.init_pure_mem(gb.GustANNConfig(meta["index_file"], meta["pq_prefix"], meta["nav_dir"]))
    nq = 513
    dq = torch.zeros((nq, 128), dtype=torch.float32, device="cuda")
    out_i = torch.zeros((nq, 10), dtype=torch.int32, device="cuda")
    out_d = torch.zeros((nq, 10), dtype=torch.float32, device="cuda")
    out_f = torch.zeros(nq, dtype=torch.int32, device="cuda")
    rc = gb.lib().gann_search_batch_noalloc(g.handle, dq.data_ptr(), nq, 10, 48, None, out_i.data_ptr(),
                                            out_d.data_ptr(), out_f.data_ptr(), None)
    assert rc == gb.GANN_ERANGE
    assert "512" in gb.lib().gann_last_error().decode()
    # FP32 tables never touch the table region: any batch size is taken
    opts = gb.GustANN._opts(gb.PREC_FP32, 4, 10)
    rc = gb.lib().gann_search_batch_noalloc(g.handle, dq.data_ptr(), nq, 10, 48, ctypes.byref(opts),
                                            out_i.data_ptr(), out_d.data_ptr(), out_f.data_ptr(), None)
    assert rc == gb.GANN_OK, gb.lib().gann_last_error()
    g.check()
    g.close()
