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


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [gb.PREC_BF16, gb.PREC_FP32])
def test_noalloc_matches_batch_device_on_two_calls(golden, precision):
    import torch

    meta = golden["u8_nav"]
    g = gb.GustANN(gb.DataType.UINT8)
    g.init_pure_mem(gb.GustANNConfig(meta["index_file"], meta["pq_prefix"], meta["nav_dir"]))
    k, L = 10, 48
    stream = torch.cuda.current_stream().cuda_stream
    opts = gb.GustANN._opts(precision, 4, 10)
    batches = [meta["queries"], np.ascontiguousarray(meta["queries"][:150][::-1])]
    for q in batches:  # two calls in a row, the second on the first call's leftovers
        nq = q.shape[0]
        dq = torch.from_numpy(q).cuda()

        def outs():
            return (torch.zeros((nq, k), dtype=torch.int32, device="cuda"),
                    torch.zeros((nq, k), dtype=torch.float32, device="cuda"),
                    torch.zeros(nq, dtype=torch.int32, device="cuda"))

        ref, got = outs(), outs()
        g.search_batch_device(dq.data_ptr(), nq, 0, 0, k, L, ref[0].data_ptr(), ref[1].data_ptr(),
                              ref[2].data_ptr(), precision=precision, beam_width=4, hash_bits=10, stream=stream)
        rc = gb.lib().gann_search_batch_noalloc(g.handle, dq.data_ptr(), nq, k, L, ctypes.byref(opts),
                                                got[0].data_ptr(), got[1].data_ptr(), got[2].data_ptr(),
                                                gb._stream(stream))
        assert rc == gb.GANN_OK, gb.lib().gann_last_error()
        g.check(stream)
        np.testing.assert_array_equal(got[0].cpu().numpy(), ref[0].cpu().numpy())
        np.testing.assert_allclose(got[1].cpu().numpy(), ref[1].cpu().numpy(), rtol=0, atol=0)
        np.testing.assert_array_equal(got[2].cpu().numpy(), ref[2].cpu().numpy())
        assert (got[2].cpu().numpy() == k).all()
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
    g.close()
