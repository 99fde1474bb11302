"""The allocation-free entry point, ipuma_gpu_compare_noalloc.

It serves callers that cannot call cudaMalloc: code running while its stream
is captured into a CUDA graph, hosts whose own pool owns all device memory,
latency-critical paths that cannot take the synchronisation cudaMalloc and
cudaFree imply.  Instead of an allocated buffer its kernel uses a fixed
16 MiB device array that every call shares, so the test runs two calls in a
row -- the second one over scratch still holding the first batch's strips --
and checks both, bit for bit, against the regular entry point
ipuma_gpu_compare_device on the same device buffers.
"""
import numpy as np
import pytest
import torch

import ipuma_b200 as ib
import workloads

pytestmark = pytest.mark.gpu


def _device_batch(wl):
    dev = torch.device("cuda", 0)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    d_codes = torch.from_numpy(wl.codes).to(dev)
    d_pairs = torch.from_numpy(pairs.view(np.uint8)).to(dev)
    return d_codes, d_pairs


def _check_against_engine(wl, forward_only):
    torch.cuda.set_device(0)
    sw = ib.sw_config(wl.gap_init, wl.gap_extend, wl.match, wl.mismatch, wl.ambiguity,
                      wl.similarity, wl.datatype)
    d_codes, d_pairs = _device_batch(wl)
    n = wl.n
    max_b = int(wl.b_len.max())
    want = torch.zeros(3, n, dtype=torch.int32, device="cuda")
    got = torch.full((3, n), -7, dtype=torch.int32, device="cuda")
    with ib.Engine(sw, ib.algo_config(forward_only=forward_only)) as e:
        e.compare_device(d_codes.data_ptr(), d_codes.numel(), d_pairs.data_ptr(), n,
                         int(wl.a_len.max()), max_b, want[0].data_ptr(), want[1].data_ptr(),
                         want[2].data_ptr())
    torch.cuda.synchronize()
    rc = ib.compare_noalloc(sw, forward_only, d_codes.data_ptr(), d_codes.numel(),
                            d_pairs.data_ptr(), n, max_b, got[0].data_ptr(), got[1].data_ptr(),
                            got[2].data_ptr())
    assert rc == ib.OK, ib.last_error()
    torch.cuda.synchronize()
    diff = (want != got).any(dim=0).nonzero()
    assert diff.numel() == 0, "noalloc differs from the engine on %d pairs" % diff.numel()


def test_two_calls_in_a_row_match_the_engine():
    # Protein pairs up to 2000 residues cross several 512-column strips, so
    # the first call fills the static scratch; the second call (other data,
    # other scoring) runs over what the first left behind.
    _check_against_engine(workloads.protein(n=600, seed=61), forward_only=False)
    _check_against_engine(workloads.dna_batched(n=4000, seed=62), forward_only=True)


def test_rejects_sizes_beyond_the_limit():
    torch.cuda.set_device(0)
    wl = workloads.dna_batched(n=64, seed=63)
    sw = ib.sw_config()
    d_codes, d_pairs = _device_batch(wl)
    out = torch.zeros(3, wl.n, dtype=torch.int32, device="cuda")
    args = (d_codes.data_ptr(), d_codes.numel(), d_pairs.data_ptr(), wl.n)
    outs = (out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr())
    rc = ib.compare_noalloc(sw, True, *args, 70_000, *outs)
    assert rc == ib.ERR_TOO_LONG and "65535" in ib.last_error()
    # a stated maximum below a real |B| is caught on the device
    rc = ib.compare_noalloc(sw, True, *args, int(wl.b_len.max()) - 1, *outs)
    assert rc == ib.ERR_TOO_LONG, ib.last_error()
    # and the entry point still works afterwards
    rc = ib.compare_noalloc(sw, True, *args, int(wl.b_len.max()), *outs)
    assert rc == ib.OK, ib.last_error()
