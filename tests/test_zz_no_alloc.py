"""The allocation-free entry point, ipuma_gpu_compare_noalloc.

It serves callers that cannot call cudaMalloc: host programs whose own
memory pool owns all device memory, and latency-critical paths that cannot
take the synchronisation cudaMalloc and cudaFree imply.  Instead of an
allocated buffer its kernel uses a fixed 16 MiB device array that every call
shares, so the test runs two calls in a row -- the second one over scratch
still holding the first batch's strips -- and checks both, bit for bit,
against the regular entry point ipuma_gpu_compare_device on the same device
buffers and against the oracle.
"""
import numpy as np
import pytest
import torch

import ipuma_b200 as ib
import oracle
import workloads

pytestmark = pytest.mark.gpu


def _device_batch(wl, pairs=None):
    dev = torch.device("cuda", 0)
    if pairs is None:
        pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    d_codes = torch.from_numpy(wl.codes).to(dev)
    d_pairs = torch.from_numpy(pairs.view(np.uint8)).to(dev)
    return d_codes, d_pairs


def _check_against_engine_and_oracle(wl, forward_only):
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
    sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
    ref = oracle.sw_batch(wl.codes, wl.a_off, wl.a_len, wl.b_off, wl.b_len, sim, wl.gap_init,
                          wl.gap_extend, forward_only=forward_only)
    g = got.cpu().numpy()
    for k, name in enumerate(("score", "arange", "brange")):
        bad = np.nonzero(g[k] != ref[k])[0]
        assert bad.size == 0, "%s differs from the oracle on %d pairs" % (name, bad.size)


def test_two_calls_in_a_row_match_the_engine_and_the_oracle():
    # Protein pairs up to 2000 residues cross several 512-column strips, so
    # the first call fills the static scratch; the second call (other data,
    # other scoring) runs over what the first left behind.
    _check_against_engine_and_oracle(workloads.protein(n=600, seed=61), forward_only=False)
    _check_against_engine_and_oracle(workloads.dna_batched(n=4000, seed=62), forward_only=True)


def _call(sw, d_codes, n_codes, d_pairs, n, max_b, out):
    return ib.compare_noalloc(sw, True, d_codes.data_ptr(), n_codes, d_pairs.data_ptr(), n, max_b,
                              out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr())


def test_rejects_sizes_beyond_the_limit():
    torch.cuda.set_device(0)
    wl = workloads.dna_batched(n=64, seed=63)
    sw = ib.sw_config()
    d_codes, d_pairs = _device_batch(wl)
    out = torch.zeros(3, wl.n, dtype=torch.int32, device="cuda")
    nc = d_codes.numel()
    rc = _call(sw, d_codes, nc, d_pairs, wl.n, 70_000, out)
    assert rc == ib.ERR_TOO_LONG and "65535" in ib.last_error()
    # a stated maximum below a real |B| is caught on the device
    rc = _call(sw, d_codes, nc, d_pairs, wl.n, int(wl.b_len.max()) - 1, out)
    assert rc == ib.ERR_TOO_LONG, ib.last_error()
    # and the entry point still works afterwards
    rc = _call(sw, d_codes, nc, d_pairs, wl.n, int(wl.b_len.max()), out)
    assert rc == ib.OK, ib.last_error()


def test_rejects_a_longer_than_65535():
    # Ranges are uint16: an A of 70,000 residues is refused on the device
    # before any code is read; the short pair beside it is still aligned.
    torch.cuda.set_device(0)
    rng = np.random.default_rng(64)
    codes = rng.integers(1, 5, 70_000 + 300, dtype=np.uint8)
    pairs = ib.make_pairs(np.array([0, 0]), np.array([70_000, 200]), np.array([70_000, 70_000]),
                          np.array([300, 300]))
    d_codes = torch.from_numpy(codes).cuda()
    d_pairs = torch.from_numpy(pairs.view(np.uint8)).cuda()
    out = torch.full((3, 2), -7, dtype=torch.int32, device="cuda")
    rc = _call(ib.sw_config(), d_codes, codes.size, d_pairs, 2, 300, out)
    assert rc == ib.ERR_TOO_LONG, ib.last_error()
    o = out.cpu().numpy()
    assert (o[:, 0] == 0).all()
    sim = oracle.select_matrix("na")
    ref = oracle.sw_batch(codes, pairs["a_off"][1:], pairs["a_len"][1:], pairs["b_off"][1:],
                          pairs["b_len"][1:], sim, 0, -1, forward_only=True)
    assert [int(r[0]) for r in ref] == [int(x) for x in o[:, 1]]


def test_rejects_pairs_outside_the_code_array():
    # The descriptors point inside a valid, larger allocation, but past the
    # n_codes residues the caller declares: the device check fires before
    # any read, so nothing reads past the declared array.
    torch.cuda.set_device(0)
    wl = workloads.dna_batched(n=32, seed=65)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    d_codes, d_pairs = _device_batch(wl, pairs)
    out = torch.full((3, wl.n), -7, dtype=torch.int32, device="cuda")
    last = int(np.argmax(pairs["b_off"] + pairs["b_len"]))
    declared = int(pairs["b_off"][last] + pairs["b_len"][last]) - 1
    rc = _call(ib.sw_config(), d_codes, declared, d_pairs, wl.n, int(wl.b_len.max()), out)
    assert rc == ib.ERR_INVALID_ARG and "outside" in ib.last_error()
    assert (out[:, last] == 0).all()
    # a negative length is refused the same way
    bad = pairs.copy()
    bad["b_len"][3] = -5
    d_codes, d_pairs = _device_batch(wl, bad)
    rc = _call(ib.sw_config(), d_codes, d_codes.numel(), d_pairs, wl.n, int(wl.b_len.max()), out)
    assert rc == ib.ERR_INVALID_ARG, ib.last_error()
    assert (out[:, 3] == 0).all()
    # the full, valid batch still aligns afterwards
    d_codes, d_pairs = _device_batch(wl, pairs)
    rc = _call(ib.sw_config(), d_codes, d_codes.numel(), d_pairs, wl.n, int(wl.b_len.max()), out)
    assert rc == ib.OK, ib.last_error()
