"""GPU parity of the chunked host-buffer path of ipuma_gpu_compare.

Large batches are split into chunks of consecutive pairs whose code ranges
upload while earlier chunks compute, on two alternating streams with their
own buffer sets.  Every case must give exactly the results of the one-upload
path (option "chunks" = 1) and of the oracle, whatever the layout of the
code array: pair-ordered (the overlapping case), shared or scattered
sequences (chunks then read ranges other chunks already uploaded).
"""
import numpy as np
import pytest

import ipuma_b200 as ib
import oracle
import workloads

pytestmark = pytest.mark.gpu


def _engine(wl, forward_only, **opts):
    sw = ib.sw_config(wl.gap_init, wl.gap_extend, wl.match, wl.mismatch, wl.ambiguity,
                      wl.similarity, wl.datatype)
    e = ib.Engine(sw, ib.algo_config(forward_only=forward_only))
    for k, v in opts.items():
        e.set_option(k, v)
    return e


def _oracle(wl, codes, pairs, forward_only, idx=None):
    if idx is not None:
        pairs = pairs[idx]
    sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
    return oracle.sw_batch(codes, pairs["a_off"], pairs["a_len"], pairs["b_off"], pairs["b_len"],
                           sim, wl.gap_init, wl.gap_extend, forward_only=forward_only)


def _same(got, want, label):
    for g, w, name in zip(got, want, ("score", "arange", "brange")):
        bad = np.nonzero(np.asarray(g) != np.asarray(w))[0]
        assert bad.size == 0, "%s %s: %d pairs differ, first %d" % (label, name, bad.size, bad[0])


def _run(wl, codes, pairs, forward_only, chunks):
    with _engine(wl, forward_only, chunks=chunks) as e:
        got = e.compare(codes, pairs)
        st = e.stats()
    return got, st


@pytest.mark.parametrize("forward_only", [True, False])
def test_chunked_equals_single_upload_and_oracle(forward_only):
    wl = workloads.dna_batched(n=9_000, seed=41)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    # empty pairs at and around chunk boundaries
    for p in (0, 1, 2999, 3000, 4499, 4500, 8999):
        pairs["a_len" if p % 2 else "b_len"][p] = 0
    want = _oracle(wl, wl.codes, pairs, forward_only)
    base, st1 = _run(wl, wl.codes, pairs, forward_only, 1)
    assert st1.chunks == 1
    _same(base, want, "single upload")
    for chunks in (2, 3, 8):
        got, st = _run(wl, wl.codes, pairs, forward_only, chunks)
        assert st.chunks == chunks
        _same(got, want, "chunks=%d" % chunks)


def test_chunked_with_scattered_and_shared_sequences():
    """Pair k aligns A of pair k against B of pair n-1-k and half the pairs
    reuse one sequence: every chunk reads ranges spread over the array."""
    wl = workloads.protein(n=3_000, seed=42)
    n = wl.n
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off[::-1].copy(), wl.b_len[::-1].copy())
    pairs["a_off"][::2] = wl.a_off[7]
    pairs["a_len"][::2] = wl.a_len[7]
    want = _oracle(wl, wl.codes, pairs, False)
    for chunks in (1, 4, 7):
        got, st = _run(wl, wl.codes, pairs, False, chunks)
        assert st.chunks == chunks
        _same(got, want, "scattered chunks=%d" % chunks)
    assert n == pairs.shape[0]


def test_chunked_overflow_reruns_are_summed():
    """s16x2 give-ups and s32 pairs land in several chunks; each chunk's
    rerun list and status are its own, and the call sums them."""
    wl = workloads.protein_mixed(n=1_200, seed=43, long_identical_frac=0.01)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    want = _oracle(wl, wl.codes, pairs, True)
    assert (want[0] > 32767).sum() >= 6
    got1, st1 = _run(wl, wl.codes, pairs, True, 1)
    got4, st4 = _run(wl, wl.codes, pairs, True, 4)
    _same(got1, want, "overflow single")
    _same(got4, want, "overflow chunks=4")
    assert st4.overflow_reruns == st1.overflow_reruns
    assert st4.cells == st1.cells


def test_chunked_into_pinned_buffers():
    """Pinned outputs take the per-chunk download path."""
    import torch
    wl = workloads.dna_batched(n=6_000, seed=44)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    h_codes = torch.from_numpy(wl.codes).pin_memory()
    h_pairs = torch.from_numpy(pairs.view(np.uint8)).pin_memory()
    h_out = torch.full((3, wl.n), -1, dtype=torch.int32).pin_memory()
    with _engine(wl, False, chunks=5) as e:
        for _ in range(2):
            h_out.fill_(-1)
            e.compare_into(h_codes.numpy(), h_pairs.numpy().view(ib.PAIR_DTYPE), h_out[0].numpy(),
                           h_out[1].numpy(), h_out[2].numpy())
            assert e.stats().chunks == 5
            out = h_out.numpy().copy()
            _same(tuple(out), _oracle(wl, wl.codes, pairs, False), "pinned")


def test_automatic_chunking_of_a_large_batch():
    """From 500,000 pairs and 32 MB of codes the call chunks by itself (one
    chunk per 333,334 pairs, at least 2); the pairs are checked on several host
    threads."""
    wl = workloads.dna_batched(n=520_000, seed=45)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    assert wl.codes.size >= 32 << 20
    auto, st = _run(wl, wl.codes, pairs, True, 0)
    assert st.chunks == 2
    single, st1 = _run(wl, wl.codes, pairs, True, 1)
    assert st1.chunks == 1
    _same(auto, single, "auto vs single")
    idx = np.random.default_rng(0).choice(wl.n, 2_000, replace=False)
    _same(tuple(a[idx] for a in auto), _oracle(wl, wl.codes, pairs, True, idx), "auto sample")


def test_bad_pair_deep_in_a_large_batch_is_reported():
    """The threaded host check reports the first pair outside the code array,
    whichever thread finds it, and the engine stays usable."""
    wl = workloads.dna_batched(n=400_000, seed=46)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    pairs["b_off"][301_234] = wl.codes.size - 3
    pairs["b_off"][350_000] = wl.codes.size + 10
    with _engine(wl, True) as e:
        with pytest.raises(ib.IpumaError) as ei:
            e.compare(wl.codes, pairs)
        assert ei.value.code == ib.ERR_INVALID_ARG
        assert "301234" in str(ei.value)
        small = pairs[:1000].copy()
        got = e.compare(wl.codes, small)
        _same(got, _oracle(wl, wl.codes, small, True), "after a rejected call")


def test_bad_pair_in_a_later_chunk_is_reported():
    """A pair outside the code array in a later chunk of a chunked call is
    reported by index, and the engine stays usable for the corrected batch."""
    wl = workloads.dna_batched(n=520_000, seed=47)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    pairs["a_off"][400_123] = wl.codes.size + 5
    with _engine(wl, True) as e:
        with pytest.raises(ib.IpumaError) as ei:
            e.compare(wl.codes, pairs)
        assert ei.value.code == ib.ERR_INVALID_ARG
        assert "400123" in str(ei.value)
        pairs["a_off"][400_123] = wl.a_off[400_123]
        got = e.compare(wl.codes, pairs)
        assert e.stats().chunks == 2
        idx = np.random.default_rng(1).choice(wl.n, 2_000, replace=False)
        _same(tuple(a[idx] for a in got), _oracle(wl, wl.codes, pairs, True, idx), "after a rejected call")
