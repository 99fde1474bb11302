"""GPU parity of ipuma_gpu_compare_packed: codes packed two (4-bit) or
four (2-bit, A/C/G/T) per byte are uploaded (whole, or per chunk of pairs)
and expanded on the device; every result must equal ipuma_gpu_compare on
the byte codes and the oracle, for sequences starting inside a byte,
ranges ending mid-byte, empty pairs, and chunks whose code ranges
overlap."""
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


def _oracle(wl, codes, pairs, forward_only):
    sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
    return oracle.sw_batch(codes, pairs["a_off"], pairs["a_len"], pairs["b_off"], pairs["b_len"],
                           sim, wl.gap_init, wl.gap_extend, forward_only=forward_only)


def _same(got, want, label):
    for g, w, name in zip(got, want, ("score", "arange", "brange")):
        bad = np.nonzero(np.asarray(g) != np.asarray(w))[0]
        assert bad.size == 0, "%s %s: %d pairs differ, first %d" % (label, name, bad.size, bad[0])


def _odd_layout(wl):
    """The workload's codes behind one extra residue (every sequence starts
    at the other nibble) and with an odd total length."""
    codes = np.concatenate([[3], wl.codes, [1, 2] if wl.codes.size % 2 == 0 else [1]]).astype(np.uint8)
    assert codes.size % 2 == 1
    pairs = ib.make_pairs(wl.a_off + 1, wl.a_len, wl.b_off + 1, wl.b_len)
    return codes, pairs


@pytest.mark.parametrize("bits", [4, 2])
@pytest.mark.parametrize("forward_only", [True, False])
def test_packed_equals_bytes_and_oracle(forward_only, bits):
    wl = workloads.dna_batched(n=9_000, seed=71)
    for shift in (0, 1):
        if shift:
            codes, pairs = _odd_layout(wl)
        else:
            codes, pairs = wl.codes, ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
        for p in (0, 4499, 4500, 8999):
            pairs["a_len" if p % 2 else "b_len"][p] = 0
        packed = ib.pack_codes(codes, bits)
        want = _oracle(wl, codes, pairs, forward_only)
        for chunks in (1, 3, 8):
            with _engine(wl, forward_only, chunks=chunks) as e:
                got_b = e.compare(codes, pairs)
                got_p = e.compare_packed(packed, codes.size, pairs, bits=bits)
                assert e.stats().chunks == chunks
            _same(got_b, want, "bytes shift=%d chunks=%d" % (shift, chunks))
            _same(got_p, want, "packed shift=%d chunks=%d" % (shift, chunks))


@pytest.mark.parametrize("bits", [4, 2])
def test_packed_with_scattered_and_shared_sequences(bits):
    """Chunks read ranges other chunks already uploaded, ranges that share a
    packed byte with their neighbours, and single residues."""
    wl = workloads.dna_batched(n=4_000, seed=72)
    codes, _ = _odd_layout(wl)
    rng = np.random.default_rng(72)
    n = wl.n
    a_off = wl.a_off[rng.permutation(n)] + 1
    b_off = wl.b_off[::-1].copy() + 1
    a_len = wl.a_len[rng.permutation(n)].copy()
    b_len = wl.b_len[::-1].copy()
    # keep every pair inside the array; some single-residue sequences
    a_len = np.minimum(a_len, codes.size - a_off).astype(np.int32)
    b_len = np.minimum(b_len, codes.size - b_off).astype(np.int32)
    a_len[::97] = 1
    b_len[5::101] = 1
    pairs = ib.make_pairs(a_off, a_len, b_off, b_len)
    packed = ib.pack_codes(codes, bits)
    want = _oracle(wl, codes, pairs, False)
    for chunks in (1, 4, 7):
        with _engine(wl, False, chunks=chunks) as e:
            got = e.compare_packed(packed, codes.size, pairs, bits=bits)
        _same(got, want, "scattered chunks=%d" % chunks)


@pytest.mark.parametrize("bits", [4, 2])
def test_packed_automatic_chunks_into_pinned_buffers(bits):
    torch = pytest.importorskip("torch")
    wl = workloads.dna_batched(n=520_000, seed=73)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    h_packed = torch.empty((wl.codes.size * bits + 7) // 8, dtype=torch.uint8).pin_memory()
    ib.pack_codes(wl.codes, bits, h_packed.numpy())
    h_pairs = torch.from_numpy(pairs.view(np.uint8)).pin_memory()
    h_out = torch.full((3, wl.n), -1, dtype=torch.int32).pin_memory()
    with _engine(wl, True) as e:
        e.compare_packed_into(h_packed.numpy(), wl.codes.size, h_pairs.numpy().view(ib.PAIR_DTYPE),
                              h_out[0].numpy(), h_out[1].numpy(), h_out[2].numpy(), bits=bits)
        assert e.stats().chunks == 2
        ref = e.compare(wl.codes, pairs)
    _same(tuple(h_out.numpy()), ref, "packed auto vs bytes")
    idx = np.random.default_rng(0).choice(wl.n, 2_000, replace=False)
    _same(tuple(a[idx] for a in h_out.numpy()), _oracle(wl, wl.codes, pairs[idx], True), "packed sample")


def test_packed_needs_a_small_alphabet():
    wl = workloads.protein(n=100, seed=74)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    with _engine(wl, True) as e:
        for bits in (4, 2, 3):
            with pytest.raises(ib.IpumaError) as ei:
                e.compare_packed(np.zeros(wl.codes.size, np.uint8), wl.codes.size, pairs, bits=bits)
            assert ei.value.code == ib.ERR_INVALID_ARG
        _same(e.compare(wl.codes, pairs), _oracle(wl, wl.codes, pairs, True), "after rejection")
