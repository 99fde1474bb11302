"""GPU parity of the packed-code calls: codes packed as a bit stream of 2-bit
(A/C/G/T), 4-bit or 5-bit (amino acid) fields are uploaded (whole, or per
chunk of pairs) and read packed by the kernels; device-resident packed
codes go straight to ipuma_gpu_compare_device_packed.  Every result must
equal the byte-code call and the oracle, for sequences starting inside a
byte, ranges ending mid-byte, empty pairs, chunks whose code ranges
overlap, reverse passes, and every kernel class (wavefront classes, the
hybrid and s32 classes with their diagonal bound, the exact kernel)."""
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
    # 25 amino-acid codes need 5 bits: 4, 2 (and 3) are refused.
    wl = workloads.protein(n=100, seed=74)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    with _engine(wl, True) as e:
        for bits in (4, 2, 3):
            with pytest.raises(ib.IpumaError) as ei:
                e.compare_packed(np.zeros(wl.codes.size, np.uint8), wl.codes.size, pairs, bits=bits)
            assert ei.value.code == ib.ERR_INVALID_ARG
        _same(e.compare(wl.codes, pairs), _oracle(wl, wl.codes, pairs, True), "after rejection")


@pytest.mark.parametrize("forward_only", [True, False])
def test_protein_5bit_host_call_equals_bytes_and_oracle(forward_only):
    wl = workloads.protein(n=3_000, seed=75)
    codes = np.concatenate([[7], wl.codes, [1, 2, 3]]).astype(np.uint8)
    pairs = ib.make_pairs(wl.a_off + 1, wl.a_len, wl.b_off + 1, wl.b_len)
    pairs["a_len"][17] = 0
    packed = ib.pack_codes(codes, 5)
    want = _oracle(wl, codes, pairs, forward_only)
    for chunks in (1, 3):
        with _engine(wl, forward_only, chunks=chunks) as e:
            got = e.compare_packed(packed, codes.size, pairs, bits=5)
        _same(got, want, "5-bit chunks=%d" % chunks)


def _device_packed(wl, codes, pairs, bits, forward_only, graphs=0, reruns=None, routed=None, **opts):
    """compare_device_packed on a device copy of the packed codes (padded as
    the call requires) and compare_device on the byte codes; `reruns` and
    `routed`, when given, collect each call's count of s16x2 pairs rerun in
    s32 and of pairs the binning sent to the s32 / hybrid classes."""
    torch = pytest.importorskip("torch")
    packed = ib.pack_codes(codes, bits)
    buf = np.zeros(ib.device_packed_bytes(codes.size, bits), np.uint8)
    buf[:packed.size] = packed
    d_packed = torch.from_numpy(buf).cuda()
    d_bytes = torch.from_numpy(codes).cuda()
    d_pairs = torch.from_numpy(pairs.view(np.uint8)).cuda()
    n = pairs.shape[0]
    outs = []
    with _engine(wl, forward_only, graphs=graphs, **opts) as e:
        for call in ("packed", "bytes"):
            out = torch.full((3, n), -7, dtype=torch.int32, device="cuda")
            args = (pairs.shape[0], int(pairs["a_len"].max()), int(pairs["b_len"].max()),
                    out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr())
            if call == "packed":
                e.compare_device_packed(d_packed.data_ptr(), codes.size, bits, d_pairs.data_ptr(), *args)
            else:
                e.compare_device(d_bytes.data_ptr(), codes.size, d_pairs.data_ptr(), *args)
            torch.cuda.synchronize()
            outs.append(tuple(out.cpu().numpy()))
            if reruns is not None:
                reruns.append(int(e.stats().overflow_reruns))
            if routed is not None:
                routed.append(int(e.stats().s32_pairs))
    return outs


@pytest.mark.parametrize("bits,kind", [(2, "dna"), (4, "dna"), (5, "protein")])
@pytest.mark.parametrize("forward_only", [True, False])
def test_device_packed_equals_bytes_and_oracle(bits, kind, forward_only):
    wl = workloads.dna_batched(n=6_000, seed=76) if kind == "dna" else workloads.protein(n=2_000, seed=76)
    codes, pairs = (_odd_layout(wl) if kind == "dna" else
                    (np.concatenate([[5], wl.codes]).astype(np.uint8),
                     ib.make_pairs(wl.a_off + 1, wl.a_len, wl.b_off + 1, wl.b_len)))
    pairs["b_len"][3] = 0
    want = _oracle(wl, codes, pairs, forward_only)
    for graphs in (0, 1):
        got_p, got_b = _device_packed(wl, codes, pairs, bits, forward_only, graphs=graphs)
        _same(got_p, want, "device %d-bit graphs=%d" % (bits, graphs))
        _same(got_b, want, "device bytes graphs=%d" % graphs)


def test_device_packed_high_scores_hybrid_and_s32():
    # Near-identical long protein pairs (scores above int16, held by the
    # 16-bit lanes), plus W/C-rich pairs scoring above the 16-bit lanes'
    # range: the diagonal bound (read packed) sends those to the hybrid
    # class, which switches to s32 strips; with option hybrid 0 they run in
    # the s32 class.
    base = workloads.protein_mixed(n=1_200, seed=77, long_identical_frac=0.01)
    rng = np.random.default_rng(77)
    wc = np.array([oracle.encode("aa", "W")[0], oracle.encode("aa", "C")[0]], dtype=np.uint8)
    extra_a = [rng.choice(wc, n).astype(np.uint8) for n in (6800, 7100)]
    extra_b = [a.copy() for a in extra_a]
    codes = np.concatenate([base.codes] + extra_a + extra_b).astype(np.uint8)
    off = base.codes.size
    a_off = np.concatenate([base.a_off, [off, off + 6800]])
    b_off = np.concatenate([base.b_off, [off + 6800 + 7100, off + 2 * 6800 + 7100]])
    a_len = np.concatenate([base.a_len, [6800, 7100]])
    b_len = np.concatenate([base.b_len, [6800, 7100]])
    pairs = ib.make_pairs(a_off, a_len, b_off, b_len)
    want = _oracle(base, codes, pairs, True)
    assert want[0].max() > 65535 - 1024 - 11 and (want[0] > 32767).sum() >= 8
    for hybrid in (1, 0):
        reruns, routed = [], []
        got_p, got_b = _device_packed(base, codes, pairs, 5, True, hybrid=hybrid, reruns=reruns,
                                      routed=routed)
        _same(got_p, want, "5-bit high scores hybrid=%d" % hybrid)
        _same(got_b, want, "byte high scores hybrid=%d" % hybrid)
        # Every pair above the s16 limit has a diagonal bound above it (checked
        # on the CPU for this batch), so none starts in s16x2 lanes and has to
        # be rerun: the warp-parallel bound routed them all.
        assert reruns == [0, 0], reruns
        # A diagonal bound never exceeds the score, so the routed pairs are
        # exactly those above the limit here (all of them caught).
        above = int((want[0] > 32767 - 11).sum())
        assert routed == [above, above], (routed, above)


def test_device_packed_exact_kernel_for_unusual_gaps():
    # gap extend > 0 runs the exact per-thread kernel, which reads packed
    # codes through the same accessor.
    wl = workloads.dna_batched(n=400, seed=78)
    wl.gap_init, wl.gap_extend = -1, 1
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    for fwd in (True, False):
        got_p, got_b = _device_packed(wl, wl.codes, pairs, 2, fwd)
        want = _oracle(wl, wl.codes, pairs, fwd)
        _same(got_p, want, "exact packed fwd=%s" % fwd)
        _same(got_b, want, "exact bytes fwd=%s" % fwd)


def test_device_packed_rejects_bad_requests():
    torch = pytest.importorskip("torch")
    wl = workloads.dna_batched(n=50, seed=79)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    d = torch.zeros(ib.device_packed_bytes(wl.codes.size, 2) + 8, dtype=torch.uint8, device="cuda")
    d_pairs = torch.from_numpy(pairs.view(np.uint8)).cuda()
    out = torch.zeros((3, wl.n), dtype=torch.int32, device="cuda")
    args = (d_pairs.data_ptr(), wl.n, 250, 1000, out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr())
    with _engine(wl, True) as e:
        for bits, ptr in ((3, d.data_ptr()), (8, d.data_ptr()), (2, d.data_ptr() + 1)):
            with pytest.raises(ib.IpumaError) as ei:
                e.compare_device_packed(ptr, wl.codes.size, bits, *args)
            assert ei.value.code == ib.ERR_INVALID_ARG
        # the per-thread class reads bytes only
        e.set_option("tile_k", 7)
        with pytest.raises(ib.IpumaError):
            e.compare_device_packed(d.data_ptr(), wl.codes.size, 2, *args)
