"""GPU parity: the CUDA engine against the CPU oracle, bit-exact.

Every case calls through the C ABI (ipuma_gpu_compare / ipuma_gpu_run_buffer)
and compares score, A range and B range of every pair with the oracle
(oracle/sw_oracle.c, pinned to the reference by tests/test_oracle_golden.py)
or with the reference codelet's own answers stored in tests/golden/.
"""
import json
import os

import numpy as np
import pytest

import ipuma_b200 as ib
import oracle
import workloads

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _engine(case, forward_only=False, **opts):
    sw = ib.sw_config(case["gapInit"], case["gapExtend"], case["match"], case["mismatch"],
                      case["ambiguity"], case["similarity"], case["datatype"])
    e = ib.Engine(sw, ib.algo_config(forward_only=forward_only))
    for k, v in opts.items():
        e.set_option(k, v)
    return e


def _pack(case):
    a = [oracle.encode(case["datatype"], s) for s in case["A"]]
    b = [oracle.encode(case["datatype"], s) for s in case["B"]]
    return oracle.pack_pairs(a, b)


def _gpu(case, forward_only=False, **opts):
    codes, a_off, a_len, b_off, b_len = _pack(case)
    with _engine(case, forward_only, **opts) as e:
        return e.compare(codes, ib.make_pairs(a_off, a_len, b_off, b_len))


def _oracle(case, forward_only=False):
    sim = oracle.select_matrix(case["similarity"], case["match"], case["mismatch"],
                               case["ambiguity"])
    return oracle.sw_batch(*_pack(case), sim, case["gapInit"], case["gapExtend"],
                           forward_only=forward_only)


def _assert_same(got, want, label=""):
    for g, w, name in zip(got, want, ("score", "arange", "brange")):
        g = np.asarray(g)
        w = np.asarray(w)
        bad = np.nonzero(g != w)[0]
        assert bad.size == 0, "%s %s: %d pairs differ, first %d: %d vs %d" % (
            label, name, bad.size, bad[0], g[bad[0]], w[bad[0]])


def _wl_case(wl):
    return {"similarity": wl.similarity, "match": wl.match, "mismatch": wl.mismatch,
            "ambiguity": wl.ambiguity, "datatype": wl.datatype, "gapInit": wl.gap_init,
            "gapExtend": wl.gap_extend}


def _wl_run(wl, forward_only=False, **opts):
    case = _wl_case(wl)
    with _engine(case, forward_only, **opts) as e:
        got = e.compare(wl.codes, ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len))
        stats = e.stats()
    sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
    want = oracle.sw_batch(wl.codes, wl.a_off, wl.a_len, wl.b_off, wl.b_len, sim, wl.gap_init,
                           wl.gap_extend, forward_only=forward_only)
    return got, want, stats


# ---------------------------------------------------------------- golden ---

@pytest.mark.parametrize("forward_only", [False, True])
def test_simple_known_answers(forward_only):
    known = json.load(open(os.path.join(GOLD, "known_answers.json")))["simple"]
    case = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1, "datatype": "na",
            "gapInit": 0, "gapExtend": -1, "A": [k["query"] for k in known],
            "B": [k["ref"] for k in known]}
    score, ar, br = _gpu(case, forward_only)
    qb, qe = oracle.unpack_range(ar)
    rb, re_ = oracle.unpack_range(br)
    for i, k in enumerate(known):
        assert score[i] == k["score"], i
        assert (qe[i], re_[i]) == (k["qend"], k["rend"]), i
        if not forward_only:
            assert (qb[i], rb[i]) == (k["qstart"], k["rstart"]), i


def test_mn_known_answers():
    mn = json.load(open(os.path.join(GOLD, "known_answers.json")))["mn"]
    case = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1, "datatype": "na",
            "gapInit": 0, "gapExtend": -1, "A": [mn["seqs"][c[0]] for c in mn["comparisons"]],
            "B": [mn["seqs"][c[1]] for c in mn["comparisons"]]}
    assert _gpu(case)[0].tolist() == mn["scores"]


@pytest.mark.parametrize("fixture", ["parity_ref.json", "random_ref.json"])
@pytest.mark.parametrize("forward_only", [False, True])
def test_reference_codelet_answers(fixture, forward_only):
    for case in json.load(open(os.path.join(GOLD, fixture)))["cases"]:
        key = "fwd_" if forward_only else ""
        want = (case["ref"][key + "score"], case["ref"][key + "arange"],
                case["ref"][key + "brange"])
        _assert_same(_gpu(case, forward_only), want, case["name"])


@pytest.mark.parametrize("tile_k", list(range(1, 22)))
def test_random_answers_each_tile_width(tile_k):
    """Forces every pair through one s16x2 kernel class (16 or 32 lanes per
    group, 4..16 columns per lane -- widths that are not whole words use
    word-padded profile rows -- or 7: one thread per two pairs with
    16-column strips), so that long pairs cross several strips (global
    scratch hand-over)."""
    for case in json.load(open(os.path.join(GOLD, "random_ref.json")))["cases"]:
        want = (case["ref"]["score"], case["ref"]["arange"], case["ref"]["brange"])
        _assert_same(_gpu(case, False, tile_k=tile_k), want, "%s class=%d" % (case["name"], tile_k))
        fwd = (case["ref"]["fwd_score"], case["ref"]["fwd_arange"], case["ref"]["fwd_brange"])
        _assert_same(_gpu(case, True, tile_k=tile_k), fwd, "%s class=%d fwd" % (case["name"], tile_k))


# ------------------------------------------------------- workload shapes ---

def test_dna_plain_workload_all_pairs():
    wl = workloads.dna_plain()
    got, want, st = _wl_run(wl, forward_only=True)
    _assert_same(got, want, wl.name)
    assert st.cells == wl.cells


@pytest.mark.parametrize("forward_only", [True, False])
def test_dna_batched_workload_sample(forward_only):
    wl = workloads.dna_batched(n=20_000, seed=11)
    got, want, _ = _wl_run(wl, forward_only)
    _assert_same(got, want, wl.name)


@pytest.mark.parametrize("forward_only", [True, False])
def test_protein_workload_sample(forward_only):
    wl = workloads.protein(n=4_000, seed=12)
    got, want, _ = _wl_run(wl, forward_only)
    _assert_same(got, want, wl.name)


def test_protein_mixed_with_s16_overflow():
    """Heavy-tailed protein lengths plus near-identical 7000+ residue pairs
    whose scores exceed int16: they must come back exact (the hybrid
    class's biased 16-bit halves hold them)."""
    wl = workloads.protein_mixed(n=1_500, seed=13, long_identical_frac=0.004)
    got, want, st = _wl_run(wl, forward_only=False)
    _assert_same(got, want, wl.name)
    assert (want[0] > 32767).sum() >= 3


# Largest score the hybrid class's biased 16-bit halves hold (BLOSUM62).
U16_LIMIT = 65535 - 1024 - 11


def test_s16_rerun_of_unpredicted_overflow():
    """A pair whose main diagonal looks unrelated (so it is not routed to
    the hybrid class up front) but whose gapped score exceeds int16 (and
    the biased halves' range): the s16x2 kernel gives up on the device and
    the pair is rerun in 32-bit."""
    rng = np.random.default_rng(5)
    w, c = oracle.encode("aa", "W")[0], oracle.encode("aa", "C")[0]
    a = np.where(rng.random(7000) < 0.5, w, c).astype(np.uint8)
    b = np.concatenate([[oracle.encode("aa", "A")[0]], a]).astype(np.uint8)
    short = a[:1000]
    codes = np.concatenate([a, b, short, short])
    pairs = ib.make_pairs([0, a.size + b.size], [a.size, 1000],
                          [a.size, a.size + b.size + 1000], [b.size, 1000])
    case = {"similarity": "blosum62", "match": 1, "mismatch": -1, "ambiguity": -1,
            "datatype": "aa", "gapInit": -10, "gapExtend": -1}
    for fwd in (False, True):
        with _engine(case, fwd) as e:
            got = e.compare(codes, pairs)
            st = e.stats()
        sim = oracle.select_matrix("blosum62")
        want = oracle.sw_batch(codes, pairs["a_off"], pairs["a_len"], pairs["b_off"],
                               pairs["b_len"], sim, -10, -1, forward_only=fwd)
        _assert_same(got, want, "overflow fwd=%s" % fwd)
        assert want[0][0] > U16_LIMIT
        assert st.overflow_reruns >= 1


# ----------------------------------------------- per-thread class (7) ---

THREAD_CLASS = 7


@pytest.mark.parametrize("forward_only", [True, False])
def test_thread_class_dna_and_protein_samples(forward_only):
    """Every pair through the per-thread class: two pairs per thread with
    different lengths, boundary columns in global scratch across strips."""
    for wl in (workloads.dna_batched(n=3_000, seed=61), workloads.protein(n=2_000, seed=62)):
        got, want, _ = _wl_run(wl, forward_only, tile_k=THREAD_CLASS)
        _assert_same(got, want, "%s thread class" % wl.name)


def test_thread_class_edges_ties_and_strip_boundaries():
    rng = np.random.default_rng(63)
    A, B = [], []
    for la in [1, 2, 15, 16, 17, 31, 32, 33, 47, 48, 49, 255, 256, 257]:
        for lb in [1, 2, 3, 4, 5, 7, 8, 9, 63, 64, 65, 300]:
            a = "".join(rng.choice(list("ACGT"), la))
            b = a[: max(1, lb // 2)] + "".join(rng.choice(list("ACGT"), max(0, lb - lb // 2)))
            A.append(a)
            B.append(b[:lb])
    A += ["", "A", "AAAA", "ACGT" * 100, "T" * 700, "ACACACACAC", "GATTACA" * 9, "A" * 300]
    B += ["A", "", "AAAA", "ACGT" * 100, "A" * 700, "ACACAC" * 5, "GATTACA" * 20, "A" * 77]
    case = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1, "datatype": "na",
            "gapInit": 0, "gapExtend": -1, "A": A, "B": B}
    for fwd in (False, True):
        _assert_same(_gpu(case, fwd, tile_k=THREAD_CLASS), _oracle(case, fwd),
                     "thread edges fwd=%s" % fwd)


def test_thread_class_s16_overflow_goes_to_s32_rerun():
    """A pair passing the s16 limit inside the per-thread class is rerun
    in 32-bit lanes; its partner in the other halfword is unaffected."""
    rng = np.random.default_rng(64)
    w, c = oracle.encode("aa", "W")[0], oracle.encode("aa", "C")[0]
    a = np.where(rng.random(3500) < 0.5, w, c).astype(np.uint8)
    b = np.concatenate([[oracle.encode("aa", "A")[0]], a]).astype(np.uint8)
    others = workloads.protein(n=63, seed=65)
    codes = np.concatenate([a, b, others.codes])
    base = a.size + b.size
    pairs = ib.make_pairs(np.concatenate([[0], base + others.a_off]),
                          np.concatenate([[a.size], others.a_len]),
                          np.concatenate([[a.size], base + others.b_off]),
                          np.concatenate([[b.size], others.b_len]))
    case = {"similarity": "blosum62", "match": 1, "mismatch": -1, "ambiguity": -1,
            "datatype": "aa", "gapInit": -10, "gapExtend": -1}
    sim = oracle.select_matrix("blosum62")
    for fwd in (False, True):
        with _engine(case, fwd, tile_k=THREAD_CLASS) as e:
            got = e.compare(codes, pairs)
            st = e.stats()
        want = oracle.sw_batch(codes, pairs["a_off"], pairs["a_len"], pairs["b_off"],
                               pairs["b_len"], sim, -10, -1, forward_only=fwd)
        _assert_same(got, want, "thread overflow fwd=%s" % fwd)
        assert want[0][0] > 32767
        assert st.overflow_reruns >= 1


def test_thread_class_chosen_automatically_for_large_batches():
    """With the class enabled (option thread_class) a large batch sends part
    of its pairs to it; results equal the run with the class disabled.  (Its
    items are long, so the latency share is widened to let it qualify.)"""
    wl = workloads.dna_batched(n=120_000, seed=66)
    case = _wl_case(wl)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    outs = []
    for on in (1, 0):
        with _engine(case, True, thread_class=on, time_launches=1, latency_share=500) as e:
            outs.append(e.compare(wl.codes, pairs))
            st = e.stats()
            kinds = {st.timed_kind[k]: st.timed_cells[k] for k in range(st.n_timed)}
        assert (kinds.get(10, 0) > 0) == bool(on)
    _assert_same(outs[0], outs[1], "thread class on/off")
    idx = np.random.default_rng(1).choice(wl.n, 2_000, replace=False)
    sim = oracle.select_matrix(wl.similarity)
    want = oracle.sw_batch(wl.codes, wl.a_off[idx], wl.a_len[idx], wl.b_off[idx], wl.b_len[idx],
                           sim, wl.gap_init, wl.gap_extend, forward_only=True)
    _assert_same(tuple(o[idx] for o in outs[0]), want, "thread class sample")


# ------------------------------------------------------- hybrid class ---

HYBRID_KIND = 20


def _mutated(rng, seq, rate, alphabet):
    out = seq.copy()
    hit = rng.random(seq.size) < rate
    out[hit] = rng.choice(alphabet, hit.sum())
    return out


@pytest.mark.parametrize("forward_only", [True, False])
def test_hybrid_class_for_scores_above_int16(forward_only):
    """Near-identical long protein pairs of different lengths, in warps with
    short pairs; their main diagonal sends them to the hybrid class.
    Ordinary near-identical pairs (scores between int16 and the biased
    halves' range) run every strip in biased 16-bit halves; pairs rich in W
    and C score above that range, so their strips run in biased halves
    while the strip bound holds, then each pair continues in s32.  Same
    results with the hybrid class on and off, equal to the oracle."""
    rng = np.random.default_rng(71)
    alpha = np.arange(20, dtype=np.uint8)
    wc = np.array([oracle.encode("aa", "W")[0], oracle.encode("aa", "C")[0]], dtype=np.uint8)
    seqs_a, seqs_b = [], []
    for la, al in ((7000, wc), (6900, wc), (7300, wc), (6500, alpha), (7200, alpha), (3600, alpha)):
        a = rng.choice(al, la).astype(np.uint8)
        seqs_a.append(a)
        seqs_b.append(_mutated(rng, a[: la - int(rng.integers(0, 300))], 0.01, al))
    for la in (40, 300, 900):
        a = rng.choice(alpha, la).astype(np.uint8)
        seqs_a.append(a)
        seqs_b.append(_mutated(rng, a, 0.3, alpha))
    codes, a_off, a_len, b_off, b_len = oracle.pack_pairs(seqs_a, seqs_b)
    pairs = ib.make_pairs(a_off, a_len, b_off, b_len)
    case = {"similarity": "blosum62", "match": 1, "mismatch": -1, "ambiguity": -1,
            "datatype": "aa", "gapInit": -10, "gapExtend": -1}
    sim = oracle.select_matrix("blosum62")
    want = oracle.sw_batch(codes, a_off, a_len, b_off, b_len, sim, -10, -1,
                           forward_only=forward_only)
    assert (want[0] > U16_LIMIT).sum() >= 3 and ((want[0] > 32767) & (want[0] <= U16_LIMIT)).sum() >= 2
    for hyb in (1, 0):
        with _engine(case, forward_only, hybrid=hyb, time_launches=1) as e:
            got = e.compare(codes, pairs)
            st = e.stats()
            kinds = {st.timed_kind[k]: st.timed_cells[k] for k in range(st.n_timed)}
        _assert_same(got, want, "hybrid=%d fwd=%s" % (hyb, forward_only))
        assert (kinds.get(HYBRID_KIND, 0) > 0) == bool(hyb)


def test_hybrid_class_switches_at_the_first_strip():
    """DNA scored +50/-40: long identical pairs score above the biased
    halves' range, so once the strip bound fails (after two strips) they
    switch to s32, and short ones never leave 16-bit lanes."""
    rng = np.random.default_rng(72)
    acgt = np.array([1, 2, 3, 4], dtype=np.uint8)
    seqs_a, seqs_b = [], []
    for la in (2100, 1800, 1300, 900, 520, 511):
        a = rng.choice(acgt, la).astype(np.uint8)
        seqs_a.append(a)
        seqs_b.append(_mutated(rng, a, 0.002, acgt))
    codes, a_off, a_len, b_off, b_len = oracle.pack_pairs(seqs_a, seqs_b)
    pairs = ib.make_pairs(a_off, a_len, b_off, b_len)
    case = {"similarity": "na", "match": 50, "mismatch": -40, "ambiguity": -40,
            "datatype": "na", "gapInit": 0, "gapExtend": -1}
    sim = oracle.select_matrix("na", 50, -40, -40)
    for fwd in (True, False):
        want = oracle.sw_batch(codes, a_off, a_len, b_off, b_len, sim, 0, -1, forward_only=fwd)
        assert (want[0] > 65535 - 1024 - 50).sum() >= 3
        for hyb in (1, 0):
            with _engine(case, fwd, hybrid=hyb) as e:
                got = e.compare(codes, pairs)
            _assert_same(got, want, "dna +50 hybrid=%d fwd=%s" % (hyb, fwd))


# ------------------------------------------------- concurrent classes ---

@pytest.mark.parametrize("forward_only", [True, False])
def test_concurrent_class_launches_equal_sequential(forward_only):
    """Classes launched concurrently on shares of the SMs (default) give the
    results of one-after-the-other launches, with s32 pairs, s16x2 give-ups
    rerun after all classes, and multi-strip pairs in several classes at
    once (each with its own scratch region)."""
    wl = workloads.protein_mixed(n=2_500, seed=67, long_identical_frac=0.004)
    outs, reruns = [], []
    for conc in (1, 0):
        got, want, st = _wl_run(wl, forward_only, concurrent=conc)
        _assert_same(got, want, "%s concurrent=%d" % (wl.name, conc))
        outs.append(got)
        reruns.append(st.overflow_reruns)
    assert reruns[0] == reruns[1]


# --------------------------------------------------------------- edges ---

def test_edge_lengths_and_strip_boundaries():
    rng = np.random.default_rng(21)
    A, B = [], []
    for la in [1, 2, 3, 31, 32, 33, 95, 96, 97, 127, 128, 129, 159, 160, 161, 223, 224, 225, 255, 256,
               257, 511, 512, 513, 1023, 1024, 1025]:
        for lb in [1, 2, 17, 63, 64, 65, 300]:
            a = "".join(rng.choice(list("ACGT"), la))
            b = a[: max(1, lb // 2)] + "".join(rng.choice(list("ACGT"), max(0, lb - lb // 2)))
            A.append(a)
            B.append(b[:lb])
    A += ["", "A", "AAAA", "ACGT" * 100, "T" * 700]
    B += ["A", "", "AAAA", "ACGT" * 100, "A" * 700]
    case = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1, "datatype": "na",
            "gapInit": 0, "gapExtend": -1, "A": A, "B": B}
    for fwd in (False, True):
        _assert_same(_gpu(case, fwd), _oracle(case, fwd), "edges fwd=%s" % fwd)


def test_ties_pick_first_cell_in_row_major_order():
    """Repeats give many equal maxima; the reference keeps the first one in
    (B index, A index) order and, in reverse, the last."""
    A = ["ACACACACAC", "AAAA", "GATTACA" * 9, "A" * 300]
    B = ["ACACAC" * 5, "AAAAAAAA", "GATTACA" * 20, "A" * 77]
    case = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1, "datatype": "na",
            "gapInit": 0, "gapExtend": -1, "A": A, "B": B}
    _assert_same(_gpu(case), _oracle(case), "ties")


@pytest.mark.parametrize("gap_init,gap_extend", [(0, 0), (2, -1), (-1, 1)])
def test_unusual_gap_configs_use_exact_path(gap_init, gap_extend):
    rng = np.random.default_rng(31)
    A = ["".join(rng.choice(list("ACGT"), n)) for n in rng.integers(1, 200, 40)]
    B = [a[::2] + "".join(rng.choice(list("ACGT"), 20)) for a in A]
    case = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1, "datatype": "na",
            "gapInit": gap_init, "gapExtend": gap_extend, "A": A, "B": B}
    _assert_same(_gpu(case), _oracle(case), "gaps %d/%d" % (gap_init, gap_extend))


def test_rejects_pairs_outside_code_array():
    case = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1, "datatype": "na",
            "gapInit": 0, "gapExtend": -1}
    with _engine(case) as e:
        with pytest.raises(ib.IpumaError) as ei:
            e.compare(np.zeros(10, np.uint8), ib.make_pairs([0], [5], [8], [5]))
        assert ei.value.code == ib.ERR_INVALID_ARG
        # the engine stays usable after a rejected call
        s, _, _ = e.compare(np.array([1, 2, 3, 4, 1, 2, 3, 4], np.uint8),
                            ib.make_pairs([0], [4], [4], [4]))
        assert s[0] == 4


@pytest.mark.parametrize("graphs", [0, 1])
def test_device_call_rejects_pairs_outside_code_array(graphs):
    # Device-resident descriptors are checked on the device before any code
    # is read.  The codes live in a valid, larger allocation; the pairs reach
    # past the n_codes residues the caller declares, or carry a negative
    # field.  The rejected pairs get a zero result, the others their real
    # one, and the call reports IPUMA_ERR_INVALID_ARG.
    import torch
    wl = workloads.dna_batched(n=300, seed=71)
    case = _wl_case(wl)
    pairs = ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len)
    last = int(np.argmax(pairs["b_off"] + pairs["b_len"]))
    declared = int(pairs["b_off"][last] + pairs["b_len"][last]) - 1
    bad = pairs.copy()
    bad["a_len"][7] = -3
    bad["b_off"][11] = -1
    sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
    want = oracle.sw_batch(wl.codes, wl.a_off, wl.a_len, wl.b_off, wl.b_len, sim, wl.gap_init,
                           wl.gap_extend, forward_only=True)
    d_codes = torch.from_numpy(wl.codes).cuda()
    with _engine(case, True, graphs=graphs) as e:
        for desc, n_codes, rejected in ((pairs, declared, [last]), (bad, wl.codes.size, [7, 11])):
            d_pairs = torch.from_numpy(desc.view(np.uint8)).cuda()
            out = torch.full((3, wl.n), -7, dtype=torch.int32, device="cuda")
            with pytest.raises(ib.IpumaError) as ei:
                e.compare_device(d_codes.data_ptr(), n_codes, d_pairs.data_ptr(), wl.n,
                                 int(wl.a_len.max()), int(wl.b_len.max()), out[0].data_ptr(),
                                 out[1].data_ptr(), out[2].data_ptr())
            assert ei.value.code == ib.ERR_INVALID_ARG and "outside" in str(ei.value)
            got = out.cpu().numpy()
            keep = np.setdiff1d(np.arange(wl.n), rejected)
            assert (got[:, rejected] == 0).all()
            for k in range(3):
                assert np.array_equal(got[k][keep], want[k][keep])
        # and a valid call on the same engine is exact
        d_pairs = torch.from_numpy(pairs.view(np.uint8)).cuda()
        out = torch.zeros((3, wl.n), dtype=torch.int32, device="cuda")
        e.compare_device(d_codes.data_ptr(), wl.codes.size, d_pairs.data_ptr(), wl.n,
                         int(wl.a_len.max()), int(wl.b_len.max()), out[0].data_ptr(),
                         out[1].data_ptr(), out[2].data_ptr())
        _assert_same(out.cpu().numpy(), want, "device call after rejections")


@pytest.mark.parametrize("tile_k", [1, 4])
def test_reverse_early_stop_over_several_strips(tile_k):
    # Full alignments whose A spans several strips of a narrow class (64 or
    # 256 columns): the reverse pass of each pair runs over [0..Aend] x
    # [0..Bend], so the two pairs of a 16-lane group get very different
    # reverse lengths; one finds its target (the forward score) and stops
    # early while the other runs out of rows.  Mixed related and unrelated
    # pairs, local alignments anywhere in the matrix.
    rng = np.random.default_rng(72 + tile_k)
    A, B = [], []
    for _ in range(600):
        a = "".join(rng.choice(list("ACGT"), int(rng.integers(100, 700))))
        if rng.random() < 0.7:
            lo = int(rng.integers(0, len(a) - 50))
            hi = int(rng.integers(lo + 30, min(len(a), lo + 400)))
            core = list(a[lo:hi])
            for k in range(len(core)):
                if rng.random() < 0.08:
                    core[k] = rng.choice(list("ACGT"))
            b = ("".join(rng.choice(list("ACGT"), int(rng.integers(0, 300)))) + "".join(core) +
                 "".join(rng.choice(list("ACGT"), int(rng.integers(0, 300)))))
        else:
            b = "".join(rng.choice(list("ACGT"), int(rng.integers(50, 900))))
        A.append(a)
        B.append(b)
    case = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1, "datatype": "na",
            "gapInit": 0, "gapExtend": -1, "A": A, "B": B}
    _assert_same(_gpu(case, forward_only=False, tile_k=tile_k), _oracle(case), "tile_k %d" % tile_k)


# ------------------------------------------------------- wire buffer ---

def _wire(wl, tiles, max_batches, bufsize):
    """Lays pairs out in the reference wire format, `max_batches` per tile."""
    algo = ib.algo_config(tiles_used=tiles, max_batches=max_batches, bufsize=bufsize)
    words = ib.input_buffer_words(algo)
    inputs = np.zeros(words, dtype=np.int32)
    seq = inputs.view(np.uint8)
    tile_bytes = ((bufsize + 3) // 4) * 4
    meta = inputs[tiles * ((bufsize + 3) // 4):].reshape(tiles, max_batches, 4)
    slot_of = np.full(wl.n, -1)
    t = s = used = 0
    for p in range(wl.n):
        need = int(wl.a_len[p] + wl.b_len[p])
        if s == max_batches or used + need > bufsize:
            t, s, used = t + 1, 0, 0
        assert t < tiles
        a, b = wl.seqs(p)
        base = t * tile_bytes
        seq[base + used: base + used + a.size] = a
        seq[base + used + a.size: base + used + need] = b
        meta[t, s] = (a.size, used, b.size, used + a.size)
        slot_of[p] = t * max_batches + s
        used += need
        s += 1
    return algo, inputs, slot_of


@pytest.mark.parametrize("scheduler", [0, 1])
@pytest.mark.parametrize("forward_only", [False, True])
def test_wire_buffer_matches_reference_codelet(scheduler, forward_only):
    wl = workloads.dna_batched(n=3_000, seed=41)
    algo, inputs, slot_of = _wire(wl, tiles=40, max_batches=80, bufsize=80_000)
    algo.forward_only = int(forward_only)
    case = _wl_case(wl)
    sw = ib.sw_config(case["gapInit"], case["gapExtend"], case["match"], case["mismatch"],
                      case["ambiguity"], case["similarity"], case["datatype"])
    with ib.Engine(sw, algo) as e:
        e.set_option("scheduler", scheduler)
        res = e.run_buffer(inputs)
    total = algo.tiles_used * algo.max_batches
    sim = oracle.select_matrix("na", 1, -1, -1)
    if oracle.have_ref():
        want = oracle.ref_codelet_run_buffer(inputs, algo.tiles_used, algo.max_batches,
                                             algo.bufsize, 300, sim, 0, -1, forward_only)
        np.testing.assert_array_equal(res[slot_of], want[slot_of])
        np.testing.assert_array_equal(res[total + slot_of], want[total + slot_of])
        np.testing.assert_array_equal(res[2 * total + slot_of], want[2 * total + slot_of])
    w = oracle.sw_batch(wl.codes, wl.a_off, wl.a_len, wl.b_off, wl.b_len, sim, 0, -1,
                        forward_only=forward_only)
    _assert_same((res[slot_of], res[total + slot_of], res[2 * total + slot_of]), w, "wire")


def test_async_jobs_poll_and_join():
    wl = workloads.dna_batched(n=800, seed=51)
    algo, inputs, slot_of = _wire(wl, tiles=10, max_batches=80, bufsize=60_000)
    sw = ib.sw_config()
    total = algo.tiles_used * algo.max_batches
    with ib.Engine(sw, algo) as e:
        outs = [np.zeros(3 * total, np.int32) for _ in range(3)]
        jobs = [e.submit_buffer(inputs, o) for o in outs]
        assert e.poll(jobs[0]) in (True, False)
        for j in jobs:
            e.join(j, timeout_ms=60_000)
        with pytest.raises(ib.IpumaError) as ei:
            e.join(12345)
        assert ei.value.code == ib.ERR_UNKNOWN_JOB
    sim = oracle.select_matrix("na", 1, -1, -1)
    w = oracle.sw_batch(wl.codes, wl.a_off, wl.a_len, wl.b_off, wl.b_len, sim, 0, -1)
    for o in outs:
        _assert_same((o[slot_of], o[total + slot_of], o[2 * total + slot_of]), w, "async")


# ------------------------------------------------------------- graphs ---

def test_graph_replay_matches_direct_launches():
    """Option "graphs": the binning + kernel pipeline is captured once and
    replayed for repeated shapes; results must equal direct launches."""
    import torch
    wl = workloads.protein(n=1500, seed=71)
    case = _wl_case(wl)
    dev = torch.device("cuda", 0)
    d_codes = torch.from_numpy(wl.codes).to(dev)
    d_pairs = torch.from_numpy(ib.make_pairs(wl.a_off, wl.a_len, wl.b_off, wl.b_len).view(np.uint8)).to(dev)
    outs = []
    for graphs in (0, 1, 1):
        out = torch.full((3, wl.n), -1, dtype=torch.int32, device=dev)
        with _engine(case, False, graphs=graphs) as e:
            for _ in range(2 if graphs else 1):
                e.compare_device(d_codes.data_ptr(), d_codes.numel(), d_pairs.data_ptr(), wl.n,
                                 int(wl.a_len.max()), int(wl.b_len.max()), out[0].data_ptr(),
                                 out[1].data_ptr(), out[2].data_ptr())
                assert e.stats().used_graph == graphs
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])
    sim = oracle.select_matrix(wl.similarity)
    want = oracle.sw_batch(wl.codes, wl.a_off, wl.a_len, wl.b_off, wl.b_len, sim, wl.gap_init,
                           wl.gap_extend)
    _assert_same(tuple(outs[1]), want, "graphs")
