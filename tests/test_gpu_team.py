"""Strip teams (k_strips<16>): the warps of a block share one item's strips.

Every case calls through the C ABI and compares score, end coordinates
and (with the reverse pass) start coordinates of every pair with the
oracle.  Option tile_k = 24 forces every s16x2 pair into the team class;
without it the cost model picks teams for long pairs of small batches.
"""
import time

import numpy as np
import pytest

import ipuma_b200 as ib
import oracle

pytestmark = pytest.mark.gpu

TEAM_TILE_K = 24          # tile_k value of the strip-team class
KIND_TEAM = 27            # IPUMA_KERNEL_S16_TEAM
PROTEIN = {"similarity": "blosum62", "match": 1, "mismatch": -1, "ambiguity": -1,
           "datatype": "aa", "gapInit": -11, "gapExtend": -1}
DNA = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1,
       "datatype": "na", "gapInit": -1, "gapExtend": -1}


def _engine(case, forward_only=True, **opts):
    sw = ib.sw_config(case["gapInit"], case["gapExtend"], case["match"], case["mismatch"],
                      case["ambiguity"], case["similarity"], case["datatype"])
    e = ib.Engine(sw, ib.algo_config(forward_only=forward_only))
    for k, v in opts.items():
        e.set_option(k, v)
    return e


def _oracle(case, codes, pairs, forward_only=True):
    sim = oracle.select_matrix(case["similarity"], case["match"], case["mismatch"],
                               case["ambiguity"])
    return oracle.sw_batch(codes, pairs["a_off"], pairs["a_len"], pairs["b_off"], pairs["b_len"],
                           sim, case["gapInit"], case["gapExtend"], forward_only=forward_only)


def _assert_same(got, want, label=""):
    for g, w, name in zip(got, want, ("score", "arange", "brange")):
        g = np.asarray(g)
        w = np.asarray(w)
        bad = np.nonzero(g != w)[0]
        assert bad.size == 0, "%s %s: %d pairs differ, first %d: %d vs %d" % (
            label, name, bad.size, bad[0], g[bad[0]], w[bad[0]])


def _mutate(rng, src, letters, sub_rate, indel_rate):
    """A copy of src with substitutions and single-residue indels."""
    out = []
    for x in src:
        r = rng.random()
        if r < indel_rate / 2:
            continue                                   # deletion
        if r < indel_rate:
            out.append(int(rng.integers(0, letters)))  # insertion before x
        out.append(int(rng.integers(0, letters)) if rng.random() < sub_rate else int(x))
    return np.array(out, dtype=np.uint8)


def _long_pairs(rng, n, letters, a_lo, a_hi, b_lo, b_hi, related=0.5):
    """n pairs with |A| in [a_lo, a_hi), |B| in [b_lo, b_hi): related pairs
    take B from a window of A (mutated), so their best cell can lie in any
    strip; the others are unrelated."""
    a_list, b_list = [], []
    for _ in range(n):
        a = rng.integers(0, letters, int(rng.integers(a_lo, a_hi))).astype(np.uint8)
        blen = int(rng.integers(b_lo, b_hi))
        if rng.random() < related and blen < a.size:
            start = int(rng.integers(0, a.size - blen))
            b = _mutate(rng, a[start:start + blen], letters, 0.15, 0.03)
        else:
            b = rng.integers(0, letters, blen).astype(np.uint8)
        a_list.append(a)
        b_list.append(b if b.size else np.zeros(1, dtype=np.uint8))
    return a_list, b_list


@pytest.mark.parametrize("forward_only", [True, False])
@pytest.mark.parametrize("warps", [2, 3, 8])
def test_forced_team_protein_parity(warps, forward_only):
    """Every pair through strip teams of 2, 3 and 8 warps: ragged couples
    (the two pairs of an item differ in both lengths), pairs of one strip
    (the other warps idle), an odd pair count (the last item holds one
    pair), and a repeat whose two equal maxima lie in different strips
    (the first in row-major order must win); forward pass alone and with
    the reverse pass."""
    rng = np.random.default_rng(700 + warps)
    a_list, b_list = _long_pairs(rng, 36, 20, 513, 3800, 40, 1400)
    short_a, short_b = _long_pairs(rng, 4, 20, 100, 512, 100, 600)
    a_list += short_a
    b_list += short_b
    s = rng.integers(0, 20, 700).astype(np.uint8)
    x = rng.integers(0, 20, 300).astype(np.uint8)
    a_list.append(np.concatenate([s, x, s]))
    b_list.append(s.copy())
    codes, a_off, a_len, b_off, b_len = oracle.pack_pairs(a_list, b_list)
    pairs = ib.make_pairs(a_off, a_len, b_off, b_len)
    assert pairs.shape[0] % 2 == 1
    with _engine(PROTEIN, forward_only, tile_k=TEAM_TILE_K, team_warps=warps) as e:
        got = e.compare(codes, pairs)
    want = _oracle(PROTEIN, codes, pairs, forward_only)
    _assert_same(got, want, "team of %d, forward_only=%s" % (warps, forward_only))
    # The repeat: equal maxima in columns 699 and 1699; the first one wins.
    assert got[0][-1] == want[0][-1] and (got[1][-1] >> 16) == 699


@pytest.mark.parametrize("forward_only", [True, False])
def test_forced_team_dna_bytes_and_2bit(forward_only):
    """DNA through teams of 8: byte codes (16-letter profile) and 2-bit
    packed codes (four-row profile)."""
    rng = np.random.default_rng(711)
    a_list, b_list = _long_pairs(rng, 30, 4, 600, 5000, 200, 2500, related=0.7)
    a_list = [x + 1 for x in a_list]  # A, C, G, T = codes 1..4
    b_list = [x + 1 for x in b_list]
    codes, a_off, a_len, b_off, b_len = oracle.pack_pairs(a_list, b_list)
    pairs = ib.make_pairs(a_off, a_len, b_off, b_len)
    want = _oracle(DNA, codes, pairs, forward_only)
    with _engine(DNA, forward_only, tile_k=TEAM_TILE_K, team_warps=8) as e:
        _assert_same(e.compare(codes, pairs), want, "dna bytes")
        packed = ib.pack_codes(codes, 2)
        _assert_same(e.compare_packed(packed, codes.size, pairs, bits=2), want, "dna 2-bit")


@pytest.mark.parametrize("forward_only", [True, False])
def test_team_overflow_goes_to_the_s32_rerun(forward_only):
    """A near-identical pair shifted by 500 residues: its main diagonal is
    unrelated (no diagonal bound sends it to 32 bits), so it runs in a
    team, passes int16 there, and the s32 rerun gives the exact result."""
    rng = np.random.default_rng(712)
    s = rng.integers(0, 20, 7000).astype(np.uint8)
    a = np.concatenate([rng.integers(0, 20, 500).astype(np.uint8), s])
    b = np.concatenate([s, rng.integers(0, 20, 300).astype(np.uint8)])
    a2, b2 = _long_pairs(rng, 3, 20, 3500, 4000, 1000, 2000)
    codes, a_off, a_len, b_off, b_len = oracle.pack_pairs([a] + a2, [b] + b2)
    pairs = ib.make_pairs(a_off, a_len, b_off, b_len)
    want = _oracle(PROTEIN, codes, pairs, forward_only)
    assert want[0][0] > 32767
    with _engine(PROTEIN, forward_only, team_warps=8, time_launches=1) as e:
        got = e.compare(codes, pairs)
        st = e.stats()
    _assert_same(got, want, "team overflow")
    assert st.overflow_reruns >= 1
    kinds = [st.timed_kind[k] for k in range(st.n_timed)]
    assert KIND_TEAM in kinds


def test_cost_model_picks_teams_for_a_small_batch_of_long_pairs():
    """Without forcing: a batch of twelve long pairs, whose one-warp
    latency is most of the batch's time, runs in teams, with and without
    start coordinates; with team_warps 0 it does not."""
    rng = np.random.default_rng(713)
    a_list, b_list = _long_pairs(rng, 12, 20, 3200, 6000, 2000, 5000)
    codes, a_off, a_len, b_off, b_len = oracle.pack_pairs(a_list, b_list)
    pairs = ib.make_pairs(a_off, a_len, b_off, b_len)
    for fwd, warps in ((True, 8), (False, 8), (True, 0)):
        with _engine(PROTEIN, fwd, time_launches=1, team_warps=warps) as e:
            got = e.compare(codes, pairs)
            st = e.stats()
        _assert_same(got, _oracle(PROTEIN, codes, pairs, fwd), "auto fwd=%s warps=%d" % (fwd, warps))
        team = [st.timed_cells[k] for k in range(st.n_timed) if st.timed_kind[k] == KIND_TEAM]
        if warps:
            assert team and sum(team) == int((pairs["a_len"].astype(np.int64) * pairs["b_len"]).sum())
        else:
            assert not team


def test_team_options_are_checked():
    with _engine(PROTEIN) as e:
        for bad in (1, 9, -1):
            with pytest.raises(ib.IpumaError):
                e.set_option("team_warps", bad)
        e.set_option("team_warps", 0)
        e.set_option("team_warps", 4)
        for bad in (22, 23, 25):
            with pytest.raises(ib.IpumaError):
                e.set_option("tile_k", bad)
        e.set_option("tile_k", TEAM_TILE_K)


def test_teams_shorten_a_small_batch_of_long_pairs():
    """64 unrelated 6000 x 6000 protein pairs (32 items: far fewer than the
    GPU's warps): teams of 8 against one warp per item."""
    rng = np.random.default_rng(714)
    a_list = [rng.integers(0, 20, 6000).astype(np.uint8) for _ in range(64)]
    b_list = [rng.integers(0, 20, 6000).astype(np.uint8) for _ in range(64)]
    codes, a_off, a_len, b_off, b_len = oracle.pack_pairs(a_list, b_list)
    pairs = ib.make_pairs(a_off, a_len, b_off, b_len)
    ms = {}
    res = {}
    for w in (0, 8):
        with _engine(PROTEIN, team_warps=w) as e:
            e.compare(codes, pairs)  # warm-up (autotuning, buffers)
            t = []
            for _ in range(3):
                t0 = time.perf_counter()
                res[w] = e.compare(codes, pairs)
                t.append(time.perf_counter() - t0)
            ms[w] = 1e3 * min(t)
    for g, w in zip(res[0], res[8]):
        assert np.array_equal(g, w)
    print("64 pairs 6000 x 6000: one warp %.1f ms, teams of 8 %.1f ms" % (ms[0], ms[8]))
    assert ms[8] * 2.0 < ms[0]


def test_forced_team_on_short_pairs_and_without_warps():
    """tile_k 24 on a batch of one-strip pairs runs teams of two (one warp
    idles); with team_warps 0 the forced class has no warps and the call is
    refused."""
    rng = np.random.default_rng(715)
    a_list, b_list = _long_pairs(rng, 9, 20, 30, 512, 30, 400)
    codes, a_off, a_len, b_off, b_len = oracle.pack_pairs(a_list, b_list)
    pairs = ib.make_pairs(a_off, a_len, b_off, b_len)
    with _engine(PROTEIN, False, tile_k=TEAM_TILE_K, time_launches=1) as e:
        got = e.compare(codes, pairs)
        st = e.stats()
    _assert_same(got, _oracle(PROTEIN, codes, pairs, False), "short pairs in teams")
    assert KIND_TEAM in [st.timed_kind[k] for k in range(st.n_timed)]
    with _engine(PROTEIN, tile_k=TEAM_TILE_K, team_warps=0) as e:
        with pytest.raises(ib.IpumaError):
            e.compare(codes, pairs)
