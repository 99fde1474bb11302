"""Pins the CPU oracle against the reference's golden vectors.

* known answers: test/simple-test.cpp:25-45 (score, query/ref start/end) and
  test/mn_cmp-test.cpp:29-57 (M x N scores);
* the reference codelet itself, compiled for the host, on the parity-test
  pairs and on seeded random pairs (fixtures made by tests/golden/make_golden.py);
* the reference's SSW on the parity-test pairs (score and end coordinates).
"""
import json
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def _run_case(case, forward_only=False):
    sim = oracle.select_matrix(case["similarity"], case["match"], case["mismatch"],
                               case["ambiguity"])
    a = [oracle.encode(case["datatype"], s) for s in case["A"]]
    b = [oracle.encode(case["datatype"], s) for s in case["B"]]
    packed = oracle.pack_pairs(a, b)
    return oracle.sw_batch(*packed, sim, case["gapInit"], case["gapExtend"],
                           forward_only=forward_only)


def test_simple_known_answers():
    known = _load("known_answers.json")["simple"]
    # compare_local(queries, refs): A = query, B = ref (simple-test.cpp:100).
    case = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1, "datatype": "na",
            "gapInit": 0, "gapExtend": -1, "A": [k["query"] for k in known],
            "B": [k["ref"] for k in known]}
    score, ar, br = _run_case(case)
    qb, qe = oracle.unpack_range(ar)
    rb, re_ = oracle.unpack_range(br)
    for i, k in enumerate(known):
        assert score[i] == k["score"], i
        assert (qb[i], qe[i], rb[i], re_[i]) == (k["qstart"], k["qend"], k["rstart"], k["rend"]), i


def test_mn_known_answers():
    mn = _load("known_answers.json")["mn"]
    seqs = mn["seqs"]
    case = {"similarity": "na", "match": 1, "mismatch": -1, "ambiguity": -1, "datatype": "na",
            "gapInit": 0, "gapExtend": -1, "A": [seqs[c[0]] for c in mn["comparisons"]],
            "B": [seqs[c[1]] for c in mn["comparisons"]]}
    score, _, _ = _run_case(case)
    assert score.tolist() == mn["scores"]


@pytest.mark.parametrize("fixture", ["parity_ref.json", "random_ref.json"])
def test_oracle_matches_reference_codelet(fixture):
    for case in _load(fixture)["cases"]:
        for fwd in (False, True):
            score, ar, br = _run_case(case, forward_only=fwd)
            key = "fwd_" if fwd else ""
            np.testing.assert_array_equal(score, case["ref"][key + "score"], err_msg=case["name"])
            np.testing.assert_array_equal(ar, case["ref"][key + "arange"], err_msg=case["name"])
            np.testing.assert_array_equal(br, case["ref"][key + "brange"], err_msg=case["name"])


def test_reference_codelet_matches_ssw_on_parity_pairs():
    """The reference's own cross-check (parity-test.cpp:70-87), on the fixtures."""
    for case in _load("parity_ref.json")["cases"]:
        ref, ssw = case["ref"], case["ssw"]
        qb, qe = oracle.unpack_range(ref["arange"])
        rb, re_ = oracle.unpack_range(ref["brange"])
        assert ref["score"] == ssw["score"], case["name"]
        assert qe.tolist() == ssw["a_end"], case["name"]
        assert re_.tolist() == ssw["b_end"], case["name"]
        assert qb.tolist() == ssw["a_begin"], case["name"]
        assert rb.tolist() == ssw["b_begin"], case["name"]


def test_tables_shape():
    t = oracle.tables()
    assert t["NA_CODE"]["N"] == 0 and t["NA_CODE"]["\\0"] == 16
    assert t["AA_CODE"]["A"] == 0 and t["AA_CODE"]["\\0"] == 24
    na = oracle.select_matrix("na", 1, -1, -1)
    assert na.shape == (16, 16) and na[1, 1] == 1 and na[1, 2] == -1 and na[0, 5] == -1
    assert oracle.select_matrix("blosum62")[0, 0] == 4
