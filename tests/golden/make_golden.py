"""Generates the golden fixtures in tests/golden/ from the reference tree.

Run where the reference tree is available (read-only; its path in
IPUMA_REF_DIR or --ref) and the reference libraries are built by
``make -C oracle ref``:

    IPUMA_REF_DIR=<reference tree> python tests/golden/make_golden.py [--ref DIR]

Outputs (committed; nothing at test time reads the reference tree):

* ``tables.json``  -- NA_CODE / AA_CODE (src/swatlib/encoding.h:26-72) and the
  NA_SUBSTITUTION / BLOSUM50 / BLOSUM62 tables (src/swatlib/similarity.h:17-94),
  parsed from the headers as text.
* ``known_answers.json`` / ``known_answers.txt`` -- the 19 (score, q/r start/end) answers of
  test/simple-test.cpp:25-45 and the 4 M x N scores of test/mn_cmp-test.cpp:29-57,
  parsed as text.
* ``parity_ref.json`` -- the DNA and protein pairs of test/parity-test.cpp:20-59,
  239-260 (no stored answers there) with the answers of the reference codelet
  compiled for the host and of the reference's SSW, for each scoring the
  reference tests use.
* ``random_ref.json`` -- seeded random pairs (DNA with IUPAC codes, protein,
  short, long, empty) with the reference codelet's answers.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))


def _strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def parse_int_table(text: str, name: str) -> list[int]:
    m = re.search(r"\b%s\s*=\s*\{(.*?)\};" % re.escape(name), text, flags=re.S)
    if not m:
        raise RuntimeError("table %s not found" % name)
    body = _strip_comments(m.group(1))
    return [int(x) for x in re.findall(r"-?\d+", body)]


def parse_code_map(text: str, name: str) -> dict[str, int]:
    m = re.search(r"\b%s\s*=\s*\{(.*?)\};" % re.escape(name), text, flags=re.S)
    if not m:
        raise RuntimeError("map %s not found" % name)
    out = {}
    for ch, val in re.findall(r"\{\s*'(\\0|.)'\s*,\s*(\d+)\s*\}", m.group(1)):
        out[ch] = int(val)
    return out


def parse_simple_data(text: str) -> list[dict]:
    m = re.search(r"simpleData\s*=\s*\{(.*?)\n\};", text, flags=re.S)
    cases = []
    for ref, query, qs, qe, rs, re_, sc in re.findall(
            r'\{\s*"([^"]*)"\s*,\s*"([^"]*)"\s*,\s*(-?\d+)\s*,\s*(-?\d+)\s*,\s*(-?\d+)\s*,\s*(-?\d+)\s*,\s*(-?\d+)\s*\}',
            m.group(1)):
        cases.append({"ref": ref, "query": query, "qstart": int(qs), "qend": int(qe),
                      "rstart": int(rs), "rend": int(re_), "score": int(sc)})
    return cases


def parse_mn(text: str) -> dict:
    m = re.search(r"TEST\(MN_Test, CompareAll\)\s*\{(.*?)\n\}", text, flags=re.S)
    body = m.group(1)
    seqs = re.findall(r'"([ACGTN]+)"', re.search(r"seqs\s*=\s*\{(.*?)\};", body, re.S).group(1))
    cmps = [[int(a), int(b)] for a, b in re.findall(
        r"\{\s*(\d+)\s*,\s*(\d+)\s*\}", re.search(r"comparisons\s*=\s*\{(.*?)\n\s*\};", body, re.S).group(1))]
    exp = {int(i): int(v) for i, v in re.findall(r"result\.scores\[(\d+)\],\s*(-?\d+)", body)}
    return {"seqs": seqs, "comparisons": cmps, "scores": [exp[i] for i in range(len(cmps))]}


def parse_parity(text: str) -> dict:
    blocks = re.findall(r"queries\s*=\s*\{(.*?)\};.*?refs\s*=\s*\{(.*?)\};", text, flags=re.S)
    dna_q = re.findall(r'"([A-Z]+)"', blocks[0][0])
    dna_r = re.findall(r'"([A-Z]+)"', blocks[0][1])
    aa_q = re.findall(r'"([A-Z]+)"', blocks[1][0])
    aa_r = re.findall(r'"([A-Z]+)"', blocks[1][1])
    return {"dna_queries": dna_q, "dna_refs": dna_r, "aa_queries": aa_q, "aa_refs": aa_r}


def run_ref(oracle, a_list, b_list, sim, gI, gE, datatype):
    a_codes = [oracle.encode(datatype, s) for s in a_list]
    b_codes = [oracle.encode(datatype, s) for s in b_list]
    packed = oracle.pack_pairs(a_codes, b_codes)
    sc, ar, br = oracle.ref_codelet_pairs(*packed, sim, gI, gE, forward_only=False, nthreads=4)
    sc_m, ar_m, br_m = oracle.ref_codelet_pairs(*packed, sim, gI, gE, forward_only=False,
                                                nthreads=4, variant="multi")
    assert (sc == sc_m).all() and (ar == ar_m).all() and (br == br_m).all(), \
        "SWAffine and MultiSWAffine disagree"
    fsc, far, fbr = oracle.ref_codelet_pairs(*packed, sim, gI, gE, forward_only=True, nthreads=4)
    return {"score": sc.tolist(), "arange": ar.tolist(), "brange": br.tolist(),
            "fwd_score": fsc.tolist(), "fwd_arange": far.tolist(), "fwd_brange": fbr.tolist()}


def run_ssw(oracle, a_list, b_list, sim, gap_open, gap_ext, datatype):
    a_codes = [oracle.encode(datatype, s) for s in a_list]
    b_codes = [oracle.encode(datatype, s) for s in b_list]
    packed = oracle.pack_pairs(a_codes, b_codes)
    sc, ae, be, ab, bb = oracle.ref_ssw_pairs(*packed, sim, gap_open, gap_ext, report_begin=True,
                                             nthreads=4)
    return {"score": sc.tolist(), "a_end": ae.tolist(), "b_end": be.tolist(),
            "a_begin": ab.tolist(), "b_begin": bb.tolist()}


def random_cases(rng, oracle):
    """Seeded random pairs covering the shapes the reference's paths see."""
    out = []
    na = "ACGT"
    iupac = "NACGTURYKMSWBDHV"
    aa = "ARNDCQEGHILKMFPSTWYV"
    aa_ext = aa + "BZX*"

    def mutate(s, alphabet, sub, indel):
        res = []
        for ch in s:
            r = rng.random()
            if r < indel / 2:
                continue
            if r < indel:
                res.append(ch)
                res.append(alphabet[rng.integers(len(alphabet))])
                continue
            if rng.random() < sub:
                res.append(alphabet[rng.integers(len(alphabet))])
            else:
                res.append(ch)
        return "".join(res)

    def rnd(alphabet, n):
        return "".join(alphabet[i] for i in rng.integers(0, len(alphabet), n))

    # DNA, +1/-1, gap open 1 / extend 1 (gapInit 0, gapExtend -1)
    a_l, b_l = [], []
    for k in range(120):
        la = int(rng.integers(1, 260))
        a = rnd(na, la)
        if k % 10 == 0:
            b = rnd(na, int(rng.integers(1, 400)))
        else:
            core = mutate(a, na, 0.08, 0.04)
            left = rnd(na, int(rng.integers(0, 60)))
            right = rnd(na, int(rng.integers(0, 60)))
            b = left + core + right
        a_l.append(a)
        b_l.append(b)
    # edge shapes
    a_l += ["A", "A", "ACGT", "T" * 40, "A" * 150, "ACGTACGT", "G" * 64, "C" * 33]
    b_l += ["A", "C", "A", "T" * 40, "T" * 150, "", "G" * 64, "C" * 31]
    a_l += ["", "ACGT"]
    b_l += ["ACGT", ""]
    out.append({"name": "dna_gap1", "datatype": "na", "similarity": "na", "match": 1,
                "mismatch": -1, "ambiguity": -1, "gapInit": 0, "gapExtend": -1, "A": a_l, "B": b_l})
    # DNA with IUPAC codes and gap open 3 (gapInit -2), match 2
    a_l, b_l = [], []
    for k in range(60):
        a = rnd(iupac, int(rng.integers(1, 200)))
        b = mutate(a, iupac, 0.1, 0.05) + rnd(iupac, int(rng.integers(0, 30)))
        a_l.append(a)
        b_l.append(b if b else "N")
    out.append({"name": "dna_iupac_gap3", "datatype": "na", "similarity": "na", "match": 2,
                "mismatch": -3, "ambiguity": -1, "gapInit": -2, "gapExtend": -1, "A": a_l,
                "B": b_l})
    # Protein, BLOSUM62, gap open 11 / extend 1 (gapInit -10, gapExtend -1)
    a_l, b_l = [], []
    for k in range(80):
        la = int(rng.integers(1, 700)) if k % 8 else int(rng.integers(700, 1300))
        a = rnd(aa, la)
        if k % 7 == 0:
            b = rnd(aa_ext, int(rng.integers(1, 700)))
        else:
            b = mutate(a, aa_ext, 0.35, 0.05)
            b = b if b else "A"
        a_l.append(a)
        b_l.append(b)
    out.append({"name": "aa_blosum62", "datatype": "aa", "similarity": "blosum62", "match": 1,
                "mismatch": -1, "ambiguity": -1, "gapInit": -10, "gapExtend": -1, "A": a_l,
                "B": b_l})
    # Protein, BLOSUM50, gap open 3 / extend 1 (gapInit -2)
    a_l, b_l = [], []
    for k in range(40):
        a = rnd(aa_ext, int(rng.integers(1, 400)))
        b = mutate(a, aa_ext, 0.3, 0.06)
        a_l.append(a)
        b_l.append(b if b else "W")
    out.append({"name": "aa_blosum50", "datatype": "aa", "similarity": "blosum50", "match": 1,
                "mismatch": -1, "ambiguity": -1, "gapInit": -2, "gapExtend": -1, "A": a_l,
                "B": b_l})
    for case in out:
        sim = oracle.select_matrix(case["similarity"], case["match"], case["mismatch"],
                                   case["ambiguity"])
        case["ref"] = run_ref(oracle, case["A"], case["B"], sim, case["gapInit"],
                              case["gapExtend"], case["datatype"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("IPUMA_REF_DIR"),
                    help="reference tree (default: $IPUMA_REF_DIR)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("pass --ref or set IPUMA_REF_DIR to the reference tree")
    ref = args.ref
    rd = lambda p: open(os.path.join(ref, p)).read()

    enc = rd("src/swatlib/encoding.h")
    simh = rd("src/swatlib/similarity.h")
    tables = {
        "source": "src/swatlib/encoding.h:26-72, src/swatlib/similarity.h:17-94",
        "NA_CODE": parse_code_map(enc, "NA_CODE"),
        "AA_CODE": parse_code_map(enc, "AA_CODE"),
        "NA_SUBSTITUTION": parse_int_table(simh, "NA_SUBSTITUTION"),
        "BLOSUM50": parse_int_table(simh, "BLOSUM50"),
        "BLOSUM62": parse_int_table(simh, "BLOSUM62"),
    }
    assert len(tables["NA_SUBSTITUTION"]) == 256
    assert len(tables["BLOSUM50"]) == 625 and len(tables["BLOSUM62"]) == 625
    assert len(tables["NA_CODE"]) == 17 and len(tables["AA_CODE"]) == 25
    with open(os.path.join(HERE, "tables.json"), "w") as f:
        json.dump(tables, f, indent=1)

    import oracle  # noqa: E402  (needs tables.json)

    known = {
        "source": "test/simple-test.cpp:25-45, test/mn_cmp-test.cpp:29-57",
        "simple": parse_simple_data(rd("test/simple-test.cpp")),
        "mn": parse_mn(rd("test/mn_cmp-test.cpp")),
    }
    assert len(known["simple"]) == 19, len(known["simple"])
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(known, f, indent=1)
    # Plain-text copy for the C++ drop-in tests (tests/cpp): one case per line.
    with open(os.path.join(HERE, "known_answers.txt"), "w") as f:
        f.write("# simple: ref query qstart qend rstart rend score\n")
        for k in known["simple"]:
            f.write("simple %s %s %d %d %d %d %d\n" % (k["ref"], k["query"], k["qstart"], k["qend"],
                                                     k["rstart"], k["rend"], k["score"]))
        f.write("# mn: seq <s> ... / cmp <indexA> <indexB> <score>\n")
        for sq in known["mn"]["seqs"]:
            f.write("mnseq %s\n" % sq)
        for (ia, ib), sc in zip(known["mn"]["comparisons"], known["mn"]["scores"]):
            f.write("mncmp %d %d %d\n" % (ia, ib, sc))

    par = parse_parity(rd("test/parity-test.cpp"))
    assert len(par["dna_queries"]) == 18 and len(par["aa_queries"]) == 4
    parity = {"source": "test/parity-test.cpp:20-59,239-260", "cases": []}
    # DNA: gap opening 1 and 3 with extend 1, +1/-1 (parity-test.cpp:160-161,217-237).
    # test_aligns_ipu(alns, refs, queries) passes refs as A (parity-test.cpp:170).
    for gap_open in (1, 3):
        gI, gE = -(gap_open - 1), -1
        sim = oracle.select_matrix("na", 1, -1, -1)
        A, B = par["dna_refs"], par["dna_queries"]
        parity["cases"].append({
            "name": "dna_gapopen%d" % gap_open, "datatype": "na", "similarity": "na",
            "match": 1, "mismatch": -1, "ambiguity": -1, "gapInit": gI, "gapExtend": gE,
            "A": A, "B": B,
            "ref": run_ref(oracle, A, B, sim, gI, gE, "na"),
            "ssw": run_ssw(oracle, A, B, sim, gap_open, 1, "na")})
    for simname, gap_open in (("blosum50", 3), ("blosum62", 11)):
        gI, gE = -(gap_open - 1), -1
        sim = oracle.select_matrix(simname)
        A, B = par["aa_refs"], par["aa_queries"]
        parity["cases"].append({
            "name": "aa_%s_gapopen%d" % (simname, gap_open), "datatype": "aa",
            "similarity": simname, "match": 1, "mismatch": -1, "ambiguity": -1, "gapInit": gI,
            "gapExtend": gE, "A": A, "B": B,
            "ref": run_ref(oracle, A, B, sim, gI, gE, "aa"),
            "ssw": run_ssw(oracle, A, B, sim, gap_open, 1, "aa")})
    with open(os.path.join(HERE, "parity_ref.json"), "w") as f:
        json.dump(parity, f)

    rng = np.random.Generator(np.random.PCG64(20261203))
    rnd = {"source": "seeded random pairs (PCG64 seed 20261203); answers from the reference "
                     "codelet compiled for the host (oracle/_ref/libref_codelet.so)",
           "cases": random_cases(rng, oracle)}
    with open(os.path.join(HERE, "random_ref.json"), "w") as f:
        json.dump(rnd, f)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
