"""The ipusw_b200 command line: input loaders, configuration, batching and
the IPUSWLOG run logs (ipusw/main.cpp, ipusw/run_comparison.hpp,
ipusw/batch.hpp, scripts/extract.py of the reference).

CPU tests run the program with --dry-run and check its batches against a
restatement of createBatches (batch.hpp) with the reference's limits
(run_comparison.hpp:93-94).  GPU tests run whole comparisons and check the
--output results against the oracle.
"""
import json
import os
import random
import subprocess

import numpy as np
import pytest

import oracle

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "ipuma-lib_b200")
EXE = os.path.join(PKG, "ipusw", "ipusw_b200")

AA = "ARNDCQEGHILKMFPSTWYVBZX"


@pytest.fixture(scope="module")
def exe():
    if not os.path.exists(EXE):
        subprocess.run(["make", "-s", "-C", PKG, "ipusw"], check=True)
    return EXE


def _config(**over):
    sw = {"gapInit": -1, "gapExtend": -1, "matchValue": 1, "mismatchValue": -1,
          "ambiguityValue": -1, "similarity": "na", "datatype": "na"}
    ipu = {"tilesUsed": 128, "maxAB": 300, "maxBatches": 4, "bufsize": 800, "vtype": "cpp",
           "fillAlgo": "fillfirst", "forwardOnly": False, "useRemoteBuffer": False,
           "transmissionPrograms": 1, "ioTiles": 0}
    top = {"numDevices": 1, "numThreads": 2, "duplicateDatasets": False, "duplicationFactor": 0,
           "repeat": 1}
    for k, v in over.items():
        (sw if k in sw else ipu if k in ipu else top)[k] = v
    return dict(top, sw=sw, ipu=ipu)


def _seqs(n, seed, alphabet="ACGT", lo=0, hi=250):
    r = random.Random(seed)
    return ["".join(r.choice(alphabet) for _ in range(r.randint(lo, hi))) for _ in range(n)]


def _write_txt(path, seqs, crlf=False):
    with open(path, "w", newline="") as f:
        for s in seqs:
            f.write(s + ("\r\n" if crlf else "\n"))


def _write_fasta(path, seqs, width=60):
    with open(path, "w") as f:
        for i, s in enumerate(seqs):
            f.write(">seq%d some description\n" % i)
            for k in range(0, len(s), width):
                f.write(s[k:k + width] + "\n")


def create_batches(A, B, cmp_limit, data_limit):
    """batch.hpp createBatches: consecutive pairs while one more comparison
    stays below cmp_limit and the bytes below data_limit."""
    out, num, size, begin = [], 0, 0, 0
    for a, b in zip(A, B):
        if num + 1 < cmp_limit and size + len(a) + len(b) < data_limit:
            num += 1
            size += len(a) + len(b)
        else:
            out.append((begin, begin + num, num, size))
            begin += num
            num, size = 1, len(a) + len(b)
    if num > 0:
        out.append((begin, begin + num, num, size))
    return out


def _limits(cfg):
    ipu = cfg["ipu"]
    total = ipu["tilesUsed"] * ipu["maxBatches"]
    bufsize32b = (ipu["bufsize"] + 3) // 4
    return total - ipu["maxBatches"], ipu["tilesUsed"] * bufsize32b * 4 - ipu["bufsize"] * 100


def _run(exe, tmp_path, cfg, ref, query, *extra, check=True):
    cpath = tmp_path / "cfg.json"
    cpath.write_text(json.dumps(cfg))
    r = subprocess.run([exe, "--config", str(cpath), *extra, str(ref), str(query)],
                       capture_output=True, text=True, timeout=900)
    if check:
        assert r.returncode == 0, r.stdout + r.stderr
    return r


def _logs(stdout):
    out = []
    for line in stdout.splitlines():
        if "IPUSWLOG" in line:
            out.append(json.loads(line.split("IPUSWLOG", 1)[1]))
    return out


def _batches(stdout):
    return [tuple(int(x) for x in line.split()[1:]) for line in stdout.splitlines()
            if line.startswith("batch ")]


@pytest.mark.parametrize("max_batches,bufsize", [(4, 800), (2, 600), (10, 2000)])
def test_dry_run_batches_follow_create_batches(exe, tmp_path, max_batches, bufsize):
    A, B = _seqs(700, 1), _seqs(700, 2, lo=1)
    _write_txt(tmp_path / "ref.txt", A)
    _write_txt(tmp_path / "query.txt", B)
    cfg = _config(maxBatches=max_batches, bufsize=bufsize)
    r = _run(exe, tmp_path, cfg, tmp_path / "ref.txt", tmp_path / "query.txt", "--dry-run")
    want = create_batches(A, B, *_limits(cfg))
    assert len(want) > 1
    assert _batches(r.stdout) == want


def test_txt_and_fasta_inputs_load_the_same_sequences(exe, tmp_path):
    """.txt is one sequence per line (CRLF tolerated); any other name is FASTA
    with wrapped lines."""
    A, B = _seqs(300, 3, AA, 1, 400), _seqs(300, 4, AA, 1, 400)
    _write_txt(tmp_path / "ref.txt", A, crlf=True)
    _write_txt(tmp_path / "query.txt", B)
    _write_fasta(tmp_path / "ref.fasta", A)
    _write_fasta(tmp_path / "query.fa", B, width=37)
    cfg = _config(similarity="blosum62", datatype="aa")
    r1 = _run(exe, tmp_path, cfg, tmp_path / "ref.txt", tmp_path / "query.txt", "--dry-run")
    r2 = _run(exe, tmp_path, cfg, tmp_path / "ref.fasta", tmp_path / "query.fa", "--dry-run")
    want = create_batches(A, B, *_limits(cfg))
    assert _batches(r1.stdout) == want
    assert _batches(r2.stdout) == want


def test_setup_log_carries_the_config_extract_reads(exe, tmp_path):
    """run_comparison_setup holds the merged config: JSON file, then --KEY
    VALUE overrides; scripts/extract.py reads numDevices, numThreads,
    duplicateDatasets, ipu.useRemoteBuffer and ipu.fillAlgo from it."""
    A = _seqs(20, 5)
    _write_txt(tmp_path / "a.txt", A)
    cfg = _config(numThreads=3, duplicateDatasets=True, numDevices=2)
    r = _run(exe, tmp_path, cfg, tmp_path / "a.txt", tmp_path / "a.txt", "--dry-run",
             "--gapInit", "-7", "--useRemoteBuffer", "true", "--fillAlgo", "greedy")
    logs = _logs(r.stdout)
    assert [l["tag"] for l in logs] == ["run_comparison_setup"]
    setup = logs[0]
    c = setup["config"]
    assert c["numDevices"] == 2 and c["numThreads"] == 3 and c["duplicateDatasets"] is True
    assert c["ipu"]["useRemoteBuffer"] is True and c["ipu"]["fillAlgo"] == "greedy"
    assert c["sw"]["gapInit"] == -7 and c["sw"]["gapExtend"] == -1
    assert setup["duplicationFactor"] == 2
    assert setup["ref_path"].endswith("a.txt") and setup["query_path"].endswith("a.txt")


def test_defaults_without_a_config_file(exe, tmp_path):
    """Without --config the scoring and batching defaults are the driver's
    SW_CONFIGURATION / ALGO_CONFIGURATION (driver.hpp)."""
    A = _seqs(10, 6)
    _write_txt(tmp_path / "a.txt", A)
    r = subprocess.run([exe, "--dry-run", str(tmp_path / "a.txt"), str(tmp_path / "a.txt")],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    c = _logs(r.stdout)[0]["config"]
    assert c["ipu"]["tilesUsed"] == 8832 and c["ipu"]["maxAB"] == 200
    assert c["ipu"]["maxBatches"] == 300 and c["ipu"]["bufsize"] == 30000
    assert c["sw"]["gapInit"] == 0 and c["sw"]["gapExtend"] == -1
    assert _batches(r.stdout) == [(0, 10, 10, 2 * sum(map(len, A)))]


@pytest.mark.parametrize("args,message", [
    (["--bogus", "1"], "unknown option --bogus"),
    (["--forwardOnly", "maybe"], "not a boolean"),
    (["--similarity", "pam250"], "similarity"),
    (["--maxAB", "300x"], "not an integer"),
    (["--numThreads", ""], "not an integer"),
])
def test_bad_options_are_reported(exe, tmp_path, args, message):
    _write_txt(tmp_path / "a.txt", ["ACGT"])
    r = subprocess.run([exe, *args, "--dry-run", str(tmp_path / "a.txt"), str(tmp_path / "a.txt")],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert message in r.stderr


def test_bad_inputs_are_reported(exe, tmp_path):
    _write_txt(tmp_path / "a.txt", ["ACGT", "AC"])
    _write_txt(tmp_path / "b.txt", ["ACGT"])
    (tmp_path / "bad.json").write_text('{"sw": {"gapInit": -1,}')
    cases = [
        ([str(tmp_path / "a.txt"), str(tmp_path / "missing.txt")], "File not found"),
        ([str(tmp_path / "a.txt"), str(tmp_path / "b.txt")], "not equal"),
        (["--config", str(tmp_path / "bad.json"), str(tmp_path / "a.txt"), str(tmp_path / "a.txt")],
         "config JSON"),
    ]
    for args, message in cases:
        r = subprocess.run([exe, "--dry-run", *args], capture_output=True, text=True, timeout=60)
        assert r.returncode == 1, args
        assert message in r.stderr, (args, r.stderr)
    r = subprocess.run([exe, str(tmp_path / "a.txt")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stdout


# ---------------------------------------------------------------------------
# GPU: whole runs against the oracle
# ---------------------------------------------------------------------------

def _oracle_tsv(A, B, datatype, similarity, cfg, forward_only):
    enc = [oracle.encode(datatype, s) for s in A], [oracle.encode(datatype, s) for s in B]
    codes, a_off, a_len, b_off, b_len = oracle.pack_pairs(*enc)
    sw = cfg["sw"]
    sim = oracle.select_matrix(similarity, sw["matchValue"], sw["mismatchValue"], sw["ambiguityValue"])
    score, ar, br = oracle.sw_batch(codes, a_off, a_len, b_off, b_len, sim, sw["gapInit"],
                                    sw["gapExtend"], forward_only=forward_only)
    a0, a1 = oracle.unpack_range(ar)
    b0, b1 = oracle.unpack_range(br)
    return np.stack([score, a0, a1, b0, b1], axis=1)


def _read_tsv(path):
    rows = np.loadtxt(path, dtype=np.int64, skiprows=1, ndmin=2)
    assert (rows[:, 0] == np.arange(rows.shape[0])).all()
    return rows[:, 1:]


@pytest.mark.gpu
@pytest.mark.parametrize("forward_only", [False, True])
def test_dna_run_matches_oracle_and_logs_every_batch(exe, tmp_path, forward_only):
    A, B = _seqs(3000, 7, hi=300), _seqs(3000, 8, lo=1, hi=300)
    A[5], A[17] = "", "ACGT" * 75
    B[17] = A[17]
    _write_txt(tmp_path / "ref.txt", A)
    _write_fasta(tmp_path / "query.fasta", B)
    cfg = _config(numThreads=4, forwardOnly=forward_only, gapInit=-2, maxBatches=8, bufsize=1200)
    r = _run(exe, tmp_path, cfg, tmp_path / "ref.txt", tmp_path / "query.fasta",
             "--output", str(tmp_path / "out.tsv"))
    got = _read_tsv(tmp_path / "out.tsv")
    want = _oracle_tsv(A, B, "na", "na", cfg, forward_only)
    if forward_only:
        got, want = got[:, [0, 2, 4]], want[:, [0, 2, 4]]
    bad = np.nonzero((got != want).any(axis=1))[0]
    assert bad.size == 0, "%d pairs differ, first %d: %s vs %s" % (
        bad.size, bad[0], got[bad[0]], want[bad[0]])

    logs = _logs(r.stdout)
    nb = len(create_batches(A, B, *_limits(cfg)))
    assert nb > 3
    perf = [l for l in logs if l["tag"] == "batch_perf"]
    final = [l for l in logs if l["tag"] == "final_log"]
    assert len(perf) == nb and len(final) == 1
    cells = sum(len(a) * len(b) for a, b in zip(A, B))
    assert sum(p["cell_count"] for p in perf) == cells
    for p in perf:
        assert p["time_inner"] > 0 and p["time_outer"] >= p["time_inner"]
        assert p["gcups_inner"] > 0
    f = final[0]
    assert f["cells"] == cells and f["cmps_orig"] == len(A)
    assert f["cmps_processed"] == f["cmps_submitted"] == len(A)
    assert f["batches_processed"] == f["batches_submitted"] == f["batches_orig"] == nb
    assert f["outer_gcups"] > 0


@pytest.mark.gpu
def test_protein_run_with_duplicated_batches(exe, tmp_path):
    """duplicateDatasets submits every batch duplicationFactor times and
    counts the duplicates' cells (run_comparison.hpp:72-75, 152-155)."""
    A, B = _seqs(1500, 9, AA, 1, 500), _seqs(1500, 10, AA, 1, 500)
    _write_fasta(tmp_path / "ref.fasta", A)
    _write_fasta(tmp_path / "query.fasta", B)
    cfg = _config(similarity="blosum62", datatype="aa", gapInit=-11, gapExtend=-1, maxAB=600,
                  maxBatches=6, bufsize=3000, duplicateDatasets=True, duplicationFactor=3,
                  numThreads=6)
    r = _run(exe, tmp_path, cfg, tmp_path / "ref.fasta", tmp_path / "query.fasta",
             "--output", str(tmp_path / "out.tsv"))
    got = _read_tsv(tmp_path / "out.tsv")
    want = _oracle_tsv(A, B, "aa", "blosum62", cfg, False)
    assert (got == want).all()
    logs = _logs(r.stdout)
    nb = len(create_batches(A, B, *_limits(cfg)))
    final = logs[-1]
    assert final["tag"] == "final_log"
    assert final["batches_submitted"] == final["batches_processed"] == 3 * nb
    assert final["cmps_submitted"] == 3 * len(A)
    assert final["cells"] == 3 * sum(len(a) * len(b) for a, b in zip(A, B))
    assert sum(1 for l in logs if l["tag"] == "batch_perf") == 3 * nb
