"""Runs the C++ drop-in host tests (tests/cpp/partition_test.cpp), which
mirror the reference's partition, M x N mapping and prepare tests."""
import os
import subprocess

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_partition_and_prepare():
    exe = os.path.join(REPO, "tests", "cpp", "partition_test")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "tests", "cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, cwd=REPO)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout


def test_reverse_pass_early_stop_is_exact():
    """tests/cpp/reverse_stop_test.c: the strip-wise early stop of the reverse
    pass gives the full reverse pass's (score, row, column) on random and
    related pairs, five scorings, strip widths 1 to 64."""
    exe = os.path.join(REPO, "tests", "cpp", "reverse_stop_test")
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "tests", "cpp"), exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, cwd=REPO, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout
