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
