"""Runs the C++ drop-in tests on the GPU (tests/cpp/dropin_test.cpp): the
reference's simple-test and mn_cmp-test known answers through
ipu::batchaffine::SWAlgorithm, the class a reference caller uses."""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu


def test_dropin_api_known_answers():
    exe = os.path.join(REPO, "tests", "cpp", "dropin_test")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "tests", "cpp")], check=True)
    env = dict(os.environ, IPUMA_GOLDEN_DIR=os.path.join(REPO, "tests", "golden"))
    r = subprocess.run([exe], capture_output=True, text=True, cwd=REPO, env=env, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout
