"""Shared pytest set-up: markers and import paths."""
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", os.path.join("ipuma-lib_b200", "python")):
    p = os.path.join(REPO, sub)
    if p not in sys.path:
        sys.path.insert(0, p)
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
