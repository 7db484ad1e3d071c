"""Shared pytest set-up: the `gpu` marker, import paths, and in-tree builds of the CPU-side
libraries (the oracle checker and the synthetic-data renderer) when they are missing."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
PKG = os.path.join(ROOT, "frame-aligner_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device (sm_100a)")
    if not os.path.exists(os.path.join(ORACLE, "liboracle.so")):
        subprocess.run(["make", "-s", "-C", ORACLE, os.path.join(ORACLE, "liboracle.so")], check=True)
    if not os.path.exists(os.path.join(PKG, "libfa_synth.so")):
        subprocess.run(["make", "-s", "-C", PKG, os.path.join(PKG, "libfa_synth.so")], check=True)


def golden_cases():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f != "phase_shifts.npz")


def load_golden(name):
    import numpy as np

    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.fixture(params=golden_cases())
def golden(request):
    return request.param, load_golden(request.param)
