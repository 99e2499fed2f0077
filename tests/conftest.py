"""Shared test setup: repo root on sys.path, the `gpu` marker, golden-fixture loaders."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


def golden_npz(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def golden_json(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


# (name, mu, eps, scatter, absorption, numStepsInt, bins, N, S) of the golden tables
LUT_SETS = {
    "A": (1.0, 0.01, 10.0, 0.0, 2000, 1024, 66, 10.0),
    "B": (1.0, 0.01, 10.0, 0.05, 2000, 2048, 34, 12.0),
    "C": (0.3, 0.0025, 50.0, 0.0, 4000, 512, 18, 6.0),
    # the benchmark configurations: plain form (N = 66 for 64: the reference bootstrapper's N)
    # and precision form (N = 258 for 256)
    "D": (1.0, 0.01, 10.0, 0.0, 4000, 4096, 66, 10.0),
    "E": (1.0, 0.01, 10.0, 0.0, 20000, 8192, 258, 20.0),
}
GEOM = {
    66: ((0, 0, 0), (1, 0, 0), (8, 0, 0), (1, 0, 0)),
    34: ((0, 0, 0), (0, 0, 1), (0, 0, 7), (0, 0, 1)),
    18: ((0, 0, 0), (1, 0, 0), (2.5, 1.0, 0.5), (0, 1, 0)),
    10: ((0, 0, 0), (1, 0, 0), (3, 0, 0), (1, 0, 0)),
    258: ((0, 0, 0), (0, 0, 1), (0, 0, 12), (0, 0, 1)),
}


@pytest.fixture(scope="session")
def oracle():
    from oracle import py_oracle
    py_oracle.build()
    return py_oracle
