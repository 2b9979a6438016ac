import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from __graft_entry__ import REFERENCE, load_package  # noqa: E402,F401  (REFERENCE: reference tree root)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through the C ABI of librbk.so")


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def golden():
    d = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(d, "cases.json")) as f:
        meta = json.load(f)
    arrays = dict(np.load(os.path.join(d, "golden.npz")))
    return meta, arrays


def as_ops(ops_json):
    """cases.json stores instruction tuples as lists."""
    return [(m, tuple(q), tuple(p)) for m, q, p in ops_json]
