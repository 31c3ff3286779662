"""Shared test setup.

Markers:
  gpu — needs a CUDA device (B200); everything else runs on the CPU.
"""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "rust-igraph_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU")


def pytest_collection_modifyitems(config, items):
    # keep the no-allocation entry point test (if present) last
    items.sort(key=lambda it: 1 if "test_zz_" in it.nodeid else 0)


@pytest.fixture(scope="session")
def golden_cases():
    with open(os.path.join(GOLDEN, "reference_fixtures.json")) as f:
        return json.load(f)["cases"]


def case_edges(case):
    e = np.asarray(case["edges"], dtype=np.uint32).reshape(-1, 2)
    f, t = e[:, 0].copy(), e[:, 1].copy()
    if not case["directed"]:
        f, t = np.minimum(f, t), np.maximum(f, t)
    return f, t


def within(actual, expected, kind, tol):
    actual = np.asarray(actual, dtype=np.float64)
    expected = np.asarray(expected, dtype=np.float64)
    if actual.shape != expected.shape:
        return False
    d = np.abs(actual - expected)
    if kind == "rel":
        scale = np.maximum(np.maximum(np.abs(actual), np.abs(expected)), 1.0)
        return bool(np.all(d <= tol * scale))
    return bool(np.all(d < tol))


@pytest.fixture(scope="session")
def cuda_ok():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return True
