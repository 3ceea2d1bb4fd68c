"""Shared test setup: import paths, the gpu marker, golden fixtures."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "sunny-batched-geneig_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_W():
    return dict(np.load(os.path.join(GOLDEN, "golden_W.npz")))


@pytest.fixture(scope="session")
def golden_U0():
    return dict(np.load(os.path.join(GOLDEN, "golden_U0.npz")))


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    if not os.path.exists(O.LIB_PATH):
        O.build()
    return O
