import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_literals.json")) as f:
        return json.load(f)


def fmajor(cats_factor_major):
    """(Q, n) lists -> F-order (n, Q) uint32 array."""
    return np.asfortranarray(np.array(cats_factor_major, dtype=np.uint32).T)


def generate_synthetic_data(n_levels, n_rows, seed=42):
    """y = D x_true (no noise), as the reference's tests/conftest.py:7-21 generator."""
    rng = np.random.default_rng(seed)
    cats = [rng.integers(0, nl, size=n_rows) for nl in n_levels]
    x_true = rng.standard_normal(sum(n_levels))
    y = np.zeros(n_rows)
    off = 0
    for f, nl in enumerate(n_levels):
        y += x_true[off + cats[f]]
        off += nl
    return np.asfortranarray(np.column_stack(cats).astype(np.uint32)), x_true, y
