import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "evoc-rs_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
FIXTURES = ("small_200", "medium_800", "large_2000")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libevoc_gpu.so")


def _has_cuda() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_cuda():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


@pytest.fixture(scope="session")
def golden():
    return {n: load_golden(n) for n in FIXTURES}


def knn_parity_counts(inds, dists, exp_inds, exp_dists, tol=1e-6):
    """The three counts of assert_knn_parity (evoc-rs tests/parity.rs:34-68)."""
    dd = np.abs(dists.astype(np.float64) - exp_dists.astype(np.float64))
    dist_m = int(np.sum(dd > tol))
    bad = int(np.sum((inds != exp_inds) & (dd > tol)))
    tie = int(np.sum((inds != exp_inds) & (dd <= tol)))
    return dist_m, bad, tie


def assert_knn_parity(inds, dists, exp_inds, exp_dists, max_ties=8):
    dist_m, bad, tie = knn_parity_counts(inds, dists, exp_inds, exp_dists)
    assert dist_m == 0, f"kNN distance mismatch count {dist_m}"
    assert bad == 0, f"kNN index mismatch with different distance {bad}"
    assert tie <= max_ties, f"excessive tied-neighbor reordering: {tie}"
