import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def built():
    """Builds the product library and the oracle in-tree if missing."""
    lib = os.path.join(ROOT, "tycho2_b200", "lib", "libtycho_b200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tycho2_b200", "csrc")], check=True)
    oracle_lib = os.path.join(ROOT, "oracle", "_build", "libtycho_oracle.so")
    if not os.path.exists(oracle_lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    return True


@pytest.fixture(scope="session")
def kuhn3_ref():
    return dict(np.load(os.path.join(GOLDEN, "kuhn3_ref.npz")))


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return tmp_path_factory.mktemp("tycho")


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def rel_linf(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))
