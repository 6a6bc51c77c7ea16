"""Shared test set-up: import paths of the package (gem-pic-3d_b200/g3d) and of the oracle, the `gpu` marker."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "gem-pic-3d_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libg3d.so")


def rel_l2(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    nb = np.linalg.norm(b.astype(np.complex128) if np.iscomplexobj(b) else b.astype(np.float64))
    d = np.linalg.norm((a.astype(np.complex128) - b.astype(np.complex128)) if np.iscomplexobj(a) or np.iscomplexobj(b)
                       else (a.astype(np.float64) - b.astype(np.float64)))
    return d / nb if nb > 0 else d


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    return load
