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


FIELDS = ["Rx", "Ry", "Ez", "Bz", "Lx", "Ly"]
CURRENTS = ["jkx", "jky", "jkz"]


def state_errors(got, ref, names):
    """Relative L2 errors of a set of spectra measured against the norm of the whole set (the field state
    vector): {name: (||got - ref|| / ||ref set||, ||got - ref|| / ||ref||)}. E_z, B_z and L are gamma^-2
    smaller than R for a relativistic bunch, so their own relative error mostly measures the cancellation
    in them; the parity bound applies to the state norm, the component bound is a sanity check."""
    total = np.sqrt(sum(np.linalg.norm(np.asarray(ref[n])) ** 2 for n in names))
    out = {}
    for n in names:
        d = np.linalg.norm(np.asarray(got[n]) - np.asarray(ref[n]))
        nr = np.linalg.norm(np.asarray(ref[n]))
        out[n] = (d / total if total > 0 else d, d / nr if nr > 0 else d)
    return out


def assert_state(got, ref, names, tol=1e-10, comp_tol=1e-6, tag=""):
    """The state bound on every component; the component bound only on components above 1e-12 of the state norm
    (a component that small is rounding noise in both codes, e.g. R_y of an x-polarised laser on the free-hand
    grid: 1.6e-11 against 5.6e4)."""
    total = np.sqrt(sum(np.linalg.norm(np.asarray(ref[n])) ** 2 for n in names))
    for n, (e_state, e_comp) in state_errors(got, ref, names).items():
        assert e_state <= tol, (tag, n, "state-relative", e_state)
        if np.linalg.norm(np.asarray(ref[n])) > 1e-12 * total:
            assert e_comp <= comp_tol, (tag, n, "component-relative", e_comp)


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    return load
