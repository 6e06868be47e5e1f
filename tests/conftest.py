import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")
    config.addinivalue_line("markers", "slow: larger CPU parity cases")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name))
    return load


def golden_sets(npz):
    """Group the flat 'name/key' arrays of a golden npz by name."""
    out = {}
    for k in npz.files:
        if "/" in k:
            name, key = k.split("/", 1)
            out.setdefault(name, {})[key] = npz[k]
    return out


def none_if_empty(a):
    return None if a.size == 0 else a.astype(np.int32)


def verify_heap(nodes):
    """The reference's verify_tree rule (kdtest.c:73-99) over a whole node
    array: a left child's coordinate in its parent's split dimension is <=
    the parent's, a right child's is >=."""
    dim = nodes["dim"].astype(np.int64)
    xyz = nodes["xyz"]
    par = np.arange(1, len(dim) // 2)
    left = par[nodes["has_l"][par] != 0]
    right = par[nodes["has_r"][par] != 0]
    assert np.all(xyz[2 * left, dim[left]] <= xyz[left, dim[left]])
    assert np.all(xyz[2 * right + 1, dim[right]] >= xyz[right, dim[right]])
