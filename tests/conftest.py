import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")


@pytest.fixture(scope="session")
def golden():
    """Golden fixtures generated from the reference's own sources (tests/golden/make_golden.py)."""
    class G:
        def __init__(self):
            self._c = {}

        def __getitem__(self, name):
            if name not in self._c:
                self._c[name] = np.load(os.path.join(GOLDEN, name + ".npz"))
            return self._c[name]
    return G()


@pytest.fixture(scope="session")
def c_oracle():
    from oracle import c_oracle
    c_oracle.lib()
    return c_oracle


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle import ref_oracle
    if not ref_oracle.available():
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    return ref_oracle


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype == np.float32 and b.dtype == np.float32:
        return np.array_equal(a.view(np.uint32), b.view(np.uint32)) or np.array_equal(a, b)
    return np.array_equal(a, b)


def csr_sets(off, idx):
    return [np.sort(idx[off[i]:off[i + 1]]) for i in range(len(off) - 1)]


def sorted_csr(off, idx):
    """The same CSR with every list sorted ascending (vectorised)."""
    off = np.asarray(off)
    seg = np.repeat(np.arange(len(off) - 1), np.diff(off))
    return off, np.asarray(idx)[np.lexsort((idx, seg))]
