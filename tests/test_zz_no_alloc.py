"""fs_query_position_noalloc: the position query that works from a fixed
device array instead of allocating. Through the C-ABI, against
fs_query_position on the same search, two calls in a row (the second reuses
the resolved array and must reset its count). Collected last on purpose:
it must pass both in a fresh process and after every other test."""
import ctypes

import numpy as np
import pytest

from fluidsolver_b200 import NeighborhoodSearch, ParticleCollection
from fluidsolver_b200 import _lib as F

pytestmark = pytest.mark.gpu


def _both(ns, q, cap=4096):
    L = F.lib()
    pos = np.zeros(3, np.float32)
    pos[:len(q)] = q
    a, b = np.zeros(cap, np.int64), np.zeros(cap, np.int64)
    ca, cb = ctypes.c_int64(-1), ctypes.c_int64(-1)
    F.check(L.fs_query_position(ns.ctx, pos.ctypes.data, a.ctypes.data, cap, ctypes.byref(ca)))
    F.check(L.fs_query_position_noalloc(ns.ctx, pos.ctypes.data, b.ctypes.data, cap, ctypes.byref(cb)))
    return a[:min(ca.value, cap)], ca.value, b[:min(cb.value, cap)], cb.value


@pytest.mark.parametrize("kind,dim", [("hashed-3d", 3), ("compressed-3d", 3), ("quadratic-3d", 3),
                                      ("hashed-2d", 2), ("quadratic-2d", 2)])
def test_noalloc_query_equals_allocating_query(kind, dim):
    rng = np.random.default_rng(21)
    n = 30000 if not kind.startswith("quadratic") else 5000
    pos = (rng.random((n, dim)) * 20).astype(np.float32)
    typ = rng.integers(0, 3, n).astype(np.uint8)
    ns = NeighborhoodSearch(kind, 1.0)
    ns.data.collection = ParticleCollection(position=pos, type=typ)
    ns.find_neighbors()
    queries = (rng.random((8, dim)) * 20).astype(np.float32)
    total = 0
    for q in queries:
        first = second = None
        for call in range(2):   # two calls in a row on the same query
            a, ca, b, cb = _both(ns, q)
            assert ca == cb and a.tolist() == b.tolist(), (kind, call)
            total += cb
            if call == 0:
                first = b.copy()
            else:
                second = b.copy()
        assert first.tolist() == second.tolist()
    assert total > 0
    ns.close()


@pytest.mark.parametrize("kind", ["hashed-3d", "quadratic-3d"])
@pytest.mark.parametrize("precision,reference_order", [("fp32-kahan", False), ("fp32", True), ("fp64", False)])
def test_noalloc_query_in_every_precision(kind, precision, reference_order):
    """The same equality in the three precision modes (FP64 positions take the
    double-precision walk) and with the reference-order layout."""
    rng = np.random.default_rng(22)
    n = 20000 if kind == "hashed-3d" else 4000
    pos = (rng.random((n, 3)) * 15).astype(np.float32)
    typ = rng.integers(0, 3, n).astype(np.uint8)
    ns = NeighborhoodSearch(kind, 1.0, precision=precision, reference_order=reference_order)
    ns.data.collection = ParticleCollection(position=pos, type=typ)
    ns.find_neighbors()
    total = 0
    for q in (rng.random((6, 3)) * 15).astype(np.float32):
        for call in range(2):
            a, ca, b, cb = _both(ns, q)
            assert ca == cb and a.tolist() == b.tolist(), (kind, precision, call)
            total += cb
    assert total > 0
    ns.close()


def test_noalloc_rejects_caps_beyond_the_fixed_array():
    ns = NeighborhoodSearch("compressed-3d", 1.0)
    ns.data.collection = ParticleCollection(position=np.zeros((4, 3), np.float32))
    ns.find_neighbors()
    L = F.lib()
    q = np.zeros(3, np.float32)
    cap = F.FS_QUERY_NOALLOC_MAX + 1
    out = np.zeros(cap, np.int64)
    cnt = ctypes.c_int64(-1)
    st = L.fs_query_position_noalloc(ns.ctx, q.ctypes.data, out.ctypes.data, cap, ctypes.byref(cnt))
    assert st == F.FS_ERR_INVALID
    assert b"65536" in L.fs_last_error()
    # at the limit it runs, and a small cap truncates but reports the full count
    st = L.fs_query_position_noalloc(ns.ctx, q.ctypes.data, out.ctypes.data, F.FS_QUERY_NOALLOC_MAX,
                                     ctypes.byref(cnt))
    assert st == F.FS_OK and cnt.value == 4 and out[:4].tolist() == [0, 1, 2, 3]
    st = L.fs_query_position_noalloc(ns.ctx, q.ctypes.data, out.ctypes.data, 2, ctypes.byref(cnt))
    assert st == F.FS_OK and cnt.value == 4
    ns.close()
