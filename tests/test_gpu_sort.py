"""The searches' own radix sort (csrc/fs_sort.cuh) on the
device, through fs_sort_keys, against numpy's stable sort: the same keys in
the same order and the same permutation (equal keys in input order), for
both key widths, both code paths (one block up to 4,096 keys, the three
kernels per digit above), digit counts that do and do not divide the key
width, and the key patterns of the search (nearly sorted runs of cells,
heavy duplicates, all keys equal)."""
import numpy as np
import pytest

from fluidsolver_b200.solver import sort_keys

pytestmark = pytest.mark.gpu


def expect(keys):
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    return keys[order], order


SIZES = [0, 1, 2, 31, 1000, 4095, 4096, 4097, 5000, 65_537, 1_000_003]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("bits", [5, 8, 17, 24, 32])
def test_uint32_keys(n, bits):
    rng = np.random.default_rng(n * 100 + bits)
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
    got_k, got_o = sort_keys(keys, bits)
    want_k, want_o = expect(keys)
    assert np.array_equal(got_k, want_k)
    assert np.array_equal(got_o, want_o)


@pytest.mark.parametrize("n", [3000, 300_000])
@pytest.mark.parametrize("bits", [40, 64])
def test_uint64_keys(n, bits):
    """The reference-order mode's keys: (region, cell) above, the order inside a cell below."""
    rng = np.random.default_rng(n + bits)
    hi = rng.integers(0, 1 << (bits - 32), n, dtype=np.uint64)
    lo = rng.integers(0, 1 << 32, n, dtype=np.uint64)
    keys = (hi << np.uint64(32)) | lo
    got_k, got_o = sort_keys(keys, bits)
    want_k, want_o = expect(keys)
    assert np.array_equal(got_k, want_k)
    assert np.array_equal(got_o, want_o)


@pytest.mark.parametrize("n", [4000, 1_000_000])
def test_search_like_keys(n):
    """Cells of the previous step's order with a few percent of particles moved one cell:
    runs of duplicates, nearly sorted; and the degenerate case of every key equal."""
    rng = np.random.default_rng(7)
    cells = np.sort(rng.integers(0, n // 8, n)).astype(np.uint32)
    moved = rng.random(n) < 0.05
    cells[moved] += rng.integers(0, 3, int(moved.sum())).astype(np.uint32)
    got_k, got_o = sort_keys(cells, 22)
    want_k, want_o = expect(cells)
    assert np.array_equal(got_k, want_k) and np.array_equal(got_o, want_o)
    same = np.full(n, 12345, np.uint32)
    got_k, got_o = sort_keys(same, 14)
    assert np.array_equal(got_o, np.arange(n, dtype=np.uint32)) and np.all(got_k == 12345)
