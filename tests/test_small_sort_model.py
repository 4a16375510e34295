"""A host model of the small-scene kernel's cluster-wide sort
(csrc/fs_small.cu, sort_small_cluster), checked against numpy's stable sort.

The device sort splits n <= 4,096 (key, index) pairs into one contiguous
share per block of the cluster, turns each pair into the unique word
(key masked to whole bytes << 12 | index), places each word of a share by
the number of the share's words below it, and then places it in the output
by the sum over all shares of the words below it (a binary search per
share, skipped for shares that lie wholly below or above the word). These
tests pin that arithmetic on the host: the result is a stable sort by the
masked key, for every cluster size the launch can choose and for the key
widths the kernel sees. The device kernel itself is compared bit for bit
with the step-by-step path and the reference on the GPU
(tests/test_gpu_small.py, tests/test_gpu_configs.py)."""
import numpy as np
import pytest

MAX_PARTICLES = 4096   # kSmallMax: the words' index field has 12 bits


def cluster_sort_model(keys, bits, blocks):
    n = len(keys)
    share = -(-n // blocks)
    rbits = (bits + 7) // 8 * 8
    mask = (1 << min(rbits, 64)) - 1
    words = [((int(k) & mask) << 12) | i for i, k in enumerate(keys)]
    assert all(w < (1 << 64) for w in words)
    runs = []
    for q in range(blocks):
        lo, hi = min(n, q * share), min(n, (q + 1) * share)
        part = words[lo:hi]
        run = [0] * len(part)
        for v in part:
            run[sum(1 for u in part if u < v)] = v
        runs.append(run)
    out = [None] * n
    for run in runs:
        for v in run:
            rank = 0
            for other in runs:
                if not other or v < other[0]:
                    continue
                if v > other[-1]:
                    rank += len(other)
                    continue
                rank += int(np.searchsorted(np.array(other, dtype=object), v))
            out[rank] = v
    return [w & 0xFFF for w in out]


@pytest.mark.parametrize("blocks", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("bits", [14, 29, 34])
def test_cluster_sort_model_is_a_stable_sort(blocks, bits):
    rng = np.random.default_rng(blocks * 100 + bits)
    for n in (2, 3, 37, 300):
        # nearly sorted keys with duplicates (the last step's order), and
        # random ones
        base = np.sort(rng.integers(0, 1 << bits, n, dtype=np.uint64))
        swaps = rng.integers(0, n, (n // 8, 2))
        for a, b in swaps:
            base[a], base[b] = base[b], base[a]
        for keys in (base, rng.integers(0, 1 << min(bits, 6), n, dtype=np.uint64)):
            order = cluster_sort_model(keys, bits, blocks)
            ref = np.argsort(keys, kind="stable")
            assert order == ref.tolist(), (n, blocks, bits)


def test_key_bits_above_the_byte_rounded_width_are_ignored():
    """sort_small_block orders by whole 8-bit digits: bits above the rounded
    width do not take part, in the model as on the device."""
    keys = np.array([(1 << 20) | 5, 3, 5, (1 << 21) | 3], dtype=np.uint64)
    order = cluster_sort_model(keys, 14, 2)   # 14 bits -> 16 bits sorted
    assert order == [1, 3, 0, 2]


def test_the_largest_scene_fits_the_index_field():
    """4,096 particles on 16 blocks: every index fits the 12-bit field."""
    rng = np.random.default_rng(7)
    keys = rng.integers(0, 1 << 12, MAX_PARTICLES, dtype=np.uint64)
    order = cluster_sort_model(keys, 14, 16)
    assert order == np.argsort(keys, kind="stable").tolist()


@pytest.mark.parametrize("regions", [1, 2, 3])
def test_binary_searched_cell_table_equals_the_scanned_counts(regions):
    """The small-scene kernel's cell-start table: entry t (region g, cell c
    at t = g (cells + 1) + c) is the first sorted index whose key's entry is
    >= t, found by binary search; the step-by-step path writes each run's
    length at its first particle's entry and scans the table. Same table."""
    rng = np.random.default_rng(regions)
    cells, key_bits = 700, 10
    for n in (0, 1, 50, 3000):
        g = rng.integers(0, regions, n)
        c = rng.integers(0, cells, n)
        keys = np.sort((g << key_bits) | c)
        te = (keys >> key_bits) * (cells + 1) + (keys & ((1 << key_bits) - 1))
        table = regions * (cells + 1)
        counts = np.zeros(table, np.int64)
        for t in te:
            counts[t] += 1
        scanned = np.concatenate([[0], np.cumsum(counts)[:-1]])
        searched = np.searchsorted(te, np.arange(table), side="left")
        assert np.array_equal(scanned, searched)
