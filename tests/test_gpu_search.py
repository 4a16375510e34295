"""GPU neighborhood-search parity: the device search (through the C-ABI)
against the reference's googletest expectations, the golden fixtures made
from the reference's own sources, and the C oracle. Neighbor lists must be
bit-exact as sorted index sets."""
import numpy as np
import pytest

from conftest import csr_sets, sorted_csr
from fluidsolver_b200 import NeighborhoodSearch, ParticleCollection, scenes
from fluidsolver_b200._lib import FS_ERR_CAPACITY, FluidSolverError

pytestmark = pytest.mark.gpu


def run_search(kind, pos, radius, typ=None):
    ns = NeighborhoodSearch(kind, radius)
    ns.data.collection = ParticleCollection(position=np.asarray(pos, np.float32), type=typ)
    ns.find_neighbors()
    off, idx = ns.neighbor_lists()
    ns.close()
    return off, idx


def same_sets(off, idx, ro, ri):
    return [s.tolist() for s in csr_sets(off, idx)] == [s.tolist() for s in csr_sets(ro, ri)]


@pytest.mark.parametrize("kind", ["quadratic-2d", "hashed-2d", "compact-hashing-2d"])
def test_googletest_grids(golden, kind):
    g = golden["search"]
    for name in ("grid11", "grid11x2"):
        off, idx = run_search(kind, g[f"{name}_quadratic-2d_pos"], float(g[f"{name}_quadratic-2d_r"]))
        assert idx[off[0]:off[1]].tolist() == [0, 1, 2, 11, 12, 22]
        assert idx[off[38]:off[39]].tolist() == [16, 26, 27, 28, 36, 37, 38, 39, 40, 48, 49, 50, 60]
        if kind != "compact-hashing-2d":
            assert same_sets(off, idx, g[f"{name}_{kind}_off"], g[f"{name}_{kind}_idx"])
    off, idx = run_search(kind, g["grid3_quadratic-2d_pos"], 2.0)
    assert idx[off[4]:off[5]].tolist() == list(range(9))
    assert idx[off[0]:off[1]].tolist() == [0, 1, 2, 3, 4, 6]


def test_single_particle():
    for kind in ("quadratic-2d", "hashed-2d"):
        off, idx = run_search(kind, [[234.56341, 6578.45]], 2.0)
        assert idx.tolist() == [0]
    off, idx = run_search("hashed-3d", [[1e3, -2e3, 5.5]], 2.0)
    assert idx.tolist() == [0]


def test_moving_grid_1024_steps(golden):
    # NeighborhoodSearchTests.cpp:301-354 (r = 2.01)
    pos = golden["search"]["grid11_quadratic-2d_pos"].copy()
    ns = NeighborhoodSearch("hashed-2d", 2.01)
    ns.data.collection = ParticleCollection(position=pos.copy())
    mv = np.array([0.34, -0.5], np.float32)
    for step in range(1024):
        pos += mv
        ns.set_positions(pos)
        ns.find_neighbors()
        if step % 16 == 15 or step < 4:
            off, idx = ns.neighbor_lists()
            assert idx[off[0]:off[1]].tolist() == [0, 1, 2, 11, 12, 22], step
            assert idx[off[38]:off[39]].tolist() == [16, 26, 27, 28, 36, 37, 38, 39, 40, 48, 49, 50, 60], step
    ns.close()


@pytest.mark.parametrize("kind", ["hashed-3d", "quadratic-3d", "compressed-3d"])
def test_3d_with_inactive_particles(golden, kind):
    g = golden["search"]
    off, idx = run_search(kind, g["dam3d_pos"], 2.0, g["dam3d_type"])
    assert same_sets(off, idx, g[f"dam3d_{kind}_off"], g[f"dam3d_{kind}_idx"])


@pytest.mark.parametrize("kind", ["quadratic-2d", "hashed-2d"])
def test_2d_with_inactive_particles(golden, kind):
    g = golden["search"]
    off, idx = run_search(kind, g["dam2d_pos"], 2.0, g["dam2d_type"])
    assert same_sets(off, idx, g[f"dam2d_{kind}_off"], g[f"dam2d_{kind}_idx"])


def test_uniform_random_points(golden):
    g = golden["search"]
    for kind in ("hashed-3d", "compressed-3d"):
        off, idx = run_search(kind, g["rand_pos"], 0.1)
        assert same_sets(off, idx, g[f"rand_{kind}_off"], g[f"rand_{kind}_idx"])


def test_compressed_capacity_is_reported(golden):
    # the reference terminates the process above 97 neighbors; the device path reports it
    g = golden["search"]
    assert int(g["blob_compressed_exit"]) != 0
    with pytest.raises(FluidSolverError) as e:
        run_search("compressed-3d", g["blob_pos"], 0.1)
    assert e.value.status == FS_ERR_CAPACITY
    off, idx = run_search("hashed-3d", g["blob_pos"], 0.1)   # no capacity limit there
    assert np.max(np.diff(off)) > 97


def test_coincident_particles():
    pos = np.zeros((50, 3), np.float32)
    pos[25:] = 7.0
    off, idx = run_search("hashed-3d", pos, 0.5)
    for i in range(50):
        assert idx[off[i]:off[i + 1]].tolist() == (list(range(25)) if i < 25 else list(range(25, 50)))


def test_empty_collection():
    off, idx = run_search("hashed-3d", np.zeros((0, 3), np.float32), 2.0)
    assert off.tolist() == [0] and len(idx) == 0


def test_far_apart_clusters_exceed_the_cell_grid(c_oracle):
    # clusters 1e5 radii apart: the cell grid clamps, the sets stay exact
    rng = np.random.default_rng(9)
    a = rng.random((3000, 3)).astype(np.float32) * 4
    b = a + np.float32(2.0e5)
    pos = np.concatenate([a, b, -b])
    off, idx = run_search("hashed-3d", pos, 0.5)
    ro, ri, _ = c_oracle.search("hashed-3d", pos, 0.5)
    assert same_sets(off, idx, ro, ri)


def test_compact_hashing_on_a_sparse_domain(c_oracle):
    """Compact hashing's hashed cell table (CompactHashingNeighborhoodSearch.cpp:342-349):
    four clusters millions of radii apart, with boundary and inactive
    particles. A dense grid over that extent would clamp nearly every
    particle into a border cell; the table holds only the occupied cells, and
    the sets equal the oracle's (active owners and candidates, <= 40)."""
    rng = np.random.default_rng(10)
    a = (rng.random((4000, 2)) * 30).astype(np.float32)
    pos = np.concatenate([a, a + np.float32(3.0e6), a - np.float32(5.0e5),
                          a + np.array([1.0e6, -2.0e6], np.float32)]).astype(np.float32)
    typ = rng.choice(np.array([0, 0, 0, 1, 2], np.uint8), len(pos))
    off, idx = run_search("compact-hashing-2d", pos, 1.0, typ)
    ro, ri, ok = c_oracle.search("compact-hashing-2d", pos, 1.0, typ)
    assert ok
    assert np.array_equal(off, ro)
    assert np.array_equal(idx, sorted_csr(ro, ri)[1])
    assert off[-1] > 5 * len(pos)


def test_compact_hashing_capacity_is_reported():
    # more than 40 neighbors: the reference throws (CompactHashingNeighborhoodSearch.cpp:5, 210-247)
    pos = (np.random.default_rng(11).random((200, 2)) * 2).astype(np.float32)
    with pytest.raises(FluidSolverError) as e:
        run_search("compact-hashing-2d", pos, 1.0)
    assert e.value.status == FS_ERR_CAPACITY


@pytest.mark.parametrize("kind", ["hashed-3d", "compressed-3d"])
def test_uniform_1m_points_match_oracle(c_oracle, kind):
    # the 3D search microbenchmark's uniform case at full size: 1,000,000 points
    pos = scenes.ns_points_uniform()
    off, idx = run_search(kind, pos, 0.02)
    ro, ri, ok = c_oracle.search(kind, pos, 0.02)
    assert ok
    assert np.array_equal(off, ro)
    assert np.array_equal(idx, sorted_csr(ro, ri)[1])


def test_gaussian_blobs_match_oracle(c_oracle):
    # the microbenchmark's clustered case (64 blobs, sigma 0.03), 200,000 points
    pos = scenes.ns_points_blobs(n=200_000)
    off, idx = run_search("hashed-3d", pos, 0.02)
    ro, ri, _ = c_oracle.search("hashed-3d", pos, 0.02)
    assert np.array_equal(off, ro)
    assert np.array_equal(idx, sorted_csr(ro, ri)[1])


@pytest.mark.parametrize("dim,kind", [(3, "hashed-3d"), (3, "quadratic-3d"), (3, "compressed-3d"), (2, "hashed-2d"),
                                      (2, "quadratic-2d")])
def test_position_queries_match_reference(golden, dim, kind):
    """get_neighbors(position) of every contract against the reference's
    (fixtures from its sources): inactive particles, the length/dot
    predicates and hashed-3d's skipped cell minimum."""
    g = golden["position_queries"]
    pos, typ, queries = g[f"pos{dim}"], g[f"type{dim}"], g[f"queries{dim}"]
    off, idx = g[f"{kind}/offsets"], g[f"{kind}/indices"]
    ns = NeighborhoodSearch(kind, 1.0)
    ns.data.collection = ParticleCollection(position=pos, type=typ)
    ns.find_neighbors()
    for i, q in enumerate(queries):
        assert ns.get_neighbors_of_position(q).tolist() == idx[off[i]:off[i + 1]].tolist(), (kind, i)
    ns.close()


def test_position_queries_at_scale(c_oracle):
    """20k points: the device query against the oracle's restatement."""
    rng = np.random.default_rng(4)
    pos = rng.random((20000, 3)).astype(np.float32)
    ns = NeighborhoodSearch("hashed-3d", 0.05)
    ns.data.collection = ParticleCollection(position=pos)
    ns.find_neighbors()
    for q in rng.random((20, 3)).astype(np.float32):
        assert ns.get_neighbors_of_position(q).tolist() == c_oracle.query_position("hashed-3d", pos, 0.05, q).tolist()
    ns.close()


def test_compact_hashing_position_query_is_rejected():
    ns = NeighborhoodSearch("compact-hashing-2d", 1.0)
    ns.data.collection = ParticleCollection(position=np.zeros((4, 2), np.float32))
    ns.find_neighbors()
    with pytest.raises(FluidSolverError):
        ns.get_neighbors_of_position(np.zeros(2, np.float32))
    ns.close()
