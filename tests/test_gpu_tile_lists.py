"""The lists the 3D IISPH fast path walks (tile lists, fs_tiles.cuh) hold
exactly the contract's neighbor sets (hashed 3D: every particle of the 27
cells with dot(d, d) <= r^2, HashedNeighborhoodSearch3D.cpp:12-110).

The tile builder leaves out cells whose box lies farther than r from the
owner; these tests compare its lists, decoded through the tile ranges, with
the search's own CSR export (itself checked against the oracle in
test_gpu_search.py), on scenes that put particles exactly on cell faces,
far from the origin, and in motion.
"""
import dataclasses

import numpy as np
import pytest

from fluidsolver_b200 import scenes
from fluidsolver_b200.solver import ParticleCollection
from test_gpu_solvers import make_solver, simulator_step

pytestmark = pytest.mark.gpu

SETTINGS = [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1]


def solver_for(col):
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS, (scenes.REFERENCE_UNITS_DT, 0.4, 0.25))
    s.data.collection = col
    return s


def assert_lists_equal(s):
    """The contract lists every active particle's neighbors; the solver walks
    lists of its fluid owners only, and they must be the contract's."""
    off_c, idx_c = s.neighbor_lists()
    off_s, idx_s = s.solver_lists()
    fluid = s.data.collection.type == 0
    len_c, len_s = np.diff(off_c), np.diff(off_s)
    assert (len_s[~fluid] == 0).all()
    assert np.array_equal(len_c[fluid], len_s[fluid]) and len_s.sum() > 0
    own_c = np.repeat(fluid, len_c)
    assert np.array_equal(idx_c[own_c], idx_s)


def shifted(col: ParticleCollection, by) -> ParticleCollection:
    return dataclasses.replace(col, position=(col.position + np.asarray(by, np.float32)).astype(np.float32))


@pytest.mark.parametrize("jitter", [0.0, 0.01])
def test_tile_lists_equal_the_contract_on_a_dam(jitter):
    # jitter 0: every fluid particle sits on a lattice of spacing 1 with cells
    # of size 2, so half of them lie exactly on cell faces and many pairs are
    # exactly r apart (dot(d, d) == r^2 is a neighbor)
    sc = scenes.breaking_dam_3d(40, 30, 30, 1.0, tank=(120, 70, 45), jitter_frac=jitter, seed=11)
    s = solver_for(sc.collection)
    s.execute_neighborhood_search()
    assert_lists_equal(s)
    for _ in range(4):
        simulator_step(s)
    s.execute_neighborhood_search()
    assert_lists_equal(s)
    s.close()


@pytest.mark.parametrize("offset", [(1000.0, -500.0, 250.0), (-4096.0, 8192.0, -2048.0)])
def test_tile_lists_equal_the_contract_far_from_the_origin(offset):
    # large coordinates: cell coordinates floor(x / r) and face positions carry
    # rounding errors of ~1e-3, which the builder's pruning margin must cover
    sc = scenes.breaking_dam_3d(32, 24, 24, 1.0, tank=(100, 60, 40), jitter_frac=0.0, seed=12)
    s = solver_for(shifted(sc.collection, offset))
    s.execute_neighborhood_search()
    assert_lists_equal(s)
    for _ in range(3):
        simulator_step(s)
    s.execute_neighborhood_search()
    assert_lists_equal(s)
    s.close()


def test_tile_lists_equal_the_contract_at_1m():
    sc = scenes.dam_1m()
    s = solver_for(sc.collection)
    for _ in range(2):
        simulator_step(s)
    s.execute_neighborhood_search()
    assert_lists_equal(s)
    s.close()
