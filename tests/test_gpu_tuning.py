"""The fast mode's launch shapes (fs_autotune, fs_set_tuning): tuning leaves
the tuned context's state as it was and reports a time for every value it
tried. The prefetch depth changes only when list entries are loaded, and the
per-particle kernels' block size only how they are launched, never the
arithmetic: steps are bit-identical under any of them. The staging cap
decides which tiles fall back to 32-bit lists, whose owners split their
lists between their two threads differently, and the threads per owner of
the pressure passes decide how an owner's sums are split: the neighbor sets
stay the contract's and the results agree to rounding."""
import numpy as np
import pytest

from conftest import bits_equal
from fluidsolver_b200 import _lib as F
from fluidsolver_b200 import scenes
from test_gpu_solvers import make_solver, simulator_step

pytestmark = pytest.mark.gpu

SETTINGS_3D = [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1]
FIELDS = ("position", "velocity", "density", "pressure", "acceleration", "mass")


def dam():
    return scenes.breaking_dam_3d(30, 24, 20, 1.0, tank=(80, 50, 40), seed=13).collection


def test_autotune_keeps_the_state_and_picks_valid_depths():
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    s.data.collection = dam()
    for _ in range(2):
        simulator_step(s)
    before = s.collection()
    t = s.autotune()
    after = s.collection()
    for f in FIELDS:
        assert bits_equal(getattr(before, f), getattr(after, f)), f
    assert t["tuned"] and 1 <= t["first_loop_prefetch"] <= 4 and 1 <= t["pressure_prefetch"] <= 4
    assert sorted(t["pressure_iteration_ms"]) == [1, 2, 3, 4] and sorted(t["first_loop_ms"]) == [1, 2]
    assert all(v > 0 for v in t["pressure_iteration_ms"].values())
    assert t["tile_cap"] in F.TILE_CAPS and sorted(t["step_ms_by_tile_cap"]) == list(F.TILE_CAPS)
    assert t["block_size"] in F.BLOCK_SIZES and sorted(t["step_ms_by_block_size"]) == list(F.BLOCK_SIZES)
    assert t["pressure_threads_per_owner"] in F.THREADS_PER_OWNER
    assert sorted(t["pressure_iteration_ms_by_threads"]) == list(F.THREADS_PER_OWNER)
    fb = [t["fallback_tiles_by_tile_cap"][c] for c in F.TILE_CAPS]
    assert all(0.0 <= x <= 1.0 for x in fb) and fb == sorted(fb, reverse=True)
    simulator_step(s)   # the tuned context steps on
    s.close()


def test_prefetch_depths_do_not_change_results():
    runs = []
    for l1, pr in ((1, 1), (2, 4), (1, 3)):
        s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
        s.data.collection = dam()
        s.set_tuning(l1, pr)
        for _ in range(3):
            s.step()
        runs.append(s.collection())
        s.close()
    for other in runs[1:]:
        for f in FIELDS:
            assert bits_equal(getattr(runs[0], f), getattr(other, f)), f


def test_block_size_does_not_change_results():
    runs = []
    for b in F.BLOCK_SIZES:
        s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
        s.data.collection = dam()
        s.set_tuning(1, 3, block_size=b)
        for _ in range(3):
            s.step()
        runs.append(s.collection())
        s.close()
    for other in runs[1:]:
        for f in FIELDS:
            assert bits_equal(getattr(runs[0], f), getattr(other, f)), f


def test_tile_cap_keeps_the_sets_and_the_results_to_rounding():
    runs, lists = [], []
    for cap in F.TILE_CAPS:
        s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
        s.data.collection = dam()
        s.set_tuning(1, 3, tile_cap=cap)
        s.execute_neighborhood_search()
        lists.append(s.solver_lists())
        for _ in range(3):
            s.step()
        runs.append(s.collection())
        s.close()
    for (o, i) in lists[1:]:
        assert np.array_equal(o, lists[0][0]) and np.array_equal(i, lists[0][1])
    for other in runs[1:]:
        for f in ("position", "density"):
            a, b = getattr(runs[0], f).astype(np.float64), getattr(other, f).astype(np.float64)
            assert np.max(np.abs(a - b)) <= 1e-5 * np.max(np.abs(a)), f


def test_threads_per_owner_keep_the_results_to_rounding():
    """1, 2 or 4 threads walk each owner's list in the pressure passes: the
    same pairs summed in other groupings, so the steps agree to rounding, with
    the same iteration counts. Positions and densities agree to 1e-5 of their
    largest magnitude; the pressures to 1e-4, since they are relaxed-Jacobi
    iterates stopped by the density-error test, and each iteration divides
    its rounding-level change of A p by the small diagonal a_ii (measured on a
    B200: 4e-5 after three steps)."""
    runs, its = [], []
    for tpo in F.THREADS_PER_OWNER:
        s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
        s.data.collection = dam()
        s.set_tuning(1, 3, pressure_threads_per_owner=tpo)
        its.append([int(s.step().iterations) for _ in range(3)])
        runs.append(s.collection())
        s.close()
    assert its[0] == its[1] == its[2]
    for other in runs[1:]:
        for f, tol in (("position", 1e-5), ("density", 1e-5), ("pressure", 1e-4)):
            a, b = getattr(runs[1], f).astype(np.float64), getattr(other, f).astype(np.float64)
            assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(a)), f


def test_invalid_shapes_are_rejected():
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    s.data.collection = dam()
    for kw in ({"tile_cap": 100}, {"tile_cap": 4096}, {"tile_cap": 1030}, {"block_size": 48}, {"block_size": 2048},
               {"pressure_threads_per_owner": 3}, {"pressure_threads_per_owner": 8}):
        with pytest.raises(Exception):
            s.set_tuning(1, 3, **kw)
    s.close()


def test_untiled_modes_report_nothing_to_tune():
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25), precision="fp32",
                    reference_order=True)
    s.data.collection = dam()
    assert not s.autotune()["tuned"]
    with pytest.raises(Exception):
        s.set_tuning(0, 5)
    s.close()
