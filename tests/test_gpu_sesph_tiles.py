"""3D SESPH in the fast mode runs on tile lists (fs_tiles.cuh:
k_tile_sesph3d_density, k_tile_sesph3d_accel; the formulas of
SESPHFluidSolver3D.hpp:49-130).

The lists it walks are the contract's neighbor sets, and over several steps
its results stay within the reference's own float error of an FP64 build: the
FP32 reference-order mode is bit-identical to the reference (tested in
test_gpu_solvers.py), so its distance to FP64 is that error, and the fast mode
may exceed it by 1e-5 of each field's scale, the bar of
test_kahan_within_tolerance_of_reference."""
import numpy as np
import pytest

from fluidsolver_b200 import scenes
from test_gpu_solvers import make_solver, simulator_step
from test_gpu_tile_lists import assert_lists_equal

pytestmark = pytest.mark.gpu

SETTINGS = [1000.0, 0.01, 1.0, 1.1, 1.1]   # stiffness, viscosity, single layer, gamma 1, gamma 2
GEN = (0.001, 0.4, 0.25)


def dam(seed=61):
    return scenes.breaking_dam_3d(30, 24, 20, 1.0, tank=(60, 40, 30), seed=seed)


def run(precision, steps, reference_order=False, settings=SETTINGS):
    s = make_solver("sesph-3d", "hashed-3d", settings, GEN, precision=precision, reference_order=reference_order)
    s.data.collection = dam().collection
    for _ in range(steps):
        simulator_step(s)
    out = s.collection()
    s.close()
    return out


def test_sesph3d_walks_the_contract_lists():
    s = make_solver("sesph-3d", "hashed-3d", SETTINGS, GEN)
    s.data.collection = dam().collection
    s.execute_neighborhood_search()
    assert_lists_equal(s)
    for _ in range(3):
        simulator_step(s)
    s.execute_neighborhood_search()
    assert_lists_equal(s)
    s.close()


@pytest.mark.parametrize("single_layer", [True, False])
def test_sesph3d_tiles_within_the_reference_float_error(single_layer):
    settings = list(SETTINGS)
    settings[2] = 1.0 if single_layer else 0.0
    steps = 5
    fast = run("fp32-kahan", steps, settings=settings)
    ref = run("fp32", steps, reference_order=True, settings=settings)
    exact = run("fp64", steps, settings=settings)
    for f in ("position", "velocity", "density", "pressure"):
        e = getattr(exact, f).astype(np.float64)
        envelope = np.max(np.abs(getattr(ref, f).astype(np.float64) - e))
        slack = 1e-5 * max(float(np.max(np.abs(e))), 1e-30)
        err = np.max(np.abs(getattr(fast, f).astype(np.float64) - e))
        assert err <= envelope + slack, (f, err, envelope, slack)
    # the fluid is in motion (5 steps of 0.001 under gravity: |v| ~ 0.05), so
    # the comparison is not of a scene at rest
    assert np.max(np.abs(fast.velocity)) > 1e-2
