"""The tile passes' prefetch depths (fs_autotune, fs_set_tuning): tuning
leaves the tuned context's state as it was, and the depth changes only when
the list entries are loaded, never the arithmetic, so steps with any depths
are bit-identical."""
import numpy as np
import pytest

from conftest import bits_equal
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
    assert all(x > 0 for x in t["pressure_iteration_ms"]) and sum(x > 0 for x in t["first_loop_ms"]) == 2
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


def test_untiled_modes_report_nothing_to_tune():
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25), precision="fp32",
                    reference_order=True)
    s.data.collection = dam()
    assert not s.autotune()["tuned"]
    with pytest.raises(Exception):
        s.set_tuning(0, 5)
    s.close()
