"""The bounded waits' error path, exercised without faulting the GPU.

The tile passes wait for their staged copies with a bounded number of tries
(fs_tiles.cuh, stage_tile_wait). fs_set_tile_wait_limit(ctx, 0) makes every
such wait give up at once: the step must return FS_ERR_TIMEOUT through the
status word, leave a finite state, and the next step, with the default limit
back, must run normally on the same context."""
import numpy as np
import pytest

from fluidsolver_b200 import IISPHFluidSolver3D, scenes
from fluidsolver_b200 import _lib as F
from fluidsolver_b200._lib import FS_ERR_TIMEOUT, FluidSolverError

pytestmark = pytest.mark.gpu


def _solver():
    sc = scenes.breaking_dam_3d(24, 20, 16, 1.0, tank=(48, 30, 24), seed=71)
    s = IISPHFluidSolver3D(search="hashed-3d", precision="fp32-kahan")
    s.parameters.rest_density, s.parameters.gravity, s.parameters.particle_size = 1.0, 9.81, 1.0
    s.settings.viscosity, s.settings.single_layer_boundary = 0.01, True
    s.timestep_generator.settings.timestep = scenes.REFERENCE_UNITS_DT
    s.data.collection = sc.collection
    return s


def test_a_wait_that_runs_out_returns_timeout_and_the_next_step_runs():
    s = _solver()
    L = F.lib()
    s.step()
    before = s.collection()
    try:
        F.check(L.fs_set_tile_wait_limit(s.ctx, 0))
        with pytest.raises(FluidSolverError) as e:
            s.step()
        assert e.value.status == FS_ERR_TIMEOUT
    finally:
        F.check(L.fs_set_tile_wait_limit(s.ctx, -1))
    mid = s.collection()
    assert np.isfinite(mid.position).all() and np.isfinite(mid.velocity).all()
    # the passes skipped their tiles: nothing moved further than one step could carry it
    assert np.max(np.abs(mid.position - before.position)) < 1.0
    st = s.step()
    assert st.status == 0 and 2 <= st.iterations <= 100
    assert np.isfinite(s.collection().position).all()
    s.close()


def test_the_default_limit_is_restored_for_other_contexts():
    """The limit belongs to the device: a context created after the reset
    steps normally."""
    s = _solver()
    F.check(F.lib().fs_set_tile_wait_limit(s.ctx, -1))
    assert s.step().status == 0
    s.close()
