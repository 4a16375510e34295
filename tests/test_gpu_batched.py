"""Batched 3D IISPH scenes (fs_batch_create / fs_batch_run): each scene of a
batch must evolve as it does when it runs alone through the same solver,
with its own convergence test and time step."""
import ctypes

import numpy as np
import pytest

from fluidsolver_b200 import BatchedIISPHFluidSolver3D, IISPHFluidSolver3D, scenes
from fluidsolver_b200 import _lib as F
from fluidsolver_b200.scenes import REFERENCE_UNITS_DT

pytestmark = pytest.mark.gpu


def _configure(s):
    s.parameters.rest_density = 1.0
    s.parameters.gravity = 9.81
    s.parameters.particle_size = 1.0
    s.settings.viscosity = 0.01
    s.settings.single_layer_boundary = True
    s.settings.single_layer_boundary_gamma_1 = 1.1
    s.settings.max_density_error_allowed = 0.001
    s.settings.min_number_of_iterations = 2
    s.settings.max_number_of_iterations = 100
    s.settings.omega = 0.5
    s.settings.gamma = 0.7
    s.timestep_generator.settings.timestep = REFERENCE_UNITS_DT


def _scenes(count, seed, f_min=800, f_max=6000):
    return scenes.batched_dams(count, seed=seed, f_min=f_min, f_max=f_max)


def _alone(scene, steps):
    s = IISPHFluidSolver3D(search="hashed-3d", precision="fp32-kahan")
    _configure(s)
    s.data.collection = scene.collection
    iters, dts = [], []
    for _ in range(steps):
        st = s.step()   # the solver's own stats object, overwritten by every step
        iters.append(int(st.iterations))
        dts.append(float(st.actual_dt))
    out = s.collection()
    s.close()
    return out, iters, dts


@pytest.mark.parametrize("count,seed", [(5, 11), (17, 12)])
def test_batched_scenes_match_scenes_run_alone(count, seed):
    sc = _scenes(count, seed)
    steps = 6
    batch = BatchedIISPHFluidSolver3D([s.collection for s in sc])
    _configure(batch)
    per_step = [batch.run(1) for _ in range(steps)]
    got = batch.collections()
    batch.close()
    for i, scene in enumerate(sc):
        ref, iters, dts = _alone(scene, steps)
        b_iters = [int(st[i].iterations) for st in per_step]
        b_dts = [float(st[i].actual_dt) for st in per_step]
        assert all(abs(x - y) <= 1 for x, y in zip(b_iters, iters)), (i, b_iters, iters)
        np.testing.assert_allclose(b_dts, dts, rtol=1e-5)
        scale = np.abs(ref.position).max()
        np.testing.assert_allclose(got[i].position, ref.position, rtol=0, atol=1e-5 * scale)
        vscale = max(np.abs(ref.velocity).max(), 1e-3)
        np.testing.assert_allclose(got[i].velocity, ref.velocity, rtol=0, atol=1e-4 * vscale)
        np.testing.assert_allclose(got[i].density, ref.density, rtol=1e-5, atol=0)
        assert (got[i].type == scene.collection.type).all()


def test_batched_run_equals_repeated_single_steps():
    sc = _scenes(9, 13)
    a = BatchedIISPHFluidSolver3D([s.collection for s in sc])
    b = BatchedIISPHFluidSolver3D([s.collection for s in sc])
    _configure(a)
    _configure(b)
    st_a = a.run(5)
    for _ in range(5):
        st_b = b.run(1)
    ca, cb = a.collections(), b.collections()
    for x, y in zip(ca, cb):
        assert np.array_equal(x.position, y.position)
        assert np.array_equal(x.velocity, y.velocity)
    assert [s.iterations for s in st_a] == [s.iterations for s in st_b]
    a.close()
    b.close()


def test_batched_scenes_keep_their_own_convergence():
    sc = _scenes(12, 14, f_min=500, f_max=20000)
    batch = BatchedIISPHFluidSolver3D([s.collection for s in sc])
    _configure(batch)
    batch.run(3)
    st = batch.run(1)
    iters = [int(s.iterations) for s in st]
    errs = [float(s.avg_density_error_fp64) for s in st]
    assert all(i >= 2 for i in iters)
    # every scene either converged below the bound or hit the cap
    assert all(e <= 0.001 + 1e-9 or i == 100 for e, i in zip(errs, iters))
    batch.close()


def test_batched_contexts_reject_what_they_do_not_support():
    L = F.lib()
    p = F.FsParams()
    L.fs_params_default(ctypes.byref(p), 3, F.FS_SOLVER_SESPH_3D, F.FS_SEARCH_HASHED_3D)
    p.max_particles = 10
    off = np.array([0, 4, 10], np.int64)
    ctx = ctypes.c_void_p()
    assert L.fs_batch_create(ctypes.byref(p), 2, off.ctypes.data, ctypes.byref(ctx)) == F.FS_ERR_INVALID
    L.fs_params_default(ctypes.byref(p), 3, F.FS_SOLVER_IISPH_3D, F.FS_SEARCH_HASHED_3D)
    bad = np.array([0, 6, 4], np.int64)
    assert L.fs_batch_create(ctypes.byref(p), 2, bad.ctypes.data, ctypes.byref(ctx)) == F.FS_ERR_INVALID
    sc = _scenes(2, 15)
    batch = BatchedIISPHFluidSolver3D([s.collection for s in sc])
    _configure(batch)
    batch.run(1)
    q = np.zeros(3, np.float32)
    out = np.zeros(16, np.int64)
    cnt = ctypes.c_int64()
    assert L.fs_query_position(batch.ctx, q.ctypes.data, out.ctypes.data, 16, ctypes.byref(cnt)) == F.FS_ERR_INVALID
    one = sc[0].collection.normalized()
    assert L.fs_upload(batch.ctx, ctypes.byref(one.as_fs())) == F.FS_ERR_INVALID
    batch.close()
