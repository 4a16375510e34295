"""The dynamic CFL time step generator on the device
(DynamicCflTimestepGenerator.cpp:6-107): the desired time step of every step
equals the oracle's generator over the state the step starts from -- the
oracle is pinned against the reference's own generator in test_oracle.py --,
and so it can run inside multi-step CUDA graphs (fs_run) and per scene in a
batch. The bit-exact comparison with libFluid's IISPHFluidSolver3D driven by
that generator is in tests/cpp/dropin_test.cpp."""
import numpy as np
import pytest

from conftest import bits_equal
from fluidsolver_b200 import BatchedIISPHFluidSolver3D, DynamicCflTimestepGenerator, scenes
from test_gpu_solvers import make_solver, simulator_step

pytestmark = pytest.mark.gpu

SETTINGS_3D = [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1]


def dynamic(s, lo=0.0001, hi=0.05, lv=0.4, la=0.25):
    g = DynamicCflTimestepGenerator()
    g.settings.min_timestep, g.settings.max_timestep = lo, hi
    g.settings.lambda_v, g.settings.lambda_a = lv, la
    s.timestep_generator = g
    return g


def moving_dam(seed=3):
    sc = scenes.breaking_dam_3d(20, 16, 12, 1.0, tank=(60, 40, 30), seed=seed)
    col = sc.collection
    rng = np.random.default_rng(seed)
    fluid = col.type == 0
    col.velocity = np.zeros_like(col.position)
    col.velocity[fluid] = rng.uniform(-1.5, 1.5, (int(fluid.sum()), 3)).astype(np.float32)
    col.acceleration = np.zeros_like(col.position)
    col.acceleration[fluid] = [0.0, -9.81, 0.0]
    return col


def expected_dt(c_oracle, s, g):
    st = g.settings
    col = s.collection()
    return np.float32(c_oracle.dynamic_timestep(col.velocity, col.acceleration, col.type,
                                                s.parameters.particle_size, st.min_timestep, st.max_timestep,
                                                st.lambda_v, st.lambda_a))


@pytest.mark.parametrize("precision", ["fp32-kahan", "fp32"])
def test_iisph3d_desired_dt_is_the_generators(c_oracle, precision):
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25), precision=precision)
    g = dynamic(s)
    s.data.collection = moving_dam()
    seen = set()
    for _ in range(8):
        s.initialize()
        want = expected_dt(c_oracle, s, g)
        tp = simulator_step(s)
        assert bits_equal(np.float32(s.last_stats.desired_dt), want)
        assert np.float32(tp.desired_time_step) == want and tp.actual_time_step <= tp.desired_time_step
        assert g.get_generated_timestep() == float(want)
        seen.add(float(want))
    assert len(seen) > 1   # the time step follows the state
    s.close()


def test_sesph2d_desired_dt_is_the_generators(c_oracle):
    s = make_solver("sesph-2d", "quadratic-2d", [1000.0, 0.01], (0.001, 0.4, 0.25), precision="fp32",
                    reference_order=True)
    g = dynamic(s, hi=0.01)
    sc = scenes.breaking_dam_2d(30, 30, seed=2)
    col = sc.collection
    col.velocity = np.random.default_rng(2).uniform(-1, 1, col.position.shape).astype(np.float32)
    s.data.collection = col
    for _ in range(5):
        s.initialize()
        want = expected_dt(c_oracle, s, g)
        simulator_step(s)
        assert bits_equal(np.float32(s.last_stats.desired_dt), want)
    s.close()


def test_run_equals_single_steps_with_the_generator():
    a = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    b = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    dynamic(a)
    dynamic(b)
    a.data.collection = moving_dam(5)
    b.data.collection = moving_dam(5)
    for _ in range(6):
        a.step()
    last = float(a.last_stats.desired_dt)
    b.run(6)
    assert float(b.last_stats.desired_dt) == last
    ca, cb = a.collection(), b.collection()
    for f in ("position", "velocity", "density", "pressure"):
        assert bits_equal(getattr(ca, f), getattr(cb, f)), f
    a.close()
    b.close()


def test_batched_scenes_choose_their_own_time_steps():
    sc = scenes.batched_dams(4, seed=7, f_min=800, f_max=4000)
    rng = np.random.default_rng(7)
    for i, x in enumerate(sc):   # scene i moves at its own speed
        fl = x.collection.type == 0
        x.collection.velocity = np.zeros_like(x.collection.position)
        x.collection.velocity[fl] = rng.uniform(-1, 1, (int(fl.sum()), 3)).astype(np.float32) * (10 * (i + 1))
        x.collection.acceleration = np.zeros_like(x.collection.position)
        x.collection.acceleration[fl] = [0.0, -9.81, 0.0]
    ref = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    batch = BatchedIISPHFluidSolver3D([x.collection for x in sc])
    for name in vars(ref.parameters):
        setattr(batch.parameters, name, getattr(ref.parameters, name))
    for name in vars(ref.settings):
        setattr(batch.settings, name, getattr(ref.settings, name))
    dynamic(batch)
    # the first step's time step follows each scene's own speed
    dts = [float(st.desired_dt) for st in batch.run(1)]
    later = [float(st.desired_dt) for st in batch.run(2)]
    for x, dt, dt3 in zip(sc, dts, later):
        alone = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
        dynamic(alone)
        alone.data.collection = x.collection
        alone.run(1)
        assert float(alone.last_stats.desired_dt) == dt
        alone.run(2)
        # later steps: the batch sums a scene's neighbors in another order (its
        # tiles are formed over the whole batch), so the states differ by rounding
        assert float(alone.last_stats.desired_dt) == pytest.approx(dt3, rel=1e-5)
        alone.close()
    assert len(set(dts)) == len(dts)
    batch.close()
    ref.close()
