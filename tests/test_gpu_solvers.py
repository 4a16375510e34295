"""GPU solver parity (through the C-ABI).

1. FP32 precision with the reference's summation order: every step is
   bit-identical to the reference's own code (golden fixtures) -- positions,
   velocities, densities, pressures, the CFL-clamped time step and the IISPH
   iteration count.
2. The default FP32+Kahan path: within tolerance of the reference. Positions,
   densities and pressures within 1e-5 of the field's scale; velocities within
   the reference's own FP32 rounding envelope (their distance to the FP64 build
   of the step), because the pressure gradient cancels strongly and the
   reference's float velocities are themselves off by more than 1e-5 there.
3. Size-independent properties at the benchmark's full size (1M fluid).
"""
import numpy as np
import pytest

from conftest import bits_equal
from fluidsolver_b200 import (IISPHFluidSolver, IISPHFluidSolver3D, SESPHFluidSolver, SESPHFluidSolver3D, Timepoint,
                              scenes)
from fluidsolver_b200._lib import FS_ERR_NAN, FS_ERR_STATE, FluidSolverError
from tests.golden.make_golden import SOLVER_CASES

pytestmark = pytest.mark.gpu

SOLVER_CLASSES = {"iisph-3d": IISPHFluidSolver3D, "sesph-3d": SESPHFluidSolver3D, "iisph-2d": IISPHFluidSolver,
                  "sesph-2d": SESPHFluidSolver}


def make_solver(solver, search, settings, gen, precision="fp32-kahan", reference_order=False, rest_density=1.0,
                particle_size=1.0, **kw):
    s = SOLVER_CLASSES[solver](search=search, precision=precision, reference_order=reference_order, **kw)
    s.parameters.rest_density = rest_density
    s.parameters.gravity = 9.81
    s.parameters.particle_size = particle_size
    g = s.timestep_generator.settings
    g.timestep, g.lambda_v, g.lambda_a = float(gen[0]), float(gen[1]), float(gen[2])
    st = list(settings)
    if solver == "iisph-3d":
        s.settings.max_density_error_allowed, s.settings.min_number_of_iterations = st[0], int(st[1])
        s.settings.max_number_of_iterations, s.settings.omega, s.settings.gamma = int(st[2]), st[3], st[4]
        s.settings.viscosity, s.settings.single_layer_boundary = st[5], st[6] != 0
        s.settings.single_layer_boundary_gamma_1 = st[7]
    elif solver == "sesph-3d":
        s.settings.StiffnessK, s.settings.Viscosity = st[0], st[1]
        s.settings.single_layer_boundary = st[2] != 0
        s.settings.single_layer_boundary_gamma_1, s.settings.single_layer_boundary_gamma_2 = st[3], st[4]
    elif solver == "iisph-2d":
        s.settings.MaxDensityErrorAllowed, s.settings.MinNumberOfIterations = st[0], int(st[1])
        s.settings.MaxNumberOfIterations, s.settings.Omega, s.settings.Gamma, s.settings.Viscosity = \
            int(st[2]), st[3], st[4], st[5]
    else:
        s.settings.StiffnessK, s.settings.Viscosity = st[0], st[1]
    return s


def simulator_step(s):
    """Simulator::execute_simulation_step without entities and sensors."""
    tp = Timepoint(desired_time_step=s.timestep_generator.get_generated_timestep())
    tp.actual_time_step = tp.desired_time_step
    s.execute_neighborhood_search()
    s.execute_simulation_step(tp)
    return tp


@pytest.mark.parametrize("name", list(SOLVER_CASES))
def test_fp32_reference_order_is_bit_exact(golden, name):
    solver, search, build, gen, settings, steps = SOLVER_CASES[name]
    g = golden["solvers"]
    col = build().collection
    s = make_solver(solver, search, g[f"{name}_settings"], g[f"{name}_generator"], precision="fp32",
                    reference_order=True)
    s.data.collection = col
    for k in range(steps):
        tp = simulator_step(s)
        out = s.collection()
        ref = g[f"{name}_stats"][k]
        assert np.float32(tp.actual_time_step) == ref[1], (name, k)
        if solver == "iisph-3d":
            assert s.stat_last_iteration_count == int(ref[2]), (name, k)
            # the residual is summed in FP64 (the reference: a serial float sum), so
            # this statistic agrees to rounding, not bit for bit
            assert abs(s.stat_last_average_predicted_density_error - ref[3]) <= 1e-5 * abs(ref[3]), (name, k)
        for f in ("position", "velocity", "density", "pressure"):
            assert bits_equal(getattr(out, f), g[f"{name}_step{k}_{f}"]), (name, k, f)
    s.close()


def _scale(a):
    return max(float(np.max(np.abs(a))), 1e-30)


@pytest.mark.parametrize("name", ["iisph3d_hashed", "sesph3d_hashed", "sesph2d_quadratic", "iisph2d_quadratic"])
def test_kahan_within_tolerance_of_reference(golden, name):
    solver, search, build, gen, settings, steps = SOLVER_CASES[name]
    g = golden["solvers"]
    runs = {}
    for prec in ("fp32-kahan", "fp64"):
        s = make_solver(solver, search, g[f"{name}_settings"], g[f"{name}_generator"], precision=prec)
        s.data.collection = build().collection
        simulator_step(s)
        runs[prec] = s.collection()
        s.close()
    k, d = runs["fp32-kahan"], runs["fp64"]
    TOL = 1e-5
    for f in ("position", "velocity", "density", "pressure"):
        ref = g[f"{name}_step0_{f}"].astype(np.float64)
        mine = getattr(k, f).astype(np.float64)
        exact = getattr(d, f).astype(np.float64)
        # the reference's own FP32 rounding, measured against the FP64 build
        envelope = np.max(np.abs(ref - exact))
        slack = TOL * _scale(ref)
        assert np.max(np.abs(mine - exact)) <= envelope + slack, f
        assert np.max(np.abs(mine - ref)) <= 2 * envelope + slack, f
    assert np.max(np.abs(k.position - g[f"{name}_step0_position"])) <= TOL * _scale(g[f"{name}_step0_position"])


@pytest.mark.parametrize("name", ["iisph3d_hashed", "iisph3d_multilayer", "sesph3d_hashed"])
def test_fast_mode_step_by_step_from_the_reference_state(golden, name):
    """Every step of the fast mode (FP32 + compensated sums, tile lists), started
    from the reference's own state after the previous step (position, velocity,
    and the density its viscosity reads): the IISPH iteration count within +-1
    of the reference's, positions within 1e-5 of their scale, and velocity,
    density and pressure within the reference's own FP32 distance to an FP64
    step from the same state, plus 1e-5 of scale."""
    import dataclasses
    solver, search, build, gen, settings, steps = SOLVER_CASES[name]
    g = golden["solvers"]
    col0 = build().collection
    TOL = 1e-5
    for k in range(1, steps):
        start = dataclasses.replace(col0, position=g[f"{name}_step{k - 1}_position"],
                                    velocity=g[f"{name}_step{k - 1}_velocity"],
                                    density=g[f"{name}_step{k - 1}_density"])
        runs = {}
        for prec in ("fp32-kahan", "fp64"):
            s = make_solver(solver, search, g[f"{name}_settings"], g[f"{name}_generator"], precision=prec)
            s.data.collection = start
            tp = simulator_step(s)
            its = s.stat_last_iteration_count if solver == "iisph-3d" else None
            runs[prec] = (s.collection(), its, tp.actual_time_step)
            s.close()
        mine, its, dt = runs["fp32-kahan"]
        exact = runs["fp64"][0]
        ref = g[f"{name}_stats"][k]
        # the CFL clamp sees the same velocities; its accelerations differ by rounding
        assert abs(dt - float(ref[1])) <= 1e-5 * float(ref[1]), (name, k, dt, ref[1])
        if its is not None:
            assert abs(its - int(ref[2])) <= 1, (name, k, its, ref[2])
        pos = g[f"{name}_step{k}_position"].astype(np.float64)
        assert np.max(np.abs(mine.position - pos)) <= TOL * _scale(pos), (name, k)
        for f in ("velocity", "density", "pressure"):
            r = g[f"{name}_step{k}_{f}"].astype(np.float64)
            e = getattr(exact, f).astype(np.float64)
            envelope = np.max(np.abs(r - e))
            assert np.max(np.abs(getattr(mine, f) - e)) <= envelope + TOL * _scale(r), (name, k, f)


def test_kahan_is_closer_to_fp64_than_plain_fp32():
    sc = scenes.breaking_dam_3d(16, 20, 12, 1.0, tank=(30, 26, 18), seed=41)
    res = {}
    for prec in ("fp32", "fp32-kahan", "fp64"):
        s = make_solver("iisph-3d", "hashed-3d", [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1], (0.005, 0.4, 0.25),
                        precision=prec)
        s.data.collection = sc.collection
        for _ in range(3):
            simulator_step(s)
        res[prec] = s.collection()
        s.close()
    e_plain = np.abs(res["fp32"].density.astype(np.float64) - res["fp64"].density).max()
    e_kahan = np.abs(res["fp32-kahan"].density.astype(np.float64) - res["fp64"].density).max()
    assert e_kahan <= e_plain


@pytest.mark.parametrize("precision", ["fp32", "fp32-kahan"])
def test_graph_loop_equals_host_driven_loop(precision):
    """The pressure loop as a conditional node of a CUDA graph (device-side
    exit) gives the same bits as the host-driven loop."""
    sc = scenes.breaking_dam_3d(12, 14, 10, 1.0, tank=(24, 20, 16), seed=61)
    outs, its = [], []
    for sync in (False, True):
        s = make_solver("iisph-3d", "hashed-3d", [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1], (0.005, 0.4, 0.25),
                        precision=precision, reference_order=precision == "fp32")
        s.sync_each_iteration = sync
        s.data.collection = sc.collection
        its.append([])
        for _ in range(6):
            simulator_step(s)
            its[-1].append(s.stat_last_iteration_count)
        outs.append(s.collection())
        s.close()
    assert its[0] == its[1]
    for f in ("position", "velocity", "density", "pressure"):
        assert bits_equal(getattr(outs[0], f), getattr(outs[1], f)), f


def test_run_equals_repeated_steps():
    """fs_run (steps enqueued as graph launches without host synchronisation)
    gives the same bits as the same number of single steps."""
    sc = scenes.breaking_dam_3d(10, 12, 9, 1.0, tank=(20, 18, 14), seed=63)
    outs = []
    for batched in (False, True):
        s = make_solver("iisph-3d", "hashed-3d", [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1], (0.005, 0.4, 0.25))
        s.data.collection = sc.collection
        if batched:
            s.run(7)
        else:
            for _ in range(7):
                s.step()
        outs.append(s.collection())
        s.close()
    for f in ("position", "velocity", "density", "pressure"):
        assert bits_equal(getattr(outs[0], f), getattr(outs[1], f)), f


def test_iteration_cap_is_honoured():
    sc = scenes.breaking_dam_3d(8, 8, 8, 1.0, tank=(16, 16, 16), seed=62)
    s = make_solver("iisph-3d", "hashed-3d", [1e-9, 2, 7, 0.5, 0.7, 0.01, 1.0, 1.1], (0.005, 0.4, 0.25))
    s.data.collection = sc.collection
    for _ in range(3):
        simulator_step(s)
        assert s.stat_last_iteration_count == 7
    s.close()


def test_solve_before_search_is_an_error():
    s = make_solver("iisph-3d", "hashed-3d", [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1], (0.005, 0.4, 0.25))
    s.data.collection = scenes.breaking_dam_3d(4, 4, 4, 1.0, tank=(8, 8, 8)).collection
    with pytest.raises(FluidSolverError) as e:
        s.execute_simulation_step(Timepoint(desired_time_step=0.005))
    assert e.value.status == FS_ERR_STATE
    s.close()


def test_neighbor_capacity_grows_automatically():
    # a compressed cluster: more neighbors than the default list capacity
    rng = np.random.default_rng(3)
    sc = scenes.breaking_dam_3d(6, 6, 6, 1.0, tank=(10, 10, 10), seed=5)
    col = sc.collection
    f = col.type == 0
    col.position[f] = (col.position[f] - col.position[f].mean(0)) * 0.45 + 5.0 + rng.uniform(-0.01, 0.01, (f.sum(), 3))
    s = make_solver("iisph-3d", "hashed-3d", [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1], (0.005, 0.4, 0.25),
                    precision="fp32", reference_order=True)
    s.data.collection = col
    stats = s.step(0.005)
    assert stats.max_neighbors > 64
    st = s.collection()
    assert np.isfinite(st.position).all()
    s.close()


def test_external_forces_are_consumed_like_the_reference(golden):
    """ExternalForces3D is added to the non-pressure acceleration of every
    active particle and reset to zero in the first loop
    (IISPHFluidSolver3D.hpp:156-175); the C oracle reproduces the reference."""
    from oracle import c_oracle
    sc = scenes.breaking_dam_3d(6, 7, 5, 1.0, tank=(12, 12, 10), seed=51)
    col = sc.collection
    rng = np.random.default_rng(1)
    col.external = rng.uniform(-3, 3, col.position.shape).astype(np.float32)
    o = c_oracle.State(col)
    o.run(c_oracle.config("iisph-3d", "hashed-3d"), 2)
    s = make_solver("iisph-3d", "hashed-3d", [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1], (0.005, 0.4, 0.25),
                    precision="fp32", reference_order=True)
    s.data.collection = col
    simulator_step(s)
    simulator_step(s)
    out = s.collection()
    for f in ("position", "velocity", "density", "pressure", "external"):
        assert bits_equal(getattr(out, f), getattr(o, f)), f
    s.close()


def test_1m_dam_properties_at_full_size():
    """The 1M-fluid benchmark scene: finite state, mass conserved, every step
    converged to <= 0.1 % average density error within the iteration cap."""
    sc = scenes.dam_1m()
    s = make_solver("iisph-3d", "hashed-3d", [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1],
                    (scenes.REFERENCE_UNITS_DT, 0.4, 0.25))
    s.data.collection = sc.collection
    for _ in range(5):
        simulator_step(s)
        st = s.last_stats
        assert st.iterations <= 100
        assert st.iterations == 100 or st.avg_density_error_fp64 <= 0.001
    out = s.collection()
    assert np.isfinite(out.position).all() and np.isfinite(out.velocity).all()
    assert np.array_equal(np.sort(out.mass), np.sort(sc.collection.mass))
    assert np.array_equal(out.type, sc.collection.type)
    # boundary particles do not move (zero velocity, zero acceleration)
    b = out.type == 1
    assert bits_equal(out.position[b], sc.collection.position[b])
    s.close()


@pytest.mark.parametrize("precision", ["fp32-kahan", "fp32"])
def test_non_finite_positions_end_the_step_with_a_nan_status(precision):
    """A NaN position stops the step with FS_ERR_NAN: the particle is kept out
    of the cell walks, and the list builders and solver phases skip their
    work, so a broken state cannot turn the search quadratic."""
    sc = scenes.breaking_dam_3d(12, 12, 12, 1.0, tank=(40, 30, 20), seed=3)
    col = sc.collection
    col.position = col.position.copy()
    col.position[7, 1] = np.nan
    s = IISPHFluidSolver3D(search="hashed-3d", precision=precision, reference_order=precision == "fp32")
    s.parameters.rest_density, s.parameters.particle_size = 1.0, 1.0
    s.timestep_generator.settings.timestep = 0.005
    s.data.collection = col
    with pytest.raises(FluidSolverError) as e:
        s.step()
    assert e.value.status == FS_ERR_NAN
    s.close()
