"""CPU tests that pin the oracle: the plain-C restatement (oracle/fs_oracle.c)
against the golden fixtures made from the reference's own sources, against the
reference's googletest expectations, and -- where the reference checkout was
available to build oracle/_ref -- against the compiled reference directly."""
import numpy as np
import pytest

from conftest import bits_equal, csr_sets
from fluidsolver_b200 import scenes


# ---------------------------------------------------------------- kernel
def test_kernel_matches_reference_bit_for_bit(golden, c_oracle):
    g = golden["kernel"]
    for dim in (2, 3):
        for support in (1.0, 2.0, 0.02, 8.5):
            key = f"d{dim}_s{support}"
            W, dW = c_oracle.kernel_eval(dim, support, g[key + "_x"])
            assert bits_equal(W, g[key + "_W"]), key
            assert bits_equal(dW, g[key + "_dW"]), key


def test_kernel_compact_support(c_oracle):
    # CubicSplineKernelTest.cpp:5-28
    cases = [(1.0, (2.0, 0.0)), (3.0, (8.0, 0.0)), (5.0, (3.0, 16.0)), (0.8, (4.0, 10.0)), (2.5, (0.0, 3.0))]
    for support, x in cases:
        W, _ = c_oracle.kernel_eval(2, support, np.array([x], np.float32))
        assert W[0] == 0.0


def test_kernel_symmetry_nonnegativity_and_gradient_antisymmetry(c_oracle):
    # CubicSplineKernelTest.cpp:30-136 (t = 0 .. 10 step 0.001)
    t = np.arange(0, 10.0005, 0.001, dtype=np.float32)
    for support, vec in [(8.5, lambda t: np.stack([t, t], 1)), (8.5, lambda t: np.stack([t, 0 * t], 1)),
                         (6.5, lambda t: np.stack([0 * t, t], 1)), (4.5, lambda t: np.stack([0.2 * t, t], 1)),
                         (4.5, lambda t: np.stack([t, 0.8 * t], 1))]:
        x = vec(t).astype(np.float32)
        W1, d1 = c_oracle.kernel_eval(2, support, x)
        W2, d2 = c_oracle.kernel_eval(2, support, -x)
        np.testing.assert_allclose(W1, W2, rtol=4 * np.finfo(np.float32).eps, atol=0)
        assert np.all(W1 >= 0.0)
        np.testing.assert_allclose(d1, -d2, rtol=4 * np.finfo(np.float32).eps, atol=1e-30)


# ---------------------------------------------------------------- CFL
def test_cfl_clamp_matches_reference(golden, c_oracle):
    g = golden["cfl"]
    for la in (0.25, 0.3):
        mine = np.array([c_oracle.cfl(0.005, 0.4, la, 1.0, a, v) for a, v in zip(g["max_acc"], g["max_vel"])],
                        np.float32)
        assert bits_equal(mine, g[f"dt_la{la}"])


def test_dynamic_timestep_generator_matches_reference(golden, c_oracle):
    """DynamicCflTimestepGenerator::generate_next_timestep (DynamicCflTimestepGenerator.cpp:45-59)
    restated in oracle/fs_oracle.c against the reference's own generator (tests/golden)."""
    g = golden["dynamic_timestep"]
    n = sum(1 for f in g.files if f.endswith("_prm"))
    kinds = set()
    for i in range(n):
        ps, lo, hi, lv, la, dt = (float(x) for x in g[f"c{i}_prm"])
        mine = c_oracle.dynamic_timestep(g[f"c{i}_vel"], g[f"c{i}_acc"], g[f"c{i}_type"], ps, lo, hi, lv, la)
        assert bits_equal(np.float32(mine), np.float32(dt)), i
        kinds.add("min" if dt == np.float32(lo) else "max" if dt == np.float32(hi) else "cfl")
    assert kinds == {"min", "max", "cfl"}   # every branch of the generator is exercised


def test_boundary_preprocessor_matches_reference(golden, c_oracle):
    """BoundaryPreprocessor (BoundaryPreprocessor.cpp:7-48) restated in oracle/fs_oracle.c against the
    reference's own entity through its hashed-3d interface (tests/golden/boundary.npz)."""
    g = golden["boundary"]
    for name in ("one_layer", "two_layers", "jittered"):
        ps = float(g[f"{name}_size"])
        mine = c_oracle.boundary_masses(g[f"{name}_pos"], g[f"{name}_mass"], g[f"{name}_type"], ps, 1.0)
        assert bits_equal(mine, g[f"{name}_out"]), name


# ---------------------------------------------------------------- searches
def _expect_sets(off, idx, i, expected):
    assert sorted(idx[off[i]:off[i + 1]].tolist()) == sorted(expected)


@pytest.mark.parametrize("kind", ["quadratic-2d", "hashed-2d"])
def test_reference_googletest_neighbor_sets(golden, c_oracle, kind):
    # NeighborhoodSearchTests.cpp:131-299: exact sets for particles 0 and 38
    g = golden["search"]
    for name in ("grid11", "grid11x2"):
        off, idx, ok = c_oracle.search(kind, g[f"{name}_{kind}_pos"], float(g[f"{name}_{kind}_r"]))
        _expect_sets(off, idx, 0, [0, 1, 2, 11, 12, 22])
        _expect_sets(off, idx, 38, [16, 26, 27, 28, 36, 37, 38, 39, 40, 48, 49, 50, 60])
    off, idx, _ = c_oracle.search(kind, g[f"grid3_{kind}_pos"], 2.0)
    expected = {0: [0, 1, 2, 3, 4, 6], 1: [0, 1, 2, 3, 4, 5, 7], 2: [0, 1, 2, 4, 5, 8], 3: [0, 1, 3, 4, 5, 6, 7],
                4: list(range(9)), 5: [1, 2, 3, 4, 5, 7, 8], 6: [0, 3, 4, 6, 7, 8], 7: [1, 3, 4, 5, 6, 7, 8],
                8: [2, 4, 5, 6, 7, 8]}
    for i, e in expected.items():
        _expect_sets(off, idx, i, e)


def test_single_particle(c_oracle):
    # NeighborhoodSearchTests.cpp:104-129
    for kind in ("quadratic-2d", "hashed-2d"):
        off, idx, _ = c_oracle.search(kind, np.array([[234.56341, 6578.45]], np.float32), 2.0)
        assert idx.tolist() == [0]


def test_moving_grid_keeps_sets(c_oracle, golden):
    # NeighborhoodSearchTests.cpp:301-354: 1,024 translations at r = 2.01
    pos = golden["search"]["grid11_quadratic-2d_pos"].copy()
    mv = np.array([0.34, -0.5], np.float32)
    for step in range(1024):
        pos += mv
        if step % 64 != 63:
            continue
        for kind in ("quadratic-2d", "hashed-2d"):
            off, idx, _ = c_oracle.search(kind, pos, 2.01)
            _expect_sets(off, idx, 0, [0, 1, 2, 11, 12, 22])
            _expect_sets(off, idx, 38, [16, 26, 27, 28, 36, 37, 38, 39, 40, 48, 49, 50, 60])


@pytest.mark.parametrize("kind", ["hashed-3d", "quadratic-3d", "compressed-3d"])
def test_3d_lists_match_reference(golden, c_oracle, kind):
    g = golden["search"]
    off, idx, ok = c_oracle.search(kind, g["dam3d_pos"], 2.0, g["dam3d_type"])
    assert ok and bool(g[f"dam3d_{kind}_ok"])
    ro, ri = g[f"dam3d_{kind}_off"], g[f"dam3d_{kind}_idx"]
    assert [s.tolist() for s in csr_sets(off, idx)] == [s.tolist() for s in csr_sets(ro, ri)]
    if kind != "compressed-3d":  # compressed lists are ordered in the reference's re-sorted index space
        assert np.array_equal(off, ro) and np.array_equal(idx, ri)


@pytest.mark.parametrize("kind", ["quadratic-2d", "hashed-2d"])
def test_2d_lists_match_reference_in_order(golden, c_oracle, kind):
    g = golden["search"]
    off, idx, _ = c_oracle.search(kind, g["dam2d_pos"], 2.0, g["dam2d_type"])
    assert np.array_equal(off, g[f"dam2d_{kind}_off"]) and np.array_equal(idx, g[f"dam2d_{kind}_idx"])


def test_random_points_and_capacity(golden, c_oracle):
    g = golden["search"]
    for kind in ("hashed-3d", "compressed-3d"):
        off, idx, ok = c_oracle.search(kind, g["rand_pos"], 0.1)
        assert ok
        assert [s.tolist() for s in csr_sets(off, idx)] == \
            [s.tolist() for s in csr_sets(g[f"rand_{kind}_off"], g[f"rand_{kind}_idx"])]
    # more than 97 neighbors: the reference process terminates, the oracle reports it
    assert int(g["blob_compressed_exit"]) != 0
    _, _, ok = c_oracle.search("compressed-3d", g["blob_pos"], 0.1)
    assert not ok


def test_empty_search(c_oracle):
    off, idx, ok = c_oracle.search("hashed-3d", np.zeros((0, 3), np.float32), 2.0)
    assert ok and len(idx) == 0 and off.tolist() == [0]


# ---------------------------------------------------------------- solvers
def _case_scene(name):
    from tests.golden.make_golden import SOLVER_CASES  # noqa: F401  (builders live beside the fixtures)
    return SOLVER_CASES[name]


CASES = ["iisph3d_hashed", "iisph3d_multilayer", "sesph3d_hashed", "sesph2d_quadratic", "sesph2d_hashed",
         "iisph2d_quadratic"]


def _oracle_cfg(c_oracle, solver, search, settings, gen):
    s = list(settings)
    if solver == "iisph-3d":
        return c_oracle.config(solver, search, max_err=s[0], min_it=s[1], max_it=s[2], omega=s[3], gamma=s[4],
                               viscosity=s[5], single_layer=s[6] != 0, gamma1=s[7], timestep=gen[0],
                               lambda_v=gen[1], lambda_a=gen[2])
    if solver == "sesph-3d":
        return c_oracle.config(solver, search, stiffness=s[0], viscosity=s[1], single_layer=s[2] != 0, gamma1=s[3],
                               gamma2=s[4], timestep=gen[0], lambda_v=gen[1], lambda_a=gen[2])
    if solver == "iisph-2d":
        return c_oracle.config(solver, search, max_err=s[0], min_it=s[1], max_it=s[2], omega=s[3], gamma=s[4],
                               viscosity=s[5], single_layer=False, timestep=gen[0])
    return c_oracle.config(solver, search, stiffness=s[0], viscosity=s[1], single_layer=False, timestep=gen[0])


@pytest.mark.parametrize("name", CASES)
def test_solver_steps_match_reference_bit_for_bit(golden, c_oracle, name):
    solver, search, build, gen, settings, steps = _case_scene(name)
    g = golden["solvers"]
    col = build().collection
    assert bits_equal(col.position, g[f"{name}_in_position"])
    st = c_oracle.State(col)
    cfg = _oracle_cfg(c_oracle, solver, search, g[f"{name}_settings"], g[f"{name}_generator"])
    for k in range(steps):
        stats = st.run(cfg, 1, abs_int=(solver == "iisph-2d"))[0]
        for f in ("position", "velocity", "density", "pressure"):
            assert bits_equal(getattr(st, f), g[f"{name}_step{k}_{f}"]), (name, k, f)
        ref = g[f"{name}_stats"][k]
        assert stats[1] == ref[1]                      # actual dt
        if solver == "iisph-3d":
            assert int(stats[2]) == int(ref[2])        # iterations
            assert stats[3] == ref[3]                  # average density error


def test_iisph2d_uses_the_truncating_abs(golden, c_oracle):
    """The reference's 2D convergence test calls the C int abs on the float
    error (IISPHFluidSolver.hpp:401): with float abs the trajectory differs."""
    solver, search, build, gen, settings, steps = _case_scene("iisph2d_quadratic")
    g = golden["solvers"]
    st = c_oracle.State(build().collection)
    cfg = _oracle_cfg(c_oracle, solver, search, g["iisph2d_quadratic_settings"], g["iisph2d_quadratic_generator"])
    st.run(cfg, 1, abs_int=False)
    assert not bits_equal(st.pressure, g["iisph2d_quadratic_step0_pressure"])


def test_oracle_against_compiled_reference(ref_oracle, c_oracle):
    """Direct comparison with the compiled reference on a fresh seed."""
    sc = scenes.breaking_dam_3d(7, 9, 6, 1.0, tank=(13, 12, 10), seed=77)
    ref = ref_oracle.RefSolver("iisph-3d", "hashed-3d", sc.collection, (1.0, 9.81, 1.0),
                               ref_oracle.iisph3d_settings(), (0.005, 0.4, 0.25))
    st = c_oracle.State(sc.collection)
    cfg = c_oracle.config("iisph-3d", "hashed-3d")
    for _ in range(3):
        r = ref.step()
        o = st.run(cfg, 1)[0]
        s = ref.state()
        assert int(o[2]) == r["iterations"]
        for f in ("position", "velocity", "density", "pressure"):
            assert bits_equal(getattr(st, f), s[f]), f


POSITION_QUERY_KINDS = [(3, "hashed-3d"), (3, "quadratic-3d"), (3, "compressed-3d"), (2, "hashed-2d"),
                        (2, "quadratic-2d")]


@pytest.mark.parametrize("dim,kind", POSITION_QUERY_KINDS)
def test_position_query_oracle_matches_reference(golden, c_oracle, dim, kind):
    """The oracle's get_neighbors(position) against the reference's, fixtures
    made from the reference's sources: inactive particles, the length/dot
    predicates and hashed-3d's skipped cell minimum."""
    g = golden["position_queries"]
    pos, typ, queries = g[f"pos{dim}"], g[f"type{dim}"], g[f"queries{dim}"]
    off, idx = g[f"{kind}/offsets"], g[f"{kind}/indices"]
    for i, q in enumerate(queries):
        got = c_oracle.query_position(kind, pos, 1.0, q, typ)
        assert got.tolist() == idx[off[i]:off[i + 1]].tolist(), (kind, i)


def test_position_query_quirk_is_pinned(golden, c_oracle):
    """hashed-3d drops members that a plain radius test keeps (and only
    those): the fixture would not pin the quirk otherwise."""
    g = golden["position_queries"]
    pos, typ, queries = g["pos3"], g["type3"], g["queries3"]
    off, idx = g["hashed-3d/offsets"], g["hashed-3d/indices"]
    dropped = 0
    for i, q in enumerate(queries):
        full = set(c_oracle.query_position("compressed-3d", pos, 1.0, q, typ).tolist())
        got = set(idx[off[i]:off[i + 1]].tolist())
        assert got <= full
        dropped += len(full - got)
    assert dropped > 0


def test_compact_hashing_has_no_position_query(c_oracle):
    with pytest.raises(ValueError):
        c_oracle.query_position("compact-hashing-2d", np.zeros((2, 2), np.float32), 1.0, np.zeros(2, np.float32))


def test_raytrace_fixture_is_the_reference_accelerator(golden, ref_oracle):
    """tests/golden/raytrace.npz holds the first hits that the reference's own
    ParticleIntersectionAccelerator (visualizer/raytracer/ParticleIntersectionAccelerator.cpp:8-206,
    compiled in oracle/_ref) gives for its rays; the device tracer is checked against it."""
    g = golden["raytrace"]
    out = ref_oracle.trace_rays(g["pos"], g["mass"], g["type"], 1.0, 1.0, g["origins"], g["directions"])
    for k in ("hit", "point", "normal", "length"):
        assert bits_equal(out[k], g[k]), k
    assert {int(t) for t in np.unique(g["hit"])} == {-1, 0, 1, 2}   # misses and every kind of hit


def test_hashed_2d_insertion_order_over_the_2d_dam(ref_oracle, c_oracle):
    """The 2D SESPH dam (2,500 fluid + 1,188 boundary, k 1000, dt 0.001) for all
    1,000 steps on hashed-2d: the oracle stays bit-identical to the compiled
    reference because it keeps the grid's history across steps -- each
    cell's particles in order of arrival (HashedNeighborhoodSearch.cpp:117-151),
    which decides the float summation order once particles change cells."""
    col = scenes.breaking_dam_2d().collection
    ref = ref_oracle.RefSolver("sesph-2d", "hashed-2d", col, (1.0, 9.81, 1.0),
                               ref_oracle.sesph2d_settings(1000.0, 0.01), (0.001, 0.4, 0.25), variant="omp")
    st = c_oracle.State(col)
    cfg = c_oracle.config("sesph-2d", "hashed-2d", stiffness=1000.0, viscosity=0.01, timestep=0.001)
    for chunk in range(20):
        st.run(cfg, 50)
        ref.run(50)
        s = ref.state()
        for f in ("position", "velocity", "density", "pressure"):
            assert bits_equal(getattr(st, f), s[f]), (50 * (chunk + 1), f)
    assert np.max(np.abs(st.position - col.position)) > 1.0
    # without the history (a fresh grid every step, ascending index in a cell)
    # the sums differ within the first steps
    fresh = c_oracle.State(col)
    ref2 = ref_oracle.RefSolver("sesph-2d", "hashed-2d", col, (1.0, 9.81, 1.0),
                                ref_oracle.sesph2d_settings(1000.0, 0.01), (0.001, 0.4, 0.25), variant="omp")
    differs = False
    for _ in range(20):
        fresh.h2d_cell[:] = np.iinfo(np.int32).max   # forget the grid
        fresh.run(cfg, 1)
        ref2.step()
        if not bits_equal(fresh.density, ref2.state()["density"]):
            differs = True
            break
    assert differs


def _stats_collections():
    """Collections for the global sensors: a moving 2D dam, a 3D dam with
    inactive particles, all-negative pressures, and one without normal
    particles."""
    from fluidsolver_b200 import ParticleCollection
    rng = np.random.default_rng(31)
    out = []
    for dim, n in ((2, 3000), (3, 4000)):
        pos = rng.uniform(-5, 40, (n, dim)).astype(np.float32)
        typ = rng.choice(np.array([0, 0, 0, 1, 2], np.uint8), n)
        out.append(ParticleCollection(position=pos, velocity=rng.normal(0, 3, (n, dim)).astype(np.float32),
                                      mass=rng.uniform(0.5, 1.5, n).astype(np.float32),
                                      density=rng.uniform(0.9, 1.1, n).astype(np.float32),
                                      pressure=rng.uniform(-2, 50, n).astype(np.float32), type=typ))
    neg = ParticleCollection(position=np.zeros((64, 2), np.float32), velocity=np.zeros((64, 2), np.float32),
                             mass=np.ones(64, np.float32), density=np.ones(64, np.float32),
                             pressure=-np.ones(64, np.float32), type=np.zeros(64, np.uint8))
    none = ParticleCollection(position=np.zeros((16, 2), np.float32), velocity=np.ones((16, 2), np.float32),
                              mass=np.ones(16, np.float32), density=np.ones(16, np.float32),
                              pressure=np.ones(16, np.float32), type=np.ones(16, np.uint8))
    return out + [neg, none]


def test_global_sensors_oracle_equals_the_compiled_reference(ref_oracle, c_oracle):
    """The C restatement of the global sensors (ParticleStatistics.cpp:17-201)
    against the reference's own sensor classes, bit for bit: maxima starting at
    FLT_MIN, minima at FLT_MAX, averages and energies as serial float sums in
    index order, the counts. Velocity and energy in 2D only (the reference's
    sensors read 2D MovementData)."""
    for col in _stats_collections():
        dim = col.position.shape[1]
        ref = ref_oracle.global_stats(col, 9.81, 1.5)
        mine = c_oracle.global_stats(col, 9.81, 1.5)
        keys = ref_oracle.STAT_NAMES if dim == 2 else [k for k in ref_oracle.STAT_NAMES
                                                       if k.startswith(("density", "pressure"))]
        for k in keys:
            assert bits_equal(np.float32(mine[k]), ref[k]), (dim, k, mine[k], ref[k])
        for k in ("normal_particles", "boundary_particles", "inactive_particles"):
            assert mine[k] == ref[k], k
