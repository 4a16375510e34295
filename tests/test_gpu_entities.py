"""Entities and sensors on the device: the boundary preprocessor
(BoundaryPreprocessor.cpp:7-48) against the reference's own entity (golden
fixtures, bit for bit in the FP32 reference-order mode) and the global
sensors (ParticleStatistics.cpp:17-201) against the oracle's restatement and
against the reference's own sensor classes compiled in oracle/_ref."""
import numpy as np
import pytest

from conftest import bits_equal
from fluidsolver_b200 import BoundaryPreprocessor, Timepoint, scenes
from fluidsolver_b200.solver import ParticleCollection
from test_gpu_solvers import make_solver, simulator_step

pytestmark = pytest.mark.gpu

SETTINGS_3D = [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1]
CASES = ("one_layer", "two_layers", "jittered")


def collection_of(g, name):
    pos = g[f"{name}_pos"]
    n = len(pos)
    return ParticleCollection(position=pos, velocity=np.zeros_like(pos), mass=g[f"{name}_mass"],
                              density=np.ones(n, np.float32), type=g[f"{name}_type"])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision,exact", [("fp32", True), ("fp32-kahan", False), ("fp64", False)])
def test_boundary_masses_match_the_reference(golden, name, precision, exact):
    g = golden["boundary"]
    ps = float(g[f"{name}_size"])
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25), precision=precision,
                    reference_order=exact, particle_size=ps)
    s.data.collection = collection_of(g, name)
    s.execute_neighborhood_search()
    BoundaryPreprocessor(s).execute_simulation_step(Timepoint(), True)
    got = s.collection().mass
    want = g[f"{name}_out"]
    if exact:   # the reference's list order and float arithmetic
        assert bits_equal(got, want)
    else:
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=0)
    s.close()


def test_boundary_preprocessor_needs_a_fresh_search(golden):
    g = golden["boundary"]
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    s.data.collection = collection_of(g, "one_layer")
    s.execute_neighborhood_search()
    simulator_step(s)   # the step moves the particles: the search's sets are stale
    with pytest.raises(Exception):
        s.boundary_preprocess()
    with pytest.raises(ValueError):
        BoundaryPreprocessor(s).execute_simulation_step(Timepoint(), False)
    s.close()


def _check_stats(got, want, col, fluid, gravity, zero):
    for k in ("density", "pressure", "velocity"):
        assert bits_equal(np.float32(got[f"{k}_max"]), want[f"{k}_max"]), k
        assert bits_equal(np.float32(got[f"{k}_min"]), want[f"{k}_min"]), k
    for k in ("normal_particles", "boundary_particles", "inactive_particles"):
        assert got[k] == want[k], k
    # sums: the device sums in FP64; the reference sums serially in float
    v = col.velocity.astype(np.float64)
    speed = np.sqrt(np.float32((v[:, 0] ** 2 + v[:, 1] ** 2) + (v[:, 2] ** 2 if v.shape[1] == 3 else 0.0)))
    exact = {"density_avg": col.density[fluid].astype(np.float64).mean(),
             "pressure_avg": col.pressure[fluid].astype(np.float64).mean(),
             "velocity_avg": speed[fluid].astype(np.float64).mean()}
    for k, e in exact.items():
        assert got[k] == pytest.approx(e, rel=1e-6, abs=1e-30), k
        assert got[k] == pytest.approx(float(want[k]), rel=1e-4, abs=1e-6), k
    m = col.mass[fluid].astype(np.float64)
    ke = (0.5 * m * speed[fluid].astype(np.float64) ** 2).sum()
    pe = (gravity * m * (col.position[fluid, 1].astype(np.float64) - zero)).sum()
    assert got["kinetic_energy"] == pytest.approx(ke, rel=1e-5)
    assert got["potential_energy"] == pytest.approx(pe, rel=1e-5)


def test_global_statistics_3d(c_oracle):
    sc = scenes.breaking_dam_3d(16, 14, 12, 1.0, tank=(50, 30, 25), seed=8)
    col = sc.collection
    col.type[::97] = 2   # a few inactive particles
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    s.data.collection = col
    for _ in range(4):
        simulator_step(s)
    got = s.global_statistics(zero_height=3.0)
    out = s.collection()
    want = c_oracle.global_stats(out, 9.81, 3.0)
    _check_stats(got, want, out, out.type == 0, 9.81, 3.0)
    assert got["pressure_max"] > 0 and got["velocity_max"] > 0
    s.close()


def test_global_statistics_2d(c_oracle):
    # the reference's velocity and energy sensors read 2D MovementData
    s = make_solver("sesph-2d", "hashed-2d", [1000.0, 0.01], (0.001, 0.4, 0.25))
    s.data.collection = scenes.breaking_dam_2d(30, 20, seed=4).collection
    for _ in range(5):
        simulator_step(s)
    got = s.global_statistics()
    out = s.collection()
    want = c_oracle.global_stats(out, 9.81, 0.0)
    _check_stats(got, want, out, out.type == 0, 9.81, 0.0)
    s.close()


@pytest.mark.parametrize("dim", [2, 3])
def test_global_statistics_against_the_reference_sensors(ref_oracle, dim):
    """fs_global_statistics against the reference's own sensor classes
    (ParticleStatistics.cpp:17-201, compiled in oracle/_ref) on the device
    state after a few steps: maxima, minima and counts bit for bit; averages
    and energies, which the device sums in FP64 and the reference serially in
    float, within the float sum's own error bound (n - 1) u sum|x_i|, u = 2^-24.
    Velocity and energy in 2D only (the reference's sensors read 2D MovementData)."""
    if dim == 3:
        sc = scenes.breaking_dam_3d(16, 14, 12, 1.0, tank=(50, 30, 25), seed=8)
        col = sc.collection
        col.type[::97] = 2
        s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    else:
        col = scenes.breaking_dam_2d(30, 20, seed=4).collection
        s = make_solver("sesph-2d", "hashed-2d", [1000.0, 0.01], (0.001, 0.4, 0.25))
    s.data.collection = col
    for _ in range(4):
        simulator_step(s)
    got = s.global_statistics(zero_height=2.0)
    out = s.collection()
    want = ref_oracle.global_stats(out, 9.81, 2.0)
    s.close()
    fields = ("density", "pressure", "velocity") if dim == 2 else ("density", "pressure")
    for k in fields:
        assert bits_equal(np.float32(got[f"{k}_max"]), want[f"{k}_max"]), k
        assert bits_equal(np.float32(got[f"{k}_min"]), want[f"{k}_min"]), k
    for k in ("normal_particles", "boundary_particles", "inactive_particles"):
        assert got[k] == want[k], k
    fluid = out.type == 0
    nf = int(fluid.sum())
    u = 2.0 ** -24
    v = out.velocity.astype(np.float64)
    speed = np.sqrt((v ** 2).sum(1))
    terms = {"density_avg": np.abs(out.density[fluid]).sum() / nf, "pressure_avg": np.abs(out.pressure[fluid]).sum() / nf}
    if dim == 2:
        m = out.mass[fluid].astype(np.float64)
        terms.update(velocity_avg=speed[fluid].sum() / nf, kinetic_energy=(0.5 * m * speed[fluid] ** 2).sum(),
                     potential_energy=np.abs(9.81 * m * (out.position[fluid, 1] - 2.0)).sum())
    for k, mag in terms.items():
        bound = (nf - 1) * u * mag + 4 * np.spacing(np.float32(abs(float(want[k]))))
        assert abs(got[k] - float(want[k])) <= bound, (k, got[k], want[k], bound)


def test_global_statistics_quirks():
    """All-negative pressures report FLT_MIN as their maximum (MaxMinAvgSensorData starts the
    maximum at std::numeric_limits<float>::min()); no normal particles: averages 0, minima FLT_MAX."""
    n = 64
    pos = np.random.default_rng(1).uniform(0, 10, (n, 3)).astype(np.float32)
    col = ParticleCollection(position=pos, velocity=np.zeros_like(pos), mass=np.ones(n, np.float32),
                             density=np.ones(n, np.float32), pressure=-np.ones(n, np.float32),
                             type=np.zeros(n, np.uint8))
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    s.data.collection = col
    st = s.global_statistics()
    assert bits_equal(np.float32(st["pressure_max"]), np.finfo(np.float32).tiny)
    assert st["pressure_min"] == -1.0 and st["normal_particles"] == n
    s.close()
    col.type[:] = 1
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    s.data.collection = col
    st = s.global_statistics()
    assert st["density_avg"] == 0.0 and st["boundary_particles"] == n
    assert bits_equal(np.float32(st["density_min"]), np.float32(np.finfo(np.float32).max))
    s.close()


def test_dump_is_the_device_state(tmp_path):
    """fs_dump: the particle file FluidConsole writes every dump interval, from the device state;
    it reads back as the collection the device holds, and a new solver continues from it."""
    from fluidsolver_b200 import read_particles
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    s.data.collection = scenes.breaking_dam_3d(12, 10, 8, 1.0, tank=(30, 20, 16), seed=9).collection
    for _ in range(3):
        simulator_step(s)
    path = tmp_path / "particle-data" / "3.data"
    path.parent.mkdir()
    s.dump(str(path))
    got, want = read_particles(str(path)), s.collection()
    for name in ("position", "velocity", "acceleration", "external", "mass", "density", "pressure", "type", "tag"):
        assert bits_equal(getattr(got, name), getattr(want, name)), name
    t = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    t.data.collection = got
    simulator_step(s)
    simulator_step(t)
    a, b = s.collection(), t.collection()
    np.testing.assert_allclose(a.position, b.position, rtol=0, atol=1e-5)
    s.close()
    t.close()
