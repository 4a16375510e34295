"""The fluid path tracer on the device (fs_trace_rays, fs_render).

Ray queries are compared with the reference's own ParticleIntersectionAccelerator
(visualizer/raytracer/ParticleIntersectionAccelerator.cpp, compiled in oracle/ref;
tests/golden/raytrace.npz): the same hit type for at least 99.5 % of the rays
(all 2,952 on a B200), and for those the same march length, the intersection
point within 1e-4 (3.8e-6 measured) and the normal within 1e-5. The densities
along a ray are float sums over the same particles in another order, which
moves a hit only where the density at a march point lies within rounding of
the surface density. The path tracer's
images are random (the reference draws from per-thread engines in pixel
order); they are checked for what holds for every sample: the white sky where
rays miss, radiance below the sky's where they hit, the normal colours of the
first hits, the tone mapping, and the same image for the same seed."""
import numpy as np
import pytest

from fluidsolver_b200 import scenes, tone_map
from fluidsolver_b200.solver import ParticleCollection
from test_gpu_solvers import make_solver

pytestmark = pytest.mark.gpu

SETTINGS_3D = [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1]


def solver_of(pos, mass, typ):
    s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25))
    n = len(pos)
    s.data.collection = ParticleCollection(position=pos, velocity=np.zeros_like(pos), mass=mass,
                                           density=np.ones(n, np.float32), type=typ)
    return s


def test_ray_hits_match_the_reference_accelerator(golden):
    g = golden["raytrace"]
    s = solver_of(g["pos"], g["mass"], g["type"])
    got = s.trace_rays(g["origins"], g["directions"])
    s.close()
    want_hit = g["hit"]
    same = got["hit"] == want_hit
    assert same.mean() >= 0.995, same.mean()
    assert (want_hit >= 0).sum() > 0.8 * len(want_hit)   # the fixture's rays mostly hit
    both = same & (want_hit >= 0)
    assert np.mean(got["length"][both] == g["length"][both]) >= 0.995
    np.testing.assert_allclose(got["point"][both], g["point"][both], atol=1e-4, rtol=0)
    dots = np.sum(got["normal"][both] * g["normal"][both], axis=1)
    assert np.all(dots > 1 - 1e-5)
    for t in (0, 1, 2):   # every kind of hit is exercised
        assert np.sum(want_hit == t) >= 5


@pytest.fixture(scope="module")
def dam_solver():
    sc = scenes.breaking_dam_3d(12, 10, 8, 1.0, tank=(24, 16, 14), seed=51, layers=2)
    col = sc.collection
    s = solver_of(col.position, col.mass, col.type)
    yield s
    s.close()


CAM = dict(position=(30.0, 18.0, 28.0), view_direction=(-24.0, -14.0, -24.0), width=40, height=30,
           field_of_view_x=0.7)


def test_render_normals_of_first_hit(dam_solver):
    rad, rgba = dam_solver.render(**CAM, samples_per_pixel=1, output_normals_of_first_hit=True, seed=3)
    n = rad.reshape(-1, 3) * 2.0 - 1.0
    lengths = np.linalg.norm(n, axis=1)
    # every pixel is a unit normal (a first hit) or the negated ray direction (a miss)
    assert np.all(np.abs(lengths - 1.0) < 1e-4)
    rad2, _ = dam_solver.render(**CAM, samples_per_pixel=1, output_normals_of_first_hit=True, seed=4)
    # the random offsets along the rays move first hits by less than a march step
    close = np.linalg.norm(rad2 - rad, axis=2) < 0.1
    assert close.mean() > 0.9


def test_render_path_tracing(dam_solver):
    rad, rgba = dam_solver.render(**CAM, samples_per_pixel=16, seed=5)
    assert np.isfinite(rad).all() and (rad >= 0).all()
    sky = np.isclose(rad, 1.0).all(axis=2)
    assert 0.02 < sky.mean() < 0.98   # both sky and surfaces in view
    assert (rad[~sky] < 1.0).all()    # lit by the sky through a diffuse bsdf with albedo < 1
    # the same seed, the same image; another seed, another estimate
    again, _ = dam_solver.render(**CAM, samples_per_pixel=16, seed=5)
    other, _ = dam_solver.render(**CAM, samples_per_pixel=16, seed=6)
    assert np.array_equal(rad, again) and not np.array_equal(rad, other)
    # tone mapping (ToneMapper.cpp:79-102): exposure, exponential curve, gamma, bytes
    v = np.clip(1.0 - np.exp(-(rad.astype(np.float32) * np.float32(0.2))), 0, 1) ** (1 / 2.2)
    assert np.abs(rgba[..., :3].astype(int) - (v * 255).astype(int)).max() <= 1
    assert (rgba[..., 3] == 255).all()
    # exactly the mapping fs_tone_map applies, which tests/test_tonemap.py pins to the
    # reference's ToneMapper byte for byte; the filmic curve through the render settings too
    assert np.array_equal(rgba, tone_map(rad))
    rad_f, rgba_f = dam_solver.render(**CAM, samples_per_pixel=16, seed=5, tone_mapper=1, exposure=0.6)
    assert np.array_equal(rad_f, rad) and np.array_equal(rgba_f, tone_map(rad, exposure=0.6, filmic=True))


def test_render_rejects_bad_arguments(dam_solver):
    from fluidsolver_b200._lib import FluidSolverError
    with pytest.raises(FluidSolverError, match="image size"):
        dam_solver.render(**dict(CAM, width=0))
    with pytest.raises(FluidSolverError, match="bad settings"):
        dam_solver.render(**CAM, samples_per_pixel=0)
    with pytest.raises(FluidSolverError, match="surface density fraction"):
        dam_solver.render(**CAM, surface_density_fraction=0.0)
    with pytest.raises(FluidSolverError, match="view direction"):
        dam_solver.render(**dict(CAM, view_direction=(0.0, 1.0, 0.0)))   # parallel to the up vector
    with pytest.raises(TypeError):
        dam_solver.render(**CAM, no_such_setting=1)
    # no rays: nothing to trace, no error
    out = dam_solver.trace_rays(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32))
    assert len(out["hit"]) == 0


def test_render_needs_a_3d_context():
    from fluidsolver_b200._lib import FluidSolverError
    sc = scenes.breaking_dam_2d(10, 10, 1.0, seed=1)
    s = make_solver("sesph-2d", "hashed-2d", [1000.0, 0.01], (0.001, 0.4, 0.25))
    s.data.collection = sc.collection
    with pytest.raises(FluidSolverError, match="3D"):
        s.trace_rays(np.zeros((1, 3), np.float32), np.ones((1, 3), np.float32))
    s.close()


def test_trace_rays_in_fp64_matches_fp32(golden):
    """The FP64 context marches the same points; its densities are double sums
    rounded to float, so hits agree up to the same rounding margin."""
    g = golden["raytrace"]
    res = {}
    for prec in ("fp32-kahan", "fp64"):
        s = make_solver("iisph-3d", "hashed-3d", SETTINGS_3D, (0.005, 0.4, 0.25), precision=prec)
        n = len(g["pos"])
        s.data.collection = ParticleCollection(position=g["pos"], velocity=np.zeros_like(g["pos"]), mass=g["mass"],
                                               density=np.ones(n, np.float32), type=g["type"])
        res[prec] = s.trace_rays(g["origins"], g["directions"])
        s.close()
    a, b = res["fp32-kahan"], res["fp64"]
    same = a["hit"] == b["hit"]
    assert same.mean() >= 0.995
    both = same & (a["hit"] >= 0)
    np.testing.assert_allclose(a["point"][both], b["point"][both], atol=1e-3, rtol=0)
