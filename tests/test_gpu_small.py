"""The small-scene step kernel (csrc/fs_small.cu): with FS_FLAG_ONE_KERNEL_STEPS,
fs_step / fs_run of a single scene of at most 4,096 particles run whole steps
in one launch of one thread-block cluster (up to 16 blocks, about 256
particles per block: the dams here take 4 to 16). Its phases call the
per-particle functions of the step-by-step kernels in the same order, on
shared-memory copies of the fields they gather, and its sort and cell table
are its own (a cluster-wide stable sort, a binary-searched table), so it must
give the same state bit for bit as the host-driven step-by-step path
(FS_FLAG_SYNC_EACH_ITERATION) in every precision mode, solver and contract it
serves (and so, in the reference-order mode, the reference's own results,
which the step-by-step path matches: tests/test_gpu_solvers.py,
tests/test_gpu_configs.py)."""
import numpy as np
import pytest

from conftest import bits_equal
from fluidsolver_b200 import _lib as F
from fluidsolver_b200 import scenes
from fluidsolver_b200.solver import ParticleCollection
from test_gpu_solvers import make_solver

pytestmark = pytest.mark.gpu

SES2 = [1000.0, 0.01]
IIS2 = [0.001, 2, 100, 0.5, 0.7, 0.01]
SES3 = [1000.0, 0.01, 1, 1.1, 1.1]
IIS3 = [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1]
GEN2 = (0.001, 0.4, 0.25)
GEN3 = (0.005, 0.4, 0.25)


def dam2d():
    return scenes.breaking_dam_2d(30, 24, width=60, height=50, seed=3).collection


def dam3d():
    return scenes.breaking_dam_3d(10, 9, 8, 1.0, tank=(20, 16, 14), seed=3).collection


CASES = {
    "sesph2d-hashed-exact": ("sesph-2d", "hashed-2d", SES2, GEN2, "fp32", True, dam2d),
    "sesph2d-quadratic-exact": ("sesph-2d", "quadratic-2d", SES2, GEN2, "fp32", True, dam2d),
    "sesph2d-hashed-fast": ("sesph-2d", "hashed-2d", SES2, GEN2, "fp32-kahan", False, dam2d),
    "sesph2d-hashed-fp64": ("sesph-2d", "hashed-2d", SES2, GEN2, "fp64", False, dam2d),
    "iisph2d-hashed-exact": ("iisph-2d", "hashed-2d", IIS2, GEN2, "fp32", True, dam2d),
    "iisph2d-quadratic-exact": ("iisph-2d", "quadratic-2d", IIS2, GEN2, "fp32", True, dam2d),
    "iisph2d-hashed-fast": ("iisph-2d", "hashed-2d", IIS2, GEN2, "fp32-kahan", False, dam2d),
    "iisph2d-hashed-fp64": ("iisph-2d", "hashed-2d", IIS2, GEN2, "fp64", False, dam2d),
    "sesph3d-hashed-exact": ("sesph-3d", "hashed-3d", SES3, GEN3, "fp32", True, dam3d),
    "iisph3d-hashed-exact": ("iisph-3d", "hashed-3d", IIS3, GEN3, "fp32", True, dam3d),
    "iisph3d-quadratic-exact": ("iisph-3d", "quadratic-3d", IIS3, GEN3, "fp32", True, dam3d),
    "iisph3d-compressed-exact": ("iisph-3d", "compressed-3d", IIS3, GEN3, "fp32", True, dam3d),
    "iisph3d-hashed-fp64": ("iisph-3d", "hashed-3d", IIS3, GEN3, "fp64", False, dam3d),
}
STEPS = 12
FIELDS = ("position", "velocity", "density", "pressure", "mass", "type", "tag")


def pair(name):
    solver, search, settings, gen, prec, exact, build = CASES[name]
    col = build()
    small = make_solver(solver, search, settings, gen, precision=prec, reference_order=exact, one_kernel_steps=True)
    steps = make_solver(solver, search, settings, gen, precision=prec, reference_order=exact, sync_each_iteration=True)
    small.data.collection = col
    steps.data.collection = ParticleCollection(**{f: getattr(col, f).copy() for f in FIELDS if getattr(col, f) is not None})
    return small, steps


@pytest.mark.parametrize("name", list(CASES))
def test_small_kernel_equals_the_step_by_step_path(name):
    small, steps = pair(name)
    for chunk in (1, 4, STEPS - 5):          # fs_step (one launch), then fs_run of several steps per launch
        a = small.run(chunk)
        for _ in range(chunk):
            b = steps.step()
        assert a.iterations == b.iterations and bits_equal(np.float32(a.actual_dt), np.float32(b.actual_dt)), name
        assert a.avg_density_error == b.avg_density_error
    x, y = small.collection(), steps.collection()
    for f in ("position", "velocity", "density", "pressure"):
        assert bits_equal(getattr(x, f), getattr(y, f)), (name, f)
    small.close()
    steps.close()


def test_small_kernel_runs_whole_steps_in_one_launch():
    small, steps = pair("iisph2d-hashed-exact")
    small.run(1)
    # 1,218 particles: a cluster of 8 blocks of about 150 (16 and 4 blocks
    # serve the other scenes here; a device that schedules no cluster that
    # large runs fewer, larger blocks)
    assert F.lib().fs_small_blocks(small.ctx) in (1, 2, 4, 8)
    before = F.lib().fs_launch_count(small.ctx)
    small.run(20)
    # fs_run: its first step settles the list capacity (one launch), the
    # other 19 go in one more
    assert F.lib().fs_launch_count(small.ctx) - before == 2
    t = small.phase_times()
    assert len(t) == 5 and all(v >= 0.0 for v in t) and sum(t) > 0.0
    small.close()
    steps.close()


def test_small_kernel_grows_the_lists():
    """A cluster denser than the default capacity: the kernel reports the
    overflow, the step is redone on grown lists, and the results match the
    step-by-step path, which grows its lists the same way."""
    rng = np.random.default_rng(11)
    i, j = np.meshgrid(np.arange(24), np.arange(24), indexing="ij")
    dense = np.stack([i.ravel(), j.ravel()], 1) * 0.5 + rng.uniform(-0.01, 0.01, (576, 2))   # ~50 neighbors
    pos = np.concatenate([dense, rng.uniform(20, 40, (200, 2))]).astype(np.float32)
    n = len(pos)
    col = ParticleCollection(position=pos, velocity=np.zeros_like(pos), mass=np.ones(n, np.float32),
                             density=np.ones(n, np.float32), type=np.zeros(n, np.uint8))
    small = make_solver("sesph-2d", "hashed-2d", SES2, GEN2, precision="fp32", reference_order=True,
                        one_kernel_steps=True)
    steps = make_solver("sesph-2d", "hashed-2d", SES2, GEN2, precision="fp32", reference_order=True,
                        sync_each_iteration=True)
    small.data.collection = col
    steps.data.collection = ParticleCollection(position=pos.copy(), velocity=np.zeros_like(pos),
                                               mass=np.ones(n, np.float32), density=np.ones(n, np.float32),
                                               type=np.zeros(n, np.uint8))
    a = small.run(3)
    for _ in range(3):
        b = steps.step()
    assert a.max_neighbors > 32 and a.max_neighbors == b.max_neighbors
    x, y = small.collection(), steps.collection()
    for f in ("position", "velocity", "density", "pressure"):
        assert bits_equal(getattr(x, f), getattr(y, f)), f
    small.close()
    steps.close()


@pytest.mark.parametrize("dims", [(6, 5, 14, 12), (12, 10, 24, 20)])
def test_small_kernel_on_one_and_two_blocks(dims):
    """Scenes of 162 and 330 particles: a cluster of one block and of two
    (about 256 particles per block), in both 2D solvers and exact order."""
    nx, ny, w, h = dims
    for solver, settings in (("sesph-2d", SES2), ("iisph-2d", IIS2)):
        col = scenes.breaking_dam_2d(nx, ny, width=w, height=h, seed=5).collection
        small = make_solver(solver, "hashed-2d", settings, GEN2, precision="fp32", reference_order=True,
                            one_kernel_steps=True)
        steps = make_solver(solver, "hashed-2d", settings, GEN2, precision="fp32", reference_order=True,
                            sync_each_iteration=True)
        small.data.collection = col
        steps.data.collection = ParticleCollection(**{f: getattr(col, f).copy() for f in FIELDS
                                                      if getattr(col, f) is not None})
        a = small.run(8)
        assert F.lib().fs_small_blocks(small.ctx) == (1 if len(col) <= 256 else 2)
        assert F.lib().fs_small_blocks(steps.ctx) == 0
        for _ in range(8):
            b = steps.step()
        assert a.iterations == b.iterations
        x, y = small.collection(), steps.collection()
        for f in ("position", "velocity", "density", "pressure"):
            assert bits_equal(getattr(x, f), getattr(y, f)), (solver, dims, f)
        small.close()
        steps.close()
