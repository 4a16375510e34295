"""Host-side mirror of libFluid's solver and neighborhood-search interfaces
over the C-ABI, so that parity tests and benchmarks drive the device path the
way libFluid's own code drives its solvers:

    solver = IISPHFluidSolver3D(search="hashed-3d")
    solver.parameters.particle_size = 0.01 ...        (IFluidSolver.hpp:18-23)
    solver.settings.omega = 0.5 ...                   (IISPHSettings3D.hpp:6-20)
    solver.timestep_generator.settings.timestep = ... (ConstantTimestepGenerator.hpp:8-13)
    solver.data.collection = ParticleCollection(...)
    solver.execute_neighborhood_search()              (IFluidSolver.hpp:31)
    solver.execute_simulation_step(timepoint)         (IFluidSolver.hpp:30)

The collection is device resident between calls; `solver.collection()` copies
it back (the reference's host ParticleCollection is authoritative only when an
entity or sensor reads it).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib as F

SEARCH_KINDS = {
    "quadratic-2d": F.FS_SEARCH_QUADRATIC_2D,
    "hashed-2d": F.FS_SEARCH_HASHED_2D,
    "compact-hashing-2d": F.FS_SEARCH_COMPACT_2D,
    "quadratic-3d": F.FS_SEARCH_QUADRATIC_3D,
    "hashed-3d": F.FS_SEARCH_HASHED_3D,
    "compressed-3d": F.FS_SEARCH_COMPRESSED_3D,
}
PRECISIONS = {"fp32": F.FS_PRECISION_FP32, "fp32-kahan": F.FS_PRECISION_FP32_KAHAN, "fp64": F.FS_PRECISION_FP64}


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


@dataclass
class ParticleCollection:
    """Dense SoA particle arrays in host order (the components of
    fluidSolver/Particle.hpp:15-50 that the hot path reads and writes)."""

    position: np.ndarray
    velocity: np.ndarray | None = None
    acceleration: np.ndarray | None = None
    external: np.ndarray | None = None
    mass: np.ndarray | None = None
    density: np.ndarray | None = None
    pressure: np.ndarray | None = None
    type: np.ndarray | None = None
    tag: np.ndarray | None = None
    # IISPH data (download only)
    predicted_velocity: np.ndarray | None = None
    non_pressure_acceleration: np.ndarray | None = None
    source_term: np.ndarray | None = None
    diagonal_element: np.ndarray | None = None

    @property
    def dim(self) -> int:
        return self.position.shape[1]

    def __len__(self) -> int:
        return self.position.shape[0]

    def size(self) -> int:
        return len(self)

    def normalized(self) -> "ParticleCollection":
        n, d = self.position.shape
        f32 = lambda a, shape: np.ascontiguousarray(a, dtype=np.float32).reshape(shape) if a is not None else None
        return ParticleCollection(
            position=f32(self.position, (n, d)), velocity=f32(self.velocity, (n, d)),
            acceleration=f32(self.acceleration, (n, d)), external=f32(self.external, (n, d)),
            mass=f32(self.mass, (n,)), density=f32(self.density, (n,)), pressure=f32(self.pressure, (n,)),
            type=np.ascontiguousarray(self.type, dtype=np.uint8) if self.type is not None else None,
            tag=np.ascontiguousarray(self.tag, dtype=np.uint32) if self.tag is not None else None)

    def as_fs(self) -> F.FsParticles:
        p = F.FsParticles()
        p.n = len(self)
        for name in ("position", "velocity", "acceleration", "external", "mass", "density", "pressure", "type", "tag",
                     "predicted_velocity", "non_pressure_acceleration", "source_term", "diagonal_element"):
            setattr(p, name, _ptr(getattr(self, name)))
        return p


@dataclass
class Timepoint:
    """time/Timepoint.hpp:7-14"""
    timestep_number: int = 0
    simulation_time: float = 0.0
    desired_time_step: float = 0.0
    actual_time_step: float = 0.0


@dataclass
class SimulationParameters:
    rest_density: float = 1000.0
    gravity: float = 9.81
    particle_size: float = 0.1


@dataclass
class ConstantTimestepGeneratorSettings:
    timestep: float = 0.001
    lambda_v: float = 0.4
    lambda_a: float = 0.25


@dataclass
class ConstantTimestepGenerator:
    """time/ConstantTimestepGenerator.hpp: generate_next_timestep() returns settings.timestep."""
    settings: ConstantTimestepGeneratorSettings = field(default_factory=ConstantTimestepGeneratorSettings)

    def generate_next_timestep(self) -> None:
        pass

    def get_generated_timestep(self) -> float:
        return self.settings.timestep


@dataclass
class DynamicCflTimestepGeneratorSettings:
    max_timestep: float = 0.02
    min_timestep: float = 0.0001
    cfl_number: float = 0.8      # a setting of the reference that its generator does not read
    lambda_v: float = 0.4
    lambda_a: float = 0.25


@dataclass
class DynamicCflTimestepGenerator:
    """time/DynamicCflTimestepGenerator.hpp: the time step follows the largest velocity and
    acceleration of the active particles (DynamicCflTimestepGenerator.cpp:45-59). The device
    generates it at the start of every step, inside the step's CUDA graph; the step calls'
    desired_dt is then ignored, and get_generated_timestep() returns the last step's choice."""
    settings: DynamicCflTimestepGeneratorSettings = field(default_factory=DynamicCflTimestepGeneratorSettings)
    generated_timestep: float = 0.0

    def generate_next_timestep(self) -> None:
        pass

    def get_generated_timestep(self) -> float:
        return self.generated_timestep if self.generated_timestep > 0 else self.settings.max_timestep


def _generator_params(g, p) -> None:
    """Copies a time step generator's settings into fs_params."""
    if isinstance(g, DynamicCflTimestepGenerator):
        st = g.settings
        p.timestep_generator = F.FS_TIMESTEP_DYNAMIC_CFL
        p.min_timestep, p.max_timestep = st.min_timestep, st.max_timestep
        p.timestep, p.lambda_v, p.lambda_a = st.max_timestep, st.lambda_v, st.lambda_a
    else:
        st = g.settings
        p.timestep_generator = F.FS_TIMESTEP_CONSTANT
        p.timestep, p.lambda_v, p.lambda_a = st.timestep, st.lambda_v, st.lambda_a


def _default_dt(g) -> float:
    return g.settings.timestep if isinstance(g, ConstantTimestepGenerator) else g.settings.max_timestep


def _note_generated(g, stats) -> None:
    if isinstance(g, DynamicCflTimestepGenerator):
        g.generated_timestep = float(stats.desired_dt)


def read_particles(path: str) -> "ParticleCollection":
    """A ParticleSerializer v1 particle file (ParticleSerializer.cpp:89-141; scenario .data files,
    FluidConsole dumps) in host order. Components the file lacks come back as None."""
    dim, n, comp = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_uint32()
    F.check(F.lib().fs_particles_file_info(str(path).encode(), ctypes.byref(dim), ctypes.byref(n), ctypes.byref(comp)))
    d, n, c = dim.value, n.value, comp.value
    mv = c & (F.FS_COMPONENT_MOVEMENT_2D | F.FS_COMPONENT_MOVEMENT_3D)
    ex = c & (F.FS_COMPONENT_EXTERNAL_2D | F.FS_COMPONENT_EXTERNAL_3D)
    vec = lambda on: np.zeros((n, d), np.float32) if on else None
    sca = lambda on: np.zeros(n, np.float32) if on else None
    info, data = c & F.FS_COMPONENT_INFO, c & F.FS_COMPONENT_DATA
    out = ParticleCollection(position=vec(mv), velocity=vec(mv), acceleration=vec(mv), external=vec(ex),
                             mass=sca(data), density=sca(data), pressure=sca(data),
                             type=np.zeros(n, np.uint8) if info else None, tag=np.zeros(n, np.uint32) if info else None)
    view = F.FsParticles()
    view.n = n
    for name in ("position", "velocity", "acceleration", "external", "mass", "density", "pressure", "type", "tag"):
        setattr(view, name, _ptr(getattr(out, name)))
    F.check(F.lib().fs_particles_file_read(str(path).encode(), ctypes.byref(view)))
    return out


def write_particles(path: str, col: "ParticleCollection") -> None:
    """Writes `col` as a ParticleSerializer v1 particle file (ParticleSerializer.cpp:41-84) with the
    components it holds."""
    c = col.normalized()
    F.check(F.lib().fs_particles_file_write(str(path).encode(), c.dim, ctypes.byref(c.as_fs())))


def tone_map(radiance, exposure: float = 0.2, gamma: float = 2.2, filmic: bool = False,
             gamma_correction: bool = True) -> np.ndarray:
    """ToneMapper::map_render_target_to_image (ToneMapper.cpp:71-102) on radiance of shape (..., 3):
    bytes of shape (..., 4) (fs_tone_map, host code; the mapping fs_render applies)."""
    rad = np.ascontiguousarray(radiance, np.float32)
    n = rad.size // 3
    rs = F.FsRenderSettings()
    F.lib().fs_render_settings_default(ctypes.byref(rs))
    rs.exposure, rs.gamma, rs.tone_mapper, rs.gamma_correction = exposure, gamma, int(filmic), int(gamma_correction)
    out = np.zeros(rad.shape[:-1] + (4,), np.uint8)
    F.check(F.lib().fs_tone_map(rad.ctypes.data, n, ctypes.byref(rs), out.ctypes.data))
    return out


def sort_keys(keys, bits: int, device: int = 0):
    """The searches' stable radix sort on keys (uint32 or uint64, each below 2**bits), on the
    device (fs_sort_keys): (sorted keys, input position of each); equal keys keep input order."""
    k = np.ascontiguousarray(keys)
    if k.dtype not in (np.uint32, np.uint64):
        raise TypeError("keys must be uint32 or uint64")
    n = k.size
    out = np.empty_like(k)
    order = np.empty(n, np.uint32)
    F.check(F.lib().fs_sort_keys(device, k.ctypes.data, k.itemsize, n, bits, out.ctypes.data, order.ctypes.data))
    return out, order


def _tuning_dict(t) -> dict:
    """fs_tuning as a dict: the values in use and every measured time, keyed by the value tried."""
    return {"tuned": bool(t.tuned), "first_loop_prefetch": t.first_loop_prefetch,
            "pressure_prefetch": t.pressure_prefetch, "tile_cap": t.tile_cap, "block_size": t.block_size,
            "pressure_threads_per_owner": t.pressure_threads_per_owner,
            "pressure_iteration_ms_by_threads": {q: v for q, v in zip(F.THREADS_PER_OWNER,
                                                                    t.pressure_iteration_ms_by_threads) if v > 0},
            "first_loop_ms": {d + 1: v for d, v in enumerate(t.first_loop_ms) if v > 0},
            "pressure_iteration_ms": {d + 1: v for d, v in enumerate(t.pressure_iteration_ms) if v > 0},
            "step_ms_by_tile_cap": {c: v for c, v in zip(F.TILE_CAPS, t.step_ms_by_tile_cap) if v > 0},
            "fallback_tiles_by_tile_cap": {c: v for c, v, m in zip(F.TILE_CAPS, t.fallback_tiles_by_tile_cap,
                                                                   t.step_ms_by_tile_cap) if m > 0},
            "step_ms_by_block_size": {b: v for b, v in zip(F.BLOCK_SIZES, t.step_ms_by_block_size) if v > 0}}


class BoundaryPreprocessor:
    """entities/BoundaryPreprocessor.hpp: an entity that runs before the solver and sets the mass of
    every boundary particle from its boundary neighbors. This one runs on the device state of
    `solver` (its last neighborhood search), so the collection need not come back to the host."""

    execution_point = "BeforeSolver"

    def __init__(self, solver):
        self.solver = solver

    def execute_simulation_step(self, timepoint: "Timepoint", before_solver: bool) -> None:
        if not before_solver:
            raise ValueError("It makes only sense to execute the preprocessor before the solver!")
        self.solver.boundary_preprocess()


@dataclass
class IISPHSettings3D:
    max_density_error_allowed: float = 0.001
    min_number_of_iterations: int = 2
    max_number_of_iterations: int = 100
    omega: float = 0.5
    gamma: float = 0.7
    viscosity: float = 5.0
    single_layer_boundary: bool = False
    single_layer_boundary_gamma_1: float = 1.1


@dataclass
class IISPHSettings:
    MaxDensityErrorAllowed: float = 0.001
    MinNumberOfIterations: int = 2
    MaxNumberOfIterations: int = 100
    Omega: float = 0.5
    Gamma: float = 0.7
    Viscosity: float = 5.0


@dataclass
class SESPHSettings3D:
    StiffnessK: float = 100000.0
    Viscosity: float = 5.0
    single_layer_boundary: bool = False
    single_layer_boundary_gamma_1: float = 1.1
    single_layer_boundary_gamma_2: float = 1.1


@dataclass
class SESPHSettings:
    StiffnessK: float = 100000.0
    Viscosity: float = 5.0


class _Data:
    def __init__(self):
        self.collection: ParticleCollection | None = None
        self.changed = True

    def notify_that_data_changed(self):
        self.changed = True


class _DeviceContext:
    """Owns one fs_ctx."""

    def __init__(self, params: F.FsParams):
        self.L = F.lib()
        self.params = params
        self.ctx = ctypes.c_void_p()
        F.check(self.L.fs_create(ctypes.byref(params), ctypes.byref(self.ctx)))

    def close(self):
        if self.ctx:
            self.L.fs_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FluidSolverBase:
    """IFluidSolverBase (IFluidSolver.hpp:16-34) over the device path."""

    DIM = 3
    SOLVER = F.FS_SOLVER_NONE
    DEFAULT_SEARCH = "hashed-3d"

    def __init__(self, search: str | None = None, precision: str = "fp32-kahan", reference_order: bool = False,
                 device: int = 0, neighbor_capacity: int = 0, sync_each_iteration: bool = False,
                 one_kernel_steps: bool = False):
        self.search = search or self.DEFAULT_SEARCH
        if self.search not in SEARCH_KINDS:
            raise ValueError(f"unknown neighborhood search {self.search!r}")
        self.precision = precision
        self.reference_order = reference_order
        self.sync_each_iteration = sync_each_iteration
        self.one_kernel_steps = one_kernel_steps   # FS_FLAG_ONE_KERNEL_STEPS
        self.device = device
        self.neighbor_capacity = neighbor_capacity
        self.parameters = SimulationParameters()
        self.timestep_generator = ConstantTimestepGenerator()
        self.data = _Data()
        self._dev: _DeviceContext | None = None
        self._key = None
        self.last_stats = F.FsStepStats()

    # ---- configuration -------------------------------------------------
    def _fill_settings(self, p: F.FsParams) -> None:
        raise NotImplementedError

    def _params(self, n: int) -> F.FsParams:
        p = F.FsParams()
        F.lib().fs_params_default(ctypes.byref(p), self.DIM, self.SOLVER, SEARCH_KINDS[self.search])
        p.precision = PRECISIONS[self.precision]
        p.flags = (F.FS_FLAG_REFERENCE_ORDER if self.reference_order else 0) | \
            (F.FS_FLAG_SYNC_EACH_ITERATION if self.sync_each_iteration else 0) | \
            (F.FS_FLAG_ONE_KERNEL_STEPS if self.one_kernel_steps else 0)
        p.device = self.device
        p.rest_density = self.parameters.rest_density
        p.gravity = self.parameters.gravity
        p.particle_size = self.parameters.particle_size
        _generator_params(self.timestep_generator, p)
        p.max_particles = max(n, 1)
        p.neighbor_capacity = self.neighbor_capacity
        self._fill_settings(p)
        return p

    def initialize(self) -> None:
        """Creates / reconfigures the device context and uploads the
        collection when data changed (IISPHFluidSolver3D.hpp:79-103)."""
        col = self.data.collection
        if col is None:
            raise F.FluidSolverError(F.FS_ERR_INVALID, "Particle collection is null.")
        p = self._params(len(col))
        key = (p.max_particles, p.precision, p.flags, p.search, p.solver)
        if self._dev is None or key != self._key:
            if self._dev is not None:
                self._dev.close()
            self._dev = _DeviceContext(p)
            self._key = key
            self.data.changed = True
        else:
            F.check(F.lib().fs_set_params(self._dev.ctx, ctypes.byref(p)))
        if self.data.changed:
            self._uploaded = col.normalized()
            F.check(F.lib().fs_upload(self._dev.ctx, ctypes.byref(self._uploaded.as_fs())))
            self.data.changed = False

    @property
    def ctx(self):
        if self._dev is None:
            self.initialize()
        return self._dev.ctx

    # ---- IFluidSolverBase ---------------------------------------------
    def execute_neighborhood_search(self) -> None:
        self.initialize()
        F.check(F.lib().fs_find_neighbors(self._dev.ctx))

    def execute_simulation_step(self, timepoint: Timepoint) -> None:
        self.initialize()
        F.check(F.lib().fs_solve_step(self._dev.ctx, float(timepoint.desired_time_step), ctypes.byref(self.last_stats)))
        _note_generated(self.timestep_generator, self.last_stats)
        if isinstance(self.timestep_generator, DynamicCflTimestepGenerator):
            timepoint.desired_time_step = float(self.last_stats.desired_dt)
        timepoint.actual_time_step = float(self.last_stats.actual_dt)

    def step(self, desired_dt: float | None = None) -> F.FsStepStats:
        """Neighborhood search + step in one call (fs_step)."""
        self.initialize()
        dt = _default_dt(self.timestep_generator) if desired_dt is None else desired_dt
        F.check(F.lib().fs_step(self._dev.ctx, float(dt), ctypes.byref(self.last_stats)))
        _note_generated(self.timestep_generator, self.last_stats)
        return self.last_stats

    def run(self, steps: int, desired_dt: float | None = None) -> F.FsStepStats:
        """`steps` steps without host synchronisation in between (fs_run);
        returns the last step's statistics."""
        self.initialize()
        dt = _default_dt(self.timestep_generator) if desired_dt is None else desired_dt
        F.check(F.lib().fs_run(self._dev.ctx, int(steps), float(dt), ctypes.byref(self.last_stats)))
        _note_generated(self.timestep_generator, self.last_stats)
        return self.last_stats

    def phase_times(self) -> list[float]:
        out = np.zeros(5, np.float32)
        F.check(F.lib().fs_last_phase_times(self.ctx, out.ctypes.data))
        return out.tolist()

    # ---- neighborhood interface ---------------------------------------
    def neighbor_lists(self) -> tuple[np.ndarray, np.ndarray]:
        """CSR (offsets, indices) of the contract's lists in host index space, each list ascending."""
        n = len(self.data.collection)
        off = np.zeros(n + 1, np.int64)
        tot = ctypes.c_int64()
        st = F.lib().fs_get_neighbors_csr(self.ctx, off.ctypes.data, None, ctypes.byref(tot))
        if st not in (F.FS_OK, F.FS_ERR_CAPACITY):
            F.check(st)
        idx = np.zeros(max(tot.value, 1), np.int64)
        F.check(F.lib().fs_get_neighbors_csr(self.ctx, off.ctypes.data, idx.ctypes.data, ctypes.byref(tot)))
        return off, idx[:tot.value]

    # ---- entities and sensors on the device ---------------------------
    def boundary_preprocess(self) -> None:
        """BoundaryPreprocessor::execute_simulation_step (BoundaryPreprocessor.cpp:7-48) on the device
        state: boundary masses from the boundary neighbors of the last search (fs_boundary_preprocess)."""
        F.check(F.lib().fs_boundary_preprocess(self.ctx))

    def global_statistics(self, zero_height: float = 0.0) -> dict:
        """The global sensors of ParticleStatistics.cpp:17-201 over the device state (fs_global_statistics)."""
        st = F.FsGlobalStats()
        F.check(F.lib().fs_global_statistics(self.ctx, float(zero_height), ctypes.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_ if name != "reserved"}

    def autotune(self) -> dict:
        """Chooses the fast mode's launch shapes (prefetch depths, staging cap, block size) by timing
        steps on a copy of this solver's device context (fs_autotune); this solver's state is left as
        it was. Returns every measured time."""
        t = F.FsTuning()
        F.check(F.lib().fs_autotune(self.ctx, ctypes.byref(t)))
        return _tuning_dict(t)

    def set_tuning(self, first_loop_prefetch: int, pressure_prefetch: int, tile_cap: int = 0,
                   block_size: int = 0, pressure_threads_per_owner: int = 0) -> None:
        """The fast mode's launch shapes (0 keeps the current cap / block size / threads per owner)."""
        t = F.FsTuning(first_loop_prefetch=first_loop_prefetch, pressure_prefetch=pressure_prefetch,
                       tile_cap=tile_cap, block_size=block_size,
                       pressure_threads_per_owner=pressure_threads_per_owner)
        F.check(F.lib().fs_set_tuning(self.ctx, ctypes.byref(t)))

    # ---- the fluid path tracer (visualizer/raytracer/FluidRaytracer3D) ----
    def trace_rays(self, origins, directions, surface_density_fraction: float = 0.8) -> dict:
        """First surface hits of rays through the SPH density (fs_trace_rays): hit (-1 none, 0/1 the
        fluid surface from outside/inside, 2 a boundary), point, normal, length."""
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        m = len(o)
        out = {"hit": np.zeros(m, np.int32), "point": np.zeros((m, 3), np.float32),
               "normal": np.zeros((m, 3), np.float32), "length": np.zeros(m, np.float32)}
        F.check(F.lib().fs_trace_rays(self.ctx, float(surface_density_fraction), m, o.ctypes.data, d.ctypes.data,
                                      out["hit"].ctypes.data, out["point"].ctypes.data, out["normal"].ctypes.data,
                                      out["length"].ctypes.data))
        return out

    def render(self, position, view_direction, view_up=(0.0, 1.0, 0.0), width: int = 320, height: int = 240,
               field_of_view_x: float = 90.0 / 360.0 * 2.0 * 3.1415, flip_y: bool = False, **settings):
        """FluidRaytracer3D::render on the device state (fs_render): (radiance, rgba) arrays of
        height x width x 3 floats and x 4 bytes. settings: samples_per_pixel, maximum_recursion_depth,
        output_normals_of_first_hit, surface_density_fraction, exposure, gamma, seed, tone_mapper (0
        exponential, 1 filmic), gamma_correction."""
        cam = F.FsCamera()
        cam.position[:], cam.view_direction[:], cam.view_up[:] = position, view_direction, view_up
        cam.field_of_view_x, cam.width, cam.height, cam.flip_y = field_of_view_x, width, height, int(flip_y)
        rs = F.FsRenderSettings()
        F.lib().fs_render_settings_default(ctypes.byref(rs))
        for k, v in settings.items():
            if not hasattr(rs, k):
                raise TypeError(f"unknown render setting {k!r}")
            setattr(rs, k, int(v) if isinstance(v, bool) else v)
        rad = np.zeros((height, width, 3), np.float32)
        rgba = np.zeros((height, width, 4), np.uint8)
        F.check(F.lib().fs_render(self.ctx, ctypes.byref(cam), ctypes.byref(rs), rad.ctypes.data, rgba.ctypes.data))
        return rad, rgba

    def dump(self, path: str) -> None:
        """The device state as a particle file (fs_dump), FluidConsole's particle dump."""
        F.check(F.lib().fs_dump(self.ctx, str(path).encode()))

    def solver_lists(self) -> tuple[np.ndarray, np.ndarray]:
        """CSR (offsets, indices) of the lists the solver's passes walk (3D IISPH fast mode: the tile
        lists), host index space, each list ascending. They must equal neighbor_lists() for the owners."""
        n = len(self.data.collection)
        off = np.zeros(n + 1, np.int64)
        tot = ctypes.c_int64()
        F.check(F.lib().fs_get_solver_lists_csr(self.ctx, off.ctypes.data, None, ctypes.byref(tot)))
        idx = np.zeros(max(tot.value, 1), np.int64)
        F.check(F.lib().fs_get_solver_lists_csr(self.ctx, off.ctypes.data, idx.ctypes.data, ctypes.byref(tot)))
        return off, idx[:tot.value]

    def get_neighbors(self, index: int) -> np.ndarray:
        off, idx = self.neighbor_lists()
        return idx[off[index]:off[index + 1]]

    def get_neighbors_of_position(self, position, cap: int = 4096) -> np.ndarray:
        pos = np.zeros(3, np.float32)
        pos[:self.DIM] = np.asarray(position, np.float32)[:self.DIM]
        cnt = ctypes.c_int64()
        while True:
            out = np.zeros(cap, np.int64)
            F.check(F.lib().fs_query_position(self.ctx, pos.ctypes.data, out.ctypes.data, cap, ctypes.byref(cnt)))
            if cnt.value <= cap:
                return out[:cnt.value]
            cap = cnt.value

    # ---- state ---------------------------------------------------------
    def collection(self, iisph: bool = False) -> ParticleCollection:
        """Downloads the device state in host order."""
        n = len(self.data.collection)
        d = self.DIM
        out = ParticleCollection(
            position=np.zeros((n, d), np.float32), velocity=np.zeros((n, d), np.float32),
            acceleration=np.zeros((n, d), np.float32), external=np.zeros((n, d), np.float32),
            mass=np.zeros(n, np.float32), density=np.zeros(n, np.float32), pressure=np.zeros(n, np.float32),
            type=np.zeros(n, np.uint8), tag=np.zeros(n, np.uint32))
        if iisph:
            out.predicted_velocity = np.zeros((n, d), np.float32)
            out.non_pressure_acceleration = np.zeros((n, d), np.float32)
            out.source_term = np.zeros(n, np.float32)
            out.diagonal_element = np.zeros(n, np.float32)
        F.check(F.lib().fs_download(self.ctx, ctypes.byref(out.as_fs())))
        return out

    def close(self):
        if self._dev is not None:
            self._dev.close()
            self._dev = None


class IISPHFluidSolver3D(FluidSolverBase):
    """IISPHFluidSolver3D (fluidSolver/solver/IISPHFluidSolver3D.hpp:22-610)."""
    DIM = 3
    SOLVER = F.FS_SOLVER_IISPH_3D
    DEFAULT_SEARCH = "hashed-3d"

    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.settings = IISPHSettings3D()

    @property
    def stat_last_iteration_count(self) -> int:
        return int(self.last_stats.iterations)

    @property
    def stat_last_average_predicted_density_error(self) -> float:
        return float(self.last_stats.avg_density_error)

    def _fill_settings(self, p):
        s = self.settings
        p.max_density_error = s.max_density_error_allowed
        p.min_iterations = s.min_number_of_iterations
        p.max_iterations = s.max_number_of_iterations
        p.omega, p.gamma, p.viscosity = s.omega, s.gamma, s.viscosity
        p.single_layer_boundary = 1 if s.single_layer_boundary else 0
        p.single_layer_gamma_1 = s.single_layer_boundary_gamma_1


class BatchedIISPHFluidSolver3D:
    """Many independent 3D IISPH scenes advanced together (fs_batch_create,
    fs_batch_run). One launch per sub-phase covers every scene. Each scene
    keeps its own pressure-loop convergence test and its own CFL-clamped time
    step, and particles of different scenes never interact. The physics of
    each scene is IISPHFluidSolver3D's (same parameter and settings objects);
    the reference has no batched form, it runs one solver object per scene.

    scenes: one ParticleCollection per scene (host order within each)."""

    def __init__(self, scenes: list, device: int = 0, neighbor_capacity: int = 0):
        self._template = IISPHFluidSolver3D(search="hashed-3d", precision="fp32-kahan", device=device,
                                            neighbor_capacity=neighbor_capacity)
        self.parameters = self._template.parameters
        self.settings = self._template.settings
        self.scenes = [c.normalized() for c in scenes]
        self.offsets = np.concatenate([[0], np.cumsum([len(c) for c in self.scenes])]).astype(np.int64)
        self._ctx = None
        self.last_stats = None

    def set_tuning(self, first_loop_prefetch: int, pressure_prefetch: int, tile_cap: int = 0,
                   block_size: int = 0, pressure_threads_per_owner: int = 0) -> None:
        """The fast mode's launch shapes, e.g. as IISPHFluidSolver3D.autotune() chose them on a
        representative scene (fs_set_tuning); 0 keeps the current cap / block size / threads per owner."""
        t = F.FsTuning(first_loop_prefetch=first_loop_prefetch, pressure_prefetch=pressure_prefetch,
                       tile_cap=tile_cap, block_size=block_size,
                       pressure_threads_per_owner=pressure_threads_per_owner)
        F.check(F.lib().fs_set_tuning(self.ctx, ctypes.byref(t)))

    @property
    def timestep_generator(self):
        """ConstantTimestepGenerator or DynamicCflTimestepGenerator (per scene on the device)."""
        return self._template.timestep_generator

    @timestep_generator.setter
    def timestep_generator(self, g) -> None:
        self._template.timestep_generator = g

    def initialize(self) -> None:
        if self._ctx is not None:
            return
        n = int(self.offsets[-1])
        p = self._template._params(n)
        ctx = ctypes.c_void_p()
        F.check(F.lib().fs_batch_create(ctypes.byref(p), len(self.scenes), self.offsets.ctypes.data, ctypes.byref(ctx)))
        self._ctx = ctx
        cat = lambda name: None if getattr(self.scenes[0], name) is None else \
            np.ascontiguousarray(np.concatenate([getattr(c, name) for c in self.scenes]))
        self._uploaded = ParticleCollection(**{name: cat(name) for name in (
            "position", "velocity", "acceleration", "external", "mass", "density", "pressure", "type", "tag")})
        F.check(F.lib().fs_upload(self._ctx, ctypes.byref(self._uploaded.as_fs())))

    @property
    def ctx(self):
        self.initialize()
        return self._ctx

    def run(self, steps: int, desired_dt: float | None = None):
        """`steps` steps of every scene; returns one FsStepStats per scene
        (the last step's)."""
        self.initialize()
        dt = _default_dt(self.timestep_generator) if desired_dt is None else desired_dt
        stats = (F.FsStepStats * len(self.scenes))()
        F.check(F.lib().fs_batch_run(self._ctx, int(steps), float(dt), ctypes.cast(stats, ctypes.c_void_p)))
        self.last_stats = list(stats)
        return self.last_stats

    def collections(self) -> list:
        """Downloads every scene's state (host order within each scene)."""
        self.initialize()
        n, d = int(self.offsets[-1]), 3
        out = ParticleCollection(
            position=np.zeros((n, d), np.float32), velocity=np.zeros((n, d), np.float32),
            acceleration=np.zeros((n, d), np.float32), external=np.zeros((n, d), np.float32),
            mass=np.zeros(n, np.float32), density=np.zeros(n, np.float32), pressure=np.zeros(n, np.float32),
            type=np.zeros(n, np.uint8), tag=np.zeros(n, np.uint32))
        F.check(F.lib().fs_download(self._ctx, ctypes.byref(out.as_fs())))
        res = []
        for a, b in zip(self.offsets[:-1], self.offsets[1:]):
            res.append(ParticleCollection(**{k: (None if v is None else v[a:b]) for k, v in out.__dict__.items()}))
        return res

    def close(self) -> None:
        if self._ctx:
            F.lib().fs_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class IISPHFluidSolver(FluidSolverBase):
    """IISPHFluidSolver, 2D (fluidSolver/solver/IISPHFluidSolver.hpp:21-548)."""
    DIM = 2
    SOLVER = F.FS_SOLVER_IISPH_2D
    DEFAULT_SEARCH = "quadratic-2d"

    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.settings = IISPHSettings()

    def _fill_settings(self, p):
        s = self.settings
        p.max_density_error = s.MaxDensityErrorAllowed
        p.min_iterations = s.MinNumberOfIterations
        p.max_iterations = s.MaxNumberOfIterations
        p.omega, p.gamma, p.viscosity = s.Omega, s.Gamma, s.Viscosity


class SESPHFluidSolver3D(FluidSolverBase):
    """SESPHFluidSolver3D (fluidSolver/solver/SESPHFluidSolver3D.hpp:12-339)."""
    DIM = 3
    SOLVER = F.FS_SOLVER_SESPH_3D
    DEFAULT_SEARCH = "hashed-3d"

    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.settings = SESPHSettings3D()

    def _fill_settings(self, p):
        s = self.settings
        p.stiffness, p.viscosity = s.StiffnessK, s.Viscosity
        p.single_layer_boundary = 1 if s.single_layer_boundary else 0
        p.single_layer_gamma_1 = s.single_layer_boundary_gamma_1
        p.single_layer_gamma_2 = s.single_layer_boundary_gamma_2


class SESPHFluidSolver(FluidSolverBase):
    """SESPHFluidSolver, 2D (fluidSolver/solver/SESPHFluidSolver.hpp:12-299)."""
    DIM = 2
    SOLVER = F.FS_SOLVER_SESPH_2D
    DEFAULT_SEARCH = "quadratic-2d"

    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.settings = SESPHSettings()

    def _fill_settings(self, p):
        s = self.settings
        p.stiffness, p.viscosity = s.StiffnessK, s.Viscosity


class NeighborhoodSearch(FluidSolverBase):
    """A neighborhood search on its own (the NS concept, IFluidSolver.hpp:36-73):
    collection, search_radius, find_neighbors(), get_neighbors(index | position).
    The search radius is 2 * particle_size as the solvers set it
    (IISPHFluidSolver3D.hpp:94)."""

    SOLVER = F.FS_SOLVER_NONE

    def __init__(self, search: str, search_radius: float, **k):
        super().__init__(search=search, **k)
        self.DIM = 2 if search.endswith("2d") else 3
        self.parameters.particle_size = search_radius / 2.0
        self.settings = None

    @property
    def search_radius(self) -> float:
        return self.parameters.particle_size * 2.0

    def _fill_settings(self, p):
        pass

    def find_neighbors(self) -> None:
        self.execute_neighborhood_search()

    def set_positions(self, position: np.ndarray) -> None:
        self.data.collection.position = np.ascontiguousarray(position, np.float32)
        self.data.changed = True
