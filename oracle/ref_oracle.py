"""TEST INFRASTRUCTURE -- the oracle. ctypes access to the reference's own
libFluid hot-path code compiled unmodified in oracle/_ref (see
oracle/ref/Makefile). Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use it, as the checker and the timed reference; the product path
never calls it.

All arrays are in tag space (input order), see oracle/ref/harness.cpp.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_float, c_int, c_int64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

NS_KINDS = {"quadratic-2d": 0, "hashed-2d": 1, "quadratic-3d": 2, "hashed-3d": 3, "compressed-3d": 4}
SOLVER_KINDS = {"sesph-2d": 0, "sesph-3d": 1, "iisph-2d": 2, "iisph-3d": 3}

_libs: dict[str, ctypes.CDLL] = {}


def available(variant: str = "serial") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libfsref_{variant}.so"))


def lib(variant: str = "serial") -> ctypes.CDLL:
    """variant: 'serial' (reference as built: StdParallelForEach, 1 core) or
    'omp' (same sources, the loop_for chunks spread over all host cores)."""
    if variant in _libs:
        return _libs[variant]
    path = os.path.join(REF_DIR, f"libfsref_{variant}.so")
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built (make -C oracle/ref)")
    L = ctypes.CDLL(path)
    L.ref_last_error.restype = ctypes.c_char_p
    L.ref_kernel_eval.argtypes = [c_int, c_float, c_int64, c_void_p, c_void_p, c_void_p]
    L.ref_cfl_timestep.argtypes = [c_float] * 4 + [c_int64, c_void_p, c_void_p, c_void_p]
    L.ref_dynamic_timestep.argtypes = [c_int, c_int64, c_void_p, c_void_p, c_void_p] + [c_float] * 5
    L.ref_dynamic_timestep.restype = c_float
    L.ref_boundary_preprocess.argtypes = [c_void_p, c_void_p, c_float, c_float, c_void_p]
    L.ref_trace_rays.argtypes = [c_int64, c_void_p, c_void_p, c_void_p, c_float, c_float, c_int64] + [c_void_p] * 6
    L.ref_tone_map.argtypes = [c_int64, c_int64, c_void_p, c_float, c_float, c_int, c_int, c_void_p]
    L.ref_global_stats.argtypes = [c_int, c_int64] + [c_void_p] * 6 + [c_float, c_float, c_void_p, c_void_p]
    L.ref_ns_create.restype = c_void_p
    L.ref_ns_create.argtypes = [c_int, c_int64, c_void_p, c_void_p, c_float]
    L.ref_ns_destroy.argtypes = [c_void_p]
    L.ref_ns_set_positions.argtypes = [c_void_p, c_void_p]
    L.ref_ns_find.argtypes = [c_void_p]
    L.ref_ns_lists.restype = c_int64
    L.ref_ns_lists.argtypes = [c_void_p, c_void_p, c_void_p]
    L.ref_ns_query_position.restype = c_int64
    L.ref_ns_query_position.argtypes = [c_void_p, c_void_p, c_void_p, c_int64]
    L.ref_solver_create.restype = c_void_p
    L.ref_solver_create.argtypes = [c_int, c_int, c_int64] + [c_void_p] * 11
    L.ref_solver_destroy.argtypes = [c_void_p]
    L.ref_solver_step.argtypes = [c_void_p, c_void_p]
    L.ref_solver_run.argtypes = [c_void_p, c_int64, c_void_p]
    L.ref_solver_state.argtypes = [c_void_p] + [c_void_p] * 9
    L.ref_solver_lists.restype = c_int64
    L.ref_solver_lists.argtypes = [c_void_p, c_void_p, c_void_p]
    _libs[variant] = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data


def kernel_eval(dim: int, support: float, x: np.ndarray):
    x = np.ascontiguousarray(x, np.float32)
    n = x.shape[0]
    W = np.zeros(n, np.float32)
    dW = np.zeros((n, dim), np.float32)
    lib().ref_kernel_eval(dim, support, n, _p(x), _p(W), _p(dW))
    return W, dW


def cfl_timestep(timestep, lambda_v, lambda_a, particle_size, max_acc, max_vel):
    a = np.ascontiguousarray(max_acc, np.float32)
    v = np.ascontiguousarray(max_vel, np.float32)
    out = np.zeros_like(a)
    lib().ref_cfl_timestep(timestep, lambda_v, lambda_a, particle_size, len(a), _p(a), _p(v), _p(out))
    return out


def dynamic_timestep(vel, acc, type_, particle_size, min_ts, max_ts, lambda_v, lambda_a) -> float:
    vel = np.ascontiguousarray(vel, np.float32)
    acc = np.ascontiguousarray(acc, np.float32)
    type_ = np.ascontiguousarray(type_, np.uint8)
    return lib().ref_dynamic_timestep(vel.shape[1], len(vel), _p(vel), _p(acc), _p(type_), particle_size, min_ts,
                                      max_ts, lambda_v, lambda_a)


def trace_rays(pos, mass, type_, particle_size, rest_density, origins, directions) -> dict:
    """ParticleIntersectionAccelerator's first hits (no random offset along the rays)."""
    f = lambda a: np.ascontiguousarray(a, np.float32)
    pos, mass, o, d = f(pos), f(mass), f(origins), f(directions)
    t = np.ascontiguousarray(type_, np.uint8)
    m = len(o)
    out = {"hit": np.zeros(m, np.int32), "point": np.zeros((m, 3), np.float32),
           "normal": np.zeros((m, 3), np.float32), "length": np.zeros(m, np.float32)}
    if lib().ref_trace_rays(len(pos), _p(pos), _p(mass), _p(t), particle_size, rest_density, m, _p(o), _p(d),
                            _p(out["hit"]), _p(out["point"]), _p(out["normal"]), _p(out["length"])) != 0:
        raise RuntimeError(lib().ref_last_error().decode())
    return out


def tone_map(radiance, exposure=0.2, gamma=2.2, filmic=False, gamma_correction=True) -> np.ndarray:
    """The reference's ToneMapper (map_render_target_to_image) on radiance of shape (h, w, 3):
    (h, w, 4) bytes."""
    rad = np.ascontiguousarray(radiance, np.float32)
    h, w = rad.shape[0], rad.shape[1]
    out = np.zeros((h, w, 4), np.uint8)
    if lib().ref_tone_map(w, h, _p(rad), exposure, gamma, 1 if gamma_correction else 0, 1 if filmic else 0,
                          _p(out)) != 0:
        raise RuntimeError(lib().ref_last_error().decode())
    return out


STAT_NAMES = ["density_max", "density_min", "density_avg", "pressure_max", "pressure_min", "pressure_avg",
              "velocity_max", "velocity_min", "velocity_avg", "kinetic_energy", "potential_energy"]


def global_stats(col, gravity: float, zero_height: float = 0.0) -> dict:
    """The reference's global sensors (ParticleStatistics.cpp: density, pressure,
    velocity, energy, particle counts) through their calculate_for_timepoint.
    Velocity and energy are NaN for 3D collections (the reference's sensors
    read 2D MovementData)."""
    f = lambda a: np.ascontiguousarray(a, np.float32)
    pos, vel = f(col.position), f(col.velocity)
    out = np.zeros(11, np.float32)
    counts = np.zeros(3, np.int64)
    if lib().ref_global_stats(pos.shape[1], len(pos), _p(pos), _p(vel), _p(f(col.mass)), _p(f(col.density)),
                              _p(f(col.pressure)), _p(np.ascontiguousarray(col.type, np.uint8)), gravity, zero_height,
                              _p(out), _p(counts)) != 0:
        raise RuntimeError(lib().ref_last_error().decode())
    d = {k: np.float32(v) for k, v in zip(STAT_NAMES, out)}
    d.update(normal_particles=int(counts[0]), boundary_particles=int(counts[1]), inactive_particles=int(counts[2]))
    return d


class RefSearch:
    """One reference neighborhood search over a fixed particle set."""

    def __init__(self, kind: str, position: np.ndarray, radius: float, type_: np.ndarray | None = None,
                 variant: str = "serial"):
        self.L = lib(variant)
        self.pos = np.ascontiguousarray(position, np.float32)
        self.n = self.pos.shape[0]
        self.type = None if type_ is None else np.ascontiguousarray(type_, np.uint8)
        self.h = self.L.ref_ns_create(NS_KINDS[kind], self.n, _p(self.pos), _p(self.type), radius)
        if not self.h:
            raise RuntimeError(self.L.ref_last_error().decode())

    def set_positions(self, position: np.ndarray):
        p = np.ascontiguousarray(position, np.float32)
        self.L.ref_ns_set_positions(self.h, _p(p))

    def find(self):
        """Returns False when the reference threw (e.g. more than 97 neighbors)."""
        return self.L.ref_ns_find(self.h) == 0

    def lists(self):
        """(offsets, indices) in tag space, each list in the reference's own order."""
        off = np.zeros(self.n + 1, np.int64)
        tot = self.L.ref_ns_lists(self.h, _p(off), None)
        if tot < 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        idx = np.zeros(max(tot, 1), np.int64)
        self.L.ref_ns_lists(self.h, _p(off), _p(idx))
        return off, idx[:tot]

    def query(self, p, cap=1 << 16):
        p = np.ascontiguousarray(p, np.float32)
        out = np.zeros(cap, np.int64)
        c = self.L.ref_ns_query_position(self.h, _p(p), _p(out), cap)
        if c < 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return out[:min(c, cap)]

    def boundary_preprocess(self, mass: np.ndarray, particle_size: float, rest_density: float) -> np.ndarray:
        """BoundaryPreprocessor on this search's collection (after find()), through its own interface."""
        mass = np.ascontiguousarray(mass, np.float32)
        out = np.zeros_like(mass)
        if self.L.ref_boundary_preprocess(self.h, _p(mass), particle_size, rest_density, _p(out)) != 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return out

    def close(self):
        if self.h:
            self.L.ref_ns_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class RefSolver:
    """A reference solver (template instantiation chosen by kind + search)
    driven like Simulator::execute_simulation_step."""

    def __init__(self, solver: str, search: str, col, params, settings, generator, variant: str = "serial"):
        """col: object with position, velocity, acceleration, external, mass,
        density, pressure, type arrays (host order).
        params: (rest_density, gravity, particle_size);
        settings: solver-specific list (see oracle/ref/harness.cpp);
        generator: (timestep, lambda_v, lambda_a)."""
        self.L = lib(variant)
        d = col.position.shape[1]
        self.dim = d
        self.n = col.position.shape[0]
        f = lambda a, shape: np.ascontiguousarray(np.zeros(shape) if a is None else a, np.float32)
        self._keep = [f(col.position, (self.n, d)), f(col.velocity, (self.n, d)), f(col.acceleration, (self.n, d)),
                      f(col.mass, (self.n,)), f(col.density, (self.n,)), f(col.pressure, (self.n,)),
                      np.ascontiguousarray(col.type, np.uint8), f(col.external, (self.n, d)),
                      np.asarray(params, np.float32), np.asarray(settings, np.float32),
                      np.asarray(generator, np.float32)]
        self.h = self.L.ref_solver_create(SOLVER_KINDS[solver], NS_KINDS[search], self.n,
                                          *[_p(a) for a in self._keep])
        if not self.h:
            raise RuntimeError(self.L.ref_last_error().decode())
        self.stats = np.zeros(4, np.float32)

    def step(self):
        if self.L.ref_solver_step(self.h, _p(self.stats)) != 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return dict(desired_dt=float(self.stats[0]), actual_dt=float(self.stats[1]),
                    iterations=int(self.stats[2]), avg_density_error=float(self.stats[3]))

    def run(self, steps: int):
        if self.L.ref_solver_run(self.h, steps, _p(self.stats)) != 0:
            raise RuntimeError(self.L.ref_last_error().decode())

    def state(self):
        n, d = self.n, self.dim
        out = dict(position=np.zeros((n, d), np.float32), velocity=np.zeros((n, d), np.float32),
                   acceleration=np.zeros((n, d), np.float32), mass=np.zeros(n, np.float32),
                   density=np.zeros(n, np.float32), pressure=np.zeros(n, np.float32), type=np.zeros(n, np.uint8),
                   external=np.zeros((n, d), np.float32), iisph=np.zeros((n, 9), np.float32))
        self.L.ref_solver_state(self.h, *[_p(out[k]) for k in ("position", "velocity", "acceleration", "mass",
                                                                "density", "pressure", "type", "external", "iisph")])
        return out

    def lists(self):
        off = np.zeros(self.n + 1, np.int64)
        tot = self.L.ref_solver_lists(self.h, _p(off), None)
        idx = np.zeros(max(tot, 1), np.int64)
        self.L.ref_solver_lists(self.h, _p(off), _p(idx))
        return off, idx[:tot]

    def close(self):
        if self.h:
            self.L.ref_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def iisph3d_settings(max_err=0.001, min_it=2, max_it=100, omega=0.5, gamma=0.7, viscosity=0.01, single_layer=True,
                     gamma1=1.1):
    return [max_err, min_it, max_it, omega, gamma, viscosity, 1.0 if single_layer else 0.0, gamma1]


def sesph3d_settings(k=1000.0, viscosity=0.01, single_layer=True, gamma1=1.1, gamma2=1.1):
    return [k, viscosity, 1.0 if single_layer else 0.0, gamma1, gamma2]


def iisph2d_settings(max_err=0.001, min_it=2, max_it=100, omega=0.5, gamma=0.7, viscosity=0.01):
    return [max_err, min_it, max_it, omega, gamma, viscosity]


def sesph2d_settings(k=1000.0, viscosity=0.01):
    return [k, viscosity]
