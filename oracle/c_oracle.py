"""TEST INFRASTRUCTURE -- ctypes access to the plain-C restatement of the
reference hot path (oracle/fs_oracle.c, built into oracle/_build by
`make -C oracle`). Used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg only, as the checker; the product never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import c_float, c_int, c_int64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libfs_oracle.so")

NS_KINDS = {"quadratic-2d": 0, "hashed-2d": 1, "compact-hashing-2d": 2, "quadratic-3d": 3, "hashed-3d": 4,
            "compressed-3d": 5}
SOLVERS = {"sesph-2d": 0, "sesph-3d": 1, "iisph-2d": 2, "iisph-3d": 3}

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.oracle_kernel_eval.argtypes = [c_int, c_float, c_int64, c_void_p, c_void_p, c_void_p]
        L.oracle_cfl.argtypes = [c_float] * 6
        L.oracle_cfl.restype = c_float
        L.oracle_dynamic_timestep.argtypes = [c_int, c_int64, c_void_p, c_void_p, c_void_p] + [c_float] * 5
        L.oracle_dynamic_timestep.restype = c_float
        L.oracle_boundary_masses.argtypes = [c_int64, c_void_p, c_void_p, c_void_p, c_float, c_float, c_void_p,
                                             c_void_p, c_void_p]
        L.oracle_global_stats.argtypes = [c_int, c_int64] + [c_void_p] * 6 + [c_float, c_float, c_void_p, c_void_p]
        L.oracle_ns.argtypes = [c_int, c_int64, c_void_p, c_void_p, c_float, c_void_p, c_void_p]
        L.oracle_ns.restype = c_int64
        L.oracle_run.argtypes = [c_void_p, c_int64, c_int] + [c_void_p] * 13 + [c_int, c_void_p, c_int] + \
            [c_void_p] * 3
        L.oracle_run.restype = c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def kernel_eval(dim, support, x):
    x = np.ascontiguousarray(x, np.float32)
    W = np.zeros(len(x), np.float32)
    dW = np.zeros((len(x), dim), np.float32)
    lib().oracle_kernel_eval(dim, support, len(x), _p(x), _p(W), _p(dW))
    return W, dW


def cfl(timestep, lambda_v, lambda_a, particle_size, max_acc, max_vel) -> float:
    return lib().oracle_cfl(timestep, lambda_v, lambda_a, particle_size, max_acc, max_vel)


def dynamic_timestep(vel, acc, type_, particle_size, min_ts, max_ts, lambda_v, lambda_a) -> float:
    """DynamicCflTimestepGenerator's time step for one collection (vel, acc: n x dim)."""
    vel = np.ascontiguousarray(vel, np.float32)
    acc = np.ascontiguousarray(acc, np.float32)
    type_ = np.ascontiguousarray(type_, np.uint8)
    return lib().oracle_dynamic_timestep(vel.shape[1], len(vel), _p(vel), _p(acc), _p(type_), particle_size,
                                         min_ts, max_ts, lambda_v, lambda_a)


def boundary_masses(position, mass, type_, particle_size, rest_density, kind="hashed-3d") -> np.ndarray:
    """BoundaryPreprocessor's masses (3D) with the contract's lists in the reference's order."""
    pos = np.ascontiguousarray(position, np.float32)
    mass = np.ascontiguousarray(mass, np.float32)
    type_ = np.ascontiguousarray(type_, np.uint8)
    off, idx, ok = search(kind, pos, 2.0 * particle_size, type_)
    assert ok
    out = np.zeros_like(mass)
    lib().oracle_boundary_masses(len(pos), _p(pos), _p(mass), _p(type_), particle_size, rest_density, _p(off),
                                 _p(np.ascontiguousarray(idx, np.int64)), _p(out))
    return out


def global_stats(col, gravity: float, zero_height: float = 0.0) -> dict:
    """The global sensors of ParticleStatistics.cpp as the reference computes them."""
    pos = np.ascontiguousarray(col.position, np.float32)
    vel = np.ascontiguousarray(col.velocity, np.float32)
    f = lambda a: np.ascontiguousarray(a, np.float32)
    out = np.zeros(11, np.float32)
    counts = np.zeros(3, np.int64)
    lib().oracle_global_stats(pos.shape[1], len(pos), _p(pos), _p(vel), _p(f(col.mass)), _p(f(col.density)),
                              _p(f(col.pressure)), _p(np.ascontiguousarray(col.type, np.uint8)), gravity, zero_height,
                              _p(out), _p(counts))
    names = ["density_max", "density_min", "density_avg", "pressure_max", "pressure_min", "pressure_avg",
             "velocity_max", "velocity_min", "velocity_avg", "kinetic_energy", "potential_energy"]
    d = {k: np.float32(v) for k, v in zip(names, out)}
    d.update(normal_particles=int(counts[0]), boundary_particles=int(counts[1]), inactive_particles=int(counts[2]))
    return d


def search(kind: str, position, radius: float, type_=None):
    """(offsets, indices, ok): lists in the contract's order; ok is False when a
    list exceeds the contract's capacity (the reference throws there)."""
    pos = np.ascontiguousarray(position, np.float32)
    n = len(pos)
    t = None if type_ is None else np.ascontiguousarray(type_, np.uint8)
    off = np.zeros(n + 1, np.int64)
    tot = lib().oracle_ns(NS_KINDS[kind], n, _p(pos), _p(t), radius, _p(off), None)
    ok = tot >= 0
    total = int(off[n])
    idx = np.zeros(max(total, 1), np.int64)
    lib().oracle_ns(NS_KINDS[kind], n, _p(pos), _p(t), radius, _p(off), _p(idx))
    return off, idx[:total], ok


def query_position(kind: str, position, radius: float, q, type_=None) -> np.ndarray:
    """Sorted host indices that NeighborhoodInterface::get_neighbors(position)
    yields for query point q, per contract (float32 arithmetic throughout):

    * hashed-3d (HashedNeighborhoodSearch3D.cpp:279-344): the 27 cells
      around floor(q / r) (:63-66), members are the non-inactive particles of
      a cell (:90-101), test glm::length(q - x_j) <= r (:335). Entering every
      cell after the first one visited (dx = dy = dz = -1), the iterator is
      advanced once more before its first test, so that cell's member with
      the smallest index is skipped.
    * quadratic-3d (QuadraticNeighborhoodSearch3D.cpp:199-219): every
      particle, inactive ones included, length test.
    * compressed-3d (CompressedNeighbors.cpp:536-590): non-inactive
      particles (:177-178) of the 27 cells, dot(x_j - q, x_j - q) <= r * r.
    * hashed-2d (HashedNeighborhoodSearch.cpp:290-340), quadratic-2d
      (QuadraticNeighborhoodSearchDynamicAllocated.cpp:190-225): every
      particle, inactive ones included, length test.
    * compact-hashing-2d has none (CompactHashingNeighborhoodSearch.cpp:92-94
      throws "Not implemented"): ValueError.
    """
    pos = np.ascontiguousarray(position, np.float32)
    q = np.asarray(q, np.float32)
    r = np.float32(radius)
    n, dim = pos.shape
    typ = np.zeros(n, np.uint8) if type_ is None else np.asarray(type_, np.uint8)
    if kind == "compact-hashing-2d":
        raise ValueError("compact hashing implements no position query")
    d = pos - q[:dim]
    dd = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]
    if dim == 3:
        dd = dd + d[:, 2] * d[:, 2]
    if kind == "compressed-3d":
        hit = (dd <= r * r) & (typ != 2)
    else:
        hit = np.sqrt(dd) <= r
    if kind == "hashed-3d":
        hit &= typ != 2
        cq = np.floor(q[:3] / r).astype(np.int64)
        cell = np.floor(pos / r).astype(np.int64)
        ordinal = 0
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    if ordinal > 0:
                        m = np.nonzero((cell == cq + np.array([dx, dy, dz])).all(1) & (typ != 2))[0]
                        if len(m):
                            hit[m.min()] = False
                    ordinal += 1
    return np.nonzero(hit)[0].astype(np.int64)


def config(solver: str, search: str, rest_density=1.0, gravity=9.81, particle_size=1.0, stiffness=1000.0,
           viscosity=0.01, single_layer=True, gamma1=1.1, gamma2=1.1, max_err=0.001, min_it=2, max_it=100, omega=0.5,
           gamma=0.7, timestep=0.005, lambda_v=0.4, lambda_a=0.25) -> np.ndarray:
    return np.array([SOLVERS[solver], NS_KINDS[search], rest_density, gravity, particle_size, stiffness, viscosity,
                     1.0 if single_layer else 0.0, gamma1, gamma2, max_err, min_it, max_it, omega, gamma, timestep,
                     lambda_v, lambda_a], np.float32)


class State:
    """A copy of a particle collection the oracle advances in place."""

    def __init__(self, col):
        n, d = col.position.shape
        f = lambda a, shape: np.array(np.zeros(shape) if a is None else a, np.float32).reshape(shape)
        self.n, self.dim = n, d
        self.position = f(col.position, (n, d))
        self.velocity = f(col.velocity, (n, d))
        self.acceleration = f(col.acceleration, (n, d))
        self.external = f(col.external, (n, d))
        self.mass = f(col.mass, (n,))
        self.density = f(col.density, (n,))
        self.pressure = f(col.pressure, (n,))
        self.type = np.array(col.type, np.uint8)
        self.predicted_velocity = np.zeros((n, d), np.float32)
        self.non_pressure_acceleration = np.zeros((n, d), np.float32)
        self.source_term = np.zeros(n, np.float32)
        self.diagonal_element = np.zeros(n, np.float32)
        self.density_error = np.zeros(n, np.float32)
        # the 2D hashed grid's history across steps (HashedNeighborhoodSearch.cpp:117-151):
        # each particle's cell (none yet) and the sequence number of its last insertion
        self.h2d_cell = np.full((n, 2), np.iinfo(np.int32).max, np.int32)
        self.h2d_seq = np.zeros(n, np.int64)
        self.h2d_counter = np.zeros(1, np.int64)

    def run(self, cfg: np.ndarray, steps: int = 1, abs_int: bool = False) -> np.ndarray:
        """Advances `steps` steps; returns per-step {desired, actual dt, iterations, avg error}."""
        stats = np.zeros((steps, 4), np.float32)
        r = lib().oracle_run(_p(cfg), self.n, self.dim, _p(self.position), _p(self.velocity), _p(self.acceleration),
                             _p(self.external), _p(self.mass), _p(self.density), _p(self.pressure), _p(self.type),
                             _p(self.predicted_velocity), _p(self.non_pressure_acceleration), _p(self.source_term),
                             _p(self.diagonal_element), _p(self.density_error), steps, _p(stats), 1 if abs_int else 0,
                             _p(self.h2d_cell), _p(self.h2d_seq), _p(self.h2d_counter))
        if r != 0:
            raise RuntimeError("oracle_run failed")
        return stats
