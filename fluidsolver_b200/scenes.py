"""Seeded synthetic scenes for the benchmark configurations and the parity
tests. They follow the reference's own scene authoring
(fluidStudio/.../InsertParticlesWindow.cpp:70-93): particles on a grid of
spacing `particle_size`, mass = particle_size^dim * rest_density, density =
rest density, zero velocity. The boundary is a tank (floor + side walls, y up).

No public dataset is involved; every scene is reproducible from its seed.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .solver import ParticleCollection

NORMAL, BOUNDARY, INACTIVE = 0, 1, 2


@dataclass
class Scene:
    collection: ParticleCollection
    particle_size: float
    rest_density: float
    description: str
    n_fluid: int
    n_boundary: int


def _collection(fluid: np.ndarray, boundary: np.ndarray, particle_size: float, rest_density: float) -> ParticleCollection:
    dim = fluid.shape[1]
    pos = np.concatenate([fluid, boundary]).astype(np.float32)
    n = pos.shape[0]
    typ = np.concatenate([np.full(len(fluid), NORMAL, np.uint8), np.full(len(boundary), BOUNDARY, np.uint8)])
    mass = np.full(n, np.float32(particle_size) ** dim * np.float32(rest_density), np.float32)
    return ParticleCollection(position=pos, velocity=np.zeros((n, dim), np.float32),
                              acceleration=np.zeros((n, dim), np.float32), external=np.zeros((n, dim), np.float32),
                              mass=mass, density=np.full(n, rest_density, np.float32),
                              pressure=np.zeros(n, np.float32), type=typ, tag=np.arange(n, dtype=np.uint32))


def fluid_block_3d(nx, ny, nz, spacing, origin=(0.0, 0.0, 0.0), jitter=0.0, rng=None) -> np.ndarray:
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    pts = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64) * spacing + np.asarray(origin)
    if jitter > 0:
        pts += rng.uniform(-jitter, jitter, pts.shape)
    return pts.astype(np.float32)


def tank_3d(lx, ly, lz, spacing, layers=1) -> np.ndarray:
    """Single- or multi-layer tank around the interior [0,lx] x [0,ly] x [0,lz]
    (floor below y = 0, walls outside x and z, open top)."""
    nx, ny, nz = int(round(lx / spacing)), int(round(ly / spacing)), int(round(lz / spacing))
    pts = []
    for L in range(1, layers + 1):
        # floor at y = -L*s spanning the walls' footprint
        xs = np.arange(-L, nx + L)
        zs = np.arange(-L, nz + L)
        X, Z = np.meshgrid(xs, zs, indexing="ij")
        pts.append(np.stack([X.ravel(), np.full(X.size, -L), Z.ravel()], 1))
        ys = np.arange(-L + 1, ny)
        # x walls (at x = -L and x = nx - 1 + L), spanning z in [-L+1, nz-1+L-1]
        for xw in (-L, nx - 1 + L):
            Y, Z = np.meshgrid(ys, np.arange(-L + 1, nz + L - 1), indexing="ij")
            pts.append(np.stack([np.full(Y.size, xw), Y.ravel(), Z.ravel()], 1))
        # z walls (at z = -L and z = nz - 1 + L), spanning x in [-L, nx-1+L]
        for zw in (-L, nz - 1 + L):
            X, Y = np.meshgrid(np.arange(-L, nx + L), ys, indexing="ij")
            pts.append(np.stack([X.ravel(), Y.ravel(), np.full(X.size, zw)], 1))
    return (np.concatenate(pts).astype(np.float64) * spacing).astype(np.float32)


def breaking_dam_3d(nx, ny, nz, spacing=1.0, tank=(180, 100, 60), jitter_frac=0.01, seed=4, layers=1,
                    rest_density=1.0) -> Scene:
    """Fluid column of nx*ny*nz particles in the corner of a tank."""
    rng = np.random.default_rng(seed)
    fluid = fluid_block_3d(nx, ny, nz, spacing, jitter=jitter_frac * spacing, rng=rng)
    bnd = tank_3d(*tank, spacing, layers=layers)
    col = _collection(fluid, bnd, spacing, rest_density)
    return Scene(col, spacing, rest_density, f"3D breaking dam {nx}x{ny}x{nz} fluid @ {spacing}, tank {tank}, "
                 f"{layers}-layer, jitter {jitter_frac} of spacing, seed {seed}", len(fluid), len(bnd))


# Units. Every scenario the reference ships uses particle-size 1 and
# rest-density 1 (scenarios/**/*.json). The benchmark scenes are therefore
# authored in those units: a spacing of 0.01 m becomes 1, lengths scale by
# 100, and the time step scales by sqrt(100) (Froude scaling: same
# dimensionless dynamics under the same gravity), 0.0005 s -> 0.005. At the
# literal 0.01 m / rho0 = 1 scale the reference's IISPH never builds pressure:
# its diagonal is ~1e-11, below the absolute FLT_EPSILON test of
# IISPHFluidSolver3D.hpp:441, so every step ends after the minimum iterations
# with p = 0 (breaking_dam_3d(..., spacing=0.01) reproduces that case).
REFERENCE_UNITS_DT = 0.005


def dam_100k(seed=4) -> Scene:
    """40 x 50 x 50 column (100,000 fluid) in a single-layer tank of
    180 x 100 x 60 spacings (59,684 boundary particles)."""
    return breaking_dam_3d(40, 50, 50, 1.0, tank=(180, 100, 60), seed=seed)


def dam_1m(seed=5) -> Scene:
    """100 x 100 x 100 block (1,000,000 fluid) in a single-layer tank of
    320 x 220 x 150 spacings (256,624 boundary particles)."""
    return breaking_dam_3d(100, 100, 100, 1.0, tank=(320, 220, 150), seed=seed)


def batched_dams(count=256, seed=6, f_min=2000, f_max=60000) -> list:
    """The batched breaking dams: `count` scenes with fluid counts drawn
    log-uniform in [f_min, f_max] and a block aspect ratio a ~ U(0.5, 2):
    nx = round((F a)^(1/3)), ny = round(F^(1/3)), nz = max(1, round(F / (nx ny)))
    (the actual count is nx ny nz). Each block sits in its own single-layer
    tank with the 1M dam's proportions (3.2 nx x 2.2 ny x 1.5 nz spacings).
    Scene i's jitter seed is seed * 100003 + i."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        f = int(round(np.exp(rng.uniform(np.log(f_min), np.log(f_max)))))
        a = rng.uniform(0.5, 2.0)
        nx = max(1, int(round((f * a) ** (1.0 / 3.0))))
        ny = max(1, int(round(f ** (1.0 / 3.0))))
        nz = max(1, int(round(f / (nx * ny))))
        tank = (max(nx + 2, int(round(3.2 * nx))), max(ny + 2, int(round(2.2 * ny))), max(nz + 2, int(round(1.5 * nz))))
        out.append(breaking_dam_3d(nx, ny, nz, 1.0, tank=tank, seed=seed * 100003 + i))
    return out


def breaking_dam_2d(nx=50, ny=50, spacing=1.0, width=150, height=120, layers=3, jitter=0.01, seed=1,
                    rest_density=1.0) -> Scene:
    """2D dam: nx x ny fluid block from (0,0) with uniform jitter, in a box
    walled by `layers` layers of boundary particles (floor + two sides)."""
    rng = np.random.default_rng(seed)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    fluid = np.stack([i.ravel(), j.ravel()], 1).astype(np.float64) * spacing
    fluid += rng.uniform(-jitter, jitter, fluid.shape)
    pts = []
    for L in range(1, layers + 1):
        xs = np.arange(-layers, width + layers)
        pts.append(np.stack([xs, np.full(xs.size, -L)], 1))
        ys = np.arange(0, height)
        pts.append(np.stack([np.full(ys.size, -L), ys], 1))
        pts.append(np.stack([np.full(ys.size, width - 1 + L), ys], 1))
    bnd = np.concatenate(pts).astype(np.float64) * spacing
    col = _collection(fluid.astype(np.float32), bnd.astype(np.float32), spacing, rest_density)
    return Scene(col, spacing, rest_density, f"2D dam {nx}x{ny} @ {spacing}, box {width}x{height}, {layers} layers, "
                 f"jitter +-{jitter}, seed {seed}", len(fluid), len(bnd))


def ns_points_uniform(n=1_000_000, seed=2) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.random((n, 3), dtype=np.float64).astype(np.float32)


def ns_points_blobs(n=1_000_000, blobs=64, sigma=0.03, seed=3) -> np.ndarray:
    """`blobs` Gaussian blobs (centres U(0.1, 0.9)^3) of n/blobs points each,
    rejection-resampled into [0,1)^3."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.1, 0.9, (blobs, 3))
    per = n // blobs
    out = []
    for c in centres:
        pts = np.empty((0, 3))
        while len(pts) < per:
            cand = rng.normal(c, sigma, (per * 2, 3))
            cand = cand[np.all((cand >= 0) & (cand < 1), axis=1)]
            pts = np.concatenate([pts, cand])
        out.append(pts[:per])
    return np.concatenate(out).astype(np.float32)
