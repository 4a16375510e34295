"""B200 implementation of libFluid's per-timestep hot path (neighborhood
search, SESPH and IISPH in 2D and 3D) behind a C-ABI; this package is the
Python host mirror of libFluid's solver interfaces over that C-ABI."""
from ._lib import FluidSolverError, lib  # noqa: F401
from .solver import (  # noqa: F401
    BatchedIISPHFluidSolver3D,
    BoundaryPreprocessor,
    ConstantTimestepGenerator,
    DynamicCflTimestepGenerator,
    IISPHFluidSolver,
    IISPHFluidSolver3D,
    NeighborhoodSearch,
    ParticleCollection,
    SESPHFluidSolver,
    SESPHFluidSolver3D,
    Timepoint,
    read_particles,
    tone_map,
    write_particles,
)
