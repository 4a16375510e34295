"""ctypes binding of the C-ABI in include/fluidsolver_b200.h.

The shared library is built in-tree (fluidsolver_b200/lib/libfluidsolver_b200.so,
see fluidsolver_b200/build.py). Loading fails loudly when it is missing: there
is no CPU fallback on the product path.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int32, c_int64, c_uint8, c_uint32, c_void_p

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libfluidsolver_b200.so")

FS_OK = 0
FS_ERR_INVALID = 1
FS_ERR_CAPACITY = 2
FS_ERR_NAN = 3
FS_ERR_TIMEOUT = 4
FS_ERR_CUDA = 5
FS_ERR_NO_DEVICE = 6
FS_ERR_STATE = 7

FS_QUERY_NOALLOC_MAX = 65536  # include/fluidsolver_b200.h

FS_SOLVER_NONE = 0
FS_SOLVER_SESPH_2D = 1
FS_SOLVER_SESPH_3D = 2
FS_SOLVER_IISPH_2D = 3
FS_SOLVER_IISPH_3D = 4

FS_COMPONENT_MOVEMENT_2D = 1 << 1
FS_COMPONENT_MOVEMENT_3D = 1 << 2
FS_COMPONENT_INFO = 1 << 3
FS_COMPONENT_DATA = 1 << 4
FS_COMPONENT_EXTERNAL_2D = 1 << 5
FS_COMPONENT_EXTERNAL_3D = 1 << 6

FS_TIMESTEP_CONSTANT = 0
FS_TIMESTEP_DYNAMIC_CFL = 1

FS_SEARCH_QUADRATIC_2D = 0
FS_SEARCH_HASHED_2D = 1
FS_SEARCH_COMPACT_2D = 2
FS_SEARCH_QUADRATIC_3D = 3
FS_SEARCH_HASHED_3D = 4
FS_SEARCH_COMPRESSED_3D = 5

FS_PRECISION_FP32 = 0
FS_PRECISION_FP32_KAHAN = 1
FS_PRECISION_FP64 = 2

FS_FLAG_REFERENCE_ORDER = 0x1
FS_FLAG_SYNC_EACH_ITERATION = 0x2
FS_FLAG_ONE_KERNEL_STEPS = 0x4

FS_TYPE_NORMAL = 0
FS_TYPE_BOUNDARY = 1
FS_TYPE_INACTIVE = 2

# symbols the header declares (checked by the CPU test suite)
EXPORTED_SYMBOLS = (
    "fs_abi_version", "fs_last_error", "fs_params_default", "fs_create", "fs_destroy", "fs_set_params",
    "fs_upload", "fs_download", "fs_find_neighbors", "fs_get_neighbors_csr", "fs_query_position", "fs_solve_step", "fs_step",
    "fs_run", "fs_last_phase_times", "fs_stream", "fs_launch_count", "fs_small_blocks", "fs_batch_create", "fs_batch_run",
    "fs_query_position_noalloc", "fs_get_solver_lists_csr", "fs_boundary_preprocess", "fs_global_statistics",
    "fs_particles_file_info", "fs_particles_file_read", "fs_particles_file_write", "fs_dump",
    "fs_autotune", "fs_set_tuning", "fs_trace_rays", "fs_render_settings_default", "fs_render",
    "fs_set_tile_wait_limit", "fs_tone_map", "fs_sort_keys",
)


class FsParams(ctypes.Structure):
    _fields_ = [
        ("dim", c_int32), ("solver", c_int32), ("search", c_int32), ("precision", c_int32),
        ("flags", c_uint32), ("device", c_int32),
        ("rest_density", c_float), ("gravity", c_float), ("particle_size", c_float),
        ("stiffness", c_float), ("viscosity", c_float), ("single_layer_boundary", c_int32),
        ("single_layer_gamma_1", c_float), ("single_layer_gamma_2", c_float),
        ("max_density_error", c_float), ("min_iterations", c_int32), ("max_iterations", c_int32),
        ("omega", c_float), ("gamma", c_float),
        ("timestep", c_float), ("lambda_v", c_float), ("lambda_a", c_float),
        ("max_particles", c_int64), ("neighbor_capacity", c_int32),
        ("timestep_generator", c_int32), ("min_timestep", c_float), ("max_timestep", c_float),
    ]


class FsParticles(ctypes.Structure):
    _fields_ = [
        ("n", c_int64),
        ("position", c_void_p), ("velocity", c_void_p), ("acceleration", c_void_p), ("external", c_void_p),
        ("mass", c_void_p), ("density", c_void_p), ("pressure", c_void_p),
        ("type", c_void_p), ("tag", c_void_p),
        ("predicted_velocity", c_void_p), ("non_pressure_acceleration", c_void_p),
        ("source_term", c_void_p), ("diagonal_element", c_void_p),
    ]


class FsStepStats(ctypes.Structure):
    _fields_ = [
        ("desired_dt", c_float), ("actual_dt", c_float), ("iterations", c_int32),
        ("avg_density_error", c_float), ("avg_density_error_fp64", c_double),
        ("max_density_error", c_float), ("max_velocity", c_float), ("max_acceleration", c_float),
        ("status", c_int32), ("max_neighbors", c_int32),
    ]


class FsGlobalStats(ctypes.Structure):
    _fields_ = [
        ("density_max", c_float), ("density_min", c_float), ("density_avg", c_float),
        ("pressure_max", c_float), ("pressure_min", c_float), ("pressure_avg", c_float),
        ("velocity_max", c_float), ("velocity_min", c_float), ("velocity_avg", c_float),
        ("kinetic_energy", c_float), ("potential_energy", c_float), ("reserved", c_int32),
        ("normal_particles", c_int64), ("boundary_particles", c_int64), ("inactive_particles", c_int64),
    ]


class FsTuning(ctypes.Structure):
    _fields_ = [
        ("tuned", c_int32), ("first_loop_prefetch", c_int32), ("pressure_prefetch", c_int32), ("tile_cap", c_int32),
        ("block_size", c_int32), ("pressure_threads_per_owner", c_int32),
        ("first_loop_ms", c_float * 4), ("pressure_iteration_ms", c_float * 4), ("step_ms_by_tile_cap", c_float * 4),
        ("step_ms_by_block_size", c_float * 3), ("fallback_tiles_by_tile_cap", c_float * 4),
        ("pressure_iteration_ms_by_threads", c_float * 3),
    ]


TILE_CAPS = (1024, 1536, 2048, 3072)   # include/fluidsolver_b200.h, fs_tuning
BLOCK_SIZES = (128, 256, 512)
THREADS_PER_OWNER = (1, 2, 4)


class FsCamera(ctypes.Structure):
    _fields_ = [("position", c_float * 3), ("view_direction", c_float * 3), ("view_up", c_float * 3),
                ("field_of_view_x", c_float), ("width", c_int32), ("height", c_int32), ("flip_y", c_int32)]


class FsRenderSettings(ctypes.Structure):
    _fields_ = [("samples_per_pixel", c_int32), ("maximum_recursion_depth", c_int32),
                ("output_normals_of_first_hit", c_int32), ("surface_density_fraction", c_float),
                ("exposure", c_float), ("gamma", c_float), ("seed", ctypes.c_uint64), ("tone_mapper", c_int32),
                ("gamma_correction", c_int32)]


class FluidSolverError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"fluidsolver_b200 status {status}: {message}")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FluidSolverError(FS_ERR_NO_DEVICE,
                               f"{LIB_PATH} is missing; build it with `python -m fluidsolver_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    ctx_p = c_void_p
    L.fs_abi_version.restype = c_int32
    L.fs_last_error.restype = c_char_p
    L.fs_params_default.argtypes = [POINTER(FsParams), c_int32, c_int32, c_int32]
    L.fs_params_default.restype = None
    L.fs_create.argtypes = [POINTER(FsParams), POINTER(ctx_p)]
    L.fs_destroy.argtypes = [ctx_p]
    L.fs_set_params.argtypes = [ctx_p, POINTER(FsParams)]
    L.fs_upload.argtypes = [ctx_p, POINTER(FsParticles)]
    L.fs_download.argtypes = [ctx_p, POINTER(FsParticles)]
    L.fs_find_neighbors.argtypes = [ctx_p]
    L.fs_get_neighbors_csr.argtypes = [ctx_p, c_void_p, c_void_p, POINTER(c_int64)]
    L.fs_get_solver_lists_csr.argtypes = [ctx_p, c_void_p, c_void_p, POINTER(c_int64)]
    L.fs_boundary_preprocess.argtypes = [ctx_p]
    L.fs_particles_file_info.argtypes = [ctypes.c_char_p, POINTER(c_int32), POINTER(c_int64), POINTER(ctypes.c_uint32)]
    L.fs_particles_file_read.argtypes = [ctypes.c_char_p, POINTER(FsParticles)]
    L.fs_particles_file_write.argtypes = [ctypes.c_char_p, c_int32, POINTER(FsParticles)]
    L.fs_dump.argtypes = [ctx_p, ctypes.c_char_p]
    L.fs_autotune.argtypes = [ctx_p, POINTER(FsTuning)]
    L.fs_trace_rays.argtypes = [ctx_p, c_float, c_int64] + [c_void_p] * 6
    L.fs_render_settings_default.argtypes = [POINTER(FsRenderSettings)]
    L.fs_render_settings_default.restype = None
    L.fs_render.argtypes = [ctx_p, POINTER(FsCamera), POINTER(FsRenderSettings), c_void_p, c_void_p]
    L.fs_set_tuning.argtypes = [ctx_p, POINTER(FsTuning)]
    L.fs_set_tile_wait_limit.argtypes = [ctx_p, c_int32]
    L.fs_tone_map.argtypes = [c_void_p, c_int64, POINTER(FsRenderSettings), c_void_p]
    L.fs_sort_keys.argtypes = [c_int32, c_void_p, c_int32, c_int64, c_int32, c_void_p, c_void_p]
    L.fs_global_statistics.argtypes = [ctx_p, c_float, POINTER(FsGlobalStats)]
    L.fs_query_position.argtypes = [ctx_p, c_void_p, c_void_p, c_int64, POINTER(c_int64)]
    L.fs_query_position_noalloc.argtypes = [ctx_p, c_void_p, c_void_p, c_int64, POINTER(c_int64)]
    L.fs_step.argtypes = [ctx_p, c_float, POINTER(FsStepStats)]
    L.fs_solve_step.argtypes = [ctx_p, c_float, POINTER(FsStepStats)]
    L.fs_run.argtypes = [ctx_p, c_int32, c_float, POINTER(FsStepStats)]
    L.fs_last_phase_times.argtypes = [ctx_p, c_void_p]
    L.fs_stream.argtypes = [ctx_p]
    L.fs_stream.restype = c_void_p
    L.fs_launch_count.argtypes = [ctx_p]
    L.fs_launch_count.restype = c_int64
    L.fs_small_blocks.argtypes = [ctx_p]
    L.fs_small_blocks.restype = c_int32
    L.fs_batch_create.argtypes = [POINTER(FsParams), c_int32, c_void_p, POINTER(ctx_p)]
    L.fs_batch_run.argtypes = [ctx_p, c_int32, c_float, c_void_p]
    for name in ("fs_create", "fs_destroy", "fs_set_params", "fs_upload", "fs_download", "fs_find_neighbors",
                 "fs_get_neighbors_csr", "fs_query_position", "fs_solve_step", "fs_step", "fs_run", "fs_last_phase_times",
                 "fs_batch_create", "fs_batch_run", "fs_query_position_noalloc", "fs_get_solver_lists_csr",
                 "fs_boundary_preprocess", "fs_global_statistics", "fs_particles_file_info",
                 "fs_particles_file_read", "fs_particles_file_write", "fs_dump", "fs_autotune", "fs_set_tuning",
                 "fs_trace_rays", "fs_render", "fs_set_tile_wait_limit", "fs_tone_map", "fs_sort_keys"):
        getattr(L, name).restype = c_int32
    _lib = L
    return L


def check(status: int) -> None:
    if status != FS_OK:
        msg = lib().fs_last_error()
        raise FluidSolverError(status, msg.decode() if msg else "")
