"""CPU tests of the C-ABI boundary: the library builds and loads, exports every
function include/fluidsolver_b200.h declares, fills libFluid's defaults, and
rejects bad configurations before touching a device."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available
from fluidsolver_b200 import _lib as F
from fluidsolver_b200 import build


@pytest.fixture(scope="module")
def L():
    build.build()
    return F.lib()


def declared_functions():
    src = open(os.path.join(ROOT, "include", "fluidsolver_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fs_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("fs_create", "fs_upload", "fs_find_neighbors", "fs_solve_step", "fs_step", "fs_download",
                 "fs_get_neighbors_csr", "fs_query_position", "fs_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol(L):
    for name in declared_functions():
        assert hasattr(L, name), name
    assert set(F.EXPORTED_SYMBOLS) <= set(declared_functions())


def test_abi_version(L):
    assert L.fs_abi_version() == 4


def test_structs_match_the_header(tmp_path):
    """The ctypes mirrors have the C compiler's layout of the header's structs."""
    src = tmp_path / "layout.c"
    classes = {"fs_params": F.FsParams, "fs_step_stats": F.FsStepStats, "fs_global_stats": F.FsGlobalStats,
               "fs_tuning": F.FsTuning, "fs_camera": F.FsCamera, "fs_render_settings": F.FsRenderSettings}
    fields = {name: [f[0] for f in cls._fields_] for name, cls in classes.items()}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "fluidsolver_b200.h"', "int main(void) {"]
    for st, names in fields.items():
        lines.append(f'printf("%zu\\n", sizeof({st}));')
        lines += [f'printf("%zu\\n", offsetof({st}, {n}));' for n in names]
    lines += ["return 0;", "}"]
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = []
    for cls in classes.values():
        want.append(ctypes.sizeof(cls))
        want += [getattr(cls, f[0]).offset for f in cls._fields_]
    assert got == want


def test_params_default_are_libfluid_defaults(L):
    p = F.FsParams()
    L.fs_params_default(ctypes.byref(p), 3, F.FS_SOLVER_IISPH_3D, F.FS_SEARCH_HASHED_3D)
    # IFluidSolver.hpp:18-23, IISPHSettings3D.hpp:6-20, ConstantTimestepGenerator.hpp:8-13
    assert (p.rest_density, round(p.gravity, 5), round(p.particle_size, 5)) == (1000.0, 9.81, 0.1)
    assert (round(p.max_density_error, 6), p.min_iterations, p.max_iterations) == (0.001, 2, 100)
    assert (p.omega, round(p.gamma, 5), p.viscosity) == (0.5, 0.7, 5.0)
    assert (p.single_layer_boundary, round(p.single_layer_gamma_1, 5)) == (0, 1.1)
    assert (round(p.timestep, 6), round(p.lambda_v, 5), p.lambda_a) == (0.001, 0.4, 0.25)
    assert p.precision == F.FS_PRECISION_FP32_KAHAN


def _params(L, **kw):
    p = F.FsParams()
    L.fs_params_default(ctypes.byref(p), 3, F.FS_SOLVER_IISPH_3D, F.FS_SEARCH_HASHED_3D)
    p.max_particles = 100
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("bad", [
    dict(dim=4), dict(search=17), dict(solver=9), dict(search=F.FS_SEARCH_HASHED_2D),
    dict(max_iterations=1, min_iterations=2), dict(max_density_error=0.0), dict(particle_size=0.0),
    dict(timestep=-1.0), dict(max_particles=0), dict(precision=7),
])
def test_invalid_configurations_are_rejected(L, bad):
    ctx = ctypes.c_void_p()
    assert L.fs_create(ctypes.byref(_params(L, **bad)), ctypes.byref(ctx)) == F.FS_ERR_INVALID
    assert not ctx.value
    assert L.fs_last_error()


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_fails_loudly(L):
    ctx = ctypes.c_void_p()
    st = L.fs_create(ctypes.byref(_params(L)), ctypes.byref(ctx))
    assert st == F.FS_ERR_NO_DEVICE
    assert not ctx.value


def test_null_arguments(L):
    assert L.fs_destroy(None) == F.FS_OK
    assert L.fs_upload(None, None) == F.FS_ERR_INVALID
    assert L.fs_step(None, ctypes.c_float(0.0), None) == F.FS_ERR_INVALID


def test_sort_keys_validates_its_arguments(L):
    """fs_sort_keys rejects bad widths and keys at or above 2^bits before it touches a device."""
    k = np.array([1, 2, 300], np.uint32)
    out = np.empty_like(k)
    order = np.empty(3, np.uint32)
    args = (out.ctypes.data, order.ctypes.data)
    assert L.fs_sort_keys(0, k.ctypes.data, 2, 3, 16, *args) == F.FS_ERR_INVALID       # key_bytes
    assert L.fs_sort_keys(0, k.ctypes.data, 4, 3, 0, *args) == F.FS_ERR_INVALID        # bits
    assert L.fs_sort_keys(0, k.ctypes.data, 4, 3, 33, *args) == F.FS_ERR_INVALID
    assert L.fs_sort_keys(0, k.ctypes.data, 4, 3, 8, *args) == F.FS_ERR_INVALID        # 300 >= 2^8
    assert b"bits" in L.fs_last_error()
    assert L.fs_sort_keys(0, None, 4, 3, 16, *args) == F.FS_ERR_INVALID
    assert L.fs_sort_keys(0, k.ctypes.data, 4, -1, 16, *args) == F.FS_ERR_INVALID
    k8 = np.array([1, 2, 1 << 40], np.uint64)
    assert L.fs_sort_keys(0, k8.ctypes.data, 8, 3, 65, *args) == F.FS_ERR_INVALID
    assert L.fs_sort_keys(0, k8.ctypes.data, 8, 3, 40, *args) == F.FS_ERR_INVALID      # 2^40 >= 2^40


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_sort_keys_without_a_device_fails_loudly(L):
    k = np.array([3, 1, 2], np.uint32)
    out = np.empty_like(k)
    order = np.empty(3, np.uint32)
    assert L.fs_sort_keys(0, k.ctypes.data, 4, 3, 8, out.ctypes.data, order.ctypes.data) == F.FS_ERR_NO_DEVICE
