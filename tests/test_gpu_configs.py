"""Parity at the benchmark configurations, against the reference's own code.

The reference here is libFluid's hot path compiled from its own sources
(oracle/_ref): the OpenMP variant (the same arithmetic per particle, its
loops spread over the host cores) for the searches, the 2D dam and the first
step of the 1M dam, the serial build for the steps of the 100k dam after its
first, whose first loop depends on the loop order once velocities are nonzero. Every case runs at the configuration's full size:

* 2D SESPH dam (2,500 fluid + 1,188 boundary, k 1000, nu 0.01, dt 0.001):
  all 1,000 steps in the FP32 reference-order mode, bit for bit, on the
  hashed-2d and the quadratic-dynamic-allocated contracts;
* 3D IISPH dam, 100k fluid: 3 steps in the FP32 reference-order mode bit for
  bit; the fast mode (FP32 + compensated sums, tile lists) started from the
  reference's own state before each of them;
* 3D IISPH dam, 1M fluid: its first step (18 pressure iterations) bit for bit
  in the reference-order mode, and the fast mode's first step within tolerance;
* 3D search microbenchmark, 10^6 points: hashed-3d lists (uniform and 64
  Gaussian blobs) and compressed lists (uniform) against the reference's
  HashedNeighborhoodSearch3D and CompressedNeighborhoodSearch themselves.

Fast-mode tolerance, per step from the same input state: the IISPH
iteration count within +-1 of the reference's, the CFL time step within 1e-5
relative, positions within 1e-5 of their scale, and velocity, density and
pressure no further from an FP64 step from that state than the reference's
own FP32 step is, plus 1e-5 of the field's scale. The measured distances are
written to $FS_PARITY_REPORT (JSON) when that variable is set.
"""
import dataclasses
import json
import os

import numpy as np
import pytest

from conftest import bits_equal
from fluidsolver_b200 import NeighborhoodSearch, ParticleCollection, scenes
from fluidsolver_b200 import _lib as F
from tests.test_gpu_solvers import make_solver, simulator_step

pytestmark = pytest.mark.gpu

TOL = 1e-5
IISPH3D_SETTINGS = [0.001, 2, 100, 0.5, 0.7, 0.01, 1.0, 1.1]
IISPH3D_GENERATOR = (scenes.REFERENCE_UNITS_DT, 0.4, 0.25)
FIELDS = ("position", "velocity", "density", "pressure")


def record(key, value):
    path = os.environ.get("FS_PARITY_REPORT")
    if not path:
        return
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data[key] = value
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)


def _scale(a):
    return max(float(np.max(np.abs(a))), 1e-30)


def fast_step_from(col, search="hashed-3d"):
    """One step of the fast mode and of the FP64 build from the same state:
    (fast state, its iterations, its dt, FP64 state)."""
    out = {}
    for prec in ("fp32-kahan", "fp64"):
        s = make_solver("iisph-3d", search, IISPH3D_SETTINGS, IISPH3D_GENERATOR, precision=prec)
        s.data.collection = col
        tp = simulator_step(s)
        out[prec] = (s.collection(), s.stat_last_iteration_count, tp.actual_time_step)
        s.close()
    return out["fp32-kahan"] + (out["fp64"][0],)


def check_fast_step(name, mine, its, dt, exact, ref, ref_stats):
    """The fast-mode tolerance (module docstring); records the distances."""
    rec = {"iterations": [int(its), int(ref_stats["iterations"])], "dt": [float(dt), float(ref_stats["actual_dt"])]}
    pos = ref["position"].astype(np.float64)
    d_pos = float(np.max(np.abs(mine.position - pos)))
    rec["position"] = {"fast_vs_ref": d_pos, "scale": _scale(pos)}
    for f in ("velocity", "density", "pressure"):
        r = ref[f].astype(np.float64)
        e = getattr(exact, f).astype(np.float64)
        m = getattr(mine, f).astype(np.float64)
        rec[f] = {"envelope_ref_vs_fp64": float(np.max(np.abs(r - e))), "fast_vs_fp64": float(np.max(np.abs(m - e))),
                  "fast_vs_ref": float(np.max(np.abs(m - r))), "scale": _scale(r)}
    record(name, rec)
    assert abs(its - ref_stats["iterations"]) <= 1, (name, its, ref_stats["iterations"])
    assert abs(dt - ref_stats["actual_dt"]) <= TOL * ref_stats["actual_dt"], (name, dt, ref_stats["actual_dt"])
    assert d_pos <= TOL * _scale(pos), (name, "position", d_pos)
    for f in ("velocity", "density", "pressure"):
        q = rec[f]
        assert q["fast_vs_fp64"] <= q["envelope_ref_vs_fp64"] + TOL * q["scale"], (name, f, q)


def with_state(col0, st):
    return dataclasses.replace(col0, position=st["position"], velocity=st["velocity"], density=st["density"])


# ---------------------------------------------------------------------------
# 2D SESPH dam, all 1,000 steps
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("path", ["graph", "cluster"])
@pytest.mark.parametrize("search", ["hashed-2d", "quadratic-2d"])
def test_sesph2d_dam_1000_steps_bit_exact(ref_oracle, search, path):
    """The 2D SESPH breaking dam for its full 1,000 steps, every field of
    every checkpoint bit for bit. On hashed-2d this holds because the device
    keeps the reference's insertion order inside a cell
    (HashedNeighborhoodSearch.cpp:117-151), which decides the float
    summation order once particles start changing cells. Both device paths:
    the CUDA graph of per-phase kernels, and the small-scene kernel
    (FS_FLAG_ONE_KERNEL_STEPS: up to 800 steps per launch of one
    thread-block cluster)."""
    sc = scenes.breaking_dam_2d()
    col = sc.collection
    gen = (0.001, 0.4, 0.25)
    ref = ref_oracle.RefSolver("sesph-2d", search, col, (1.0, 9.81, 1.0), ref_oracle.sesph2d_settings(1000.0, 0.01),
                               gen, variant="omp")
    s = make_solver("sesph-2d", search, [1000.0, 0.01], gen, precision="fp32", reference_order=True,
                    one_kernel_steps=path == "cluster")
    s.data.collection = col
    done, blocks = 0, []
    for chk in (1, 2, 10, 50, 100, 200, 400, 600, 800, 1000):
        s.run(chk - done)
        blocks.append(int(F.lib().fs_small_blocks(s.ctx)))
        ref.run(chk - done)
        done = chk
        out, r = s.collection(), ref.state()
        for f in FIELDS:
            assert bits_equal(getattr(out, f), r[f]), (search, chk, f)
    # the dam has moved: the order within cells has had to follow arrivals
    assert np.max(np.abs(out.position - col.position)) > 1.0
    # the path the steps took
    assert max(blocks) > 0 if path == "cluster" else max(blocks) == 0, blocks
    record(f"sesph2d_dam/{search}/{path}", {"steps": done, "bit_identical": True})
    s.close()
    ref.close()


# ---------------------------------------------------------------------------
# 3D IISPH dams
# ---------------------------------------------------------------------------
def _iisph3d_exact_vs_reference(ref_oracle, col, steps, name, variant="serial"):
    # The reference as built (serial loops): its first loop reads neighbor
    # densities while it overwrites them (IISPHFluidSolver3D.hpp:60-64 vs
    # :210), so its result depends on the loop order, which only the serial
    # build fixes; the OpenMP variant races there once velocities are nonzero.
    ref = ref_oracle.RefSolver("iisph-3d", "hashed-3d", col, (1.0, 9.81, 1.0), IISPH3D_SETTINGS, IISPH3D_GENERATOR,
                               variant=variant)
    s = make_solver("iisph-3d", "hashed-3d", IISPH3D_SETTINGS, IISPH3D_GENERATOR, precision="fp32",
                    reference_order=True)
    s.data.collection = col
    states, stats = [], []
    for k in range(steps):
        tp = simulator_step(s)
        st = ref.step()
        r = ref.state()
        out = s.collection()
        assert np.float32(tp.actual_time_step) == np.float32(st["actual_dt"]), (name, k)
        assert s.stat_last_iteration_count == st["iterations"], (name, k)
        for f in FIELDS:
            assert bits_equal(getattr(out, f), r[f]), (name, k, f)
        states.append(r)
        stats.append(st)
    record(f"{name}/exact", {"steps": steps, "iterations": [int(x["iterations"]) for x in stats],
                             "bit_identical": True})
    s.close()
    ref.close()
    return states, stats


def test_iisph3d_100k_dam_exact_and_fast(ref_oracle):
    col = scenes.dam_100k().collection
    states, stats = _iisph3d_exact_vs_reference(ref_oracle, col, 3, "iisph3d_100k")
    starts = [dict(position=col.position, velocity=col.velocity, density=col.density)] + states[:-1]
    for k in range(3):
        mine, its, dt, exact = fast_step_from(with_state(col, starts[k]))
        check_fast_step(f"iisph3d_100k/fast_step{k}", mine, its, dt, exact, states[k], stats[k])


def test_iisph3d_1m_dam_exact_and_fast(ref_oracle):
    """The first step of the 1M dam (it needs 18 pressure iterations): bit for
    bit in the reference-order mode, the fast mode within tolerance, both from
    the same state. The reference runs its OpenMP build here: the serial build
    takes too long at a million particles, and from rest every velocity is 0,
    so the first loop's order-dependent density read does not enter the step."""
    col = scenes.dam_1m().collection
    states, stats = _iisph3d_exact_vs_reference(ref_oracle, col, 1, "iisph3d_1m", variant="omp")
    mine, its, dt, exact = fast_step_from(col)
    check_fast_step("iisph3d_1m/fast_step0", mine, its, dt, exact, states[0], stats[0])


# ---------------------------------------------------------------------------
# 3D search microbenchmark, 10^6 points
# ---------------------------------------------------------------------------
_MIX1, _MIX2 = np.uint64(0x9E3779B97F4A7C15), np.uint64(0xBF58476D1CE4E5B9)


def set_digests(off, idx, chunk=1 << 26):
    """Per list: (count, order-independent 64-bit digest of its members)."""
    acc = np.zeros(len(off), np.uint64)
    run = np.uint64(0)
    bounds = np.asarray(off, np.int64)
    with np.errstate(over="ignore"):
        for a in range(0, len(idx), chunk):
            x = np.asarray(idx[a:a + chunk]).astype(np.uint64) * _MIX1
            x ^= x >> np.uint64(29)
            x *= _MIX2
            x ^= x >> np.uint64(32)
            c = np.cumsum(x, dtype=np.uint64) + run
            sel = (bounds > a) & (bounds <= a + len(x))
            acc[sel] = c[bounds[sel] - a - 1]
            run = c[-1]
        diff = acc[1:] - acc[:-1]
    return np.diff(bounds), diff


def device_lists(kind, pos, radius):
    ns = NeighborhoodSearch(kind, radius)
    ns.data.collection = ParticleCollection(position=pos)
    ns.find_neighbors()
    off, idx = ns.neighbor_lists()
    ns.close()
    return off, idx


@pytest.mark.parametrize("case,kind", [("uniform", "hashed-3d"), ("blobs", "hashed-3d"), ("uniform", "compressed-3d")])
def test_search_1m_points_match_reference(ref_oracle, case, kind):
    """Sets of all 10^6 lists equal the reference's own search's: counts
    exactly, members through a 64-bit digest per list. The compressed search
    is compared on the uniform points only: above 97 neighbors (the blobs'
    cores) the reference throws, which ends its process."""
    pos = scenes.ns_points_uniform() if case == "uniform" else scenes.ns_points_blobs()
    off, idx = device_lists(kind, pos, 0.02)
    dc, dd = set_digests(off, idx)
    del idx
    rs = ref_oracle.RefSearch(kind, pos, 0.02, variant="omp")
    assert rs.find()
    ro, ri = rs.lists()
    rs.close()
    rc, rd = set_digests(ro, ri)
    del ri
    assert np.array_equal(dc, rc)
    assert np.array_equal(dd, rd)
    record(f"search_1m/{case}/{kind}", {"neighbors_mean": float(dc.mean()), "neighbors_max": int(dc.max()),
                                        "entries": int(dc.sum())})


def test_set_digests_helper():
    """The digest is order-independent per list and changes with a member."""
    rng = np.random.default_rng(0)
    cnt = rng.integers(0, 7, 1000)
    off = np.concatenate([[0], np.cumsum(cnt)])
    idx = rng.integers(0, 10 ** 6, off[-1])
    c1, d1 = set_digests(off, idx, chunk=37)
    shuffled = idx.copy()
    for i in range(1000):
        shuffled[off[i]:off[i + 1]] = rng.permutation(shuffled[off[i]:off[i + 1]])
    c2, d2 = set_digests(off, shuffled, chunk=101)
    assert np.array_equal(c1, cnt) and np.array_equal(d1, d2)
    shuffled[5] += 1
    assert (set_digests(off, shuffled)[1] != d1).sum() == 1
