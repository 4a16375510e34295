"""Generates the golden fixtures in tests/golden/ from the reference's own
libFluid sources compiled in oracle/_ref (make -C oracle/ref, which needs the
reference checkout). Run from the repository root:

    python tests/golden/make_golden.py

Every fixture records the inputs (seeded) and the reference's outputs, so the
CPU tests can pin the C restatement (oracle/fs_oracle.c) and the GPU tests can
check the device path where the reference checkout is absent.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from fluidsolver_b200 import scenes  # noqa: E402
from oracle import ref_oracle as R  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def sample_grid(start, step, stop):
    """GetSampleGrid of tests/NeighborhoodSearchTests.cpp:51-62 (float loop
    counters, row-major with x fastest)."""
    pts = []
    y = np.float32(start)
    while y <= np.float32(stop):
        x = np.float32(start)
        while x <= np.float32(stop):
            pts.append((x, y))
            x = np.float32(x + np.float32(step))
        y = np.float32(y + np.float32(step))
    return np.array(pts, np.float32)


def kernel_fixture():
    rng = np.random.default_rng(11)
    out = {}
    for dim in (2, 3):
        for support in (1.0, 2.0, 0.02, 8.5):
            h = support / 2
            x = (rng.uniform(-2.2, 2.2, (2000, dim)) * h).astype(np.float32)
            x[:5] = 0.0  # |x| <= FLT_EPSILON branch
            W, dW = R.kernel_eval(dim, support, x)
            key = f"d{dim}_s{support}"
            out[key + "_x"] = x
            out[key + "_W"] = W
            out[key + "_dW"] = dW
    np.savez_compressed(os.path.join(OUT, "kernel.npz"), **out)


def cfl_fixture():
    rng = np.random.default_rng(12)
    a = (10 ** rng.uniform(-3, 4, 4000)).astype(np.float32)
    v = (10 ** rng.uniform(-3, 2, 4000)).astype(np.float32)
    a[:10] = 0.0
    v[10:20] = 0.0
    out = {}
    for la in (0.25, 0.3):
        out[f"dt_la{la}"] = R.cfl_timestep(0.005, 0.4, la, 1.0, a, v)
    np.savez_compressed(os.path.join(OUT, "cfl.npz"), max_acc=a, max_vel=v, **out)


def dynamic_timestep_fixture():
    """DynamicCflTimestepGenerator on random collections: velocity and
    acceleration magnitudes over many decades, zero fields, inactive
    particles carrying the largest values, 2D and 3D."""
    rng = np.random.default_rng(21)
    cases = []
    for c in range(64):
        dim = 3 if c % 4 else 2
        n = int(rng.integers(1, 400))
        vel = (rng.standard_normal((n, dim)) * 10 ** rng.uniform(-4, 2)).astype(np.float32)
        acc = (rng.standard_normal((n, dim)) * 10 ** rng.uniform(-4, 3)).astype(np.float32)
        typ = rng.choice(np.array([0, 1, 2], np.uint8), n, p=[0.7, 0.2, 0.1])
        if c % 7 == 0:
            vel[:] = 0.0
        if c % 11 == 0:
            acc[:] = 0.0
        if c % 5 == 0:   # the fastest particle is inactive
            k = int(rng.integers(n))
            typ[k] = 2
            vel[k] = 1e3
            acc[k] = 1e4
        ps = float(rng.choice([1.0, 0.1, 0.01]))
        lo, hi = float(10 ** rng.uniform(-6, -3)), float(10 ** rng.uniform(-3, 0))
        lv, la = float(rng.uniform(0.1, 0.9)), float(rng.uniform(0.1, 0.9))
        dt = R.dynamic_timestep(vel, acc, typ, ps, lo, hi, lv, la)
        cases.append((dim, vel, acc, typ, np.array([ps, lo, hi, lv, la, dt], np.float32)))
    out = {}
    for i, (dim, vel, acc, typ, prm) in enumerate(cases):
        out[f"c{i}_vel"], out[f"c{i}_acc"], out[f"c{i}_type"], out[f"c{i}_prm"] = vel, acc, typ, prm
    np.savez_compressed(os.path.join(OUT, "dynamic_timestep.npz"), **out)


def boundary_fixture():
    """BoundaryPreprocessor (BoundaryPreprocessor.cpp:7-48) through the reference's
    hashed-3d interface: single- and two-layer tanks, a jittered tank at another
    particle size, and initial masses that differ from particle to particle."""
    rng = np.random.default_rng(31)
    out = {}
    cases = [("one_layer", 1.0, 1, 0.0), ("two_layers", 1.0, 2, 0.0), ("jittered", 0.5, 1, 0.05)]
    for name, ps, layers, jitter in cases:
        sc = scenes.breaking_dam_3d(6, 5, 4, ps, tank=(14, 9, 8), layers=layers, seed=41)
        col = sc.collection
        pos = col.position.astype(np.float32)
        if jitter:
            pos = (pos + rng.uniform(-jitter, jitter, pos.shape) * ps).astype(np.float32)
        mass = (col.mass * rng.uniform(0.5, 1.5, len(pos))).astype(np.float32)
        typ = col.type.astype(np.uint8)
        typ[rng.choice(len(typ), 5, replace=False)] = 2   # some inactive particles
        s = R.RefSearch("hashed-3d", pos, 2.0 * ps, typ)
        assert s.find()
        res = s.boundary_preprocess(mass, ps, 1.0)
        s.close()
        out[f"{name}_pos"], out[f"{name}_mass"], out[f"{name}_type"] = pos, mass, typ
        out[f"{name}_size"], out[f"{name}_out"] = np.float32(ps), res
    np.savez_compressed(os.path.join(OUT, "boundary.npz"), **out)


def camera_rays(position, target, width, height, fov_x=np.pi / 2):
    """Pinhole rays through pixel centres (the construction of Camera.cpp:10-39, y flipped)."""
    f = np.asarray(target, np.float64) - position
    f /= np.linalg.norm(f)
    up = np.array([0.0, 1.0, 0.0])
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    x, y = np.meshgrid((np.arange(width) + 0.5) / width * 2 - 1, -((np.arange(height) + 0.5) / height * 2 - 1))
    t = np.tan(fov_x / 2)
    d = x[..., None] * t * s + y[..., None] * t * u + f
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    o = np.broadcast_to(np.asarray(position, np.float64), d.shape)
    return o.reshape(-1, 3).astype(np.float32), d.reshape(-1, 3).astype(np.float32)


def raytrace_fixture():
    """ParticleIntersectionAccelerator (ParticleIntersectionAccelerator.cpp:8-206): first hits of camera
    rays on a breaking dam in a tank (fluid from outside, walls, misses) and of rays that start inside
    the fluid (the surface from inside)."""
    sc = scenes.breaking_dam_3d(12, 10, 8, 1.0, tank=(24, 16, 14), seed=51, layers=2)
    col = sc.collection
    pos, mass, typ = col.position.astype(np.float32), col.mass.astype(np.float32), col.type.astype(np.uint8)
    o1, d1 = camera_rays((30.0, 18.0, 28.0), (6.0, 4.0, 4.0), 48, 36, fov_x=0.7)
    o3, d3 = camera_rays((6.5, 30.0, 5.5), (6.0, 4.0, 4.0), 32, 32, fov_x=0.9)   # from above the open tank
    rng = np.random.default_rng(52)
    fl = pos[typ == 0]
    o2 = fl[rng.choice(len(fl), 200, replace=False)] + rng.uniform(-0.3, 0.3, (200, 3)).astype(np.float32)
    d2 = rng.standard_normal((200, 3))
    d2 = (d2 / np.linalg.norm(d2, axis=1, keepdims=True)).astype(np.float32)
    o, d = np.concatenate([o1, o2, o3]), np.concatenate([d1, d2, d3])
    res = R.trace_rays(pos, mass, typ, 1.0, 1.0, o, d)
    np.savez_compressed(os.path.join(OUT, "raytrace.npz"), pos=pos, mass=mass, type=typ, origins=o, directions=d,
                        **res)


def _lists(kind, pos, radius, typ, calls=1, moves=None):
    s = R.RefSearch(kind, pos, radius, typ)
    ok = s.find()
    off, idx = s.lists() if ok else (np.zeros(len(pos) + 1, np.int64), np.zeros(0, np.int64))
    return ok, off, idx


def search_fixture():
    out = {}
    # the reference's googletest grids (NeighborhoodSearchTests.cpp:131-299)
    grids = {"grid11": (sample_grid(-5, 1, 5), 2.0), "grid3": (sample_grid(-1, 1, 1), 2.0),
             "grid11x2": (sample_grid(-10, 2, 10), 4.0)}
    for name, (pos, r) in grids.items():
        for kind in ("quadratic-2d", "hashed-2d"):
            ok, off, idx = _lists(kind, pos, r, None)
            out[f"{name}_{kind}_pos"] = pos
            out[f"{name}_{kind}_off"] = off.astype(np.int32)
            out[f"{name}_{kind}_idx"] = idx.astype(np.int32)
            out[f"{name}_{kind}_r"] = np.float32(r)
    # 3D sets with every particle type, including inactive ones
    sc = scenes.breaking_dam_3d(8, 9, 7, 1.0, tank=(14, 12, 11), seed=21)
    typ = sc.collection.type.copy()
    typ[::23] = 2
    for kind in ("hashed-3d", "quadratic-3d", "compressed-3d"):
        ok, off, idx = _lists(kind, sc.collection.position, 2.0, typ)
        out[f"dam3d_{kind}_ok"] = np.int32(ok)
        out[f"dam3d_{kind}_off"] = off.astype(np.int32)
        out[f"dam3d_{kind}_idx"] = idx.astype(np.int32)
    out["dam3d_pos"] = sc.collection.position
    out["dam3d_type"] = typ
    # 2D with inactive particles
    sc2 = scenes.breaking_dam_2d(12, 10, width=20, height=16)
    t2 = sc2.collection.type.copy()
    t2[::11] = 2
    for kind in ("quadratic-2d", "hashed-2d"):
        ok, off, idx = _lists(kind, sc2.collection.position, 2.0, t2)
        out[f"dam2d_{kind}_off"] = off.astype(np.int32)
        out[f"dam2d_{kind}_idx"] = idx.astype(np.int32)
    out["dam2d_pos"] = sc2.collection.position
    out["dam2d_type"] = t2
    # uniform random 3D points (the microbenchmark's distribution, 4096 points)
    rng = np.random.default_rng(2)
    pts = rng.random((4096, 3)).astype(np.float32)
    for kind in ("hashed-3d", "compressed-3d"):
        ok, off, idx = _lists(kind, pts, 0.1, None)
        out[f"rand_{kind}_ok"] = np.int32(ok)
        out[f"rand_{kind}_off"] = off.astype(np.int32)
        out[f"rand_{kind}_idx"] = idx.astype(np.int32)
    out["rand_pos"] = pts
    # a dense cluster: more than 97 neighbors. The compressed search's
    # std::bitset::set throws inside std::for_each(std::execution::par, ...),
    # which ends the process through std::terminate; run it in a child process
    # and record how it ended.
    blob = (rng.normal(0.5, 0.02, (600, 3))).astype(np.float32)
    np.save(os.path.join(OUT, "_blob_tmp.npy"), blob)
    code = ("import sys, numpy as np; sys.path.insert(0, %r); from oracle import ref_oracle as R; "
            "p = np.load(%r); s = R.RefSearch('compressed-3d', p, 0.1); sys.exit(0 if s.find() else 3)"
            % (ROOT, os.path.join(OUT, "_blob_tmp.npy")))
    rc = subprocess.run([sys.executable, "-c", code], capture_output=True).returncode
    os.remove(os.path.join(OUT, "_blob_tmp.npy"))
    out["blob_pos"] = blob
    out["blob_compressed_exit"] = np.int32(rc)
    np.savez_compressed(os.path.join(OUT, "search.npz"), **out)


SOLVER_CASES = {
    # name: (solver, search, scene builder, generator, settings, steps)
    "iisph3d_hashed": ("iisph-3d", "hashed-3d", lambda: scenes.breaking_dam_3d(6, 8, 5, 1.0, tank=(12, 12, 10), seed=31),
                       (0.005, 0.4, 0.25), R.iisph3d_settings(), 4),
    "iisph3d_multilayer": ("iisph-3d", "quadratic-3d",
                           lambda: scenes.breaking_dam_3d(5, 6, 5, 1.0, tank=(10, 10, 8), seed=32, layers=2),
                           (0.005, 0.4, 0.25), R.iisph3d_settings(single_layer=False, viscosity=5.0), 3),
    "sesph3d_hashed": ("sesph-3d", "hashed-3d", lambda: scenes.breaking_dam_3d(6, 8, 5, 1.0, tank=(12, 12, 10), seed=33),
                       (0.001, 0.4, 0.25), R.sesph3d_settings(k=1000.0), 4),
    "sesph2d_quadratic": ("sesph-2d", "quadratic-2d", lambda: scenes.breaking_dam_2d(12, 10, width=20, height=16, seed=1),
                          (0.001, 0.4, 0.25), R.sesph2d_settings(k=1000.0), 4),
    "sesph2d_hashed": ("sesph-2d", "hashed-2d", lambda: scenes.breaking_dam_2d(12, 10, width=20, height=16, seed=2),
                       (0.001, 0.4, 0.25), R.sesph2d_settings(k=1000.0), 4),
    "iisph2d_quadratic": ("iisph-2d", "quadratic-2d", lambda: scenes.breaking_dam_2d(12, 10, width=20, height=16, seed=3),
                          (0.005, 0.4, 0.25), R.iisph2d_settings(), 4),
}


def solver_fixture():
    out = {}
    for name, (solver, search, build, gen, settings, steps) in SOLVER_CASES.items():
        sc = build()
        col = sc.collection
        ref = R.RefSolver(solver, search, col, (1.0, 9.81, 1.0), settings, gen)
        out[f"{name}_in_position"] = col.position
        out[f"{name}_in_type"] = col.type
        stats = []
        for k in range(steps):
            st = ref.step()
            stats.append([st["desired_dt"], st["actual_dt"], st["iterations"], st["avg_density_error"]])
            s = ref.state()
            for f in ("position", "velocity", "density", "pressure"):
                out[f"{name}_step{k}_{f}"] = s[f]
        out[f"{name}_stats"] = np.array(stats, np.float32)
        out[f"{name}_settings"] = np.array(settings, np.float32)
        out[f"{name}_generator"] = np.array(gen, np.float32)
    np.savez_compressed(os.path.join(OUT, "solvers.npz"), **out)


def position_query_fixture():
    """NeighborhoodInterface::get_neighbors(position) of every contract that
    has one, on random points with a third of them inactive."""
    out = {}
    rng = np.random.default_rng(14)
    for dim, kinds in ((3, ("hashed-3d", "quadratic-3d", "compressed-3d")), (2, ("hashed-2d", "quadratic-2d"))):
        pos = (rng.random((3000, dim)) * 10).astype(np.float32)
        typ = rng.integers(0, 3, 3000).astype(np.uint8)
        queries = (rng.random((40, dim)) * 10).astype(np.float32)
        out[f"pos{dim}"], out[f"type{dim}"], out[f"queries{dim}"] = pos, typ, queries
        for kind in kinds:
            s = R.RefSearch(kind, pos, 1.0, typ)
            assert s.find()
            res = [np.sort(s.query(q)) for q in queries]
            s.close()
            out[f"{kind}/offsets"] = np.concatenate([[0], np.cumsum([len(a) for a in res])]).astype(np.int64)
            out[f"{kind}/indices"] = np.concatenate(res).astype(np.int64)
    np.savez_compressed(os.path.join(OUT, "position_queries.npz"), **out)


TONE_CASES = {"exponential": dict(exposure=0.2, gamma=2.2, filmic=False, gamma_correction=True),
              "filmic": dict(exposure=0.7, gamma=2.2, filmic=True, gamma_correction=True),
              "exponential_linear": dict(exposure=1.5, gamma=1.0, filmic=False, gamma_correction=False),
              "filmic_linear": dict(exposure=0.05, gamma=1.8, filmic=True, gamma_correction=False)}


def tone_radiance():
    """Fixed radiance for the tone mapper: log-spread values over 1e-4..1e3,
    zeros, negatives, values at the byte boundaries, one infinity."""
    rng = np.random.default_rng(15)
    r = np.exp(rng.uniform(np.log(1e-4), np.log(1e3), (48, 64, 3))).astype(np.float32)
    r[0, :8] = 0.0
    r[1, :8] = -rng.uniform(0, 5, (8, 3))
    r[2, :16] = (np.arange(16 * 3).reshape(16, 3) / 47.0 * 20.0).astype(np.float32)
    r[3, 0] = np.inf
    return r


def tonemap_fixture():
    """ToneMapper::map_render_target_to_image (ToneMapper.cpp:71-102) through the reference's own class."""
    rad = tone_radiance()
    out = {"radiance": rad}
    for name, kw in TONE_CASES.items():
        out[name] = R.tone_map(rad, **kw)
    np.savez_compressed(os.path.join(OUT, "tonemap.npz"), **out)


if __name__ == "__main__":
    if not R.available():
        sys.exit("oracle/_ref is not built; run `make -C oracle/ref REF=<reference checkout>` where it is available")
    fixtures = {"kernel": kernel_fixture, "cfl": cfl_fixture, "search": search_fixture, "solvers": solver_fixture,
                "position_queries": position_query_fixture, "dynamic_timestep": dynamic_timestep_fixture,
                "boundary": boundary_fixture, "raytrace": raytrace_fixture, "tonemap": tonemap_fixture}
    for name in sys.argv[1:] or fixtures:
        fixtures[name]()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)), "bytes")
