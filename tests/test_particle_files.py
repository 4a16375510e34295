"""Particle files: ParticleSerializer's version-1 layout (ParticleSerializer.cpp:41-141) in an
LZ4 frame, read and written by this library's own LZ4 coder (csrc/fs_lz4.cpp, csrc/fs_io.cpp).

The checkers: the system's lz4 library (liblz4 1.9.x, the library the reference's
Lz4CompressedStream calls, loaded here with ctypes) for the frame layer, and a numpy
restatement of the v1 layout for the records. The reference's own shipped particle files
(scenarios/**, test-series/*.data, written by the reference through liblz4 with linked
blocks) are decoded where the reference checkout is present. Host code only: no GPU."""
import ctypes
import ctypes.util
import glob
import os

import numpy as np
import pytest

from fluidsolver_b200 import _lib as F
from fluidsolver_b200 import read_particles, write_particles
from fluidsolver_b200.solver import ParticleCollection

from oracle.reference_path import reference_dir

REFERENCE = reference_dir()


def _liblz4():
    for name in (ctypes.util.find_library("lz4"), "liblz4.so.1"):
        if not name:
            continue
        try:
            L = ctypes.CDLL(name)
        except OSError:
            continue
        L.LZ4F_compressFrameBound.restype = ctypes.c_size_t
        L.LZ4F_compressFrameBound.argtypes = [ctypes.c_size_t, ctypes.c_void_p]
        L.LZ4F_compressFrame.restype = ctypes.c_size_t
        L.LZ4F_compressFrame.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                         ctypes.c_void_p]
        L.LZ4F_isError.argtypes = [ctypes.c_size_t]
        L.LZ4F_createDecompressionContext.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint]
        L.LZ4F_decompress.restype = ctypes.c_size_t
        L.LZ4F_decompress.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                      ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p]
        L.LZ4F_freeDecompressionContext.argtypes = [ctypes.c_void_p]
        return L
    return None


LZ4 = _liblz4()
needs_lz4 = pytest.mark.skipif(LZ4 is None, reason="the system lz4 library (the checker) is absent")


def lz4_compress(data: bytes) -> bytes:
    """A frame from liblz4 with its default preferences (64 KB linked blocks), as the reference writes."""
    cap = LZ4.LZ4F_compressFrameBound(len(data), None)
    dst = ctypes.create_string_buffer(cap)
    n = LZ4.LZ4F_compressFrame(dst, cap, data, len(data), None)
    assert not LZ4.LZ4F_isError(n)
    return dst.raw[:n]


def lz4_decompress(frame: bytes) -> bytes:
    ctx = ctypes.c_void_p()
    assert not LZ4.LZ4F_isError(LZ4.LZ4F_createDecompressionContext(ctypes.byref(ctx), 100))
    out, pos = bytearray(), 0
    buf = ctypes.create_string_buffer(1 << 20)
    src = ctypes.create_string_buffer(frame, len(frame))
    while pos < len(frame):
        dst_n, src_n = ctypes.c_size_t(len(buf)), ctypes.c_size_t(len(frame) - pos)
        r = LZ4.LZ4F_decompress(ctx, buf, ctypes.byref(dst_n), ctypes.byref(src, pos), ctypes.byref(src_n), None)
        assert not LZ4.LZ4F_isError(r)
        out += buf.raw[:dst_n.value]
        pos += src_n.value
        if r == 0 and src_n.value == 0 and dst_n.value == 0:
            break
    LZ4.LZ4F_freeDecompressionContext(ctx)
    return bytes(out)


# ---- numpy restatement of the v1 records (ParticleSerializer.cpp:41-141) ----------------------
def record_dtype(components, dim):
    f = []
    if components & (F.FS_COMPONENT_MOVEMENT_2D | F.FS_COMPONENT_MOVEMENT_3D):
        f += [("position", "<f4", (dim,)), ("velocity", "<f4", (dim,)), ("acceleration", "<f4", (dim,))]
    if components & F.FS_COMPONENT_INFO:
        f += [("type", "u1"), ("tag", "<u4")]
    if components & F.FS_COMPONENT_DATA:
        f += [("density", "<f4"), ("mass", "<f4"), ("pressure", "<f4")]
    if components & (F.FS_COMPONENT_EXTERNAL_2D | F.FS_COMPONENT_EXTERNAL_3D):
        f += [("external", "<f4", (dim,))]
    return np.dtype(f)


def parse_v1(payload: bytes):
    version, count = np.frombuffer(payload[:8], "<u4")
    assert version == 1
    ids = np.frombuffer(payload[8:8 + 4 * count], "<u4")
    comp = int(sum(1 << int(i) for i in ids))
    n = int(np.frombuffer(payload[8 + 4 * count:16 + 4 * count], "<u8")[0])
    dim = 2 if comp & (F.FS_COMPONENT_MOVEMENT_2D | F.FS_COMPONENT_EXTERNAL_2D) else 3
    rec = np.frombuffer(payload[16 + 4 * count:], record_dtype(comp, dim))
    assert len(rec) == n
    return comp, dim, rec


def serialize_v1(col: ParticleCollection) -> bytes:
    dim = col.dim
    comp = (F.FS_COMPONENT_MOVEMENT_2D if dim == 2 else F.FS_COMPONENT_MOVEMENT_3D) | F.FS_COMPONENT_INFO | \
        F.FS_COMPONENT_DATA | (F.FS_COMPONENT_EXTERNAL_2D if dim == 2 else F.FS_COMPONENT_EXTERNAL_3D)
    ids = [i for i in range(1, 7) if comp & (1 << i)]
    rec = np.zeros(len(col), record_dtype(comp, dim))
    for name in rec.dtype.names:
        rec[name] = getattr(col, name)
    head = np.array([1, len(ids)] + ids, "<u4").tobytes() + np.array([len(col)], "<u8").tobytes()
    return head + rec.tobytes()


def random_collection(n, dim, seed):
    rng = np.random.default_rng(seed)
    f = lambda *s: rng.standard_normal(s).astype(np.float32)
    return ParticleCollection(position=np.round(f(n, dim) * 20, 1).astype(np.float32), velocity=f(n, dim),
                              acceleration=f(n, dim), external=f(n, dim), mass=np.ones(n, np.float32),
                              density=f(n), pressure=f(n), type=rng.integers(0, 3, n).astype(np.uint8),
                              tag=rng.permutation(n).astype(np.uint32))


def assert_same(a: ParticleCollection, b: ParticleCollection):
    for name in ("position", "velocity", "acceleration", "external", "mass", "density", "pressure", "type", "tag"):
        x, y = getattr(a, name), getattr(b, name)
        assert (x is None) == (y is None), name
        if x is not None:
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8)), name


@pytest.mark.parametrize("dim,n", [(3, 1), (3, 1000), (2, 777), (3, 200_000)])
def test_round_trip(tmp_path, dim, n):
    col = random_collection(n, dim, seed=n + dim)
    path = tmp_path / "p.data"
    write_particles(path, col)
    assert_same(read_particles(path), col)


@needs_lz4
@pytest.mark.parametrize("dim,n", [(3, 1000), (2, 500), (3, 300_000)])
def test_frames_against_liblz4(tmp_path, dim, n):
    """Our frames decode with liblz4 to the v1 bytes; liblz4's frames (linked blocks, as the
    reference writes them) decode with ours."""
    col = random_collection(n, dim, seed=7 * n)
    payload = serialize_v1(col)
    ours = tmp_path / "ours.data"
    write_particles(ours, col)
    assert lz4_decompress(ours.read_bytes()) == payload
    theirs = tmp_path / "theirs.data"
    theirs.write_bytes(lz4_compress(payload))
    assert_same(read_particles(theirs), col)


@needs_lz4
def test_repetitive_payload_compresses(tmp_path):
    # the reference's own large-data pattern (Lz4CompressedStreamTests.cpp: byte i % 127) as particle
    # positions, plus a lattice: long matches, overlapping copies, several 64 KB blocks
    n = 100_000
    pos = (np.arange(3 * n) % 127).astype(np.float32).reshape(n, 3)
    col = ParticleCollection(position=pos, velocity=np.zeros_like(pos), acceleration=np.zeros_like(pos),
                             external=np.zeros_like(pos), mass=np.ones(n, np.float32), density=np.ones(n, np.float32),
                             pressure=np.zeros(n, np.float32), type=np.zeros(n, np.uint8),
                             tag=np.arange(n, dtype=np.uint32))
    path = tmp_path / "lattice.data"
    write_particles(path, col)
    raw = path.read_bytes()
    assert len(raw) < len(serialize_v1(col)) // 4
    assert lz4_decompress(raw) == serialize_v1(col)
    assert_same(read_particles(path), col)


@needs_lz4
@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="the reference checkout is absent")
def test_reference_particle_files():
    files = sorted(glob.glob(f"{REFERENCE}/scenarios/**/*.data", recursive=True) +
                   glob.glob(f"{REFERENCE}/test-series/*.data"))
    assert len(files) >= 10
    for f in files:
        raw = open(f, "rb").read()
        comp, dim, rec = parse_v1(lz4_decompress(raw))
        got = read_particles(f)
        assert got.dim == dim and len(got) == len(rec), f
        for name in rec.dtype.names:
            assert np.array_equal(np.asarray(getattr(got, name)).view(np.uint8),
                                  np.ascontiguousarray(rec[name]).view(np.uint8)), (f, name)


def test_errors(tmp_path):
    col = random_collection(50, 3, seed=1)
    path = tmp_path / "p.data"
    write_particles(path, col)
    raw = bytearray(path.read_bytes())
    bad = tmp_path / "bad.data"
    for mutate, msg in ((lambda b: b[:len(b) // 2], "truncated"), (lambda b: b[:5] + bytes([b[5] ^ 0x10]) + b[6:], "checksum"),
                        (lambda b: b"\0\0\0\0" + b[4:], "not an LZ4 frame")):
        bad.write_bytes(bytes(mutate(raw)))
        with pytest.raises(F.FluidSolverError, match=msg):
            read_particles(bad)
    with pytest.raises(F.FluidSolverError, match="cannot open"):
        read_particles(tmp_path / "missing.data")
