"""The path tracer's tone mapping (host code of the library, fs_tone_map)
against the reference's own ToneMapper (ToneMapper.cpp:7-102): exposure,
the exponential and the ACES filmic curves, the clamp, the gamma correction
on and off, the byte conversion. Byte-identical on the golden fixture made
through the reference's class (tests/golden/make_golden.py) and, where
oracle/_ref is built, on fresh inputs. No GPU: the mapping runs on the host."""
import numpy as np
import pytest

from fluidsolver_b200 import tone_map
from tests.golden.make_golden import TONE_CASES


@pytest.mark.parametrize("name", list(TONE_CASES))
def test_tone_map_equals_the_reference_fixture(golden, name):
    g = golden["tonemap"]
    assert np.array_equal(tone_map(g["radiance"], **TONE_CASES[name]), g[name])


@pytest.mark.parametrize("name", list(TONE_CASES))
def test_tone_map_equals_the_compiled_reference(ref_oracle, name):
    rng = np.random.default_rng(91)
    rad = np.exp(rng.uniform(np.log(1e-5), np.log(50.0), (33, 17, 3))).astype(np.float32)
    assert np.array_equal(tone_map(rad, **TONE_CASES[name]), ref_oracle.tone_map(rad, **TONE_CASES[name]))


def test_tone_map_rejects_an_unknown_curve():
    import ctypes
    from fluidsolver_b200 import _lib as F
    rs = F.FsRenderSettings()
    F.lib().fs_render_settings_default(ctypes.byref(rs))
    assert rs.tone_mapper == 0 and rs.gamma_correction == 1 and abs(rs.exposure - 0.2) < 1e-7
    rs.tone_mapper = 2
    rad = np.zeros(3, np.float32)
    out = np.zeros(4, np.uint8)
    assert F.lib().fs_tone_map(rad.ctypes.data, 1, ctypes.byref(rs), out.ctypes.data) == F.FS_ERR_INVALID
