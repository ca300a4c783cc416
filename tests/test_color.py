"""The renderer's colour tables (pyro_b200/color.py, a restatement of
src/color.rs) against the reference's own known-answer tests
(src/color.rs:78-114)."""
import numpy as np

from pyro_b200 import color


def _lum_at(lut, off, t):
    i = int(round((t - 300.0) / 3000.0 * 1023.0))
    c = lut[off + i]
    return 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]


def test_blackbody_luminance_matches_known_values():
    # about 6e5 cd/m^2 at 2042 K, the platinum point of the old candela
    lut = color.build_lut()
    assert 4.5e5 <= _lum_at(lut, 1024, 2042.0) <= 8.0e5
    assert _lum_at(lut, 1024, 1500.0) < _lum_at(lut, 1024, 2000.0)


def test_blackbody_colour_turns_from_red_to_yellow():
    lut = color.build_lut()
    at = lambda t: lut[1024 + int(round((t - 300.0) / 3000.0 * 1023.0))]  # noqa: E731
    c1, c2 = at(1000.0), at(2500.0)
    assert c1[1] / c1[0] < c2[1] / c2[0]
    assert c1[0] > c1[2]


def test_soot_extinction_scale():
    # 1 ppm of soot at 550 nm: about 15 /m
    e = color.soot_extinction(0.25)
    assert 12.0 <= e[1] <= 20.0
    assert e[2] > e[1] > e[0]


def test_lut_shape_and_soot_rows():
    lut = color.build_lut()
    assert lut.shape == (2048, 4) and lut.dtype == np.float32
    assert np.all(lut[:, 3] == 0) and np.all(lut[:, :3] >= 0)
    ls = 0.2126 * lut[:1024, 0] + 0.7152 * lut[:1024, 1] + 0.0722 * lut[:1024, 2]
    assert np.all(np.diff(ls) > 0)  # soot emission grows with temperature
