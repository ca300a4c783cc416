"""Image development (src/post.rs) on the CPU: the vectorised restatement in
pyro_b200.post against a scalar, pixel-by-pixel FP32 restatement of the
reference's loops (bit for bit), and the curves against their formulas."""
import math

import numpy as np
import pytest

from pyro_b200 import post

F = np.float32


def _hash_int(v):
    """post.rs:83-88 in Python integers."""
    x = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    x = (((x >> ((x >> 28) + 4)) ^ x) * 277803737) & 0xFFFFFFFF
    x = (x >> 22) ^ x
    return (x >> 8) / 16777216.0


def _box_h_scalar(b, r):
    h, w = b.shape[:2]
    out = b.copy()
    norm = F(1.0) / F(2 * r + 1)
    for y in range(h):
        line = b[y]
        acc = [F(0.0)] * 3
        for i in range(min(r, w - 1) + 1):
            acc = [F(acc[c] + line[i][c]) for c in range(3)]
        acc = [F(acc[c] + F(line[0][c] * F(r))) for c in range(3)]
        for x in range(w):
            out[y, x] = [F(a * norm) for a in acc]
            add, rem = line[min(x + r + 1, w - 1)], line[max(x - r, 0)]
            acc = [F(acc[c] + F(add[c] - rem[c])) for c in range(3)]
    return out


def _box_v_scalar(b, r):
    return _box_h_scalar(b.transpose(1, 0, 2).copy(), r).transpose(1, 0, 2).copy()


def _img(h, w, seed, scale=3.0):
    rng = np.random.default_rng(seed)
    return (rng.exponential(scale, (h, w, 3)) * (rng.random((h, w, 1)) < 0.7)).astype(F)


def test_curves():
    assert post.aces(F(0.0)) == 0.0
    x = np.linspace(0, 50, 1001, dtype=F)
    a = post.aces(x)
    assert np.all(np.diff(a) >= 0) and a[-1] == 1.0
    xd = x.astype(np.float64) * 0.6
    ad = np.clip(xd * (2.51 * xd + 0.03) / (xd * (2.43 * xd + 0.59) + 0.14), 0, 1)
    np.testing.assert_allclose(a, ad, atol=2e-7)
    assert post.srgb(F(0.001)) == F(12.92) * F(0.001)
    assert abs(float(post.srgb(F(1.0))) - 1.0) < 1e-6
    s = post.srgb(np.linspace(0.0032, 1, 100, dtype=F)).astype(np.float64)
    np.testing.assert_allclose(s, 1.055 * np.linspace(0.0032, 1, 100) ** (1 / 2.4) - 0.055,
                               atol=1e-6)
    v = np.array([0, 1, 2, 12345, 2**32 - 1], np.uint32)
    assert list(post.hash01(v)) == [F(_hash_int(int(i))) for i in v]


@pytest.mark.parametrize("h,w,r", [(5, 9, 1), (7, 4, 3), (3, 20, 6), (1, 1, 2), (6, 6, 10)])
def test_box_filters_match_the_running_sums(h, w, r):
    b = _img(h, w, h * 31 + w)
    assert np.array_equal(post.box_h(b, r), _box_h_scalar(b, r))
    assert np.array_equal(post.box_v(b, r), _box_v_scalar(b, r))
    # and, for r < w, the clamp-to-edge window mean (up to the running
    # sum's rounding); the reference's first sum takes texels 0 .. w - 1
    # once when r >= w, and so does the restatement
    if r >= w:
        return
    xs = np.clip(np.arange(w)[:, None] + np.arange(-r, r + 1)[None, :], 0, w - 1)
    want = b.astype(np.float64)[:, xs].mean(axis=2)
    np.testing.assert_allclose(post.box_h(b, r), want, rtol=1e-5, atol=1e-5 * b.max())


def _develop_scalar(cam, img, frame_dt):
    """post.rs:25-69 pixel by pixel (np.float32 scalars)."""
    h, w = img.shape[:2]
    k = np.power(F(2.0), cam.exposure(img, frame_dt))
    lin = (img * k).astype(F)
    if cam.glare > 0:
        g = np.zeros_like(lin)
        for r, wt in post.GLARE_SCALES:
            rad = max(int(F(r) * F(w)), 1)
            buf = lin.copy()
            for _ in range(3):
                buf = _box_v_scalar(_box_h_scalar(buf, rad), rad)
            g = (g + buf * F(wt)).astype(F)
        lin = (lin * (F(1.0) - cam.glare) + g * cam.glare).astype(F)
    out = np.zeros((h, w, 3), np.uint8)
    for i in range(h * w):
        n = F(F(F(_hash_int(i)) - F(0.5)) / F(255.0))
        for c in range(3):
            x = lin.reshape(-1, 3)[i, c]
            v = F(post.srgb(post.aces(x)) + n)
            out.reshape(-1, 3)[i, c] = int(F(min(max(v, F(0.0)), F(1.0)) * F(255.0) + F(0.5)))
    return out


@pytest.mark.parametrize("auto,glare", [(True, 0.04), (False, 0.0), (True, 0.0)])
def test_develop_matches_the_scalar_restatement(auto, glare):
    img = _img(12, 40, 3)
    a = post.Camera(auto, 0.5, glare)
    b = post.Camera(auto, 0.5, glare)
    for _ in range(2):  # the second frame uses the smoothed exposure
        got = a.develop(img, 1.0 / 30.0)
        want = _develop_scalar(b, img, 1.0 / 30.0)
        assert got.dtype == np.uint8 and got.shape == (12, 40, 3)
        assert np.array_equal(got, want)
        img = img * F(1.5)


def test_auto_exposure_targets_the_995th_percentile_and_smooths():
    img = np.zeros((20, 50, 3), F)
    img[..., :] = 0.1
    img[0, :4, :] = 8.0  # 4 of 1000 pixels bright: value 995 in order stays 0.1
    cam = post.Camera(True, 0.0, 0.0)
    ev0 = cam.exposure(img, 1 / 30)
    assert ev0 == pytest.approx(math.log2(4.0 / 0.1), rel=1e-6)
    ev1 = cam.exposure(img * F(4.0), 1 / 30)
    target = math.log2(4.0 / 0.4)
    assert ev1 == pytest.approx(ev0 + (target - ev0) * (1 - math.exp(-1 / 30 / 0.6)), rel=1e-5)
    assert post.Camera(False, -1.5, 0.0).exposure(img, 1 / 30) == F(-1.5)
