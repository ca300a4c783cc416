"""Image development after the path tracer: host-side restatement of the
reference's `post` module (src/post.rs:1-160), which also runs on the CPU
there.  Auto exposure (the 99.5th percentile of luminance, smoothed over
time like a video camera), lens glare (three box-blurred scales), the ACES
film curve, sRGB encoding and dithering to 8 bits.

Arithmetic is FP32 in the reference's expression order.  The box blurs keep
its running sums (add the entering texel, subtract the leaving one), which
are vectorised here across rows (columns) instead of looping over them.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

F32 = np.float32
# glare scales: (radius as a fraction of the width, weight)  (post.rs:93)
GLARE_SCALES = ((0.003, 0.5), (0.012, 0.3), (0.04, 0.2))


def aces(x: np.ndarray) -> np.ndarray:
    """Narkowicz's fit of the ACES film curve, clamped to [0, 1]
    (post.rs:72-75)."""
    x = np.asarray(x, F32) * F32(0.6)
    num = x * (F32(2.51) * x + F32(0.03))
    den = x * (F32(2.43) * x + F32(0.59)) + F32(0.14)
    return np.clip(num / den, F32(0.0), F32(1.0))


def srgb(x: np.ndarray) -> np.ndarray:
    """Linear to sRGB transfer (post.rs:76-82)."""
    x = np.asarray(x, F32)
    with np.errstate(invalid="ignore"):
        hi = F32(1.055) * np.power(x, F32(1.0) / F32(2.4)) - F32(0.055)
    return np.where(x <= F32(0.0031308), F32(12.92) * x, hi).astype(F32)


def hash01(v: np.ndarray) -> np.ndarray:
    """The PCG hash of v in [0, 1) with 24 bits (post.rs:83-88)."""
    x = np.asarray(v, np.uint32) * np.uint32(747796405) + np.uint32(2891336453)
    x = ((x >> ((x >> np.uint32(28)) + np.uint32(4))) ^ x) * np.uint32(277803737)
    x = (x >> np.uint32(22)) ^ x
    return (x >> np.uint32(8)).astype(F32) / F32(16777216.0)


def box_h(b: np.ndarray, r: int) -> np.ndarray:
    """Box filter of radius r along x with clamp-to-edge, b (h, w, 3)
    float32: the reference's running sum per row (post.rs:109-133)."""
    h, w = b.shape[:2]
    norm = F32(1.0) / F32(2 * r + 1)
    acc = np.zeros((h, 3), F32)
    for i in range(min(r, w - 1) + 1):
        acc = acc + b[:, i]
    acc = acc + b[:, 0] * F32(r)
    out = np.empty_like(b)
    for x in range(w):
        out[:, x] = acc * norm
        acc = acc + (b[:, min(x + r + 1, w - 1)] - b[:, max(x - r, 0)])
    return out


def box_v(b: np.ndarray, r: int) -> np.ndarray:
    """Box filter of radius r along y, as box_h (post.rs:135-160)."""
    h, w = b.shape[:2]
    norm = F32(1.0) / F32(2 * r + 1)
    acc = np.zeros((w, 3), F32)
    for i in range(min(r, h - 1) + 1):
        acc = acc + b[i]
    acc = acc + b[0] * F32(r)
    out = np.empty_like(b)
    for y in range(h):
        out[y] = acc * norm
        acc = acc + (b[min(y + r + 1, h - 1)] - b[max(y - r, 0)])
    return out


def percentile_rank(n: int) -> int:
    """Rank (from 0) of the auto exposure's 99.5th luminance percentile
    among n pixels (post.rs:31-35)."""
    return min(int(F32(n) * F32(0.995)), n - 1)


def glare(img: np.ndarray) -> np.ndarray:
    """Lens glare: three scales of three box passes per axis, weighted
    (post.rs:90-107)."""
    h, w = img.shape[:2]
    out = np.zeros_like(img)
    for r, wt in GLARE_SCALES:
        rad = max(int(F32(r) * F32(w)), 1)
        buf = img
        for _ in range(3):
            buf = box_v(box_h(buf, rad), rad)
        out = out + buf * F32(wt)
    return out


class Camera:
    """post::Camera (src/post.rs:6-69): the exposure state of a frame
    sequence.  `develop` turns mean radiance (h, w, 3) into sRGB bytes."""

    def __init__(self, auto: bool, ev_offset: float, glare: float):
        self.ev: Optional[np.float32] = None  # smoothed log2 exposure
        self.auto = bool(auto)
        self.ev_offset = F32(ev_offset)
        self.glare = F32(glare)

    def exposure(self, img: np.ndarray, frame_dt: float) -> np.float32:
        """log2 exposure: the 99.5th luminance percentile mapped to 4,
        approached with a 0.6 s time constant (post.rs:26-46)."""
        if not self.auto:
            return self.ev_offset
        p = img.reshape(-1, 3)
        l = F32(0.2126) * p[:, 0] + F32(0.7152) * p[:, 1] + F32(0.0722) * p[:, 2]
        k = percentile_rank(l.size)
        return self.exposure_from(np.partition(l, k)[k], frame_dt)

    def exposure_from(self, v, frame_dt: float) -> np.float32:
        """The exposure state's update from the frame's 99.5th luminance
        percentile v (the GPU development selects v on the device)."""
        if not self.auto:
            return self.ev_offset
        v = F32(v)
        target = np.log2(F32(4.0) / max(v, F32(1e-3)))
        if self.ev is None:
            ev = F32(target)
        else:
            ev = F32(self.ev + (target - self.ev) *
                     (F32(1.0) - np.exp(F32(-F32(frame_dt) / F32(0.6)))))
        self.ev = ev
        return F32(ev + self.ev_offset)

    def develop(self, img: np.ndarray, frame_dt: float) -> np.ndarray:
        """(h, w, 3) uint8 sRGB (post.rs:25-69)."""
        img = np.ascontiguousarray(img, F32)
        h, w = img.shape[:2]
        k = np.power(F32(2.0), self.exposure(img, frame_dt))
        lin = img * k
        if self.glare > 0.0:
            g = glare(lin)
            lin = lin * (F32(1.0) - self.glare) + g * self.glare
        n = ((hash01(np.arange(h * w, dtype=np.uint32)) - F32(0.5)) / F32(255.0)).reshape(h, w, 1)
        v = srgb(aces(lin)) + n
        return (np.clip(v, F32(0.0), F32(1.0)) * F32(255.0) + F32(0.5)).astype(np.uint8)
