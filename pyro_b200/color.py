"""Spectral colour tables of the renderer (src/color.rs), in FP64 on the host.

The renderer's emission kernel reads a look-up table of soot emission
colour against temperature; this module builds it the way the reference
does. The CIE 1931 2-degree colour matching functions come from the
multi-lobe Gaussian fit of Wyman, Sloan and Shirley (JCGT 2013), as in
color.rs:15-21. They are integrated against Planck's law from 360 to
830 nm in 5 nm steps (color.rs:46-70), and the result goes to linear
sRGB with a luminance-preserving gamut clip (color.rs:29-44).

    lut = build_lut()          # (2048, 4) float32: soot, then blackbody
    se = soot_extinction(0.25) # 1/m per ppm of soot at 610, 550, 465 nm
"""
from __future__ import annotations

import numpy as np

H = 6.62607015e-34     # J s
C = 2.99792458e8       # m / s
KB = 1.380649e-23      # J / K
SOOT_K = 6.97          # soot Rayleigh absorption 6 pi E(m), E(m) = 0.37 (color.rs:7)


def _lobe(l, mu, s1, s2):
    s = np.where(l < mu, s1, s2)
    q = (l - mu) / s
    return np.exp(-0.5 * (q * q))


def cmf(l):
    """x, y, z colour matching values at wavelength l in nm (color.rs:15-21)."""
    x = (1.056 * _lobe(l, 599.8, 37.9, 31.0) + 0.362 * _lobe(l, 442.0, 16.0, 26.7)
         - 0.065 * _lobe(l, 501.1, 20.4, 26.2))
    y = 0.821 * _lobe(l, 568.8, 46.9, 40.5) + 0.286 * _lobe(l, 530.9, 16.3, 31.1)
    z = 1.217 * _lobe(l, 437.0, 11.8, 36.0) + 0.681 * _lobe(l, 459.0, 26.0, 13.8)
    return x, y, z


def planck(lm, t):
    """Spectral radiance W / (m^2 sr m) at wavelength lm in m, temperature t (color.rs:24-26)."""
    l2 = lm * lm
    return 2.0 * H * C * C / (l2 * l2 * lm) / (np.exp(H * C / (lm * KB * t)) - 1.0)


def xyz_to_rgb(x, y, z):
    """CIE XYZ to linear sRGB (color.rs:28-34)."""
    return (3.2406 * x - 1.5372 * y - 0.4986 * z,
            -0.9689 * x + 1.8758 * y + 0.0415 * z,
            0.0557 * x - 0.2040 * y + 1.0570 * z)


def _gamut(r, g, b, y):
    """Negative components to zero, then rescaled to the luminance y (color.rs:37-42)."""
    c = [np.maximum(v, 0.0) for v in (r, g, b)]
    ly = 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]
    k = np.where(ly > 0.0, y / np.where(ly > 0.0, ly, 1.0), 0.0)
    return [(v * k).astype(np.float32) for v in c]


def build_lut() -> np.ndarray:
    """(2048, 4) float32 (color.rs:46-70): rows 0..1023 soot emission per
    unit volume fraction and metre of path, rows 1024..2047 blackbody
    surface luminance, for T = 300 + 3000 i / 1023 K; the last channel 0."""
    t = 300.0 + 3000.0 * np.arange(1024, dtype=np.float64) / 1023.0
    out = np.zeros((2048, 4), np.float32)
    for p in range(2):
        xyz = [np.zeros(1024), np.zeros(1024), np.zeros(1024)]
        l = 360.0
        while l <= 830.0:
            lm = l * 1e-9
            e = planck(lm, t) * 1e-9 * 5.0
            if p == 0:
                e = e * (SOOT_K / lm)
            c = cmf(l)
            for k in range(3):
                xyz[k] = xyz[k] + 683.0 * e * c[k]
            l += 5.0
        rgb = _gamut(*xyz_to_rgb(*xyz), xyz[1])
        for k in range(3):
            out[p * 1024:(p + 1) * 1024, k] = rgb[k]
    return out


def soot_extinction(albedo: float) -> np.ndarray:
    """Extinction per ppm of soot at 610, 550 and 465 nm in 1/m
    (absorption / (1 - albedo), color.rs:73-75)."""
    return np.array([SOOT_K / (l * 1e-9) * 1e-6 / (1.0 - albedo) for l in (610.0, 550.0, 465.0)],
                    dtype=np.float32)


def chemi_block(chemi: float = 0.05, soot_albedo: float = 0.25) -> np.ndarray:
    """The emission kernel's uniform (src/render.rs:153-174): chemiluminescence
    strength, soot extinction per ppm at 550 nm, smoke extinction per g/m^3
    (5), 0."""
    return np.array([chemi, soot_extinction(soot_albedo)[1], 5.0, 0.0], dtype=np.float32)
