"""Host logic of the --sim-only frame loop (src/main.rs:121-279) with a fake
simulation: CFL substep counts, the averaging window, heat-release heights,
Heskestad, and the slice image / PNG writer."""
import math
import os
import struct
import zlib

import numpy as np

from pyro_b200.run import height_at, run_frames, slice_image, substeps_for, write_png
from pyro_b200.scene import Scene
from pyro_b200.sim import Stats

SCENE = """[domain]
size = [1.6, 3.2, 1.6]
cell = 0.1
[sim]
fps = 10
duration = 2.0
cfl = 1.5
[[object]]
kind = "pool"
material = "heptane"
center = [0.8, 0.0, 0.8]
radius = 0.25
[output]
preroll = 0.5
"""


class FakeSim:
    def __init__(self, dims, dx, umax):
        self.dims = dims
        self.dx = dx
        self.time = np.float32(0.0)
        self.umax = umax
        self.calls = []

    def step(self, dt, want_stats):
        self.calls.append((float(dt), bool(want_stats)))
        self.time = np.float32(self.time + np.float32(dt))

    def read_stats(self):
        ny = self.dims[1]
        layers = [0.0] * ny
        layers[2], layers[5], layers[9] = 100.0, 300.0, 600.0
        return Stats(hrr=1000.0, rad=300.0, pyro=0.01, soot=0.0, max_t=1500.0,
                     max_u=self.umax, solid=1.0, area=0.2, resid=1e-3, layers=layers)


def test_substep_rule_matches_reference_formula():
    n, dt = substeps_for(1.5, 0.02, 30.0, 7.0)
    assert n == math.ceil((1 / 30) / (1.5 * 0.02 / 7.0))
    assert np.float32(dt) == np.float32(np.float32(1.0 / 30.0) / np.float32(n))
    assert substeps_for(1.5, 0.1, 10.0, 0.2)[0] == 1  # max(u, 1)


def test_frame_loop_counts_and_averages():
    sc = Scene.from_toml_str(SCENE)
    sim = FakeSim([16, 32, 16], 0.1, umax=7.0)
    s = run_frames(sc, sim)
    frames = round(2.5 * 10)
    n0 = substeps_for(1.5, 0.1, 10.0, 2.0)[0]   # first frame: max_u starts at 2
    n = substeps_for(1.5, 0.1, 10.0, 7.0)[0]
    assert s.frames == frames and s.substeps == n0 + (frames - 1) * n
    # statistics on the last substep of every frame only
    flags = [w for _, w in sim.calls]
    assert flags.count(True) == frames
    assert flags[n0 - 1] and all(flags[n0 + i * n + n - 1] for i in range(frames - 1))
    # the window starts at max(preroll, 0.4 * total) = 1.0 s
    assert s.avg_from == 1.0
    assert 15 <= s.frames_averaged <= 16
    assert abs(s.hrr_w - 1000.0) < 1e-6 and abs(s.rad_fraction - 0.3) < 1e-9
    assert abs(s.burning_rate_kg_m2s - 0.05) < 1e-9
    # cumulative heights: 10 %, 40 %, 100 % at layers 2, 5, 9
    assert abs(s.h50_m - 1.0) < 1e-9 and abs(s.h90_m - 1.0) < 1e-9
    assert abs(height_at(np.array([0, 0, 100, 0, 0, 300, 0, 0, 0, 600.0]), 0.4, 0.1) - 0.6) < 1e-12
    assert len(s.heskestad_m) == 1
    assert abs(s.heskestad_m[0] - (0.235 * 1.0 ** 0.4 - 1.02 * 0.5)) < 1e-9


def test_slice_image_and_png(tmp_path):
    nz, ny, nx = 4, 6, 5
    s0 = np.zeros((nz, ny, nx, 4), np.float32)
    s1 = np.zeros((nz, ny, nx, 4), np.float32)
    s0[..., 0] = 2000.0          # hot -> white in panel 0
    s0[..., 2] = 0.233
    img = slice_image(s0, s1)
    assert img.shape == (ny, 5 * nx + 8, 3)
    assert np.all(img[:, :nx] == 255)            # T panel saturated
    assert np.all(img[:, 2 * (nx + 2):2 * (nx + 2) + nx] == 255)  # Y_O2 = 1
    p = os.path.join(tmp_path, "s.png")
    write_png(p, img)
    data = open(p, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    w, h = struct.unpack(">II", data[16:24])
    assert (w, h) == (5 * nx + 8, ny)
    idat = data[data.index(b"IDAT") + 4:data.index(b"IEND") - 8]
    raw = zlib.decompress(idat)
    assert len(raw) == ny * (1 + 3 * w)


def test_rendered_frames_follow_the_reference_rule():
    """src/main.rs:122-128, 158-161: every frame once the preroll has passed;
    with a still at t, a run of t + half a frame and only its last frame."""
    sc = Scene.from_toml_str(SCENE)
    sim = FakeSim([16, 32, 16], 0.1, umax=7.0)
    seen, times = [], []

    def rec(f):
        seen.append(f)
        times.append(float(sim.time))

    s = run_frames(sc, sim, on_render=rec)
    assert seen == list(range(seen[0], s.frames)) and min(times) >= 0.5 - 1e-4
    assert seen[0] == 4  # t = 0.5 s after the fifth frame (fps 10)
    sim = FakeSim([16, 32, 16], 0.1, umax=7.0)
    seen.clear()
    s = run_frames(sc, sim, still=1.2, on_render=seen.append)
    # f32: 1.2 + 0.05 = 1.25, x 10 = 12.5, rounded half away from zero
    assert s.frames == 13 and seen == [s.frames - 1]
