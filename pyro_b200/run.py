"""The frame loop of the reference (src/main.rs:56-279).

    python -m pyro_b200.run scene.toml [--sim-only] [--duration S] [--cell M]
                                       [--preroll S] [--out DIR] [--slice] [--quiet]
                                       [--spp N] [--res WxH] [--ev EV] [--still T]

Per output frame: CFL substep count n = ceil(frame_dt / (cfl*dx/max(u,1))),
n substeps with statistics on the last, one statistics read (the frame's
only device synchronisation), time averages over t >= max(preroll,
0.4*total), then the summary: HRR, radiative fraction, pyrolysis rate,
burning area and rate per area, 50/90/99 % cumulative heat-release heights
and the Heskestad height for pools.  `--slice` writes the 5-panel mid-z
image (T, Y_F, Y_O2, soot volume fraction, heat release) of src/main.rs:
201-239 as a PNG.  Without --sim-only every frame from the end of the preroll
on (or one still with --still T) is rendered by the GPU path tracer
(pyro_b200.render), developed (pyro_b200.post) and written as a PNG, with
--spp, --res WxH and --ev as in the reference CLI.

`run_frames` works on any object with the Sim interface (step, read_stats,
time, dx, dims), so the host logic is tested without a GPU.
"""
from __future__ import annotations

import argparse
import math
import os
import struct
import sys
import time
import zlib
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

F = np.float32


@dataclass
class Summary:
    """Time averages of the --sim-only run (src/main.rs:240-279)."""
    frames_averaged: int = 0
    avg_from: float = 0.0
    hrr_w: float = 0.0
    rad_fraction: float = 0.0
    pyro_kg_s: float = 0.0
    area_m2: float = 0.0
    burning_rate_kg_m2s: float = 0.0
    h50_m: float = 0.0
    h90_m: float = 0.0
    h99_m: float = 0.0
    heskestad_m: List[float] = field(default_factory=list)
    substeps: int = 0
    frames: int = 0
    wall_s: float = 0.0


def substeps_for(cfl: float, dx: float, fps: float, max_u: float):
    """src/main.rs:140-142 in f32: (n, dt)."""
    frame_dt = F(1.0) / F(fps)
    dt_cfl = F(cfl) * F(dx) / F(max(max_u, 1.0))
    n = max(int(math.ceil(float(F(frame_dt / dt_cfl)))), 1)
    return n, F(frame_dt / F(n))


def height_at(layers_avg: np.ndarray, frac: float, dx: float) -> float:
    """First layer where the cumulative HRR reaches frac of the total
    (src/main.rs:244-253)."""
    tot = float(np.sum(layers_avg))
    acc = 0.0
    for j, v in enumerate(layers_avg):
        acc += float(v)
        if acc >= frac * tot:
            return (j + 1.0) * dx
    return 0.0


def run_frames(scene, sim, duration: Optional[float] = None, preroll: Optional[float] = None,
               on_frame: Optional[Callable] = None, quiet: bool = True,
               still: Optional[float] = None,
               on_render: Optional[Callable[[int], None]] = None) -> Summary:
    """The frame loop (src/main.rs:121-197) on `sim`.  `on_render(f)` is
    called for the frames the reference renders: every frame from the end
    of the preroll on, or with `still` = t only the last frame of a run of
    t + half a frame."""
    fps = scene.sim.fps
    frame_dt = F(1.0) / F(fps)
    # f32 as in src/main.rs:121-130; f32::round rounds halves away from zero
    pre = F(scene.output.preroll if preroll is None else preroll)
    dur = F(scene.sim.duration if duration is None else duration)
    total = F(pre + dur)
    if still is not None:
        pre, total = F(still), F(F(still) + frame_dt * F(0.5))
    frames = int(math.floor(float(F(total * F(fps))) + 0.5))
    max_u = 2.0
    avg_from = float(max(pre, F(F(0.4) * total)))
    render_from = float(F(pre - F(1e-4)))
    n_avg = 0
    hrr = rad = pyro = area = 0.0
    ny = sim.dims[1]
    layers = np.zeros(ny, np.float64)
    t_start = time.time()
    sub = 0
    for f in range(frames):
        n, dt = substeps_for(scene.sim.cfl, sim.dx, fps, max_u)
        for s in range(n):
            sim.step(dt, s == n - 1)
        sub += n
        st = sim.read_stats()
        max_u = max(st.max_u, 1.0)
        if float(sim.time) >= avg_from:
            n_avg += 1
            hrr += st.hrr
            rad += st.rad
            pyro += st.pyro
            area += st.area
            lay = np.asarray(st.layers, np.float64)
            layers[:len(lay)] += lay
        if on_frame is not None:
            on_frame(f, n, st)
        rendering = (f == frames - 1) if still is not None else float(sim.time) >= render_from
        if on_render is not None and rendering:
            on_render(f)
        if not quiet:
            print(f"t={float(sim.time):5.2f}s substeps {n:2d} HRR {st.hrr / 1e3:7.1f} kW "
                  f"rad {100.0 * st.rad / st.hrr if st.hrr > 0 else 0.0:4.0f}% "
                  f"pyro {st.pyro:6.3f} kg/s Tmax {st.max_t:4.0f} K umax {st.max_u:4.1f} "
                  f"flame {st.flame_height(sim.dx):4.2f} m soot {st.soot * 1e3:5.1f} g "
                  f"fuel {st.solid:.1f} kg resid {st.resid:.0e}  [{time.time() - t_start:.0f}s]")
    out = Summary(frames_averaged=n_avg, avg_from=avg_from, substeps=sub, frames=frames,
                  wall_s=time.time() - t_start)
    if n_avg > 0:
        nn = float(n_avg)
        out.hrr_w = hrr / nn
        out.rad_fraction = rad / max(hrr, 1.0)
        out.pyro_kg_s = pyro / nn
        out.area_m2 = area / nn
        out.burning_rate_kg_m2s = pyro / max(area, 1e-9)
        out.h50_m = height_at(layers, 0.5, sim.dx)
        out.h90_m = height_at(layers, 0.9, sim.dx)
        out.h99_m = height_at(layers, 0.99, sim.dx)
        for o in scene.objects:
            if o.kind == "pool":
                d = 2.0 * o.radius
                out.heskestad_m.append(0.235 * (out.hrr_w / 1e3) ** 0.4 - 1.02 * d)
    return out


def slice_image(s0: np.ndarray, s1: np.ndarray) -> np.ndarray:
    """5 panels side by side of the mid-z plane (src/main.rs:201-234):
    T 300-2000 K, Y_F 0-0.3, Y_O2 0-0.233, soot f_v 0-3 ppm, q 0-5 MW/m^3;
    returns (ny, 5*nx+8, 3) uint8."""
    nz, ny, nx = s0.shape[:3]
    k = nz // 2
    a = s0[k].astype(np.float32)   # (ny, nx, 4)
    b = s1[k].astype(np.float32)
    rho = F(1.204) * F(293.0) / np.maximum(a[..., 0], F(200.0))
    vals = [(a[..., 0] - F(300.0)) / F(1700.0), a[..., 1] / F(0.3), a[..., 2] / F(0.233),
            rho * a[..., 3] / F(1800.0) * F(1e6) / F(3.0), b[..., 1] / F(5e6)]
    pw = nx * 5 + 8
    img = np.zeros((ny, pw, 3), np.uint8)
    for pi, v in enumerate(vals):
        v = np.clip(v, 0.0, 1.0)
        col = np.stack([np.minimum(v * 3.0, 1.0), np.clip(v * 3.0 - 1.0, 0.0, 1.0),
                        np.clip(v * 3.0 - 2.0, 0.0, 1.0)], -1)
        x0 = pi * (nx + 2)
        img[:, x0:x0 + nx] = (col * 255.0).astype(np.uint8)[::-1]   # y up
    return img


def write_png(path: str, img: np.ndarray) -> None:
    """Minimal RGB8 PNG writer (zlib, no filter)."""
    h, w = img.shape[:2]
    raw = b"".join(b"\x00" + img[y].tobytes() for y in range(h))

    def chunk(tag, data):
        c = struct.pack(">I", len(data)) + tag + data
        return c + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    png = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0))
    png += chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b"")
    with open(path, "wb") as fh:
        fh.write(png)


def print_summary(scene, s: Summary) -> None:
    print(f"--- averages (t >= {s.avg_from:.1f} s, {s.frames_averaged} frames) ---")
    print(f"HRR {s.hrr_w / 1e3:.0f} kW  radiative fraction {s.rad_fraction:.2f}  "
          f"pyrolysis {s.pyro_kg_s:.4f} kg/s  burning area {s.area_m2:.3f} m^2  -> per area "
          f"{s.burning_rate_kg_m2s:.4f} kg/m^2s")
    print(f"cumulative heat release 50% height {s.h50_m:.2f} m  90% {s.h90_m:.2f} m  "
          f"99% {s.h99_m:.2f} m")
    for o, l in zip([o for o in scene.objects if o.kind == "pool"], s.heskestad_m):
        d = 2.0 * o.radius
        print(f"Heskestad mean flame height (from the simulated HRR) {l:.2f} m, "
              f"puffing frequency {1.5 / math.sqrt(d):.2f} Hz")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="pyro_b200.run", description=__doc__.split("\n")[0])
    ap.add_argument("scene")
    ap.add_argument("--sim-only", action="store_true", help="simulate and print statistics only")
    ap.add_argument("--duration", type=float)
    ap.add_argument("--cell", type=float)
    ap.add_argument("--preroll", type=float)
    ap.add_argument("--out")
    ap.add_argument("--slice", action="store_true")
    ap.add_argument("--quiet", action="store_true")
    ap.add_argument("--spp", type=int, help="samples per pixel")
    ap.add_argument("--res", help="image size, e.g. 1920x1080")
    ap.add_argument("--ev", type=float, help="exposure compensation (EV)")
    ap.add_argument("--still", type=float, help="render one still at t seconds")
    a = ap.parse_args(argv)
    from .scene import Scene
    from .sim import Sim
    sc = Scene.load(a.scene)
    if a.duration is not None:
        sc.sim.duration = a.duration
    if a.cell is not None:
        sc.domain.cell = a.cell
    if a.preroll is not None:
        sc.output.preroll = a.preroll
    if a.spp is not None:
        sc.render.spp = a.spp
    if a.res:
        v = [int(x) for x in a.res.split("x") if x.isdigit()]
        if len(v) == 2:
            sc.render.width, sc.render.height = v
    if a.ev is not None:
        sc.render.exposure = a.ev
    g = sc.grid()
    print(f"grid {g.dims[0]}x{g.dims[1]}x{g.dims[2]} ({np.prod(g.dims) / 1e6:.1f} M cells, "
          f"{g.dx * 100:.1f} cm)")
    sim = Sim(sc)
    out_dir = a.out or os.path.join(os.path.dirname(os.path.abspath(a.scene)), sc.output.dir)
    on_render = None
    if not a.sim_only:  # src/main.rs:100-104, 113-119, 180-197
        from .develop import Developer
        from .post import Camera
        from .render import Renderer
        os.makedirs(out_dir, exist_ok=True)
        rend = Renderer(sc, sim)
        dev = Developer(rend.w, rend.h)
        cam = Camera(sc.render.auto_exposure, sc.render.exposure, sc.render.glare)
        frame_dt = float(F(1.0) / F(sc.sim.fps))
        idx = [0]

        def on_render(f):
            # trace and develop on the GPU; one 8-bit image comes back
            rend.render_device(sim, f, sc.render.spp)
            rgb8 = dev.develop(cam, rend.accum.data_ptr(), frame_dt, sim.stream())
            name = (f"still_{float(sim.time):.1f}s.png" if a.still is not None
                    else f"frame_{idx[0]:05d}.png")
            path = os.path.join(out_dir, name)
            write_png(path, rgb8)
            idx[0] += 1
            if not a.quiet:
                print(f"  rendered {path}")
    s = run_frames(sc, sim, quiet=a.quiet, still=a.still, on_render=on_render)
    if a.slice:
        os.makedirs(out_dir, exist_ok=True)
        s0, s1 = sim.read_scalars()
        p = os.path.join(out_dir, "slice.png")
        write_png(p, slice_image(s0, s1))
        print(f"slice: {p}")
    if s.frames_averaged > 0:
        print_summary(sc, s)
    sim.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
