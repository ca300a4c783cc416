"""Flame statistics of one scene under two pressure solvers.

    python -m pyro_b200.solver_drift scene.toml [--cell M] [--preroll S]
        [--duration S] [--tol T] [--learned WEIGHTS] [--out FILE.json]

The scene runs twice through the reference frame loop (src/main.rs:121-157,
`pyro_b200.run.run_frames`) from the same voxelized start:

* `fp32_vcycle`: the reference's pressure solve, a fixed count of FP32
  V-cycles (src/sim.rs:451-491);
* `bf16_mgpcg`: flexible CG to the relative residual `--tol` (default 1e-4)
  with a V-cycle preconditioner that stores phi and b in BF16 (FP32
  arithmetic) and solves its coarsest level directly in FP64; dot products
  and norms are FP64.  With `--learned WEIGHTS` the CG starts from the
  learned warm start of that network (kept only when it cuts the
  residual), as the large-scene configuration asks.

Each run reports the reference's time-averaged summary (src/main.rs:240-268:
HRR, burning rate per area, 50/90/99 % cumulative heat-release heights) over
t >= max(preroll, 0.4 t_total), its wall time, and the second run's relative
drift from the first.  The two runs decorrelate like any two turbulent
runs, so only these windowed statistics are comparable.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

from . import _abi
from .run import run_frames
from .scene import Scene
from .sim import Sim

KEYS = ("hrr_w", "burning_rate_kg_m2s", "pyro_kg_s", "h50_m", "h90_m", "h99_m")


def run_mode(scene, mode, tol, preroll, duration, sol=None, max_iters=100, net=None):
    """One frame-loop run with pressure solver `mode`; returns (summary
    dict, the solid state it started from)."""
    sim = Sim(scene, sol)
    start = sim.read_field(_abi.F_SOL)
    if net is not None:
        sim.set_net(net)
    if mode != _abi.SOLVER_VCYCLE:
        sim.set_solver(mode, tol, max_iters)
    t0 = time.time()
    s = run_frames(scene, sim, duration=duration, preroll=preroll)
    sim.close()
    out = {k: float(getattr(s, k)) for k in KEYS}
    out.update(frames=s.frames, frames_averaged=s.frames_averaged, substeps=s.substeps,
               avg_from_s=s.avg_from, wall_s=time.time() - t0)
    return out, start


def compare(scene, preroll, duration, tol=1e-4, net=None):
    """Both runs and the drift of bf16_mgpcg from fp32_vcycle per statistic
    (`net`: the learned warm start for the CG run)."""
    ref, sol = run_mode(scene, _abi.SOLVER_VCYCLE, 0.0, preroll, duration)
    mode = _abi.SOLVER_MGPCG_LEARNED if net is not None else _abi.SOLVER_MGPCG_BF16
    mix, _ = run_mode(scene, mode, tol, preroll, duration, sol=sol, net=net)
    drift = {k: (mix[k] - ref[k]) / ref[k] if ref[k] != 0.0 else None for k in KEYS}
    g = scene.grid()
    return {"scene": {"dims": list(g.dims), "cell_m": float(g.dx), "preroll_s": preroll,
                      "duration_s": duration, "fps": scene.sim.fps},
            "tol": tol, "learned": net is not None, "fp32_vcycle": ref, "bf16_mgpcg": mix,
            "drift": drift}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="pyro_b200.solver_drift",
                                 description=__doc__.split("\n")[0])
    ap.add_argument("scene")
    ap.add_argument("--cell", type=float)
    ap.add_argument("--preroll", type=float)
    ap.add_argument("--duration", type=float)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--learned", metavar="WEIGHTS",
                    help="start each CG solve from this network's warm start")
    ap.add_argument("--out")
    a = ap.parse_args(argv)
    sc = Scene.load(a.scene)
    if a.cell:
        sc.domain.cell = a.cell
    pre = sc.output.preroll if a.preroll is None else a.preroll
    dur = sc.sim.duration if a.duration is None else a.duration
    net = None
    if a.learned:
        from .learned import Net
        net = Net.load(a.learned)
    res = compare(sc, pre, dur, a.tol, net)
    txt = json.dumps(res, indent=1)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(txt + "\n")
    print(txt)
    return 0


if __name__ == "__main__":
    sys.exit(main())
