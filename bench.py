"""Benchmark of the fire-simulation step (one substep = Sim::step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload pool_2cm|pool_small_8cm|pallets_5cm|bonfire_10cm|
                                pool_2cm_exact]
                    [--solver vcycle|mgpcg|mgpcg_bf16] [--tol T]

Workload (default): the 1 m n-heptane pool fire on a 2 cm grid,
160 x 320 x 160 = 8.19 M cells (x, y up, z; scene file
pyro_b200/scenes/pool_2cm.toml, synthetic: random-free scene geometry, no
dataset).  Before
timing, the scene is simulated for --preroll-s seconds (default 1.0 s) so the
flame and plume are developed; then W warm-up substeps; then exactly K timed
substeps with dt from the CFL rule of the reference frame loop
(src/main.rs:140-145, 30 frames/s) and statistics on the last substep of
every frame.  The working set (~1.9 GB) is far larger than the 126 MB L2, so
no flush is needed between steps.

One JSON line on stdout (rank 0).  `value` is device time per substep (ms,
lower is better) from CUDA events on the simulation's stream, max over
ranks.  `e2e` is the same metric through the public Python API (Sim.step
every substep, each substep's statistics read on the host while the next
one runs with Sim.read_stats_prev: the 576-byte parameter block goes host
-> device and the 4160-byte statistics block device -> host each substep).
`roofline` is the dominant single kernel's algorithmic bytes per launch over
its CUDA-event duration, against the measured HBM copy bandwidth.
`cpu_baseline` is the CPU oracle (a C++ restatement of the reference's
kernels) on the host cores, timed on rank 0 over whole substeps of the same
state.

--impl reference times that CPU restatement alone (the reference itself is
Rust + wgpu, with no Rust toolchain or graphics stack on the box): each step
is one full substep of the same workload on all host cores.

Multi-GPU (torchrun, one process per GPU): replicas only -- each rank steps
its own copy of the scene; `value` is max over ranks and `throughput` sums
cells*substeps/s over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import faulthandler
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

faulthandler.enable()
METRIC = "2cm pool-fire ms/step"
UNIT = "ms/step"
# Scene files with the reference's grid rule (every dimension a multiple of
# 16): the reference V-cycle needs dimensions that halve evenly at every
# level, and diverges on odd coarse dimensions (e.g. 150 x 365 x 150).
WORKLOADS = {
    "pool_2cm": "pool_2cm.toml",              # 160 x 320 x 160 = 8.19 M cells
    "pool_small_8cm": "pool_small_8cm.toml",  # 32 x 80 x 32
    "pallets_5cm": "pallets_5cm.toml",        # 128 x 240 x 128
    "bonfire_10cm": "bonfire_10cm.toml",      # 160 x 240 x 160
    # the 2 cm pool at the exact 3.0 x 7.3 x 3.0 m shape, 150 x 365 x 150 =
    # 8.21 M cells (no rounding): CG pressure solves only
    "pool_2cm_exact": "pool_2cm_exact.toml",
}
EXACT_DIMS = {"pool_2cm_exact": [150, 365, 150]}
SOLVERS = {"vcycle": 0, "mgpcg": 2, "mgpcg_bf16": 3}
# Algorithmic bytes per cell per launch (each distinct array element read or
# written once at the reference's width; read-modify-write twice).
ALG_BYTES = {"solid": 68, "curl": 28, "adv_vel1": 24, "adv_vel2": 40, "adv_s1": 76,
             "adv_s2": 108, "react": 116, "forces": 76, "divergence": 36, "project": 32}
# the renderer's input pack per cell: s0, s1, sol (16 each), flags (4) and the
# cell's three faces (4 each) in, three binary16 volumes (8 each) out; the
# bricks read two of those volumes once
RENDER_PACK_BYTES = 16 * 3 + 4 + 12 + 24
RENDER_BRICKS_BYTES = 16
MG_LEVEL_BYTES = 122.5   # 4 sweeps (96) + restrict (13.5) + prolong (13) per level cell
COARSE_SWEEP_BYTES = 24.0


def mg_cycle_bytes(dims_list):
    n0 = dims_list[0][0] * dims_list[0][1] * dims_list[0][2]
    b = 0.0
    for d in dims_list[:-1]:
        b += MG_LEVEL_BYTES * d[0] * d[1] * d[2]
    dc = dims_list[-1]
    b += 80 * COARSE_SWEEP_BYTES * dc[0] * dc[1] * dc[2]
    return b, n0


def mg_class_bytes(dims_list, cycles):
    """Algorithmic bytes of each V-cycle launch class over one pressure
    solve of `cycles` V-cycles (the classes of pyro_sim_profile_pressure):
    12 B per level cell per colour pass, 13.5 per restriction and 13 per
    prolongation (per fine cell), 80 sweeps of 24 B on the coarsest level;
    the preparation reads each level's u32 flags and writes its mask byte,
    and per coarse level reads the fine flags and writes the coarse ones."""
    n = [d[0] * d[1] * d[2] for d in dims_list]
    L = len(n)
    out = {"mg_prepare": sum(5.0 * m for m in n) + sum(4.0 * n[l - 1] + 4.0 * n[l]
                                                     for l in range(1, L)),
           "mg_pass_l0": cycles * 8 * 12.0 * n[0],
           "mg_restrict_l0": cycles * 13.5 * n[0] if L > 1 else 0.0,
           "mg_prolong_l0": cycles * 13.0 * n[0] if L > 1 else 0.0,
           "mg_pass_mid": cycles * sum(8 * 12.0 * n[l] for l in range(1, L - 1)),
           "mg_restrict_mid": cycles * sum(13.5 * n[l] for l in range(1, L - 1)),
           "mg_prolong_mid": cycles * sum(13.0 * n[l] for l in range(1, L - 1)),
           "mg_coarse": cycles * 80 * COARSE_SWEEP_BYTES * n[-1]}
    return out


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_tensor_peak():
    """Dense BF16 TFLOP/s for a kernel timed on its own (burst figure)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def net_roofline(net, bd, fd, dims, h, reps=5):
    """The learned stage's network forward on this pressure system, timed
    alone with CUDA events, as tensor-core throughput (the FLOPs of its nine
    3x3x3 convolutions per voxel, pyro_b200.learned.flops_per_voxel) against
    the measured dense BF16 peak."""
    import torch
    from pyro_b200.learned import flops_per_voxel
    phi = torch.empty_like(bd)
    s = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        net.forward(bd.data_ptr(), fd.data_ptr(), dims, 1, h, phi.data_ptr(), stream=s)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.forward(bd.data_ptr(), fd.data_ptr(), dims, 1, h, phi.data_ptr(), stream=s)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    vox = dims[0] * dims[1] * dims[2]
    tf = flops_per_voxel() * vox / (ms * 1e-3) / 1e12
    peak, kind = load_tensor_peak()
    return {"bound": "tensor", "forward_ms": round(ms, 3), "achieved": tf, "peak": peak,
            "peak_kind": kind, "unit": "TFLOP/s", "frac": tf / peak,
            "flops_per_voxel": flops_per_voxel(), "voxels": vox}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed
    region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                  "--format=csv,noheader,nounits", "-lms", "100"],
                                 stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return
        try:
            while not self._stop.is_set():
                line = p.stdout.readline()
                if not line:
                    break
                self.samples.append([x.strip() for x in line.split(",")])
        finally:
            p.terminate()
            try:
                p.wait(timeout=2)
            except Exception:
                p.kill()

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=3)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[0]))
                mx = float(s[1])
                for n, v in zip(names, s[3:7]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(name):
    from pyro_b200.scene import Scene
    sc = Scene.load(os.path.join(ROOT, "pyro_b200", "scenes", WORKLOADS[name]))
    if name in EXACT_DIMS:
        sc.dims_override = list(EXACT_DIMS[name])
    return sc


def solver_for(args):
    """The pressure solver of the run: --solver, else the reference's fixed
    V-cycles, except on shapes whose levels do not halve evenly (CG)."""
    if args.solver:
        return args.solver
    return "mgpcg_bf16" if args.workload in EXACT_DIMS else "vcycle"


def cfl_substeps(sc, max_u):
    """src/main.rs:140-142."""
    frame_dt = np.float32(1.0) / np.float32(sc.sim.fps)
    dt_cfl = np.float32(sc.sim.cfl) * np.float32(sc.domain.cell) / np.float32(max(max_u, 1.0))
    n = max(int(math.ceil(float(frame_dt / dt_cfl))), 1)
    return n, np.float32(frame_dt / np.float32(n))


def cpu_baseline_run(sc, P, sol, fields, n_steps, dt, t0, threads=None):
    """Time whole oracle substeps of the given state; returns (ms/step, cores)."""
    import oracle
    if threads:
        oracle.set_threads(threads)
    cores = oracle.max_threads()
    o = oracle.OracleSim(P, sol, sc.sim.pressure_cycles)
    for f, a in fields.items():
        o.write_field(f, a)
    t = np.float32(t0)
    times = []
    for k in range(n_steps):
        s = time.perf_counter()
        o.step(float(dt), float(t), 1.0, k == n_steps - 1)
        times.append(time.perf_counter() - s)
        t = np.float32(t + dt)
    o.close()
    return 1e3 * float(np.mean(times)), cores


def max_over_ranks(values, device):
    """The slowest rank's figures: an all-reduce MAX of `values` over the
    process group when one is running with more than one rank (the timing
    rule for N replicas), else the values themselves."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


TIMED_SUBSTEPS_PER_FRAME = 6


def timed_substeps(sc):
    """Substeps per 1/fps frame and their dt in the timed region of both
    arms: 6, the frame loop's CFL count for the developed 2 cm pool
    (src/main.rs:140-142 at max |u| ~ 6 m/s), so the two arms time the same
    substep."""
    n = TIMED_SUBSTEPS_PER_FRAME
    return n, np.float32(np.float32(1.0) / np.float32(sc.sim.fps) / np.float32(n))


def bench_config(args, dims, cycles, levels, solver, n, dt):
    """The `config` object of both arms' lines."""
    return {"workload": f"{args.workload} {dims[0]}x{dims[1]}x{dims[2]} (x,y-up,z)",
            "cells": int(dims[0] * dims[1] * dims[2]), "substeps_per_frame": n,
            "dt": float(dt),
            "pressure": (f"{cycles} V-cycles, {levels} levels" if solver == "vcycle" else
                         f"{solver} to {args.tol:g}"),
            "l2": "working set 1.9 GB > L2, no flush",
            "parallelism": f"replicas x{args.gpus}"}


def run_reference(args):
    """CPU restatement of the reference step on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    from pyro_b200.scene import shapes_array
    sc = build_workload(args.workload)
    P = sc.params()
    g = sc.grid()
    sh = sc.shapes()
    dens, kind = sc.slot_tables()
    sol = oracle.voxelize(shapes_array(sh), len(sh), g.dims[0], g.dims[1], g.dims[2], g.dx,
                          float(np.float32(sc.sim.ambient_temp)), sc.sim.seed, dens, kind)
    n, dt = timed_substeps(sc)
    cores = oracle.max_threads()
    o = oracle.OracleSim(P, sol, sc.sim.pressure_cycles)
    t = np.float32(0.0)
    for k in range(args.warmup):
        o.step(float(dt), float(t), 1.0, False)
        t = np.float32(t + dt)
    times = []
    for k in range(args.steps):
        s = time.perf_counter()
        o.step(float(dt), float(t), 1.0, (k % n) == n - 1)
        times.append(time.perf_counter() - s)
        t = np.float32(t + dt)
    ms = 1e3 * float(np.mean(times))
    cells = g.dims[0] * g.dims[1] * g.dims[2]
    line = {
        "impl": "reference", "metric": METRIC, "value": ms, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": bench_config(args, g.dims, sc.sim.pressure_cycles,
                               len(oracle.mg_levels(*g.dims)), "vcycle", n, dt),
        "state": "from ignition (the oracle's cost per substep hardly depends on the state)",
        "cpu_baseline": {"value": ms, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} full substeps of the workload from ignition "
                                   "(C++ oracle restating the reference's WGSL kernels, OpenMP)"},
        "e2e": {"value": ms, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "throughput": {"value": cells / (ms * 1e-3), "unit": "cells*substeps/s"},
    }
    print(json.dumps(line), flush=True)
    return 0


def log(msg):
    sys.stderr.write(f"[bench {time.strftime('%H:%M:%S')}] {msg}\n")
    sys.stderr.flush()


def load_traffic():
    """Per-launch DRAM bytes (read + write) of kernels captured with ncu,
    from the committed summary profiles/ncu_traffic.json ({} if absent)."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles",
                        "ncu_traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _learned_net():
    from pyro_b200.learned import Net
    w = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pyro_b200", "weights",
                     "warmstart.pnet")
    return Net.load(w) if os.path.exists(w) else None


def solve_runs(ps, bd, runs, net=None):
    """Each (name, mode, tol, cap) solved twice from phi = 0 into the same
    array, as a simulation calls it; the second solve's device time (CUDA
    events inside the solver) is reported.  The first allocates lazily and
    captures the CG modes' iteration graph for that array."""
    import torch
    from pyro_b200 import _abi
    res = {}
    phi = torch.zeros_like(bd)
    for name, mode, tol, cap in runs:
        if mode == _abi.SOLVER_MGPCG_LEARNED and net is None:
            continue
        best = None
        for rep in range(2):
            phi.zero_()
            torch.cuda.synchronize()
            best = ps.solve(bd.data_ptr(), phi.data_ptr(), mode, tol, cap, allow_cap=True)
        r = {"ms": round(best.ms, 3), "iterations": best.iterations,
             "rel_resid": best.rel_resid, "converged": bool(best.converged)}
        if mode == _abi.SOLVER_MGPCG_LEARNED:
            r.update(learned=best.learned, learned_ms=round(best.learned_ms, 3),
                     rel_resid_after_learned=best.rel_resid_learned)
        res[name] = r
    return res


def metric_runs():
    from pyro_b200 import _abi
    return [("vcycle_fp32_to_1e-3", _abi.SOLVER_VCYCLE_TOL, 1e-3, 60),
            ("mgpcg_fp32_to_1e-3", _abi.SOLVER_MGPCG, 1e-3, 200),
            ("mgpcg_fp32_to_1e-4", _abi.SOLVER_MGPCG, 1e-4, 200),
            ("mgpcg_bf16_to_1e-4", _abi.SOLVER_MGPCG_BF16, 1e-4, 200),
            ("mgpcg_bf16_learned_to_1e-4", _abi.SOLVER_MGPCG_LEARNED, 1e-4, 200)]


def render_frames(sc, sim, stream, spp=64, reps=2):
    """The path tracer's frame (pyro_b200.render.Renderer.render: input
    pack, emission tables, light caches and blur in light-cache mode, then
    the camera rays) on the developed state at the scene's render settings
    (1280 x 720, `spp` samples), in light-cache and pure path-tracing mode.
    Device time from CUDA events on the simulation's stream around each
    frame, after one untimed frame per mode; the image read-back at the end
    of a frame is included."""
    import torch
    from pyro_b200.render import Renderer
    out = {"width": int(sc.render.width), "height": int(sc.render.height), "spp": spp}
    for mode in ("cache", "path"):
        cfg = type(sc.render)(**{**sc.render.__dict__, "mode": mode})
        r = Renderer(sc, sim, cfg)
        r.render(sim, frame=0, spp=spp)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        times = []
        for k in range(reps):
            e0.record(stream)
            t0 = time.perf_counter()
            img = r.render(sim, frame=k + 1, spp=spp)
            wall = time.perf_counter() - t0
            e1.record(stream)
            e1.synchronize()
            times.append((e0.elapsed_time(e1), wall * 1e3))
        ms = min(t[0] for t in times)
        out[mode] = {"frame_ms": ms, "frame_wall_ms": min(t[1] for t in times),
                     "mean_radiance": float(np.mean(img)),
                     "pixel_samples_per_s": out["width"] * out["height"] * spp / (ms * 1e-3)}
        log(f"render {mode}: {ms:.1f} ms per {out['width']}x{out['height']} frame at {spp} spp")
        del r
    return out


def sim_solver_bench(sim):
    """The pressure system of the simulation's last substep (its b and
    flags; reference boundaries), solved from phi = 0 by each solver."""
    import torch
    from pyro_b200 import _abi
    from pyro_b200.poisson import PoissonSolver
    b = sim.read_field(_abi.F_B)
    f = sim.read_field(_abi.F_FLAGS)
    bd = torch.from_numpy(b).cuda()
    fd = torch.from_numpy(f.astype(np.int32)).cuda()
    ps = PoissonSolver(tuple(sim.dims), sim.dx, 0)
    ps.set_flags(fd.data_ptr())
    net = _learned_net()
    if net is not None:
        ps.set_net(net)
    res = solve_runs(ps, bd, metric_runs(), net)
    # where a BF16 CG iteration's time goes: the same iterations one launch
    # at a time, an event after each step (per iteration, event overhead
    # included)
    cg_classes = None
    b16 = res.get("mgpcg_bf16_to_1e-4")
    if b16:
        phi = torch.zeros_like(bd)
        torch.cuda.synchronize()  # the solver's stream does not wait for torch's
        k = max(int(b16["iterations"]), 1)
        prof = ps.profile_cg(bd.data_ptr(), phi.data_ptr(), _abi.SOLVER_MGPCG_BF16, k)
        cg_classes = {c: {"ms_per_iteration": round(v["ms"] / k, 4),
                          "steps_per_iteration": v["steps"] / k} for c, v in prof.items()}
        log("cg classes per iteration " + " ".join(
            f"{c}={v['ms_per_iteration']:.3f}" for c, v in cg_classes.items()))
    ps.set_net(None)
    ps.close()
    v, l = res.get("vcycle_fp32_to_1e-3"), res.get("mgpcg_bf16_learned_to_1e-4")
    out = {"config": f"the bench's last substep, {sim.dims[0]}x{sim.dims[1]}x{sim.dims[2]}, "
                     "phi0 = 0", "runs": res, "cg_classes_bf16": cg_classes}
    if net is not None:
        out["net_roofline"] = net_roofline(net, bd, fd, tuple(sim.dims), sim.dx)
    if v and l:
        out["speedup_learned_1e-4_vs_vcycle_1e-3"] = v["ms"] / l["ms"]
    b16 = res.get("mgpcg_bf16_to_1e-4")
    if v and b16:
        out["speedup_bf16_1e-4_vs_vcycle_1e-3"] = v["ms"] / b16["ms"]
    return out


def solver_bench(n=256, seed=1):
    """The pressure system in isolation: n^3 cells, h = 2 cm, ~5 % solid
    boxes, N(0,1) zero-mean rhs (pyro_b200.poisson.poisson_case).  Device
    time of each solve from CUDA events inside the solver, from phi = 0."""
    import torch
    from pyro_b200 import _abi
    from pyro_b200.poisson import PoissonSolver, poisson_case
    f, b = poisson_case(n, n, n, seed=seed)
    fd = torch.from_numpy(f).cuda()
    bd = torch.from_numpy(b).cuda()
    out = {"config": f"poisson {n}^3 h=0.02 solid={float(f.mean()):.3f} seed={seed}"}
    runs = metric_runs() + [("mgpcg_fp32_to_1e-6", _abi.SOLVER_MGPCG, 1e-6, 200),
                            ("mgpcg_bf16_to_1e-6", _abi.SOLVER_MGPCG_BF16, 1e-6, 200)]
    net = _learned_net()
    for bc in (0, 1):
        ps = PoissonSolver((n, n, n), 0.02, bc)
        ps.set_flags(fd.data_ptr())
        if net is not None:
            ps.set_net(net)
        res = solve_runs(ps, bd, runs, net)
        ps.set_net(None)
        ps.close()
        out["bc_reference" if bc == 0 else "bc_top_dirichlet"] = res
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    from pyro_b200 import _abi
    from pyro_b200.sim import Sim

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    sc = build_workload(args.workload)
    log(f"creating {args.workload} {sc.grid().dims}")
    sim = Sim(sc)
    cells = sim.cells()
    solver = solver_for(args)
    if solver != "vcycle":
        sim.set_solver(SOLVERS[solver], args.tol, 200)
    log(f"created; pressure solver {solver}")
    lib = _abi.load()
    stream = torch.cuda.ExternalStream(sim.stream())

    # preroll: develop the flame (frame loop of src/main.rs:139-147)
    max_u = 2.0
    t_pre = 0.0
    while t_pre < args.preroll_s:
        n, dt = cfl_substeps(sc, max_u)
        for s in range(n):
            sim.step(dt, s == n - 1)
        st = sim.read_stats()
        max_u = max(st.max_u, 1.0)
        t_pre += float(n * dt)
    log(f"preroll done t={t_pre:.3f}s max_u={max_u:.2f} (CFL substeps per frame "
        f"{cfl_substeps(sc, max_u)[0]})")
    n, dt = timed_substeps(sc)
    for k in range(args.warmup):
        sim.step(dt, (k % n) == n - 1)
    sim.sync()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- timed region: device-resident substeps
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(dev) as clocks:
        e0.record(stream)
        for k in range(args.steps):
            sim.step(dt, (k % n) == n - 1)
        e1.record(stream)
        e1.synchronize()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    log(f"timed {ms:.3f} ms/step")

    # ---- e2e through the public API: every substep uploads its parameters
    # and brings its statistics back to the host; the host reads substep
    # k - 1's statistics while substep k runs (Sim.read_stats_prev) and the
    # last substep's after the loop
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    barrier()
    e2.record(stream)
    for k in range(args.steps):
        sim.step(dt, True)
        if k:
            st = sim.read_stats_prev()
    st = sim.read_stats()
    e3.record(stream)
    e3.synchronize()
    barrier()
    ms_e2e = e2.elapsed_time(e3) / args.steps
    log(f"e2e {ms_e2e:.3f} ms/step")

    # ---- per-kernel device times (CUDA events around each launch)
    phases = np.zeros(12)
    nprof = max(3, min(args.steps, 10))
    buf = (np.zeros(12, np.float32))
    for k in range(nprof):
        rc = lib.pyro_sim_profile_step(sim._h, float(dt), float(sim.time), 0.0, 1 if k == 0 else 0,
                                       buf.ctypes.data_as(ctypes.c_void_p), 12)
        _abi.check("pyro_sim_profile_step", rc)
        sim.time = np.float32(sim.time + dt)
        phases += buf
    phases /= nprof
    log("profiled " + " ".join(f"{v:.3f}" for v in phases))
    names = _abi.PROFILE_PHASES
    kern = {names[i]: float(phases[i]) for i in range(12)}
    peak, peak_kind = load_peaks()
    info = sim.info()
    lvl = [tuple(info.level_dims[l]) for l in range(info.levels)]
    cyc_bytes, _ = mg_cycle_bytes(lvl)
    if solver == "vcycle":
        step_bytes = sum(ALG_BYTES.values()) * cells + sc.sim.pressure_cycles * cyc_bytes
    else:
        # per CG iteration one V-cycle of the preconditioner's hierarchy
        # (counted at FP32 width, the reference rule's levels) plus the
        # matrix-vector product and vector updates (about 48 B per cell)
        cg_it = max(sim.last_solve().iterations, 1)
        step_bytes = sum(ALG_BYTES.values()) * cells + cg_it * (cyc_bytes + 48.0 * cells)
    # the pressure solve per launch class, an event after every launch (the
    # fixed V-cycle schedule; the CG solver is timed as one phase)
    mg_ms = np.zeros(len(_abi.MG_CLASSES))
    mg_n = np.zeros(len(_abi.MG_CLASSES), np.int32)
    ms_buf = np.zeros(len(_abi.MG_CLASSES), np.float32)
    for k in range(nprof if solver == "vcycle" else 0):
        _abi.check("pyro_sim_profile_pressure", lib.pyro_sim_profile_pressure(
            sim._h, ms_buf.ctypes.data_as(ctypes.c_void_p), mg_n.ctypes.data_as(ctypes.c_void_p),
            len(_abi.MG_CLASSES)))
        mg_ms += ms_buf
    mg_ms /= nprof
    mg_bytes = mg_class_bytes(lvl, sc.sim.pressure_cycles)
    # every launch class of the substep: launches, device ms per substep and
    # per launch, algorithmic bytes per launch and the HBM fraction
    classes = {}
    for k in ALG_BYTES:
        classes[k] = {"launches": 1, "ms": kern[k], "alg_bytes": ALG_BYTES[k] * cells}
    if solver != "vcycle":
        classes["pressure_cg"] = {"launches": 1, "ms": kern["pressure"],
                                  "alg_bytes": step_bytes - sum(ALG_BYTES.values()) * cells}
    for i, k in enumerate(_abi.MG_CLASSES):
        if mg_n[i] > 0:
            classes[k] = {"launches": int(mg_n[i]), "ms": float(mg_ms[i]),
                          "alg_bytes": mg_bytes[k] / int(mg_n[i])}
    for k, c in classes.items():
        c["ms_per_launch"] = c["ms"] / c["launches"]
        c["gbs"] = c["alg_bytes"] / (c["ms_per_launch"] * 1e-3) / 1e9
        c["frac"] = c["gbs"] / peak
    log("pressure classes " + " ".join(f"{k}={c['ms']:.3f}" for k, c in classes.items()
                                       if k.startswith("mg_")))
    dom = max(classes, key=lambda k: classes[k]["ms"])
    dom_bytes = classes[dom]["alg_bytes"]
    achieved = classes[dom]["gbs"]
    traffic = load_traffic().get(dom, {}).get("dram_bytes_per_launch")

    # ---- the renderer's per-frame input pack (render.wgsl:3-61): the pack
    # alone, then pack + bricks; inputs (0.5 GB) exceed L2 between launches
    sim.render_pack(True)  # first call allocates the volumes
    sim.sync()
    reps = 20
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(stream)
    for _ in range(reps):
        _abi.check("pyro_sim_render_pack", lib.pyro_sim_render_pack(sim._h, 0))
    ev[1].record(stream)
    for _ in range(reps):
        _abi.check("pyro_sim_render_pack", lib.pyro_sim_render_pack(sim._h, 1))
    ev[2].record(stream)
    ev[2].synchronize()
    pack_ms = ev[0].elapsed_time(ev[1]) / reps
    bricks_ms = max(ev[1].elapsed_time(ev[2]) / reps - pack_ms, 1e-6)
    frame_pack = {
        "pack_ms": pack_ms, "bricks_ms": bricks_ms,
        "alg_bytes_per_cell": {"pack": RENDER_PACK_BYTES, "bricks": RENDER_BRICKS_BYTES},
        "pack_gbs": RENDER_PACK_BYTES * cells / (pack_ms * 1e-3) / 1e9,
        "bricks_gbs": RENDER_BRICKS_BYTES * cells / (bricks_ms * 1e-3) / 1e9,
    }
    frame_pack["pack_frac"] = frame_pack["pack_gbs"] / load_peaks()[0]
    # the fire-light sampling tables: ecells and the FP64 CDF scan
    from pyro_b200 import color
    lut_dev = torch.from_numpy(color.build_lut()).cuda()
    chemi = color.chemi_block()
    chp = chemi.ctypes.data_as(ctypes.c_void_p)
    _abi.check("pyro_sim_render_emission",
               lib.pyro_sim_render_emission(sim._h, ctypes.c_void_p(lut_dev.data_ptr()), chp))  # first call allocates
    sim.sync()
    ev[0].record(stream)
    for _ in range(reps):
        _abi.check("pyro_sim_render_emission", lib.pyro_sim_render_emission(
            sim._h, ctypes.c_void_p(lut_dev.data_ptr()), chp))
    ev[1].record(stream)
    ev[1].synchronize()
    frame_pack["emission_ms"] = ev[0].elapsed_time(ev[1]) / reps
    ecell = sim.read_field(_abi.F_ECELL)
    frame_pack["emitting_cells"] = int((ecell > 0).sum())
    log(f"render emission (ecells + CDF) {frame_pack['emission_ms']:.3f} ms, "
        f"{frame_pack['emitting_cells']} emitting cells")
    log(f"render pack {pack_ms:.3f} ms ({frame_pack['pack_gbs']:.0f} GB/s), "
        f"bricks {bricks_ms:.3f} ms")
    frame_render = None
    if not args.no_render:
        frame_render = render_frames(sc, sim, stream)

    # gather max over ranks
    ms, ms_e2e = max_over_ranks([ms, ms_e2e], "cuda")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from pyro_b200 import _abi as A
        fields = {A.F_S0: sim.read_field(A.F_S0), A.F_S1: sim.read_field(A.F_S1),
                  A.F_SOL: sim.read_field(A.F_SOL), A.F_U: sim.read_field(A.F_U),
                  A.F_V: sim.read_field(A.F_V), A.F_W: sim.read_field(A.F_W),
                  A.F_PHI: sim.read_field(A.F_PHI)}
        log("cpu baseline")
        for f, a in fields.items():
            bad = int(np.size(a) - np.isfinite(a).sum())
            if bad:
                log(f"field {f}: {bad} non-finite values")
        cms, cores = cpu_baseline_run(sc, sim.p, fields[A.F_SOL], fields, args.cpu_steps, dt,
                                      float(sim.time))
        # the reference forms the emission CDF on the CPU from a read-back
        # buffer (src/render.rs:316-333): its loop, timed here on the same
        # emission values (the copies to and from the device not included)
        import oracle
        t0_ = time.perf_counter()
        oracle.render_cdf(ecell)
        frame_pack["cdf_cpu_ms_reference_loop"] = (time.perf_counter() - t0_) * 1e3
        cpu = {"value": cms, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{args.cpu_steps} full substeps of the same developed state "
                         "(C++ oracle restating the reference's WGSL kernels, OpenMP)"}

    solver_runs = None
    if rank == 0 and not args.no_solver:
        log("solver bench")
        solver_runs = {"sim_pressure": sim_solver_bench(sim), "poisson_256": solver_bench()}
    # kernels per substep: 11 step kernels (solid, curl, adv_vel1/2, adv_s1/2,
    # react, confine, forces, divergence, project), the level preparation
    # (flags_down per coarse level, a mask per level) and per V-cycle 4 + 1 + 5
    # per non-coarsest level plus the coarsest solve; mg_resid on the
    # statistics substeps (checked against the ncu launch list)
    L = info.levels
    launches_per_step = 11 + (L - 1) + L + sc.sim.pressure_cycles * (10 * (L - 1) + 1)
    stats_steps = sum(1 for k in range(args.steps) if (k % n) == n - 1)
    line = {
        "metric": METRIC, "value": ms, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(args, sim.dims, sc.sim.pressure_cycles, info.levels, solver, n,
                               dt),
        "state": f"developed flame after a {args.preroll_s:g} s preroll of the frame loop",
        "ms_per_frame": ms * n,
        "cg_iterations_last_solve": (sim.last_solve().iterations if solver != "vcycle"
                                     else None),
        "e2e": {"value": ms_e2e, "unit": UNIT, "h2d_bytes_per_step": 576,
                "d2h_bytes_per_step": 4 * _abi.STATS_N},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "alg_bytes_per_launch": dom_bytes,
                     "launch_ms": classes[dom]["ms_per_launch"],
                     "launches_per_substep": classes[dom]["launches"]},
        "step_roofline": {"alg_bytes": step_bytes, "achieved_gbs": step_bytes / (ms * 1e-3) / 1e9,
                          "frac": step_bytes / (ms * 1e-3) / 1e9 / peak},
        "kernels_ms": kern,
        "kernel_classes": classes,
        "frame_pack": frame_pack,
        "frame_render": frame_render,
        "throughput": {"value": world * cells / (ms * 1e-3), "unit": "cells*substeps/s"},
        "cpu_baseline": cpu,
        "solver": solver_runs,
        "gpu_launches": launches_per_step * args.steps + stats_steps,
        "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pool_2cm", choices=sorted(WORKLOADS))
    ap.add_argument("--preroll-s", type=float, default=1.0)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-solver", action="store_true")
    ap.add_argument("--no-render", action="store_true")
    ap.add_argument("--solver", choices=sorted(SOLVERS), default=None,
                    help="pressure solver of the timed substeps (default: the reference's "
                         "fixed V-cycles; CG on shapes that do not halve evenly)")
    ap.add_argument("--tol", type=float, default=1e-4, help="CG relative residual")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
