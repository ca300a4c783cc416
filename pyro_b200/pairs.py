"""Training pairs for the learned pressure stage: (b, phi, flags) of the
level-0 pressure system, taken after the multigrid solve of a plain-solver
run (the reference's L0.b and L0.phi after `vcycles`, src/sim.rs:405) and
cut into cubic tiles.

    python -m pyro_b200.pairs SCENE.toml --out DIR [--pairs N] [--every K]
                              [--tile 128] [--tiles-per-pair 4] [--preroll S]

The simulation's own phi (4 V-cycles from the previous substep's pressure)
is refined by FP32 MGPCG to a relative residual of 1e-6 on the same system
(reference boundaries) so that the targets are converged pressures; both
residuals are recorded.  Files are .npz with b and phi as bfloat16 bits
(uint16, round to nearest even), the solid mask as uint8 and the metadata
(h, scene, time, substep, tile offset, residuals).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
from typing import Dict, Iterator, List, Optional

import numpy as np

from . import _abi


def bf16_bits(a: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 bits (uint16), round to nearest even."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def from_bf16_bits(u: np.ndarray) -> np.ndarray:
    return (np.asarray(u, np.uint16).astype(np.uint32) << 16).view(np.float32)


def collect(scene_path: str, n_pairs: int, every: int = 4, preroll: Optional[float] = None,
            cell: Optional[float] = None, refine_tol: float = 1e-6, refine_iters: int = 200,
            quiet: bool = True) -> Iterator[Dict]:
    """Run the scene with the plain solver and yield `n_pairs` full-domain
    pairs, one every `every` substeps once the time passes `preroll`
    (default: the scene's preroll).  Arrays are (nz, ny, nx) numpy."""
    import torch

    from .poisson import PoissonSolver
    from .run import substeps_for
    from .scene import Scene
    from .sim import Sim

    sc = Scene.load(scene_path)
    if cell is not None:
        sc.domain.cell = cell
    pre = sc.output.preroll if preroll is None else preroll
    name = os.path.splitext(os.path.basename(scene_path))[0]
    sim = Sim(sc)
    nx, ny, nz = sim.dims
    ps = PoissonSolver((nx, ny, nz), sim.dx, bc_mode=0)
    fps = sc.sim.fps
    max_u = 2.0
    sub = 0
    got = 0
    try:
        while got < n_pairs:
            n, dt = substeps_for(sc.sim.cfl, sim.dx, fps, max_u)
            for s in range(n):
                sim.step(dt, s == n - 1)
                sub += 1
                if float(sim.time) < pre or sub % every or got >= n_pairs:
                    continue
                sim.sync()
                b = sim.read_field(_abi.F_B)
                phi_sim = sim.read_field(_abi.F_PHI)
                flags = sim.read_field(_abi.F_FLAGS)
                fd = torch.from_numpy(flags.astype(np.int32)).cuda()
                bd = torch.from_numpy(b).cuda()
                pd = torch.from_numpy(phi_sim.copy()).cuda()
                torch.cuda.synchronize()
                ps.set_flags(fd.data_ptr())
                info = ps.solve(bd.data_ptr(), pd.data_ptr(), _abi.SOLVER_MGPCG, refine_tol,
                                refine_iters, allow_cap=True)
                torch.cuda.synchronize()
                phi = pd.cpu().numpy()
                got += 1
                if not quiet:
                    print(f"{name}: pair {got}/{n_pairs} t={float(sim.time):.2f}s substep {sub} "
                          f"sim resid {info.rel_resid_start:.2e} -> {info.rel_resid:.2e}",
                          flush=True)
                yield dict(b=b, phi=phi, flags=(flags == 1).astype(np.uint8), h=sim.dx,
                           scene=name, time=float(sim.time), substep=sub,
                           resid_sim=float(info.rel_resid_start), resid=float(info.rel_resid))
            st = sim.read_stats()
            max_u = max(st.max_u, 1.0)
    finally:
        ps.close()
        sim.close()


def tiles(pair: Dict, tile: int, count: int, rng: np.random.Generator) -> List[Dict]:
    """`count` random tile^3 crops of a full-domain pair (x and z offsets
    uniform, y offset uniform from the floor)."""
    nz, ny, nx = pair["b"].shape
    t = [min(tile, nz), min(tile, ny), min(tile, nx)]
    out = []
    for _ in range(count):
        o = [int(rng.integers(0, d - s + 1)) for d, s in zip((nz, ny, nx), t)]
        sl = tuple(slice(a, a + s) for a, s in zip(o, t))
        d = {k: v for k, v in pair.items() if not isinstance(v, np.ndarray)}
        d.update(b=pair["b"][sl].copy(), phi=pair["phi"][sl].copy(),
                 flags=pair["flags"][sl].copy(), offset=o)
        out.append(d)
    return out


def write_pair(path: str, d: Dict) -> None:
    meta = {k: v for k, v in d.items() if not isinstance(v, np.ndarray)}
    np.savez_compressed(path, b=bf16_bits(d["b"]), phi=bf16_bits(d["phi"]), flags=d["flags"],
                        meta=np.frombuffer(json.dumps(meta).encode(), np.uint8))


def read_pair(path: str) -> Dict:
    with np.load(path) as z:
        d = json.loads(bytes(z["meta"]).decode())
        d.update(b=from_bf16_bits(z["b"]), phi=from_bf16_bits(z["phi"]),
                 flags=z["flags"].astype(np.uint8))
    return d


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="pyro_b200.pairs", description=__doc__.split("\n")[0])
    ap.add_argument("scene")
    ap.add_argument("--out", required=True)
    ap.add_argument("--pairs", type=int, default=8)
    ap.add_argument("--every", type=int, default=4)
    ap.add_argument("--tile", type=int, default=128)
    ap.add_argument("--tiles-per-pair", type=int, default=4)
    ap.add_argument("--preroll", type=float)
    ap.add_argument("--cell", type=float)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    rng = np.random.default_rng(a.seed)
    k = 0
    for pair in collect(a.scene, a.pairs, a.every, a.preroll, a.cell, quiet=False):
        for t in tiles(pair, a.tile, a.tiles_per_pair, rng):
            write_pair(os.path.join(a.out, f"{t['scene']}_{k:05d}.npz"), t)
            k += 1
    print(f"{k} tiles written to {a.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
