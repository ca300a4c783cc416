"""Train the learned pressure stage on the GPU and measure what it gains.

    python -m pyro_b200.train_net --out warmstart.pnet [--scenes a.toml,b.toml]
        [--pairs 12] [--holdout 2] [--every 6] [--steps 1500] [--tile 128]
        [--batch 2] [--lr 2e-4] [--w-phi 0] [--w-res 1] [--json report.json]

Pairs come from plain-solver runs of the scenes (pyro_b200.pairs.collect),
stay in device memory, and the last `holdout` pairs of every scene are held
out.  Each step takes `batch` random tile^3 crops of one training pair,
flipped in x and z and transposed x<->z at random (the pressure system is
symmetric under those, not under y: gravity and the floor), and runs one
forward/backward/Adam step through the C ABI (cosine learning-rate decay).
The default loss is the normalised residual alone: a pressure MSE on crops
is dominated by far-field pressure the network cannot see (and by crops
whose rms(b) is tiny), which made training diverge.
The evaluation solves every held-out system to a relative residual of 1e-4
from a zero guess, with BF16 MGPCG and with the learned warm start, and
reports iterations and device time of both.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time
from typing import Dict, List

import numpy as np

from . import _abi
from .learned import Net

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_SCENES = [os.path.join(HERE, "scenes", s) for s in
                  ("pool_2cm.toml", "pallets_5cm.toml", "bonfire_10cm.toml")]
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "warmstart.pnet")


def to_device(pair: Dict) -> Dict:
    import torch
    d = {k: v for k, v in pair.items() if not isinstance(v, np.ndarray)}
    d.update(b=torch.from_numpy(np.ascontiguousarray(pair["b"], np.float32)).cuda(),
             phi=torch.from_numpy(np.ascontiguousarray(pair["phi"], np.float32)).cuda(),
             flags=torch.from_numpy(pair["flags"].astype(np.int32)).cuda())
    return d


def target_scale(pairs: List[Dict]) -> float:
    """Root mean square of phi / (rms(b) h^2) over the fluid cells: the
    network's output unit (out_scale)."""
    acc, n = 0.0, 0
    for p in pairs:
        fl = p["flags"] == 0
        b = p["b"][fl].astype(np.float64)
        s = math.sqrt(float((b * b).mean())) if b.size else 0.0
        if s <= 0:
            continue
        t = p["phi"][fl].astype(np.float64) / (s * p["h"] ** 2)
        acc += float((t * t).sum())
        n += t.size
    return math.sqrt(acc / n) if n else 1.0


def _crop(p: Dict, tile: int, rng, flips: bool):
    import torch
    nz, ny, nx = p["b"].shape
    o = [int(rng.integers(0, d - tile + 1)) for d in (nz, ny, nx)]
    sl = (slice(o[0], o[0] + tile), slice(o[1], o[1] + tile), slice(o[2], o[2] + tile))
    out = [p["b"][sl], p["phi"][sl], p["flags"][sl]]
    if flips:
        if rng.random() < 0.5:
            out = [torch.flip(t, (2,)) for t in out]
        if rng.random() < 0.5:
            out = [torch.flip(t, (0,)) for t in out]
        if rng.random() < 0.5:
            out = [t.permute(2, 1, 0) for t in out]
    return out


def train(net: Net, pairs: List[Dict], steps: int, tile: int = 128, batch: int = 2,
          lr: float = 1e-3, lr_min: float = 1e-5, clip: float = 1.0, seed: int = 0,
          log_every: int = 100, quiet: bool = False) -> Dict:
    import torch
    rng = np.random.default_rng(seed)
    for p in pairs:
        if min(p["b"].shape) < tile:
            raise ValueError(f"tile {tile} larger than a pair of shape {tuple(p['b'].shape)}")
    hist = []
    t0 = time.time()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for it in range(steps):
        p = pairs[int(rng.integers(len(pairs)))]
        crops = [_crop(p, tile, rng, True) for _ in range(batch)]
        b = torch.stack([c[0] for c in crops]).contiguous()
        phi = torch.stack([c[1] for c in crops]).contiguous()
        fl = torch.stack([c[2] for c in crops]).contiguous()
        a = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * it / max(steps, 1)))
        net.train_step(b.data_ptr(), fl.data_ptr(), phi.data_ptr(), (tile, tile, tile), batch,
                       p["h"], a, clip, stream=torch.cuda.current_stream().cuda_stream)
        if (it + 1) % log_every == 0 or it == steps - 1:
            loss = net.last_loss(stream=torch.cuda.current_stream().cuda_stream)
            hist.append((it + 1, loss))
            if not quiet:
                print(f"step {it + 1}/{steps} loss {loss:.4e} lr {a:.2e} "
                      f"[{time.time() - t0:.0f}s]", flush=True)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    return dict(steps=steps, tile=tile, batch=batch, lr=lr, history=hist,
                ms_per_step=ms / max(steps, 1), voxels_per_step=batch * tile ** 3)


def evaluate(net: Net, pairs: List[Dict], tol: float = 1e-4, max_iters: int = 100) -> List[Dict]:
    """Solve every pair's system from zero with BF16 MGPCG and with the
    learned warm start; the second of two identical solves is timed."""
    import torch

    from .poisson import PoissonSolver
    res = []
    solvers = {}
    for p in pairs:
        nz, ny, nx = p["b"].shape
        key = (nx, ny, nz, p["h"])
        if key not in solvers:
            solvers[key] = PoissonSolver((nx, ny, nz), p["h"], bc_mode=0)
            solvers[key].set_net(net)
        ps = solvers[key]
        ps.set_flags(p["flags"].data_ptr())
        phi = torch.zeros_like(p["b"])
        r = dict(scene=p.get("scene"), time=p.get("time"))
        for mode, tag in ((_abi.SOLVER_MGPCG_BF16, "mgpcg_bf16"),
                          (_abi.SOLVER_MGPCG_LEARNED, "mgpcg_bf16_learned")):
            for _ in range(2):
                phi.zero_()
                torch.cuda.synchronize()
                info = ps.solve(p["b"].data_ptr(), phi.data_ptr(), mode, tol, max_iters,
                                allow_cap=True)
            r[tag] = dict(iterations=info.iterations, ms=round(info.ms, 3),
                          rel_resid=info.rel_resid, converged=bool(info.converged))
            if mode == _abi.SOLVER_MGPCG_LEARNED:
                r[tag].update(learned=info.learned, learned_ms=round(info.learned_ms, 3),
                              rel_resid_after_learned=info.rel_resid_learned)
        res.append(r)
    for ps in solvers.values():
        ps.set_net(None)
        ps.close()
    return res


def main(argv=None) -> int:
    from .pairs import collect
    ap = argparse.ArgumentParser(prog="pyro_b200.train_net", description=__doc__.split("\n")[0])
    ap.add_argument("--scenes", default=",".join(DEFAULT_SCENES))
    ap.add_argument("--pairs", type=int, default=12, help="pairs per scene")
    ap.add_argument("--holdout", type=int, default=2, help="held-out pairs per scene")
    ap.add_argument("--every", type=int, default=6)
    ap.add_argument("--preroll", type=float)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--tile", type=int, default=128)
    ap.add_argument("--batch", type=int, default=2)
    ap.add_argument("--lr", type=float, default=2e-4)
    ap.add_argument("--clip", type=float, default=1.0)
    ap.add_argument("--w-phi", type=float, default=0.0, help="weight of the pressure MSE")
    ap.add_argument("--w-res", type=float, default=1.0, help="weight of the residual MSE")
    ap.add_argument("--out-scale", type=float,
                    help="output unit (default: rms of the scaled pressure when --w-phi > 0, "
                         "else 1)")
    ap.add_argument("--log-every", type=int, default=50)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--init", help="start from this weights file")
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--json")
    a = ap.parse_args(argv)
    t0 = time.time()
    tr, ho = [], []
    for sc in [s for s in a.scenes.split(",") if s]:
        got = list(collect(sc, a.pairs, a.every, a.preroll, quiet=False))
        tr += got[:len(got) - a.holdout]
        ho += got[len(got) - a.holdout:]
    print(f"{len(tr)} training and {len(ho)} held-out pairs [{time.time() - t0:.0f}s]",
          flush=True)
    scale = a.out_scale or (target_scale(tr) if a.w_phi > 0 else 1.0)
    net = Net.load(a.init) if a.init else Net(seed=a.seed)
    if not a.init:
        p, _ = net.get_params()
        net.set_params(p, scale)
    net.set_loss(a.w_phi, a.w_res)
    dtr = [to_device(p) for p in tr]
    dho = [to_device(p) for p in ho]
    rep = dict(out_scale=scale, w_phi=a.w_phi, w_res=a.w_res, train_pairs=len(tr),
               holdout_pairs=len(ho),
               pair_meta=[{k: v for k, v in p.items() if not isinstance(v, np.ndarray)}
                          for p in tr + ho])
    rep["before"] = evaluate(net, dho)
    for r in rep["before"]:
        print("before:", json.dumps(r), flush=True)
    rep["train"] = train(net, dtr, a.steps, a.tile, a.batch, a.lr, clip=a.clip, seed=a.seed,
                         log_every=a.log_every)
    rep["after"] = evaluate(net, dho)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    net.save(a.out)
    rep["weights"] = a.out
    rep["wall_s"] = time.time() - t0
    s = json.dumps(rep, indent=1)
    if a.json:
        with open(a.json, "w") as fh:
            fh.write(s)
    for r in rep["after"]:
        print("after:", json.dumps(r))
    return 0


if __name__ == "__main__":
    sys.exit(main())
