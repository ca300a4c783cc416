"""The learned pressure stage over the C ABI (pyro_net_*).

    net = Net(seed=0)                     # or Net.load("warmstart.pnet")
    net.forward(b_ptr, flags_ptr, (nx, ny, nz), nb, h, phi_ptr)
    loss, grad = net.loss_grad(...)       # gradient check
    net.train_step(..., lr=1e-3)          # asynchronous; net.last_loss()
    ps.set_net(net); ps.solve(..., mode=SOLVER_MGPCG_LEARNED, ...)

Device pointers are plain ints (e.g. torch.Tensor.data_ptr()).  The
network has no counterpart in the reference; it stands beside the
multigrid solve of src/sim.rs:451-491, which remains the fallback.

Weights file (little endian): b"PYRONET1", u32 version (1), u32 count,
f32 out_scale, u32 reserved, then `count` f32 parameters (every layer's
weights [Cout][27][Cin], then every layer's biases).
"""
from __future__ import annotations

import ctypes
import os
import struct
from typing import Optional, Tuple

import numpy as np

from . import _abi

MAGIC = b"PYRONET1"
# (cin, cout, level, relu) of conv1 .. conv9, as in csrc/net.h
SPEC = [(2, 16, 0, 1), (16, 16, 0, 1), (16, 32, 1, 1), (32, 32, 1, 1), (32, 64, 2, 1),
        (64, 64, 2, 1), (96, 32, 1, 1), (48, 16, 0, 1), (16, 1, 0, 0)]


def _vp(p):
    return ctypes.c_void_p(int(p)) if p else None


class Net:
    def __init__(self, seed: int = 0):
        self._lib = _abi.load()
        h = ctypes.c_void_p()
        _abi.check("pyro_net_create", self._lib.pyro_net_create(seed, ctypes.byref(h)))
        self._h = h
        n = ctypes.c_uint64()
        _abi.check("pyro_net_param_count", self._lib.pyro_net_param_count(h, ctypes.byref(n)))
        self.n_params = int(n.value)

    @property
    def handle(self):
        return self._h

    # ---------------------------------------------------------- parameters
    def get_params(self) -> Tuple[np.ndarray, float]:
        p = np.empty(self.n_params, np.float32)
        s = ctypes.c_float()
        _abi.check("pyro_net_get_params", self._lib.pyro_net_get_params(
            self._h, p.ctypes.data_as(ctypes.c_void_p), self.n_params, ctypes.byref(s)))
        return p, float(s.value)

    def set_params(self, p: np.ndarray, out_scale: float = 1.0) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.size}")
        _abi.check("pyro_net_set_params", self._lib.pyro_net_set_params(
            self._h, p.ctypes.data_as(ctypes.c_void_p), self.n_params, float(out_scale)))

    def save(self, path: str) -> None:
        p, s = self.get_params()
        with open(path, "wb") as fh:
            fh.write(MAGIC + struct.pack("<IIfI", 1, p.size, s, 0) + p.astype("<f4").tobytes())

    @staticmethod
    def read_file(path: str) -> Tuple[np.ndarray, float]:
        with open(path, "rb") as fh:
            data = fh.read()
        if data[:8] != MAGIC:
            raise ValueError(f"{path}: not a pyro network file")
        ver, count, scale, _ = struct.unpack("<IIfI", data[8:24])
        if ver != 1:
            raise ValueError(f"{path}: unsupported version {ver}")
        p = np.frombuffer(data[24:24 + 4 * count], "<f4").astype(np.float32)
        if p.size != count:
            raise ValueError(f"{path}: truncated")
        return p, float(scale)

    @classmethod
    def load(cls, path: str) -> "Net":
        p, s = cls.read_file(path)
        net = cls()
        net.set_params(p, s)
        return net

    def set_loss(self, w_phi: float = 1.0, w_res: float = 0.0) -> None:
        """Training loss weights: pressure MSE and normalised residual
        (pyro_net_set_loss)."""
        _abi.check("pyro_net_set_loss", self._lib.pyro_net_set_loss(self._h, w_phi, w_res))
        self.loss_weights = (float(w_phi), float(w_res))

    # ------------------------------------------------------------- compute
    def forward(self, b_ptr: int, flags_ptr: int, dims, nb: int, h: float, phi_ptr: int,
                stream: Optional[int] = None) -> None:
        nx, ny, nz = dims
        _abi.check("pyro_net_forward", self._lib.pyro_net_forward(
            self._h, _vp(b_ptr), _vp(flags_ptr), nx, ny, nz, nb, h, _vp(phi_ptr), _vp(stream)))

    def loss_grad(self, b_ptr: int, flags_ptr: int, phi_ptr: int, dims, nb: int, h: float,
                  want_grad: bool = True, stream: Optional[int] = None):
        nx, ny, nz = dims
        loss = ctypes.c_double()
        g = np.empty(self.n_params, np.float32) if want_grad else None
        _abi.check("pyro_net_loss_grad", self._lib.pyro_net_loss_grad(
            self._h, _vp(b_ptr), _vp(flags_ptr), _vp(phi_ptr), nx, ny, nz, nb, h,
            ctypes.byref(loss), g.ctypes.data_as(ctypes.c_void_p) if g is not None else None,
            _vp(stream)))
        return float(loss.value), g

    def train_step(self, b_ptr: int, flags_ptr: int, phi_ptr: int, dims, nb: int, h: float,
                   lr: float, clip: float = 1.0, stream: Optional[int] = None) -> None:
        nx, ny, nz = dims
        _abi.check("pyro_net_train_step", self._lib.pyro_net_train_step(
            self._h, _vp(b_ptr), _vp(flags_ptr), _vp(phi_ptr), nx, ny, nz, nb, h, lr, clip,
            _vp(stream)))

    def last_loss(self, stream: Optional[int] = None) -> float:
        loss = ctypes.c_double()
        _abi.check("pyro_net_last_loss",
                   self._lib.pyro_net_last_loss(self._h, ctypes.byref(loss), _vp(stream)))
        return float(loss.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.pyro_net_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def learned_accept(re: float, eae: float, rae: float, aeae: float, rr: float):
    """The keep-or-discard rule of the learned stage (pyro_learned_accept):
    (keep, alpha, rr_new)."""
    lib = _abi.load()
    a = ctypes.c_double()
    n = ctypes.c_double()
    keep = lib.pyro_learned_accept(re, eae, rae, aeae, rr, ctypes.byref(a), ctypes.byref(n))
    return bool(keep), float(a.value), float(n.value)


# Per-voxel multiply-adds of the network, x2 for FLOPs: level 0 convs 1, 2,
# 8, 9 (K = 27 Cin, N = Cout), level 1 convs 3, 4, 7 (1/8 of the voxels),
# level 2 convs 5, 6 (1/64).
def flops_per_voxel() -> float:
    f = 0.0
    for ci, co, lvl, _ in SPEC:
        f += 2.0 * 27 * ci * co / (8 ** lvl)
    return f


def evaluate(scene_path: str, net: "Net", n_systems: int, every: int, after: float,
             tol: float = 1e-4) -> dict:
    """The learned stage on pressure systems of a scene it was not trained
    on: `n_systems` systems, one every `every` substeps once the time
    passes the scene's preroll + `after` seconds (later than the training
    pairs), each solved from zero to `tol` by BF16 MGPCG without and with
    the stage (warm timing: the second of two solves).  Returns per system
    the iterations, device ms, the residual after the stage and whether
    the stage was kept, and the fallback rate (systems where it was
    discarded)."""
    import torch

    from . import _abi
    from .pairs import collect
    from .poisson import PoissonSolver
    from .scene import Scene
    sc = Scene.load(scene_path)
    rows = []
    ps = None
    for pair in collect(scene_path, n_systems, every=every, preroll=sc.output.preroll + after,
                        refine_iters=1):
        nz, ny, nx = pair["b"].shape
        if ps is None:
            ps = PoissonSolver((nx, ny, nz), pair["h"], bc_mode=0)
            ps.set_net(net)
        b = torch.from_numpy(pair["b"]).cuda()
        ps.set_flags(torch.from_numpy(pair["flags"].astype(np.int32)).cuda().data_ptr())
        phi = torch.zeros_like(b)
        row = {"time_s": pair["time"]}
        for mode, tag in ((_abi.SOLVER_MGPCG_BF16, "without"), (_abi.SOLVER_MGPCG_LEARNED, "with")):
            for _ in range(2):
                phi.zero_()
                torch.cuda.synchronize()
                info = ps.solve(b.data_ptr(), phi.data_ptr(), mode, tol, 100, allow_cap=True)
            row[tag] = {"iterations": info.iterations, "ms": round(info.ms, 3),
                        "rel_resid": info.rel_resid}
            if tag == "with":
                row[tag].update(kept=int(info.learned), learned_ms=round(info.learned_ms, 3),
                                resid_after_stage=info.rel_resid_learned)
        rows.append(row)
    if ps is not None:
        ps.set_net(None)
        ps.close()
    kept = [r["with"]["kept"] for r in rows]
    return {"scene": os.path.basename(scene_path), "systems": rows,
            "fallback_rate": 1.0 - sum(kept) / max(len(kept), 1),
            "mean_iterations": {t: sum(r[t]["iterations"] for r in rows) / max(len(rows), 1)
                                for t in ("without", "with")},
            "mean_ms": {t: sum(r[t]["ms"] for r in rows) / max(len(rows), 1)
                        for t in ("without", "with")}}


def main(argv=None) -> int:
    """python -m pyro_b200.learned bench [--dims NX,NY,NZ] [--reps N]
    [--weights FILE]: device time of the network's forward pass on a seeded
    Poisson right-hand side.
    python -m pyro_b200.learned eval SCENE.toml ... [--systems N] [--every K]
    [--after S] [--weights FILE]: the learned stage on held-out pressure
    systems of each scene (evaluate)."""
    import argparse
    import json

    import torch

    from .poisson import poisson_case
    ap = argparse.ArgumentParser(prog="pyro_b200.learned")
    ap.add_argument("cmd", choices=["bench", "eval"])
    ap.add_argument("scenes", nargs="*")
    ap.add_argument("--dims", default="160,320,160")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--weights")
    ap.add_argument("--systems", type=int, default=4)
    ap.add_argument("--every", type=int, default=12)
    ap.add_argument("--after", type=float, default=3.0)
    a = ap.parse_args(argv)
    if a.cmd == "eval":
        if not a.weights:
            ap.error("eval needs --weights")
        net = Net.load(a.weights)
        out = [evaluate(sp, net, a.systems, a.every, a.after) for sp in a.scenes]
        print(json.dumps(out, indent=1))
        return 0
    nx, ny, nz = (int(v) for v in a.dims.split(","))
    f, b = poisson_case(nx, ny, nz, seed=1)
    net = Net.load(a.weights) if a.weights else Net(seed=0)
    bd = torch.from_numpy(b).cuda()
    fd = torch.from_numpy(f.astype(np.int32)).cuda()
    phi = torch.empty_like(bd)
    s = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        net.forward(bd.data_ptr(), fd.data_ptr(), (nx, ny, nz), 1, 0.02, phi.data_ptr(), stream=s)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        net.forward(bd.data_ptr(), fd.data_ptr(), (nx, ny, nz), 1, 0.02, phi.data_ptr(), stream=s)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    vox = nx * ny * nz
    print(json.dumps(dict(dims=[nx, ny, nz], ms=ms, voxels=vox,
                          tflops=flops_per_voxel() * vox / ms * 1e-9,
                          flops_per_voxel=flops_per_voxel())))
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
