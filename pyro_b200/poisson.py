"""The stand-alone pressure solver over the C ABI, and the seeded Poisson
workload (a 256^3 grid, h = 2 cm, ~5 % of the cells solid in random
axis-aligned boxes of 2-20 cells per edge, an N(0,1) right-hand side with
zero mean over the fluid cells).

    ps = PoissonSolver((nx, ny, nz), h, bc_mode=0)
    ps.set_flags(flags_dev)                       # device uint32 array
    info = ps.solve(b_dev, phi_dev, mode, tol, max_iters)

bc_mode 0 is the reference's boundaries (Dirichlet sides and top, Neumann
floor, src/shaders/mg.wgsl:2); 1 keeps only the top face Dirichlet.
"""
from __future__ import annotations

import ctypes
from typing import Tuple

import numpy as np

from . import _abi


def poisson_case(nx: int, ny: int, nz: int, seed: int = 1, solid: float = 0.05,
                 edge: Tuple[int, int] = (2, 20)):
    """(flags uint32, b float32) in (z, y, x) layout."""
    rng = np.random.default_rng(seed)
    f = np.zeros((nz, ny, nx), np.uint32)
    target = solid * f.size
    count = 0
    while count < target:
        e = rng.integers(edge[0], edge[1] + 1, size=3)
        o = [int(rng.integers(0, max(1, d - int(e[i]) + 1))) for i, d in enumerate((nx, ny, nz))]
        box = f[o[2]:o[2] + e[2], o[1]:o[1] + e[1], o[0]:o[0] + e[0]]
        count += int((box == 0).sum())
        box[...] = 1
    b = rng.normal(0.0, 1.0, (nz, ny, nx)).astype(np.float32)
    b[f == 1] = 0.0
    fl = f == 0
    b[fl] -= np.float32(b[fl].mean(dtype=np.float64))
    return f, b


class PoissonSolver:
    def __init__(self, dims, h: float, bc_mode: int = 0):
        self._lib = _abi.load()
        self.dims = tuple(int(v) for v in dims)
        self.h = float(h)
        h_ = ctypes.c_void_p()
        _abi.check("pyro_poisson_create", self._lib.pyro_poisson_create(
            self.dims[0], self.dims[1], self.dims[2], self.h, bc_mode, ctypes.byref(h_)))
        self._h = h_

    def set_flags(self, flags_dev_ptr: int) -> None:
        _abi.check("pyro_poisson_set_flags",
                   self._lib.pyro_poisson_set_flags(self._h, ctypes.c_void_p(flags_dev_ptr)))

    def solve(self, b_dev_ptr: int, phi_dev_ptr: int, mode: int, tol: float,
              max_iters: int, allow_cap: bool = False) -> _abi.PyroSolveInfo:
        info = _abi.PyroSolveInfo()
        rc = self._lib.pyro_poisson_solve(self._h, ctypes.c_void_p(b_dev_ptr),
                                          ctypes.c_void_p(phi_dev_ptr), mode, tol, max_iters,
                                          ctypes.byref(info))
        if not (allow_cap and rc == _abi.PYRO_E_NOCONV):
            _abi.check("pyro_poisson_solve", rc)
        return info

    def profile_cg(self, b_dev_ptr: int, phi_dev_ptr: int, mode: int, iters: int) -> dict:
        """Device time and step count per launch class of `iters` CG
        iterations run one launch at a time (pyro_poisson_profile_cg);
        phi is updated in place."""
        n = len(_abi.CG_CLASSES)
        ms = (ctypes.c_float * n)()
        cnt = (ctypes.c_int * n)()
        _abi.check("pyro_poisson_profile_cg", self._lib.pyro_poisson_profile_cg(
            self._h, ctypes.c_void_p(b_dev_ptr), ctypes.c_void_p(phi_dev_ptr), mode, iters, ms,
            cnt, n))
        return {k: {"ms": float(ms[i]), "steps": int(cnt[i])}
                for i, k in enumerate(_abi.CG_CLASSES)}

    def set_net(self, net) -> None:
        """Network for mode SOLVER_MGPCG_LEARNED (None detaches); the
        caller keeps `net` alive while it is attached."""
        self._net = net
        _abi.check("pyro_poisson_set_net",
                   self._lib.pyro_poisson_set_net(self._h, net.handle if net else None))

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _abi.check("pyro_poisson_stream", self._lib.pyro_poisson_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.pyro_poisson_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


MODES = {"vcycle": _abi.SOLVER_VCYCLE, "vcycle_tol": _abi.SOLVER_VCYCLE_TOL,
         "mgpcg": _abi.SOLVER_MGPCG, "mgpcg_bf16": _abi.SOLVER_MGPCG_BF16}


def main(argv=None) -> None:
    """Solve the seeded n^3 case on cuda:0 and print one JSON line: the
    iterations, relative residual and device time of the last of `reps`
    solves from a zero guess (a small, fixed case for profilers)."""
    import argparse
    import json

    import torch
    ap = argparse.ArgumentParser(prog="pyro_b200.poisson",
                                 description="Solve the seeded n^3 Poisson case on cuda:0.")
    ap.add_argument("--n", type=int, default=128, help="cells per edge")
    ap.add_argument("--h", type=float, default=0.02)
    ap.add_argument("--mode", choices=sorted(MODES), default="vcycle")
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--iters", type=int, default=1, help="V-cycles, or CG iterations at most")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--profile", action="store_true",
                    help="after the solves, run --iters CG iterations one launch at a time "
                         "(pyro_poisson_profile_cg) and print device time per launch class")
    a = ap.parse_args(argv)
    f, b = poisson_case(a.n, a.n, a.n, seed=1)
    fd, bd = torch.from_numpy(f).cuda(), torch.from_numpy(b).cuda()
    ps = PoissonSolver((a.n, a.n, a.n), a.h, 0)
    ps.set_flags(fd.data_ptr())
    phi = torch.zeros_like(bd)
    for _ in range(a.reps):
        phi.zero_()
        torch.cuda.synchronize()
        info = ps.solve(bd.data_ptr(), phi.data_ptr(), MODES[a.mode], a.tol, a.iters,
                        allow_cap=True)
    torch.cuda.synchronize()
    out = {"n": a.n, "mode": a.mode, "iterations": info.iterations,
           "rel_resid": info.rel_resid, "ms": info.ms}
    if a.profile:
        if a.mode not in ("mgpcg", "mgpcg_bf16"):
            raise SystemExit("--profile needs --mode mgpcg or mgpcg_bf16")
        phi.zero_()
        torch.cuda.synchronize()
        out["profile"] = ps.profile_cg(bd.data_ptr(), phi.data_ptr(), MODES[a.mode], a.iters)
    print(json.dumps(out))
    ps.close()


if __name__ == "__main__":
    main()
