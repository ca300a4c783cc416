"""The pressure solve across GPUs by z-slabs: the reference's V-cycles
(src/sim.rs:451-491, level rule src/sim.rs:142-168) with each rank holding
a slab of planes of every fine level, one-plane halo exchanges after every
smoother pass, and the coarse levels gathered onto every rank.

The reference runs on one device and has no decomposition; this follows
the layout its kernels imply.  Rank r of N owns level-0 planes
[r nz/N, (r+1) nz/N).  Level l < Lg (the distributed levels) keeps the
rank's own planes plus g_l = 2^(Lg-l) ghost planes on each side that has a
neighbour, so that every local array starts at an even global plane and the
unchanged single-domain kernels (pyro_k_mg_pass, pyro_k_mg_restrict_m,
pyro_k_mg_prolong_m, pyro_k_mg_meta, pyro_k_mg_flags_down) map coarse plane
Z to fine planes 2Z, 2Z+1 in local indices as they do globally.  The
kernels treat a local array's first and last plane as the domain's (a
Dirichlet face in bc_mode 0, no neighbour beyond); only ghost cells touch
those planes, and an own cell reads its neighbours no further than the
innermost ghost plane, which holds the neighbouring rank's current values:

  * flags: level-0 ghosts are exchanged once per set_flags; the coarse
    flags of the distributed levels follow locally (a coarse ghost plane
    k needs fine ghost planes 2k, 2k+1, present since g_l = 2 g_{l+1});
  * phi: after every smoother pass and after the prolongation the
    innermost plane is exchanged in both directions (the restriction
    zeroes a coarse level's phi everywhere, ghosts included);
  * b: never exchanged (an own cell reads only its own b).

Level Lg is the first gathered level: the restriction from Lg - 1 fills
the rank's own planes of it, an all-gather assembles the whole level on
every rank, and every rank runs the rest of the V-cycle (the levels below,
the 80 SOR sweeps of the coarsest) on whole arrays, then takes its slab of
level Lg back for the prolongation.  Lg is the largest level count with
nz divisible by N 2^Lg (every slab then halves exactly) below the coarsest
level; with N = 1 it is 0 and the solve is the single-domain one.

Every own cell sees the same inputs as in the single-domain V-cycle, so the
result equals it bit for bit.  Ranks exchange planes with
torch.distributed point-to-point operations (NCCL over NVLink between
GPUs; with a gloo group the planes pass through host memory) and meet in
one all-gather per V-cycle.  No kernel waits on another rank.

The arithmetic runs through a level-operations object: LevelOps, the CUDA
kernels behind the C ABI on torch tensors of one device.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Tuple

import torch
import torch.distributed as dist

from . import _abi

Dims = Tuple[int, int, int]
MAX_LEVELS = 4
COARSE_SWEEPS, COARSE_OMEGA = 80, 1.6


def level_dims(d0: Dims, max_levels: int = MAX_LEVELS) -> List[Dims]:
    """The reference's hierarchy (src/sim.rs:142-168): at most 4 levels,
    stop after the first whose smallest dimension is below 16, halve with
    ceil."""
    out = []
    d = tuple(int(v) for v in d0)
    for _ in range(max_levels):
        out.append(d)
        if min(d) < 16:
            break
        d = tuple((v + 1) // 2 for v in d)
    return out


@dataclass
class SlabLevel:
    dims: Dims           # the level's global dimensions
    z0: int              # own planes [z0, z1) (global)
    z1: int
    lo: int              # ghost planes below / above the own ones
    hi: int

    @property
    def zlo(self) -> int:
        return self.z0 - self.lo

    @property
    def planes(self) -> int:
        return self.z1 - self.z0 + self.lo + self.hi

    @property
    def local_dims(self) -> Dims:
        return (self.dims[0], self.dims[1], self.planes)


def plan(d0: Dims, world: int, rank: int) -> Tuple[List[Dims], int, List[SlabLevel]]:
    """(global level dims, Lg, the rank's slab of levels 0..Lg)."""
    dims = level_dims(d0)
    nz = d0[2]
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world size or rank")
    if nz % world:
        raise ValueError(f"nz = {nz} does not split into {world} equal slabs")
    lg = 0
    while lg + 1 < len(dims) and nz % (world * 2 ** (lg + 1)) == 0:
        lg += 1
    if world == 1:
        lg = 0
    slabs = []
    for l in range(lg + 1):
        s = nz // (world * 2 ** l)
        g = 2 ** (lg - l)
        slabs.append(SlabLevel(dims[l], rank * s, (rank + 1) * s, g if rank > 0 else 0,
                               g if rank + 1 < world else 0))
    return dims, lg, slabs


class LevelOps:
    """The level kernels on CUDA tensors through the C ABI (stream: the
    current torch stream of the tensors' device)."""

    def __init__(self, bc_mode: int = 0):
        self.lib = _abi.load()
        self.bc_mode = bc_mode

    @staticmethod
    def _p(t: torch.Tensor) -> ctypes.c_void_p:
        return ctypes.c_void_p(t.data_ptr())

    def _st(self):
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def _ok(self, name, rc):
        if rc != 0:
            raise RuntimeError(f"{name}: {self.lib.pyro_last_error().decode()}")

    def empty(self, dims: Dims, dtype) -> torch.Tensor:
        return torch.zeros((dims[2], dims[1], dims[0]), dtype=dtype, device="cuda")

    def meta(self, d: Dims, flags: torch.Tensor) -> torch.Tensor:
        m = self.empty(d, torch.uint8)
        self._ok("pyro_k_mg_meta", self.lib.pyro_k_mg_meta(*d, self._p(flags), self._p(m),
                                                           self._st()))
        return m

    def flags_down(self, fd: Dims, ff: torch.Tensor, cd: Dims) -> torch.Tensor:
        fc = self.empty(cd, torch.int32)
        self._ok("pyro_k_mg_flags_down", self.lib.pyro_k_mg_flags_down(
            *fd, self._p(ff), *cd, self._p(fc), self._st()))
        return fc

    def smooth_pass(self, d: Dims, h: float, b, meta, phi, color: int, omega: float):
        self._ok("pyro_k_mg_pass", self.lib.pyro_k_mg_pass(
            *d, h, self._p(b), self._p(meta), self._p(phi), color, omega, self.bc_mode,
            _abi.MG_F32, self._st()))

    def restrict(self, fd: Dims, h: float, pf, bf, mf, cd: Dims, bc, pc):
        self._ok("pyro_k_mg_restrict_m", self.lib.pyro_k_mg_restrict_m(
            *fd, h, self._p(pf), self._p(bf), self._p(mf), *cd, self._p(bc), self._p(pc),
            self.bc_mode, _abi.MG_F32, self._st()))

    def prolong(self, fd: Dims, pc, mf, pf, cd: Dims, mc):
        self._ok("pyro_k_mg_prolong_m", self.lib.pyro_k_mg_prolong_m(
            *fd, self._p(pc), self._p(mf), self._p(pf), *cd, self._p(mc), _abi.MG_F32,
            self._st()))

    def apply(self, d: Dims, h: float, flags, p, q):
        """q = A p (pyro_k_mg_apply)."""
        self._ok("pyro_k_mg_apply", self.lib.pyro_k_mg_apply(
            *d, h, self._p(flags), self._p(p), self._p(q), self.bc_mode, self._st()))

    def coarse(self, d: Dims, h: float, b, flags, meta, phi):
        if self.bc_mode == 0:
            self._ok("pyro_k_mg_coarse", self.lib.pyro_k_mg_coarse(
                *d, h, self._p(b), self._p(flags), self._p(phi), COARSE_SWEEPS, COARSE_OMEGA,
                self._st()))
            return
        for _ in range(COARSE_SWEEPS):
            for c in (0, 1):
                self.smooth_pass(d, h, b, meta, phi, c, COARSE_OMEGA)


class SlabPoisson:
    """V-cycles of the pressure system on this rank's z-slab.

        sp = SlabPoisson((nx, ny, nz), h, bc_mode=0, group=None)
        sp.set_flags(flags_own)          # (nz/N, ny, nx) int32/uint32 planes
        sp.vcycles(phi_own, b_own, 4)    # phi_own updated in place

    flags_own, b_own and phi_own are this rank's own level-0 planes
    (z-major, x fastest), on the device of `ops`.  Collective: every rank
    of the group calls each method in the same order."""

    def __init__(self, dims: Dims, h: float, bc_mode: int = 0, group=None,
                 ops: Optional[LevelOps] = None):
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.ops = ops if ops is not None else LevelOps(bc_mode)
        self.dims, self.lg, self.slabs = plan(tuple(dims), self.world, self.rank)
        self.h = [float(h) * 2 ** l for l in range(len(self.dims))]
        self._flags: List[torch.Tensor] = []
        self._meta: List[torch.Tensor] = []
        self._phi: List[torch.Tensor] = []
        self._b: List[torch.Tensor] = []
        self._fluid: Optional[torch.Tensor] = None  # own fluid cells, for the CG dots
        # host staging for groups whose backend cannot move device tensors
        self._via_host = (dist.is_initialized() and dist.get_backend(group) == "gloo")

    # ------------------------------------------------------------ exchange
    def _peer(self, r: int) -> int:
        return dist.get_global_rank(self.group, r) if self.group is not None else r

    def _swap(self, t: torch.Tensor, s: SlabLevel, width: int) -> None:
        """Copy `width` boundary planes of the own region into the
        neighbours' ghost planes (the innermost `width` of them)."""
        if self.world == 1:
            return
        ops = []
        recv = []
        plane = t.shape[1] * t.shape[2]
        flat = t.view(-1)
        own0, own1 = s.lo, s.lo + (s.z1 - s.z0)

        def buf(a, b_):
            v = flat[a * plane:b_ * plane]
            return v.cpu() if self._via_host else v

        if s.lo:
            snd = buf(own0, own0 + width)
            rcv = torch.empty_like(snd)
            ops += [dist.P2POp(dist.isend, snd.contiguous(), self._peer(self.rank - 1), self.group),
                    dist.P2POp(dist.irecv, rcv, self._peer(self.rank - 1), self.group)]
            recv.append((own0 - width, rcv))
        if s.hi:
            snd = buf(own1 - width, own1)
            rcv = torch.empty_like(snd)
            ops += [dist.P2POp(dist.isend, snd.contiguous(), self._peer(self.rank + 1), self.group),
                    dist.P2POp(dist.irecv, rcv, self._peer(self.rank + 1), self.group)]
            recv.append((own1, rcv))
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        for z, rcv in recv:
            flat[z * plane:(z + width) * plane].copy_(rcv)

    def _gather_own(self, own: torch.Tensor) -> torch.Tensor:
        """The whole level from every rank's own planes (equal slabs)."""
        own = own.contiguous()
        if self.world == 1:
            return own.clone()
        src = own.cpu() if self._via_host else own
        parts = [torch.empty_like(src) for _ in range(self.world)]
        dist.all_gather(parts, src, group=self.group)
        full = torch.cat(parts, 0)
        return full.to(own.device) if self._via_host else full

    def _gather(self, t: torch.Tensor, s: SlabLevel) -> torch.Tensor:
        return self._gather_own(t[s.lo:s.lo + (s.z1 - s.z0)])

    # ---------------------------------------------------------------- set-up
    def set_flags(self, flags_own: torch.Tensor) -> None:
        ops, s0 = self.ops, self.slabs[0]
        f0 = ops.empty(s0.local_dims, torch.int32)
        f0[s0.lo:s0.lo + (s0.z1 - s0.z0)].copy_(flags_own.view(torch.int32))
        self._swap(f0, s0, min(s0.lo or s0.hi, s0.z1 - s0.z0) if self.world > 1 else 0)
        flags = [f0]
        for l in range(1, self.lg + 1):
            flags.append(ops.flags_down(self.slabs[l - 1].local_dims, flags[-1],
                                        self.slabs[l].local_dims))
        # the gathered levels: level Lg whole, then halved on whole arrays
        whole = [self._gather(flags[self.lg], self.slabs[self.lg])]
        for l in range(self.lg + 1, len(self.dims)):
            whole.append(ops.flags_down(self.dims[l - 1], whole[-1], self.dims[l]))
        self._flags = flags[:self.lg] + whole
        ld = [s.local_dims for s in self.slabs[:self.lg]] + self.dims[self.lg:]
        self._ld = ld
        self._meta = [ops.meta(d, f) for d, f in zip(ld, self._flags)]
        self._lgmeta_local = ops.meta(self.slabs[self.lg].local_dims, flags[self.lg])
        self._phi = [ops.empty(d, torch.float32) for d in ld]
        self._b = [ops.empty(d, torch.float32) for d in ld]
        s = self.slabs[self.lg]
        self._phi_lg_local = ops.empty(s.local_dims, torch.float32)
        self._b_lg_local = ops.empty(s.local_dims, torch.float32)

    # ------------------------------------------------------------- V-cycles
    def _smooth(self, l: int, distributed: bool) -> None:
        d, ops = self._ld[l], self.ops
        for _ in range(2):
            for c in (0, 1):
                ops.smooth_pass(d, self.h[l], self._b[l], self._meta[l], self._phi[l], c, 1.0)
                if distributed:
                    self._swap(self._phi[l], self.slabs[l], 1)

    def _tail(self) -> None:
        """Levels Lg .. L-1 on whole arrays (every rank the same)."""
        ops, L = self.ops, len(self.dims)
        for l in range(self.lg, L - 1):
            self._smooth(l, False)
            ops.restrict(self.dims[l], self.h[l], self._phi[l], self._b[l], self._meta[l],
                         self.dims[l + 1], self._b[l + 1], self._phi[l + 1])
        c = L - 1
        ops.coarse(self.dims[c], self.h[c], self._b[c], self._flags[c], self._meta[c],
                   self._phi[c])
        for l in range(L - 2, self.lg - 1, -1):
            ops.prolong(self.dims[l], self._phi[l + 1], self._meta[l], self._phi[l],
                        self.dims[l + 1], self._meta[l + 1])
            self._smooth(l, False)

    def _dot(self, a: torch.Tensor, b: torch.Tensor) -> float:
        """Sum over this rank's fluid cells, all-reduced, in FP64."""
        v = torch.sum(a.double() * b.double() * self._fluid).reshape(1)
        if self.world > 1:
            src = v.cpu() if self._via_host else v
            dist.all_reduce(src, group=self.group)
            v = src
        return float(v.item())

    def mgpcg(self, phi_own: torch.Tensor, b_own: torch.Tensor, tol: float,
              max_iters: int) -> Tuple[int, float]:
        """Flexible preconditioned CG (Polak-Ribiere beta) on the slabs:
        phi_own (the initial guess) is updated in place until
        |b - A phi| <= tol |b| over the fluid cells or after max_iters
        iterations.  The operator reads the neighbours' boundary plane of
        the search direction (one exchange per iteration); the
        preconditioner is one slab V-cycle from zero; every dot product is
        this rank's FP64 sum all-reduced across the group.  The fluid cells
        must reach a Dirichlet face (otherwise the system is singular).
        Returns (iterations, relative residual)."""
        if not self._phi:
            raise RuntimeError("SlabPoisson.mgpcg: set_flags first")
        ops, s0 = self.ops, self.slabs[0]
        n0, lo = s0.z1 - s0.z0, s0.lo
        d0 = s0.local_dims if self.lg else self.dims[0]
        f0 = self._flags[0]
        # local extended arrays for the vectors the operator reads
        if self.lg:
            own = slice(lo, lo + n0)
            fl_own = f0[own]
        else:
            own = slice(s0.z0, s0.z1)
            fl_own = f0[own]
        self._fluid = (fl_own != 1).double()
        ext = ops.empty(d0, torch.float32)
        q = ops.empty(d0, torch.float32)

        def apply_own(x_own):
            """A x on the own planes (x_own: own planes)."""
            if self.lg:
                ext[own].copy_(x_own)
                self._swap(ext, s0, 1)
            else:
                ext.copy_(self._gather_own(x_own))
            ops.apply(d0, self.h[0], f0, ext, q)
            return q[own].clone()

        r = b_own - apply_own(phi_own)
        bn = self._dot(b_own, b_own) ** 0.5
        if bn == 0.0:
            phi_own.zero_()
            return 0, 0.0
        rn = self._dot(r, r) ** 0.5
        if rn <= tol * bn:
            return 0, rn / bn
        z = torch.zeros_like(r)
        self.vcycles(z, r, 1)
        p = z.clone()
        rz = self._dot(r, z)
        it = 0
        while it < max_iters:
            it += 1
            ap = apply_own(p)
            alpha = rz / self._dot(p, ap)
            phi_own.add_(p, alpha=alpha)
            r_old = r.clone()
            r.sub_(ap, alpha=alpha)
            rn = self._dot(r, r) ** 0.5
            if rn <= tol * bn:
                break
            z.zero_()
            self.vcycles(z, r, 1)
            rz_new = self._dot(r, z)
            beta = (rz_new - self._dot(r_old, z)) / rz
            rz = rz_new
            p.mul_(beta).add_(z)
        return it, rn / bn

    def vcycles(self, phi_own: torch.Tensor, b_own: torch.Tensor, cycles: int) -> None:
        if not self._phi:
            raise RuntimeError("SlabPoisson.vcycles: set_flags first")
        ops, lg = self.ops, self.lg
        s0 = self.slabs[0]
        n0 = s0.z1 - s0.z0
        if lg == 0:
            self._phi[0].copy_(self._gather_own(phi_own))
            self._b[0].copy_(self._gather_own(b_own))
        else:
            self._phi[0][s0.lo:s0.lo + n0].copy_(phi_own)
            self._b[0][s0.lo:s0.lo + n0].copy_(b_own)
            self._swap(self._phi[0], s0, 1)
        for _ in range(cycles):
            for l in range(lg):
                self._smooth(l, True)
                tgt_b = self._b[l + 1] if l + 1 < lg else self._b_lg_local
                tgt_p = self._phi[l + 1] if l + 1 < lg else self._phi_lg_local
                cd = self.slabs[l + 1].local_dims
                ops.restrict(self._ld[l], self.h[l], self._phi[l], self._b[l], self._meta[l],
                             cd, tgt_b, tgt_p)
            if lg:
                self._b[lg].copy_(self._gather(self._b_lg_local, self.slabs[lg]))
                self._phi[lg].zero_()
            self._tail()
            for l in range(lg - 1, -1, -1):
                if l + 1 == lg:
                    s = self.slabs[lg]
                    src = self._phi_lg_local
                    src.copy_(self._phi[lg][s.zlo:s.zlo + s.planes])
                    mc = self._lgmeta_local
                else:
                    src, mc = self._phi[l + 1], self._meta[l + 1]
                ops.prolong(self._ld[l], src, self._meta[l], self._phi[l],
                            self.slabs[l + 1].local_dims, mc)
                self._swap(self._phi[l], self.slabs[l], 1)
                self._smooth(l, True)
        if lg == 0:
            phi_own.copy_(self._phi[0][s0.z0:s0.z1])
        else:
            phi_own.copy_(self._phi[0][s0.lo:s0.lo + n0])


def main(argv=None) -> None:
    """Under torchrun, one rank per GPU: the seeded Poisson case
    (pyro_b200.poisson.poisson_case) split into z-slabs, `--cycles`
    V-cycles timed with CUDA events (max over ranks), and on rank 0 the
    gathered result compared with the single-GPU V-cycles of the same
    system.  Prints one JSON line on rank 0."""
    import argparse
    import datetime
    import json
    import os

    import numpy as np

    from .poisson import PoissonSolver, poisson_case
    ap = argparse.ArgumentParser(prog="pyro_b200.slab",
                                 description="z-slab V-cycles across the ranks of torchrun")
    ap.add_argument("--dims", default="160,320,160")
    ap.add_argument("--h", type=float, default=0.02)
    ap.add_argument("--cycles", type=int, default=4)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args(argv)
    dims = tuple(int(v) for v in a.dims.split(","))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    rank = dist.get_rank() if dist.is_initialized() else 0
    f, b = poisson_case(*dims, seed=1)
    n = dims[2] // world
    own = slice(rank * n, (rank + 1) * n)
    sp = SlabPoisson(dims, a.h)
    sp.set_flags(torch.from_numpy(f[own].view(np.int32).copy()).cuda())
    bo = torch.from_numpy(b[own].copy()).cuda()
    phi = torch.zeros_like(bo)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(a.reps):
        phi.zero_()
        if dist.is_initialized():
            dist.barrier()
        torch.cuda.synchronize()
        e0.record()
        sp.vcycles(phi, bo, a.cycles)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = torch.tensor([min(times)], device="cuda")
    full = sp._gather_own(phi)
    if dist.is_initialized():
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    if rank == 0:
        ps = PoissonSolver(dims, a.h, 0)
        fd = torch.from_numpy(f.view(np.int32)).cuda()
        ps.set_flags(fd.data_ptr())
        bd = torch.from_numpy(b).cuda()
        ref = torch.zeros_like(bd)
        ps.solve(bd.data_ptr(), ref.data_ptr(), _abi.SOLVER_VCYCLE, 0.0, a.cycles,
                 allow_cap=True)
        torch.cuda.synchronize()
        ps.close()
        print(json.dumps({"dims": dims, "ranks": world, "distributed_levels": sp.lg,
                          "cycles": a.cycles, "ms": float(ms.item()),
                          "equal_to_single_gpu": bool(torch.equal(full, ref))}))
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
