"""Level operations for pyro_b200.slab.SlabPoisson computed by the oracle
(test infrastructure): the reference's per-flag multigrid kernels on CPU
tensors, so the slab decomposition runs as gloo ranks without a GPU and
is compared with the oracle's single-domain V-cycles.  The "mask" of a
level is its flag array itself (the oracle's kernels read the flags)."""
import numpy as np
import torch

import oracle


def _u32(t):
    return np.ascontiguousarray(t.numpy()).view(np.uint32)


def _f32(t):
    return np.ascontiguousarray(t.numpy())


class OracleOps:
    def __init__(self, bc_mode=0):
        self.bc_mode = bc_mode

    def empty(self, dims, dtype):
        return torch.zeros((dims[2], dims[1], dims[0]), dtype=dtype)

    def meta(self, d, flags):
        return flags

    def flags_down(self, fd, ff, cd):
        shape = (fd[2], fd[1], fd[0])
        z = np.zeros(shape, np.float32)
        _, _, fc = oracle.mg_restrict(fd, 1.0, z, z, _u32(ff), self.bc_mode)
        return torch.from_numpy(fc.view(np.int32).copy())

    def smooth_pass(self, d, h, b, meta, phi, color, omega):
        out = oracle.mg_smooth(d, h, _f32(b), _u32(meta), _f32(phi), color, omega,
                               bc_mode=self.bc_mode)
        phi.copy_(torch.from_numpy(out))

    def restrict(self, fd, h, pf, bf, mf, cd, bc, pc):
        b_, p_, _ = oracle.mg_restrict(fd, h, _f32(pf), _f32(bf), _u32(mf), self.bc_mode)
        bc.copy_(torch.from_numpy(b_))
        pc.copy_(torch.from_numpy(p_))

    def prolong(self, fd, pc, mf, pf, cd, mc):
        out = oracle.mg_prolong(fd, _f32(pc), _u32(mf), _f32(pf), _u32(mc))
        pf.copy_(torch.from_numpy(out))

    def coarse(self, d, h, b, flags, meta, phi):
        for _ in range(80):
            for c in (0, 1):
                self.smooth_pass(d, h, b, meta, phi, c, 1.6)

    def apply(self, d, h, flags, p, q):
        """q = A p: (sum of fluid neighbours - count p) / h^2 in FP64, the
        Dirichlet faces counted as mg.wgsl:25-35 does (bc_mode 0: every face
        but the floor; 1: the top), 0 in solids."""
        f = _u32(flags).reshape(d[2], d[1], d[0])
        v = _f32(p).astype(np.float64).reshape(f.shape)
        fluid = f != 1
        s = np.zeros_like(v)
        cnt = np.zeros_like(v)
        for axis, side in ((2, 1), (2, -1), (1, 1), (1, -1), (0, 1), (0, -1)):
            nb = np.roll(v, -side, axis=axis)
            nf = np.roll(fluid, -side, axis=axis)
            edge = np.zeros(f.shape, bool)
            idx = [slice(None)] * 3
            idx[axis] = -1 if side == 1 else 0
            edge[tuple(idx)] = True
            floor = axis == 1 and side == -1
            top = axis == 1 and side == 1
            dirichlet = edge & (not floor) & (self.bc_mode == 0 or top)
            inside = ~edge & nf
            s += np.where(inside, nb, 0.0)
            cnt += inside + dirichlet
        out = np.where(fluid, (s - cnt * v) / (float(np.float32(h)) ** 2), 0.0)
        q.copy_(torch.from_numpy(out.astype(np.float32)))
