"""The pressure solve across ranks by z-slabs (pyro_b200.slab) on the CPU:
gloo ranks whose level operations are the oracle's kernels, against the
oracle's single-domain V-cycles, bit for bit; and the slab plan's
alignment rules."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

import oracle  # noqa: E402
from pyro_b200 import slab  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def case(dims, seed):
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    f = (rng.random((nz, ny, nx)) < 0.15).astype(np.uint32)
    f[:, 0, :] = 0
    b = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    p = rng.normal(0, 0.1, (nz, ny, nx)).astype(np.float32)
    return f, b, p


@pytest.mark.parametrize("dims", [(160, 320, 160), (32, 36, 40), (64, 64, 64), (24, 40, 32)])
@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_plan_keeps_every_local_array_aligned(dims, world):
    if dims[2] % world:
        pytest.skip("unequal slabs")
    levels = slab.level_dims(dims)
    assert levels == oracle.mg_levels(*dims)
    for rank in range(world):
        d, lg, slabs = slab.plan(dims, world, rank)
        assert d == levels and 0 <= lg < len(levels)
        assert len(slabs) == lg + 1
        for l, s in enumerate(slabs):
            own = s.z1 - s.z0
            assert own * world == levels[l][2]
            assert s.lo <= own and s.hi <= own       # ghosts come from one neighbour
            if l < lg:
                assert s.lo in (0, 2 ** (lg - l)) and s.hi in (0, 2 ** (lg - l))
                c = slabs[l + 1]
                # coarse local plane Z has the fine local children 2Z, 2Z+1
                assert s.zlo == 2 * c.zlo and s.planes == 2 * c.planes
            if lg:
                assert (s.lo > 0) == (rank > 0) and (s.hi > 0) == (rank < world - 1)


def _rank(rank, world, port, dims, cycles, bc_mode, q):
    sys.path[:0] = [ROOT, HERE]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist
    from slab_oracle_ops import OracleOps
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    f, b, p = case(dims, 7)
    n = dims[2] // world
    own = slice(rank * n, (rank + 1) * n)
    sp = slab.SlabPoisson(dims, 0.05, bc_mode, ops=OracleOps(bc_mode))
    sp.set_flags(torch.from_numpy(f[own].view(np.int32).copy()))
    phi = torch.from_numpy(p[own].copy())
    sp.vcycles(phi, torch.from_numpy(b[own].copy()), cycles)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, phi.numpy().copy(), sp.lg))


@pytest.mark.parametrize("dims,world,bc_mode,lg", [((24, 40, 32), 2, 0, 1),
                                                   ((32, 64, 64), 4, 1, 2),
                                                   ((32, 36, 40), 4, 0, 1),
                                                   ((16, 24, 21), 3, 0, 0)])
def test_slab_vcycles_equal_the_single_domain_oracle(dims, world, bc_mode, lg):
    """(24, 40, 32) on 2 ranks: level 0 on slabs, the coarsest level
    gathered; (32, 64, 64) on 4: levels 0 and 1 on slabs, top-only
    Dirichlet; (32, 36, 40) on 4: level 1 gathered and smoothed whole;
    (16, 24, 21) on 3: no level halves evenly, everything gathered."""
    cycles = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, dims, cycles, bc_mode, q))
             for r in range(world)]
    for pr in procs:
        pr.start()
    res = dict((r, (phi, lg)) for r, phi, lg in (q.get(timeout=300) for _ in procs))
    for pr in procs:
        pr.join(timeout=60)
    assert all(pr.exitcode == 0 for pr in procs)
    assert all(res[r][1] == lg for r in range(world))
    got = np.concatenate([res[r][0] for r in range(world)], 0)
    f, b, p = case(dims, 7)
    want = oracle.vcycles(dims, 0.05, p, b, f, cycles, bc_mode=bc_mode)
    assert np.array_equal(got, want), np.abs(got - want).max()


def _rank_cg(rank, world, port, dims, bc_mode, q):
    sys.path[:0] = [ROOT, HERE]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist
    from slab_oracle_ops import OracleOps
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    f, b, _ = cg_case(dims, 11)
    n = dims[2] // world
    own = slice(rank * n, (rank + 1) * n)
    sp = slab.SlabPoisson(dims, 0.05, bc_mode, ops=OracleOps(bc_mode))
    sp.set_flags(torch.from_numpy(f[own].view(np.int32).copy()))
    phi = torch.zeros((n, dims[1], dims[0]), dtype=torch.float32)
    it, rel = sp.mgpcg(phi, torch.from_numpy(b[own].copy()), 1e-6, 50)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, phi.numpy().copy(), it, rel))


def cg_case(dims, seed):
    """Sparse single solid cells (no enclosed fluid), b zero in solids."""
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    f = (rng.random((nz, ny, nx)) < 0.02).astype(np.uint32)
    b = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    b[f == 1] = 0
    return f, b, None


def test_oracle_ops_apply_matches_the_oracle_residual():
    from slab_oracle_ops import OracleOps
    import torch
    dims = (12, 10, 8)
    f, b, p = case(dims, 3)
    for bc_mode in (0, 1):
        q = torch.zeros((dims[2], dims[1], dims[0]))
        OracleOps(bc_mode).apply(dims, 0.1, torch.from_numpy(f.view(np.int32)),
                                 torch.from_numpy(p), q)
        r = np.where(f != 1, b.astype(np.float64) - q.numpy(), 0.0)
        rel = np.sqrt((r ** 2).sum() / (np.where(f != 1, b, 0.0).astype(np.float64) ** 2).sum())
        assert abs(rel - oracle.poisson_relres(dims, 0.1, p, b, f, bc_mode=bc_mode)) < 1e-5 * rel


@pytest.mark.parametrize("dims,world,bc_mode", [((24, 40, 32), 2, 0), ((32, 36, 40), 4, 1)])
def test_slab_mgpcg_converges_like_one_rank(dims, world, bc_mode):
    """CG on slabs with all-reduced dot products: converges to 1e-6 and
    agrees with the one-rank run of the same solver."""
    runs = {}
    for w in (1, world):
        ctx = mp.get_context("spawn")
        q = ctx.Queue()
        port = _free_port()
        procs = [ctx.Process(target=_rank_cg, args=(r, w, port, dims, bc_mode, q))
                 for r in range(w)]
        for pr in procs:
            pr.start()
        res = dict((r, (phi, it, rel)) for r, phi, it, rel in (q.get(timeout=300) for _ in procs))
        for pr in procs:
            pr.join(timeout=60)
        assert all(pr.exitcode == 0 for pr in procs)
        runs[w] = (np.concatenate([res[r][0] for r in range(w)], 0), res[0][1], res[0][2])
    (p1, it1, rel1), (pw, itw, relw) = runs[1], runs[world]
    f, b, _ = cg_case(dims, 11)
    assert rel1 <= 1e-6 and relw <= 1e-6 and abs(it1 - itw) <= 1
    assert oracle.poisson_relres(dims, 0.05, pw, b, f, bc_mode=bc_mode) <= 2e-6
    assert np.abs(pw - p1).max() <= 1e-4 * np.abs(p1).max()
