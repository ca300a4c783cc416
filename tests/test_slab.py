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
