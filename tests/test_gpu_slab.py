"""The z-slab pressure solve (pyro_b200.slab) through the CUDA kernels:
one rank against the library's own V-cycles, and two ranks sharing one
GPU (gloo, planes exchanged through host memory; no kernel waits on the
other rank) against the same, bit for bit."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

from gpu_util import require_cuda  # noqa: E402
from pyro_b200 import _abi, slab  # noqa: E402
from pyro_b200.poisson import PoissonSolver  # noqa: E402
from test_slab import case  # noqa: E402

pytestmark = pytest.mark.gpu
H = 0.05


def single_domain(dims, cycles, bc_mode):
    f, b, p = case(dims, 7)
    ps = PoissonSolver(dims, H, bc_mode)
    fd = torch.from_numpy(f.view(np.int32)).cuda()
    ps.set_flags(fd.data_ptr())
    bd = torch.from_numpy(b).cuda()
    phi = torch.from_numpy(p).cuda()
    ps.solve(bd.data_ptr(), phi.data_ptr(), _abi.SOLVER_VCYCLE, 0.0, cycles, allow_cap=True)
    torch.cuda.synchronize()
    ps.close()
    return phi.cpu().numpy()


@pytest.mark.parametrize("dims,bc_mode", [((64, 96, 64), 0), ((48, 40, 32), 1)])
def test_one_rank_equals_the_library_vcycles(dims, bc_mode):
    require_cuda()
    f, b, p = case(dims, 7)
    sp = slab.SlabPoisson(dims, H, bc_mode)
    sp.set_flags(torch.from_numpy(f.view(np.int32)).cuda())
    phi = torch.from_numpy(p).cuda()
    sp.vcycles(phi, torch.from_numpy(b).cuda(), 2)
    torch.cuda.synchronize()
    assert np.array_equal(phi.cpu().numpy(), single_domain(dims, 2, bc_mode))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, dims, cycles, bc_mode, q):
    sys.path[:0] = [ROOT, HERE]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    f, b, p = case(dims, 7)
    n = dims[2] // world
    own = slice(rank * n, (rank + 1) * n)
    sp = slab.SlabPoisson(dims, H, bc_mode)
    sp.set_flags(torch.from_numpy(f[own].view(np.int32).copy()).cuda())
    phi = torch.from_numpy(p[own].copy()).cuda()
    sp.vcycles(phi, torch.from_numpy(b[own].copy()).cuda(), cycles)
    torch.cuda.synchronize()
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, phi.cpu().numpy(), sp.lg))


@pytest.mark.parametrize("dims,bc_mode", [((64, 96, 64), 0), ((48, 40, 32), 1)])
def test_two_ranks_on_one_gpu_equal_the_library_vcycles(dims, bc_mode):
    require_cuda()
    world, cycles = 2, 2
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
    assert res[0][1] > 0  # some levels ran on slabs
    got = np.concatenate([res[r][0] for r in range(world)], 0)
    assert np.array_equal(got, single_domain(dims, cycles, bc_mode))


def test_operator_apply_against_the_oracle_operator():
    require_cuda()
    from slab_oracle_ops import OracleOps
    lib = _abi.load()
    dims = (40, 24, 16)
    f, b, p = case(dims, 5)
    for bc_mode in (0, 1):
        fd = torch.from_numpy(f.view(np.int32)).cuda()
        pd = torch.from_numpy(p).cuda()
        qd = torch.zeros_like(pd)
        assert lib.pyro_k_mg_apply(*dims, 0.1, fd.data_ptr(), pd.data_ptr(), qd.data_ptr(),
                                   bc_mode, None) == 0
        want = torch.zeros((dims[2], dims[1], dims[0]))
        OracleOps(bc_mode).apply(dims, 0.1, torch.from_numpy(f.view(np.int32)),
                                 torch.from_numpy(p), want)
        got = qd.cpu().numpy()
        assert np.allclose(got, want.numpy(), rtol=1e-6, atol=1e-6 * np.abs(got).max())


def _rank_cg(rank, world, port, dims, q):
    sys.path[:0] = [ROOT, HERE]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch.distributed as dist
    from test_slab import cg_case
    if world > 1:
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=120))
    f, b, _ = cg_case(dims, 11)
    n = dims[2] // world
    own = slice(rank * n, (rank + 1) * n)
    sp = slab.SlabPoisson(dims, H, 0)
    sp.set_flags(torch.from_numpy(f[own].view(np.int32).copy()).cuda())
    phi = torch.zeros((n, dims[1], dims[0]), dtype=torch.float32, device="cuda")
    it, rel = sp.mgpcg(phi, torch.from_numpy(b[own].copy()).cuda(), 1e-6, 50)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    q.put((rank, phi.cpu().numpy(), it, rel))


def test_slab_mgpcg_on_one_and_two_ranks():
    require_cuda()
    import oracle
    from test_slab import cg_case
    dims = (64, 96, 64)
    runs = {}
    for w in (1, 2):
        ctx = mp.get_context("spawn")
        q = ctx.Queue()
        port = _free_port()
        procs = [ctx.Process(target=_rank_cg, args=(r, w, port, dims, q)) for r in range(w)]
        for pr in procs:
            pr.start()
        res = dict((r, (phi, it, rel)) for r, phi, it, rel in (q.get(timeout=300) for _ in procs))
        for pr in procs:
            pr.join(timeout=60)
        assert all(pr.exitcode == 0 for pr in procs)
        runs[w] = (np.concatenate([res[r][0] for r in range(w)], 0), res[0][1], res[0][2])
    f, b, _ = cg_case(dims, 11)
    for w, (phi, it, rel) in runs.items():
        assert rel <= 1e-6, (w, it, rel)
        assert oracle.poisson_relres(dims, H, phi, b, f) <= 2e-6
    assert np.abs(runs[2][0] - runs[1][0]).max() <= 1e-4 * np.abs(runs[1][0]).max()
