"""The learned pressure stage on the GPU against the float64 oracle
(oracle/learned.py): forward pass and gradients with BF16 rounding emulated
at the GPU's storage points, gradients against float64 central finite
differences, a short training run, and the solver's fallback when the
network's correction is useless (NaN or zero weights)."""
import numpy as np
import pytest
import torch

from gpu_util import dev, host, require_cuda
from oracle import learned as L
from pyro_b200 import _abi
from pyro_b200.learned import Net
from pyro_b200.poisson import PoissonSolver, poisson_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    return require_cuda()


def _case(seed, nb, dims):
    """b, flags, phi_t of shape (nb, nz, ny, nx); phi_t is another random
    network's prediction so that the loss is of order one."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = dims
    flags = (rng.random((nb, nz, ny, nx)) < 0.12).astype(np.uint32)
    b = (rng.normal(0, 1, (nb, nz, ny, nx)) * 5.0).astype(np.float32)
    b[flags == 1] = 0.0
    phi = L.predict(L.init_params(seed + 100), b, flags, 0.05, out_scale=1.0)
    phi += rng.normal(0, 0.3 * np.abs(phi).mean() + 1e-9, phi.shape)
    return b, flags, phi.astype(np.float32)


def _dev_case(b, flags, phi):
    return dev(b), dev(flags.astype(np.int32)), dev(phi)


def _net(seed, out_scale=1.0, w_phi=1.0, w_res=0.0):
    net = Net(seed=0)
    p = L.init_params(seed)
    rng = np.random.default_rng(seed + 1)
    p[L.n_params() - 273:] = rng.normal(0, 0.05, 273)     # non-zero biases
    net.set_params(p.astype(np.float32), out_scale)
    net.set_loss(w_phi, w_res)
    return net, net.get_params()[0].astype(np.float64)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("dims,nb", [((8, 12, 16), 2), ((5, 9, 7), 1)])
def test_forward_matches_oracle(lib, dims, nb):
    b, flags, _ = _case(1, nb, dims)
    net, p = _net(2)
    bd, fd, _ = _dev_case(b, flags, b)
    phi = torch.empty_like(bd)
    h = 0.05
    nz, ny, nx = dims
    net.forward(bd.data_ptr(), fd.data_ptr(), (nx, ny, nz), nb, h, phi.data_ptr())
    got = host(phi).astype(np.float64)
    ref = L.predict(p, b, flags, h, bf=True)
    assert np.all(got[flags == 1] == 0.0)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-2 * scale, np.abs(got - ref).max() / scale
    assert _rel(got, ref) < 5e-3
    # the float64 network without BF16 rounding is close too
    assert _rel(got, L.predict(p, b, flags, h)) < 5e-2


@pytest.mark.parametrize("w_phi,w_res,scale", [(1.0, 0.0, 1.0), (0.3, 2.0, 2.0)])
def test_gradient_matches_oracle_and_finite_differences(lib, w_phi, w_res, scale):
    dims, nb, h = (8, 8, 12), 2, 0.05
    b, flags, phi_t = _case(3, nb, dims)
    phi_t *= scale
    net, p = _net(4, scale, w_phi, w_res)
    kw = dict(w_phi=w_phi, w_res=w_res)
    bd, fd, pd = _dev_case(b, flags, phi_t)
    nz, ny, nx = dims
    loss, g = net.loss_grad(bd.data_ptr(), fd.data_ptr(), pd.data_ptr(), (nx, ny, nz), nb, h)
    g = g.astype(np.float64)
    loss_bf, g_bf = L.loss_grad(p, b, flags, phi_t, h, scale, bf=True, **kw)
    loss_64, g_64 = L.loss_grad(p, b, flags, phi_t, h, scale, **kw)
    assert abs(loss - loss_bf) <= 1e-3 * loss_bf, (loss, loss_bf)
    assert abs(loss - loss_64) <= 3e-2 * loss_64, (loss, loss_64)
    wo = np.cumsum([0] + [co * 27 * ci for ci, co, _, _ in L.SPEC])
    bo = wo[-1] + np.cumsum([0] + [co for _, co, _, _ in L.SPEC])
    for l in range(9):
        for sl in (slice(wo[l], wo[l + 1]), slice(bo[l], bo[l + 1])):
            assert _rel(g[sl], g_bf[sl]) < 2e-2, (l, _rel(g[sl], g_bf[sl]))
            assert _rel(g[sl], g_64[sl]) < 1e-1, (l, _rel(g[sl], g_64[sl]))
    # float64 central differences on sampled entries of every layer
    rng = np.random.default_rng(5)
    idx = [int(rng.integers(wo[l], wo[l + 1])) for l in range(9) for _ in range(3)]
    idx += [int(i) for i in rng.integers(wo[-1], L.n_params(), 8)]
    eps = 1e-5
    fd_g, gpu_g = [], []
    for i in idx:
        pp = p.copy()
        pp[i] += eps
        lp = L.loss(pp, b, flags, phi_t, h, scale, **kw)
        pp[i] -= 2 * eps
        lm = L.loss(pp, b, flags, phi_t, h, scale, **kw)
        fd_g.append((lp - lm) / (2 * eps))
        gpu_g.append(g[i])
    fd_g, gpu_g = np.array(fd_g), np.array(gpu_g)
    err = np.abs(fd_g - gpu_g)
    assert np.all(err <= 0.05 * np.abs(fd_g).max() + 0.1 * np.abs(fd_g)), (fd_g, gpu_g)
    assert _rel(gpu_g, fd_g) < 0.05


@pytest.mark.parametrize("w_phi,w_res", [(1.0, 0.0), (0.0, 1.0)])
def test_training_lowers_loss(lib, w_phi, w_res):
    dims, nb, h = (16, 16, 16), 2, 0.05
    b, flags, phi_t = _case(6, nb, dims)
    net, _ = _net(7, 1.0, w_phi, w_res)
    bd, fd, pd = _dev_case(b, flags, phi_t)
    nz, ny, nx = dims
    l0, _ = net.loss_grad(bd.data_ptr(), fd.data_ptr(), pd.data_ptr(), (nx, ny, nz), nb, h,
                          want_grad=False)
    for _ in range(150):
        net.train_step(bd.data_ptr(), fd.data_ptr(), pd.data_ptr(), (nx, ny, nz), nb, h,
                       lr=2e-3, clip=10.0)
    l1 = net.last_loss()
    assert np.isfinite(l1) and l1 < 0.4 * l0, (l0, l1)
    # weights round-trip through a file
    import os
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "w.pnet")
        net.save(path)
        p2, s2 = Net.read_file(path)
        p1, s1 = net.get_params()
        assert np.array_equal(p1, p2) and s1 == s2


def _solve(ps, bd, phi, mode, tol=1e-4, iters=60):
    phi.zero_()
    torch.cuda.synchronize()
    return ps.solve(bd.data_ptr(), phi.data_ptr(), mode, tol, iters)


@pytest.mark.parametrize("bc", [0, 1])
def test_solver_fallback_on_useless_networks(lib, bc):
    n = 40
    f, b = poisson_case(n, n, n, seed=3)
    ps = PoissonSolver((n, n, n), 0.05, bc_mode=bc)
    fd = dev(f.astype(np.int32))
    ps.set_flags(fd.data_ptr())
    bd = dev(b)
    phi = torch.zeros_like(bd)
    with pytest.raises(_abi.PyroError):          # no network attached
        _solve(ps, bd, phi, _abi.SOLVER_MGPCG_LEARNED)
    base = _solve(ps, bd, phi, _abi.SOLVER_MGPCG_BF16)
    assert base.converged and base.learned == -1
    net = Net(seed=1)
    ps.set_net(net)
    for params in (np.full(net.n_params, np.nan, np.float32),
                   np.zeros(net.n_params, np.float32)):
        net.set_params(params, 1.0)
        info = _solve(ps, bd, phi, _abi.SOLVER_MGPCG_LEARNED)
        assert info.learned == 0
        assert info.rel_resid_learned == info.rel_resid_start == pytest.approx(1.0, abs=1e-12)
        assert info.converged and info.iterations == base.iterations
        assert np.all(np.isfinite(host(phi)))
    # an untrained network: kept only if it lowers the residual
    net.set_params(L.init_params(9).astype(np.float32), 1.0)
    info = _solve(ps, bd, phi, _abi.SOLVER_MGPCG_LEARNED)
    assert info.learned in (0, 1) and info.converged
    assert info.rel_resid_learned <= info.rel_resid_start
    if info.learned == 1:
        assert info.rel_resid_learned < 1.0
    ps.set_net(None)
    ps.close()
