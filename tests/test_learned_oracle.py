"""CPU checks of the learned stage: the float64 oracle's analytic gradient
against central finite differences, the adjoint pairs it is built from, and
the keep-or-discard rule of the solver (pyro_learned_accept) on injected bad
warm starts (NaN, zeros, noise) with the dot products formed on the host."""
import numpy as np
import pytest

from oracle import learned as L


def _case(seed, nb=2, dims=(5, 6, 7)):
    rng = np.random.default_rng(seed)
    nz, ny, nx = dims
    flags = (rng.random((nb, nz, ny, nx)) < 0.15).astype(np.uint32)
    b = rng.normal(0, 1, (nb, nz, ny, nx)) * 3.0
    phi = rng.normal(0, 1, (nb, nz, ny, nx)) * 0.02
    return b, flags, phi


def test_adjoint_pairs():
    rng = np.random.default_rng(1)
    x = rng.normal(size=(2, 5, 6, 7, 8))
    c = rng.normal(size=(2, 3, 3, 4, 8))
    # <up(c), x> = <c, up_back(x)>
    assert np.isclose((L.up(c, x.shape) * x).sum(), (c * L.up_back(x, c.shape)).sum())
    # <pool(x), c> = <x, pool_back(c)>
    assert np.isclose((L.pool(x) * c).sum(), (x * L.pool_back(c, x.shape)).sum())
    # pooling a constant keeps it
    assert np.allclose(L.pool(np.ones_like(x)), 1.0)
    # conv adjoint: <conv(x), y> = <x, conv^T(y)>, and dw by linearity
    w = rng.normal(size=(4, 27, 8))
    y = rng.normal(size=(2, 5, 6, 7, 4))
    dx, dw, db = L.conv3_back(x, w, y)
    assert np.isclose((L.conv3(x, w, np.zeros(4)) * y).sum(), (x * dx).sum())
    assert np.isclose((L.conv3(x, w, np.zeros(4)) * y).sum(), (w * dw).sum())
    assert np.allclose(db, y.reshape(-1, 4).sum(0))


def test_conv_tap_order():
    # tap t = (dz+1)*9 + (dy+1)*3 + (dx+1) reads x[z+dz][y+dy][x+dx]
    x = np.zeros((1, 3, 3, 3, 1))
    x[0, 2, 1, 0, 0] = 1.0          # z=2, y=1, x=0
    w = np.zeros((1, 27, 1))
    w[0, (1 + 1) * 9 + (0 + 1) * 3 + (-1 + 1), 0] = 1.0   # dz=+1, dy=0, dx=-1
    y = L.conv3(x, w, np.zeros(1))
    assert y[0, 1, 1, 1, 0] == 1.0 and y.sum() == 1.0


@pytest.mark.parametrize("dims,w_phi,w_res,scale", [((5, 6, 7), 1.0, 0.0, 1.0),
                                                     ((4, 4, 8), 1.0, 0.0, 1.0),
                                                     ((5, 6, 7), 0.0, 1.0, 2.0),
                                                     ((6, 5, 6), 0.3, 2.0, 0.5)])
def test_gradient_finite_differences(dims, w_phi, w_res, scale):
    b, flags, phi = _case(2, dims=dims)
    p = L.init_params(3)
    p[L.n_params() - 40:] = np.random.default_rng(4).normal(0, 0.05, 40)  # non-zero biases
    h = 0.05
    kw = dict(w_phi=w_phi, w_res=w_res)
    loss, g = L.loss_grad(p, b, flags, phi, h, scale, **kw)
    assert np.isfinite(loss) and loss > 0
    rng = np.random.default_rng(5)
    # a few entries of every layer's weights and of the biases
    ws_off = np.cumsum([0] + [co * 27 * ci for ci, co, _, _ in L.SPEC])
    idx = [int(rng.integers(ws_off[l], ws_off[l + 1])) for l in range(9) for _ in range(3)]
    idx += [int(i) for i in rng.integers(ws_off[-1], L.n_params(), 6)]
    eps = 1e-6
    for i in idx:
        pp = p.copy()
        pp[i] += eps
        lp = L.loss(pp, b, flags, phi, h, scale, **kw)
        pp[i] -= 2 * eps
        lm = L.loss(pp, b, flags, phi, h, scale, **kw)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g).max()) + 1e-4 * abs(fd), (i, fd, g[i])


def test_residual_loss_is_the_solver_residual():
    """res of the loss = (b - A phi) / rms(b) for phi = the prediction,
    with A the pressure operator (fluid neighbours, no Dirichlet faces
    inside the volume)."""
    b, flags, _ = _case(9, nb=1, dims=(6, 7, 8))
    p = L.init_params(10)
    h, scale = 0.05, 3.0
    phi = L.predict(p, b, flags, h, scale)
    fl = (flags != 1).astype(np.float64)
    Aphi = L._lap(phi, fl) / (h * h)
    s = L._vol_rms(b, flags)[0][0]
    interior = np.zeros(b.shape, bool)
    interior[:, 1:-1, 1:-1, 1:-1] = True
    interior &= flags != 1
    ref = np.mean(((b - Aphi) / s)[interior] ** 2)
    got = L.loss(p, b, flags, np.zeros_like(b), h, scale, w_phi=0.0, w_res=1.0)
    assert np.isclose(got, ref, rtol=1e-6)


def test_scale_invariance():
    """The prediction scales with b (the Poisson solution is linear)."""
    b, flags, _ = _case(6, nb=1)
    p = L.init_params(7)
    y1 = L.predict(p, b, flags, 0.1)
    y2 = L.predict(p, 4.0 * b, flags, 0.1)
    assert np.allclose(y2, 4.0 * y1)
    assert np.all(y1[flags == 1] == 0.0)


def test_bf16_rounding():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 1e-3, 0.0])
    r = L.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0          # tie to even
    assert r[2] == 1.0 + 2 ** -7                # above the tie rounds up
    assert r[3] == -2.5 and r[5] == 0.0
    assert abs(r[4] - 1e-3) <= 1e-3 * 2 ** -8


# ---------------------------------------------------------------- fallback
def _poisson_1d(n, h=0.1):
    """A small negative-definite operator like the pressure system."""
    A = np.zeros((n, n))
    for i in range(n):
        A[i, i] = -2.0
        if i > 0:
            A[i, i - 1] = 1.0
        if i < n - 1:
            A[i, i + 1] = 1.0
    return A / (h * h)


def _decide(A, r, e):
    from pyro_b200.learned import learned_accept
    with np.errstate(invalid="ignore", over="ignore"):
        Ae = A @ e
        dots = (float(r @ e), float(e @ Ae), float(r @ Ae), float(Ae @ Ae), float(r @ r))
    return learned_accept(*dots)


def test_fallback_rule_on_injected_warm_starts():
    rng = np.random.default_rng(8)
    A = _poisson_1d(64)
    r = rng.normal(size=64)
    exact = np.linalg.solve(A, r)
    # the exact correction is kept with alpha 1 and residual ~0
    keep, a, rr = _decide(A, r, exact)
    assert keep and abs(a - 1.0) < 1e-9 and rr < 1e-12 * (r @ r)
    # NaN and all-zero corrections are discarded
    keep, a, rr = _decide(A, r, np.full(64, np.nan))
    assert not keep and a == 0.0 and rr == r @ r
    keep, a, rr = _decide(A, r, np.zeros(64))
    assert not keep and rr == r @ r
    # noise: whatever is decided, a kept correction really lowers |r|
    for s in range(20):
        e = np.random.default_rng(100 + s).normal(size=64)
        keep, a, rr = _decide(A, r, e)
        true = float(np.sum((r - a * (A @ e)) ** 2))
        if keep:
            assert true < r @ r and np.isclose(true, rr, rtol=1e-8)
        else:
            assert rr == r @ r
    # a correction of the wrong sign still gets the optimal (negative) alpha
    keep, a, rr = _decide(A, r, -exact)
    assert keep and abs(a + 1.0) < 1e-9
    # infinities are discarded
    assert not _decide(A, r, np.full(64, np.inf))[0]
