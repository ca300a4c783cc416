"""CPU oracle of the learned pressure stage (test infrastructure only).

A float64 NumPy restatement of the network of pyro_b200/csrc/net.h and
net.cu: forward pass, mean-squared loss and its analytic backward pass.
Only tests may import it: the product computes on the GPU.

The network has no counterpart in the reference (it is an addition beside
the multigrid solve of src/sim.rs:451-491), so nothing external pins it.
This oracle is pinned by central finite differences of its own loss
(tests/test_learned_oracle.py), and the GPU gradients are compared with it.

    bf16=True rounds to bfloat16 (round to nearest even) wherever the GPU
    stores BF16: the network input, every convolution output but the last,
    the pooled maps, the loss gradient and every back-propagated map.

Layout: volumes (nb, nz, ny, nx); activations (nb, nz, ny, nx, C); weights
[Cout][27][Cin] with tap t = (dz+1)*9 + (dy+1)*3 + (dx+1); parameters flat:
all weights (layers in order), then all biases.
"""
from __future__ import annotations

import numpy as np

# (cin, cout, level, relu) of conv1 .. conv9
SPEC = [(2, 16, 0, 1), (16, 16, 0, 1), (16, 32, 1, 1), (32, 32, 1, 1), (32, 64, 2, 1),
        (64, 64, 2, 1), (96, 32, 1, 1), (48, 16, 0, 1), (16, 1, 0, 0)]


def n_params() -> int:
    return sum(co * 27 * ci + co for ci, co, _, _ in SPEC)


def unpack(p: np.ndarray):
    p = np.asarray(p, np.float64)
    ws, bs, o = [], [], 0
    for ci, co, _, _ in SPEC:
        n = co * 27 * ci
        ws.append(p[o:o + n].reshape(co, 27, ci))
        o += n
    for ci, co, _, _ in SPEC:
        bs.append(p[o:o + co])
        o += co
    return ws, bs


def pack(ws, bs) -> np.ndarray:
    return np.concatenate([w.ravel() for w in ws] + [b.ravel() for b in bs])


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def _taps():
    for t in range(27):
        yield t, t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1


def _shift(xp, dx, dy, dz, nz, ny, nx):
    return xp[:, 1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx, :]


def conv3(x, w, b):
    """y[v][co] = sum_t,ci w[co][t][ci] x[v + tap(t)][ci] + b[co] (zero outside)."""
    nb, nz, ny, nx, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((nb, nz, ny, nx, w.shape[0]))
    for t, dx, dy, dz in _taps():
        y += _shift(xp, dx, dy, dz, nz, ny, nx) @ w[:, t, :].T
    return y + b


def conv3_back(x, w, dy):
    """(dx, dw, db) of conv3 for the output gradient dy."""
    nb, nz, ny, nx, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    flat = dy.reshape(-1, dy.shape[-1])
    for t, ox, oy, oz in _taps():
        xs = _shift(xp, ox, oy, oz, nz, ny, nx)
        dw[:, t, :] = flat.T @ xs.reshape(-1, xs.shape[-1])
        _shift(dxp, ox, oy, oz, nz, ny, nx)[...] += dy @ w[:, t, :]
    return dxp[:, 1:-1, 1:-1, 1:-1, :], dw, flat.sum(0)


def _half(shape):
    nb, nz, ny, nx = shape[:4]
    return (nb, (nz + 1) // 2, (ny + 1) // 2, (nx + 1) // 2)


def _counts(fine):
    """children per coarse cell, broadcast to the fine grid"""
    nb, nz, ny, nx = fine[:4]
    cz = np.minimum(2, nz - 2 * np.arange((nz + 1) // 2))
    cy = np.minimum(2, ny - 2 * np.arange((ny + 1) // 2))
    cx = np.minimum(2, nx - 2 * np.arange((nx + 1) // 2))
    return cz[:, None, None] * cy[None, :, None] * cx[None, None, :]


def up(x, fine):
    """nearest up-sampling of (nb, cz, cy, cx, C) to the fine shape"""
    _, nz, ny, nx = fine[:4]
    return x.repeat(2, 1).repeat(2, 2).repeat(2, 3)[:, :nz, :ny, :nx]


def up_back(g, coarse):
    """adjoint of up: sum of the children"""
    nb, cz, cy, cx = coarse[:4]
    nz, ny, nx = g.shape[1:4]
    gp = np.zeros((nb, 2 * cz, 2 * cy, 2 * cx, g.shape[-1]))
    gp[:, :nz, :ny, :nx] = g
    return gp.reshape(nb, cz, 2, cy, 2, cx, 2, -1).sum((2, 4, 6))


def pool(x):
    """mean of the children inside the volume"""
    c = _half(x.shape)
    return up_back(x, c) / _counts(x.shape)[None, :, :, :, None]


def pool_back(g, fine):
    return up(g / _counts(fine)[None, :, :, :, None], fine)


def _vol_rms(b, flags):
    fl = flags != 1
    n = fl.reshape(fl.shape[0], -1).sum(1).astype(np.float64)
    s2 = (np.where(fl, b.astype(np.float64), 0.0) ** 2).reshape(b.shape[0], -1).sum(1)
    return np.where((n > 0) & (s2 > 0), np.sqrt(s2 / np.maximum(n, 1)), 0.0), n


def forward(p, b, flags, bf=False):
    """Network output (nb, nz, ny, nx) and the cache for backward."""
    r = bf16 if bf else (lambda a: a)
    ws, bs = unpack(p)
    if bf:
        ws = [bf16(w) for w in ws]
    b = np.asarray(b, np.float64)
    flags = np.asarray(flags)
    s, n = _vol_rms(b, flags)
    solid = flags == 1
    inv = np.where(s > 0, 1.0 / np.where(s > 0, s, 1.0), 0.0)[:, None, None, None]
    xin = np.stack([np.where(solid, 0.0, b * inv), solid.astype(np.float64)], -1)
    xin = r(xin)

    def cv(x, l):
        y = conv3(x, ws[l], bs[l])
        if SPEC[l][3]:
            y = np.maximum(y, 0.0)
        return r(y) if l < 8 else y

    c = {"in0": xin, "ws": ws, "s": s, "n": n, "flags": flags}
    c["e0a"] = cv(xin, 0)
    c["e0"] = cv(c["e0a"], 1)
    c["p1"] = r(pool(c["e0"]))
    c["e1a"] = cv(c["p1"], 2)
    c["e1"] = cv(c["e1a"], 3)
    c["p2"] = r(pool(c["e1"]))
    c["e2a"] = cv(c["p2"], 4)
    c["e2"] = cv(c["e2a"], 5)
    c["c1"] = np.concatenate([up(c["e2"], c["e1"].shape), c["e1"]], -1)
    c["d1"] = cv(c["c1"], 6)
    c["c0"] = np.concatenate([up(c["d1"], c["e0"].shape), c["e0"]], -1)
    c["d0"] = cv(c["c0"], 7)
    if bf:  # the last layer's output is FP32 on the GPU
        c["out"] = conv3(c["d0"], ws[8], bs[8])[..., 0].astype(np.float32).astype(np.float64)
    else:
        c["out"] = conv3(c["d0"], ws[8], bs[8])[..., 0]
    return c["out"], c


def predict(p, b, flags, h, out_scale=1.0, bf=False):
    """phi = out * out_scale * rms(b) * h^2 on fluid cells, 0 in solids."""
    out, c = forward(p, b, flags, bf)
    s = c["s"][:, None, None, None]
    return np.where(np.asarray(flags) == 1, 0.0, out * out_scale * s * h * h)


def _lap(q, fluid):
    """(L q)_i = sum over in-volume fluid neighbours j of q_j - their count
    * q_i on fluid cells, 0 on solids (the solver's operator times h^2)."""
    s = np.zeros_like(q)
    c = np.zeros_like(q)
    for ax in (1, 2, 3):
        for sh in (1, -1):
            qs = np.zeros_like(q)
            fs = np.zeros_like(q)
            src = [slice(None)] * 4
            dst = [slice(None)] * 4
            if sh == 1:
                src[ax], dst[ax] = slice(1, None), slice(0, -1)
            else:
                src[ax], dst[ax] = slice(0, -1), slice(1, None)
            qs[tuple(dst)] = q[tuple(src)]
            fs[tuple(dst)] = fluid[tuple(src)]
            s += qs * fs
            c += fs
    return np.where(fluid > 0, s - c * q, 0.0)


def loss(p, b, flags, phi_t, h, out_scale=1.0, bf=False, w_phi=1.0, w_res=0.0):
    return loss_grad(p, b, flags, phi_t, h, out_scale, bf, grad=False, w_phi=w_phi,
                     w_res=w_res)[0]


def loss_grad(p, b, flags, phi_t, h, out_scale=1.0, bf=False, grad=True, w_phi=1.0, w_res=0.0):
    """(loss, d loss / d params) with loss =
      w_phi * mean over fluid cells of (out - phi_t / (out_scale rms(b) h^2))^2
    + w_res * mean over the fluid cells with all six neighbours inside the
      volume of res^2, res = b / rms(b) - out_scale * L(out)."""
    r = bf16 if bf else (lambda a: a)
    out, c = forward(p, b, flags, bf)
    fl = c["flags"] != 1
    scale = (c["s"] * out_scale * h * h)[:, None, None, None]
    t = np.where(scale > 0, np.asarray(phi_t, np.float64) / np.where(scale > 0, scale, 1.0), 0.0)
    ntot = c["n"].sum()
    inv_n = 1.0 / ntot if ntot > 0 else 0.0
    d = np.where(fl, out - t, 0.0)
    L = float(w_phi * (d * d).sum() * inv_n)
    gout = 2.0 * w_phi * d * inv_n
    if w_res > 0:
        s = c["s"][:, None, None, None]
        bh = np.where(s > 0, np.asarray(b, np.float64) / np.where(s > 0, s, 1.0), 0.0)
        bh = bh.astype(np.float32).astype(np.float64)
        interior = np.zeros_like(fl)
        interior[:, 1:-1, 1:-1, 1:-1] = True
        interior &= fl
        fluid = fl.astype(np.float64)
        res = np.where(interior, bh - out_scale * _lap(out, fluid), 0.0)
        if bf:
            res = res.astype(np.float32).astype(np.float64)
        nres = interior.sum()
        if nres > 0:
            L += float(w_res * (res * res).sum() / nres)
            gout = gout - 2.0 * out_scale * w_res / nres * _lap(res, fluid)
    if not grad:
        return L, None
    ws = c["ws"]
    gw = [None] * 9
    gb = [None] * 9
    g9 = r(gout)[..., None]
    relu = lambda g, a: np.where(a > 0, g, 0.0)  # noqa: E731

    def back(x, l, g, act):
        dx, gw[l], gb[l] = conv3_back(x, ws[l], g)
        return None if act is None else r(relu(dx, act)) if act is not False else r(dx)

    g8 = back(c["d0"], 8, g9, c["d0"])
    gc0 = back(c["c0"], 7, g8, c["c0"])
    g7 = r(up_back(gc0[..., :32], c["d1"].shape))
    gc1 = back(c["c1"], 6, g7, c["c1"])
    g6 = r(up_back(gc1[..., :64], c["e2"].shape))
    g5 = back(c["e2a"], 5, g6, c["e2a"])
    gp2 = back(c["p2"], 4, g5, False)
    g4 = r(relu(pool_back(gp2, c["e1"].shape) + gc1[..., 64:], c["e1"]))
    g3 = back(c["e1a"], 3, g4, c["e1a"])
    gp1 = back(c["p1"], 2, g3, False)
    g2 = r(relu(pool_back(gp1, c["e0"].shape) + gc0[..., 32:], c["e0"]))
    g1 = back(c["e0a"], 1, g2, c["e0a"])
    back(c["in0"], 0, g1, None)
    return L, pack(gw, gb)


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights (last layer x0.1), zero biases; float64."""
    rng = np.random.default_rng(seed)
    ws, bs = [], []
    for ci, co, _, relu in SPEC:
        sd = np.sqrt(2.0 / (27.0 * ci)) * (1.0 if relu else 0.1)
        ws.append(rng.normal(0.0, sd, (co, 27, ci)))
        bs.append(np.zeros(co))
    return pack(ws, bs)
