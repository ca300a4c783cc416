"""Seeded synthetic simulation states for the parity tests.

Values span the ranges a burning scene reaches (temperatures to 2200 K,
fuel and soot fractions, velocities of several cells per substep so that
traces leave the domain) and include every solid kind of the material
table: charring (wood), liquid pool (heptane), non-charring (pmma) and inert
(steel), with some cells just above and below the burnout threshold.
"""
import numpy as np

from pyro_b200 import _abi
from pyro_b200.scene import Domain, Ignition, Object, Scene, SimCfg, Wind


def scene_for(nx, ny, nz, dx=0.05, wind=0.0):
    sc = Scene(domain=Domain([nx * dx, ny * dx, nz * dx], dx),
               sim=SimCfg(vorticity=6.0),
               wind=Wind(speed=wind, dir=30.0),
               ignition=Ignition(pos=[0.5 * nx * dx, 0.1, 0.5 * nz * dx], radius=0.3,
                                 flux=30000.0, temp=1300.0, until=4.0, fuel=0.01),
               objects=[Object(kind="pool", material="heptane", center=[0.3, 0.0, 0.3],
                               radius=0.2, depth=0.05),
                        Object(kind="box", material="wood", center=[0.5, 0.3, 0.5],
                               size=[0.2, 0.1, 0.2]),
                        Object(kind="box", material="pmma", center=[0.2, 0.4, 0.6],
                               size=[0.1, 0.1, 0.1]),
                        Object(kind="box", material="steel", center=[0.6, 0.2, 0.2],
                               size=[0.1, 0.1, 0.1])])
    sc.dims_override = [nx, ny, nz]
    return sc


def params_for(nx, ny, nz, dx=0.05, dt=0.01, ign_on=1.0, wind=0.0, sponge=None):
    P = scene_for(nx, ny, nz, dx, wind).params()
    P.dt = dt
    P.ign_on = ign_on
    if sponge is not None:
        P.sponge = sponge
    return P


def random_state(P, seed=0, vmax=6.0, solid_frac=0.12):
    """Dict of fields in the reference layout (z, y, x[, 4])."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = int(P.nx), int(P.ny), int(P.nz)
    n = (nz, ny, nx)
    nv = (nz + 1, ny + 1, nx + 1)
    t0 = P.t0
    # solids: slot 1 heptane, 2 wood, 3 pmma, 4 steel
    sol = np.zeros(n + (4,), np.float32)
    sol[..., 3] = t0
    solid = rng.random(n) < solid_frac
    slot = rng.integers(1, 5, size=n)
    dens = np.array([0.0, 684.0, 480.0, 1190.0, 7850.0], np.float32)
    mass = dens[slot] * rng.uniform(0.0, 1.15, size=n).astype(np.float32)
    near = rng.random(n) < 0.15
    mass = np.where(near, rng.uniform(0.5, 3.5, size=n), mass).astype(np.float32)
    chr_ = np.where(slot == 2, rng.uniform(0.0, 80.0, size=n), 0.0).astype(np.float32)
    chr_ = np.where(near & (slot == 2), rng.uniform(0.0, 1.0, size=n), chr_).astype(np.float32)
    ts = rng.uniform(290.0, 900.0, size=n).astype(np.float32)
    sol[..., 0] = np.where(solid, slot, 0)
    sol[..., 1] = np.where(solid, np.where(slot == 4, 1.0, mass), 0.0)
    sol[..., 2] = np.where(solid, chr_, 0.0)
    sol[..., 3] = np.where(solid, ts, t0)
    # a solid floor patch (a pool) so surface logic sees gas above
    sol[:nz // 3, 0, :nx // 3, 0] = 1
    sol[:nz // 3, 0, :nx // 3, 1] = 600.0
    sol[:nz // 3, 0, :nx // 3, 3] = rng.uniform(300, 372, size=(nz // 3, nx // 3))
    s0 = np.empty(n + (4,), np.float32)
    s0[..., 0] = rng.uniform(293.0, 2200.0, size=n)
    s0[..., 1] = rng.uniform(-0.01, 0.2, size=n)
    s0[..., 2] = rng.uniform(0.0, 0.24, size=n)
    s0[..., 3] = rng.uniform(-0.001, 0.02, size=n)
    s1 = np.zeros(n + (4,), np.float32)
    s1[..., 0] = rng.uniform(-0.001, 0.02, size=n)
    s1[..., 1] = rng.uniform(0.0, 2e6, size=n)
    s1[..., 2] = rng.uniform(-5.0, 5.0, size=n)

    def smooth_field(shape):
        a = rng.normal(0.0, 1.0, size=shape).astype(np.float32)
        for ax in range(3):
            a = 0.5 * a + 0.25 * (np.roll(a, 1, ax) + np.roll(a, -1, ax))
        a /= np.abs(a).max() + 1e-12
        return (vmax * a + rng.normal(0.0, 0.3, size=shape)).astype(np.float32)

    u, v, w = smooth_field(nv), smooth_field(nv), smooth_field(nv)
    curl = np.zeros(n + (4,), np.float32)
    curl[..., :3] = rng.normal(0.0, 40.0, size=n + (3,))
    curl[..., 3] = np.sqrt((curl[..., :3].astype(np.float32) ** 2).sum(-1))
    pyr = np.zeros(n + (4,), np.float32)
    pyr[..., 0] = np.where(rng.random(n) < 0.5, rng.uniform(0.0, 0.05, size=n), 0.0)
    pyr[..., 1] = np.where(rng.random(n) < 0.3, rng.uniform(0.0, 0.01, size=n), 0.0)
    pyr[..., 2] = rng.integers(0, 6, size=n)
    flags = (sol[..., 1] > 0.5).astype(np.uint32) * solid.astype(np.uint32)
    flags[:nz // 3, 0, :nx // 3] = 1
    phi = rng.normal(0.0, 1.0, size=n).astype(np.float32)
    b = rng.normal(0.0, 1.0, size=n).astype(np.float32)
    return dict(sol=sol, s0=s0, s1=s1, u=u, v=v, w=w, curl=curl, pyr=pyr, flags=flags,
                phi=phi, b=b)


def close(got, exp, rtol=1e-5, floor=1e-6, name=""):
    """|got - exp| <= rtol*|exp| + floor*max|exp| per trailing channel."""
    got = np.asarray(got, np.float64)
    exp = np.asarray(exp, np.float64)
    assert got.shape == exp.shape, (name, got.shape, exp.shape)
    if exp.ndim == 4:
        scale = np.abs(exp).reshape(-1, exp.shape[-1]).max(0)
    else:
        scale = np.abs(exp).max()
    tol = rtol * np.abs(exp) + floor * scale + 1e-30
    bad = np.abs(got - exp) > tol
    if bad.any():
        idx = np.argwhere(bad)[:5]
        det = [(tuple(i), float(got[tuple(i)]), float(exp[tuple(i)])) for i in idx]
        raise AssertionError(f"{name}: {int(bad.sum())} of {bad.size} values out of tolerance; "
                             f"first {det}")


def dims_of(P):
    return int(P.nx), int(P.ny), int(P.nz)


def face_valid_mask(P, k):
    """Valid positions of staggered component k in the padded face grid."""
    nx, ny, nz = dims_of(P)
    m = np.zeros((nz + 1, ny + 1, nx + 1), bool)
    hx, hy, hz = nx - 1 + (k == 0), ny - 1 + (k == 1), nz - 1 + (k == 2)
    m[:hz + 1, :hy + 1, :hx + 1] = True
    return m
