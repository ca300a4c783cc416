"""CPU oracle: internal consistency of the restatement (no GPU).

The oracle is pinned to the reference by tests/test_golden.py (golden
vectors from interpreting the reference's own WGSL); these tests check its
host schedule and the FP64 pressure oracle.
"""
import numpy as np

import oracle
from fields import params_for, random_state, scene_for


def test_level_rule_matches_reference_examples():
    # src/sim.rs:142-168 examples
    assert oracle.mg_levels(160, 320, 160) == [(160, 320, 160), (80, 160, 80), (40, 80, 40),
                                               (20, 40, 20)]
    assert oracle.mg_levels(32, 80, 32) == [(32, 80, 32), (16, 40, 16), (8, 20, 8)]
    assert oracle.mg_levels(256, 256, 256)[-1] == (32, 32, 32)
    assert oracle.mg_levels(150, 365, 150) == [(150, 365, 150), (75, 183, 75), (38, 92, 38),
                                               (19, 46, 19)]
    assert oracle.mg_levels(12, 40, 40) == [(12, 40, 40)]


def _poisson_case(nx, ny, nz, seed=0, solid=0.05):
    rng = np.random.default_rng(seed)
    f = (rng.random((nz, ny, nx)) < solid).astype(np.uint32)
    b = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    b[f == 1] = 0
    return f, b


def test_vcycle_reduces_residual_and_f64_solve_converges():
    dims = (32, 48, 32)
    f, b = _poisson_case(*dims)
    h = 0.05
    phi0 = np.zeros((dims[2], dims[1], dims[0]), np.float32)
    r0 = oracle.poisson_relres(dims, h, phi0, b, f)
    assert abs(r0 - 1.0) < 1e-12
    rels = []
    phi = phi0
    for _ in range(4):
        phi = oracle.vcycles(dims, h, phi, b, f, 1)
        rels.append(oracle.poisson_relres(dims, h, phi, b, f))
    assert rels[0] < 0.3 and all(rels[i + 1] < rels[i] for i in range(3)), rels
    x, it, rel = oracle.poisson_f64(dims, h, b, f, tol=1e-12)
    assert rel < 1e-10, (it, rel)
    # the V-cycle converges toward the FP64 solution
    err = np.abs(phi - x).max() / np.abs(x).max()
    assert err < 0.05, err


def test_smoother_colours_are_independent():
    dims = (16, 20, 18)
    f, b = _poisson_case(*dims, seed=3)
    p = np.random.default_rng(4).normal(0, 1, (18, 20, 16)).astype(np.float32)
    a = oracle.mg_smooth(dims, 0.1, b, f, p, 0, 1.0)
    # cells of colour 1 unchanged by the colour-0 pass
    z, y, x = np.meshgrid(np.arange(18), np.arange(20), np.arange(16), indexing="ij")
    col1 = ((x + y + z) & 1) == 1
    assert np.array_equal(a[col1], p[col1])
    assert not np.array_equal(a[~col1 & (f == 0)], p[~col1 & (f == 0)])


def test_restrict_and_prolong_shapes_and_flags():
    dims = (17, 33, 9)
    f, b = _poisson_case(*dims, seed=5, solid=0.3)
    p = np.zeros((9, 33, 17), np.float32)
    bc, pc, fc = oracle.mg_restrict(dims, 0.1, p, b, f)
    assert bc.shape == (5, 17, 9)
    assert np.all(pc == 0)
    # a coarse cell is solid iff all its in-domain children are solid
    for (z, y, x) in [(0, 0, 0), (4, 16, 8), (2, 7, 3)]:
        ch = f[2 * z:2 * z + 2, 2 * y:2 * y + 2, 2 * x:2 * x + 2]
        assert fc[z, y, x] == (1 if ch.min() == 1 else 0)
    pf = oracle.mg_prolong(dims, np.ones_like(bc), f, np.zeros_like(p), fc)
    fluid = f == 0
    # a constant coarse correction prolongs to the same constant
    touched = pf[fluid] != 0
    assert np.allclose(pf[fluid][touched], 1.0, atol=1e-6)


def test_whole_step_runs_and_conserves_layout():
    P = params_for(24, 32, 20, dx=0.05, dt=0.004)
    st = random_state(P, seed=1, vmax=3.0)
    sim = oracle.OracleSim(P, st["sol"], 4)
    sim.write_field(oracle.F_S0, st["s0"])
    for k in range(3):
        sim.step(0.004, 0.004 * k, 1.0, k == 2)
    s0 = sim.read_field(oracle.F_S0)
    s1 = sim.read_field(oracle.F_S1)
    assert np.isfinite(s0).all() and np.isfinite(s1).all()
    assert s0[..., 0].min() >= 250.0 and s0[..., 0].max() <= 2600.0
    stats = sim.read_stats()
    assert stats[4] > 0 and stats[11] > 0


def test_quiescent_scene_stays_quiescent_without_ignition():
    sc = scene_for(16, 32, 16, dx=0.1)
    sc.ignition = None
    P = sc.params()
    sol = np.zeros((16, 32, 16, 4), np.float32)
    sol[..., 3] = P.t0
    sim = oracle.OracleSim(P, sol, 4)
    for k in range(3):
        sim.step(0.01, 0.01 * k, 0.0, True)
    s0 = sim.read_field(oracle.F_S0)
    assert np.allclose(s0[..., 0], P.t0)
    assert np.abs(sim.read_field(oracle.F_V)).max() < 1e-6


def test_f16_conversion_matches_ieee_round_to_nearest_even():
    """The oracle's binary32 -> binary16 conversion (the renderer's texture
    stores) against numpy's, which rounds to nearest even: normal,
    subnormal and overflowing values, the ties at both ends of the range."""
    rng = np.random.default_rng(3)
    x = np.concatenate([
        rng.normal(0, 1, 100000), rng.normal(0, 1e4, 100000), rng.normal(0, 1e-5, 100000),
        np.array([65504, 65519.99, 65520, 65535, 1e6, -1e6, 5.96e-8, 2.98e-8, 2.9802322e-08,
                  2.9802326e-08, 1e-9, 0.0, -0.0, 6.1035156e-05, 6.1e-05, np.inf, -np.inf]),
    ]).astype(np.float32)
    with np.errstate(over="ignore"):
        ref = x.astype(np.float16).view(np.uint16)
    assert np.array_equal(oracle.f32_to_f16(x), ref)
    # ties: halfway between two binary16 values rounds to the even one
    lo = np.arange(0x3c00, 0x3c40, dtype=np.uint16).view(np.float16).astype(np.float64)
    mid = ((lo[:-1] + lo[1:]) / 2).astype(np.float32)
    assert np.array_equal(oracle.f32_to_f16(mid), mid.astype(np.float16).view(np.uint16))
    bits = np.arange(65536, dtype=np.uint16)
    fin = np.isfinite(bits.view(np.float16))
    assert np.array_equal(oracle.f16_to_f32(bits)[fin], bits.view(np.float16).astype(np.float32)[fin])
