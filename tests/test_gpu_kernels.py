"""Per-kernel parity of the CUDA kernels against the CPU oracle on
identical seeded inputs, through the C ABI.

Kernels without transcendental functions keep the reference's FP32
expression order on both sides (the library is built with --fmad=false, the
oracle with -ffp-contract=off), so their outputs must agree bit for bit;
kernels calling exp() (solid, react, forces) agree within 1e-5 relative with
an absolute floor of 1e-6 of each channel's magnitude.  Masks (flags,
coarse flags) are bit-exact.  Statistics are float atomics on the GPU and
FP64 sums in the oracle: 1e-4 relative.
"""
import numpy as np
import pytest

import oracle
from fields import close, face_valid_mask, params_for, random_state
from gpu_util import dev, host, params_dev, ptr, require_cuda, stats_dev
from pyro_b200 import _abi

pytestmark = pytest.mark.gpu

CASES = [(24, 32, 20, 0), (19, 23, 17, 1), (40, 16, 33, 2)]


@pytest.fixture(scope="module")
def lib():
    return require_cuda()


def _setup(nx, ny, nz, seed, **kw):
    P = params_for(nx, ny, nz, **kw)
    return P, random_state(P, seed=seed)


def _stats_close(gpu, ora, idx, rtol=1e-4):
    for i in idx:
        e = ora[i]
        assert abs(gpu[i] - e) <= rtol * abs(e) + 1e-30 + 1e-6 * abs(e), (i, gpu[i], e)


@pytest.mark.parametrize("nx,ny,nz,seed", CASES)
def test_solid(lib, nx, ny, nz, seed):
    P, S = _setup(nx, ny, nz, seed, dt=0.02)
    st = np.zeros(1040)
    sol_o, pyr_o, fl_o = oracle.solid(P, S["sol"], S["s0"], st)
    Pd = params_dev(P)
    sol_in, s0 = dev(S["sol"]), dev(S["s0"])
    sol_out, pyr, flags = dev(np.zeros_like(S["sol"])), dev(np.zeros_like(S["sol"])), \
        dev(np.zeros((nz, ny, nx), np.uint32))
    sd = stats_dev()
    assert lib.pyro_k_solid(ptr(Pd), nx, ny, nz, ptr(sol_in), ptr(sol_out), ptr(pyr), ptr(flags),
                            ptr(s0), ptr(sd), None) == 0
    assert np.array_equal(host(flags), fl_o)
    close(host(sol_out), sol_o, name="sol")
    close(host(pyr), pyr_o, name="pyr")
    _stats_close(host(sd), st, [2, 7, 9])


@pytest.mark.parametrize("nx,ny,nz,seed", CASES)
def test_curl(lib, nx, ny, nz, seed):
    P, S = _setup(nx, ny, nz, seed)
    st = np.zeros(1040)
    c_o = oracle.curl(P, S["u"], S["v"], S["w"], st)
    Pd = params_dev(P)
    u, v, w = dev(S["u"]), dev(S["v"]), dev(S["w"])
    c = dev(np.zeros_like(c_o))
    sd = stats_dev()
    assert lib.pyro_k_curl(ptr(Pd), nx, ny, nz, ptr(u), ptr(v), ptr(w), ptr(c), ptr(sd), None) == 0
    assert np.array_equal(host(c), c_o)
    assert host(sd)[5] == np.float32(st[5])


@pytest.mark.parametrize("nx,ny,nz,seed", CASES)
def test_adv_vel(lib, nx, ny, nz, seed):
    P, S = _setup(nx, ny, nz, seed, dt=0.02)
    (hu_o, hv_o, hw_o), (ou_o, ov_o, ow_o) = oracle.adv_vel(P, S["u"], S["v"], S["w"],
                                                            S["flags"])
    Pd = params_dev(P)
    u, v, w = dev(S["u"]), dev(S["v"]), dev(S["w"])
    z = np.zeros_like(S["u"])
    hu, hv, hw, ou, ov, ow = (dev(z) for _ in range(6))
    fl = dev(S["flags"])
    assert lib.pyro_k_adv_vel(ptr(Pd), nx, ny, nz, ptr(u), ptr(v), ptr(w), ptr(hu), ptr(hv),
                              ptr(hw), ptr(ou), ptr(ov), ptr(ow), ptr(fl), None) == 0
    for k, (g, e) in enumerate([(hu, hu_o), (hv, hv_o), (hw, hw_o)]):
        m = face_valid_mask(P, k)
        assert np.array_equal(host(g)[m], e[m]), f"hat {k}"
    for k, (g, e) in enumerate([(ou, ou_o), (ov, ov_o), (ow, ow_o)]):
        m = face_valid_mask(P, k)
        assert np.array_equal(host(g)[m], e[m]), f"out {k}"


@pytest.mark.parametrize("nx,ny,nz,seed", CASES)
def test_adv_scalars(lib, nx, ny, nz, seed):
    P, S = _setup(nx, ny, nz, seed, dt=0.02)
    (h0_o, h1_o), (o0_o, o1_o) = oracle.adv_scalars(P, S["u"], S["v"], S["w"], S["s0"], S["s1"])
    Pd = params_dev(P)
    u, v, w = dev(S["u"]), dev(S["v"]), dev(S["w"])
    s0, s1 = dev(S["s0"]), dev(S["s1"])
    z = np.zeros_like(S["s0"])
    h0, h1, o0, o1 = (dev(z) for _ in range(4))
    assert lib.pyro_k_adv_scalars(ptr(Pd), nx, ny, nz, ptr(u), ptr(v), ptr(w), ptr(s0), ptr(s1),
                                  ptr(h0), ptr(h1), ptr(o0), ptr(o1), None) == 0
    assert np.array_equal(host(h0), h0_o)
    assert np.array_equal(host(h1), h1_o)
    assert np.array_equal(host(o0), o0_o)
    assert np.array_equal(host(o1), o1_o)


@pytest.mark.parametrize("nx,ny,nz,seed", CASES)
@pytest.mark.parametrize("ign_on", [0.0, 1.0])
def test_react(lib, nx, ny, nz, seed, ign_on):
    P, S = _setup(nx, ny, nz, seed, dt=0.01, ign_on=ign_on)
    st = np.zeros(1040)
    o0_o, o1_o = oracle.react(P, S["s0"], S["s1"], S["flags"], S["sol"], S["pyr"], S["curl"], st)
    Pd = params_dev(P)
    args = [dev(S[k]) for k in ("s0", "s1")]
    o0, o1 = dev(np.zeros_like(S["s0"])), dev(np.zeros_like(S["s1"]))
    fl, sol, pyr, curl = dev(S["flags"]), dev(S["sol"]), dev(S["pyr"]), dev(S["curl"])
    sd = stats_dev()
    assert lib.pyro_k_react(ptr(Pd), nx, ny, nz, ptr(args[0]), ptr(args[1]), ptr(o0), ptr(o1),
                            ptr(fl), ptr(sol), ptr(pyr), ptr(curl), ptr(sd), None) == 0
    close(host(o0), o0_o, name="s0")
    close(host(o1), o1_o, name="s1")
    g = host(sd)
    _stats_close(g, st, [0, 1, 3, 6, 8])
    assert abs(g[4] - st[4]) <= 1e-5 * st[4]
    lay = g[16:16 + ny]
    close(lay, st[16:16 + ny].astype(np.float32), rtol=1e-4, floor=1e-6, name="layers")


@pytest.mark.parametrize("nx,ny,nz,seed", CASES)
def test_forces(lib, nx, ny, nz, seed):
    P, S = _setup(nx, ny, nz, seed, dt=0.01, wind=2.0, sponge=3.0)
    uo, vo, wo = oracle.forces(P, S["u"], S["v"], S["w"], S["s0"], S["s1"], S["curl"],
                               S["flags"])
    Pd = params_dev(P)
    u, v, w = dev(S["u"]), dev(S["v"]), dev(S["w"])
    s0, s1, curl, fl = dev(S["s0"]), dev(S["s1"]), dev(S["curl"]), dev(S["flags"])
    assert lib.pyro_k_forces(ptr(Pd), nx, ny, nz, ptr(u), ptr(v), ptr(w), ptr(s0), ptr(s1),
                             ptr(curl), ptr(fl), None) == 0
    for k, (g, e) in enumerate([(u, uo), (v, vo), (w, wo)]):
        m = face_valid_mask(P, k)
        close(host(g)[m], e[m], name=f"vel{k}")


@pytest.mark.parametrize("nx,ny,nz,seed", CASES)
def test_divergence_and_project(lib, nx, ny, nz, seed):
    P, S = _setup(nx, ny, nz, seed)
    b_o = oracle.divergence(P, S["u"], S["v"], S["w"], S["s1"], S["flags"])
    Pd = params_dev(P)
    u, v, w = dev(S["u"]), dev(S["v"]), dev(S["w"])
    s1, fl = dev(S["s1"]), dev(S["flags"])
    b = dev(np.zeros((nz, ny, nx), np.float32))
    assert lib.pyro_k_divergence(ptr(Pd), nx, ny, nz, ptr(u), ptr(v), ptr(w), ptr(s1), ptr(fl),
                                 ptr(b), None) == 0
    assert np.array_equal(host(b), b_o)
    uo, vo, wo = oracle.project(P, S["u"], S["v"], S["w"], S["phi"], S["flags"])
    phi = dev(S["phi"])
    assert lib.pyro_k_project(ptr(Pd), nx, ny, nz, ptr(u), ptr(v), ptr(w), ptr(phi), ptr(fl),
                              None) == 0
    for k, (g, e) in enumerate([(u, uo), (v, vo), (w, wo)]):
        m = face_valid_mask(P, k)
        assert np.array_equal(host(g)[m], e[m]), f"project {k}"


MG_CASES = [(32, 48, 32, 0, 0.05), (19, 46, 19, 1, 0.16), (17, 33, 9, 2, 0.1)]


@pytest.mark.parametrize("nx,ny,nz,seed,h", MG_CASES)
def test_mg_kernels(lib, nx, ny, nz, seed, h):
    rng = np.random.default_rng(seed)
    f = (rng.random((nz, ny, nx)) < 0.2).astype(np.uint32)
    b = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    p = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    bd, fd = dev(b), dev(f)
    for color, om in [(0, 1.0), (1, 1.0), (0, 1.6), (1, 1.6)]:
        e = oracle.mg_smooth((nx, ny, nz), h, b, f, p, color, om)
        pd = dev(p)
        assert lib.pyro_k_mg_smooth(nx, ny, nz, h, ptr(bd), ptr(fd), ptr(pd), color, om,
                                    None) == 0
        assert np.array_equal(host(pd), e), (color, om)
    cx, cy, cz = (nx + 1) // 2, (ny + 1) // 2, (nz + 1) // 2
    bc_o, pc_o, fc_o = oracle.mg_restrict((nx, ny, nz), h, p, b, f)
    bc, pc, fc = dev(np.ones_like(bc_o)), dev(np.ones_like(pc_o)), dev(np.ones_like(fc_o))
    pd = dev(p)
    assert lib.pyro_k_mg_restrict(nx, ny, nz, h, ptr(pd), ptr(bd), ptr(fd), cx, cy, cz, ptr(bc),
                                  ptr(pc), ptr(fc), None) == 0
    assert np.array_equal(host(fc), fc_o)
    assert np.array_equal(host(bc), bc_o)
    assert np.array_equal(host(pc), pc_o)
    pcv = rng.normal(0, 1, bc_o.shape).astype(np.float32)
    pf_o = oracle.mg_prolong((nx, ny, nz), pcv, f, p, fc_o)
    pcd = dev(pcv)
    assert lib.pyro_k_mg_prolong(nx, ny, nz, ptr(pcd), ptr(fd), ptr(pd), cx, cy, cz, ptr(fc),
                                 None) == 0
    assert np.array_equal(host(pd), pf_o)
    r2, b2 = oracle.mg_resid((nx, ny, nz), h, p, b, f)
    sd = stats_dev()
    pd = dev(p)
    assert lib.pyro_k_mg_resid(nx, ny, nz, h, ptr(pd), ptr(bd), ptr(fd), ptr(sd), None) == 0
    g = host(sd)
    assert abs(g[10] - r2) <= 1e-4 * r2 and abs(g[11] - b2) <= 1e-4 * b2


def _bf16_bits(x):
    """float32 -> BF16 bit patterns, round to nearest even (as
    __float2bfloat16_rn for finite values)."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def _bf16_val(bits):
    return (bits.astype(np.uint32) << 16).view(np.float32)


# the shapes the V-cycle meets: rows of a multiple of 4 cells (4-cell
# chunks in the pass, even row pairs in the transfers), of another even
# length (2-cell aligned chunks: 10, 38, 150, 130) and odd (2-cell scalar
# chunks, the last of a row with one cell: 19, 17, 75, 33, 129); the
# chunked passes take one plane per thread below 256 Ki cells, two up to
# 4 Mi, four from there
MASK_CASES = MG_CASES + [(64, 40, 24, 3, 0.04), (20, 40, 20, 4, 0.16), (10, 20, 10, 5, 0.32),
                         (80, 64, 64, 7, 0.04), (256, 128, 128, 6, 0.02),
                         (38, 40, 20, 8, 0.16), (150, 96, 24, 9, 0.02),
                         (130, 256, 128, 10, 0.02), (75, 64, 64, 11, 0.04),
                         (33, 8, 6, 12, 0.2), (129, 256, 128, 13, 0.02)]


@pytest.mark.parametrize("nx,ny,nz,seed,h", MASK_CASES)
@pytest.mark.parametrize("bc_mode", [0, 1])
@pytest.mark.parametrize("storage", [_abi.MG_F32, _abi.MG_BF16])
def test_mg_mask_kernels_as_the_vcycle_runs_them(lib, nx, ny, nz, seed, h, bc_mode, storage):
    """The smoother pass, restriction and prolongation on the level's
    neighbour masks, both boundary modes, FP32 or BF16 storage of phi and b,
    against the oracle's per-flag kernels (mg.wgsl).  BF16: the inputs are
    BF16 values, the arithmetic is FP32 on both sides and the oracle's
    result is rounded to BF16, so the bits must agree exactly."""
    rng = np.random.default_rng(100 + seed)
    f = (rng.random((nz, ny, nx)) < 0.2).astype(np.uint32)
    b = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    p = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    lo = storage == _abi.MG_BF16
    if lo:
        b, p = _bf16_val(_bf16_bits(b)), _bf16_val(_bf16_bits(p))
    enc = (lambda a: _bf16_bits(a)) if lo else (lambda a: np.ascontiguousarray(a, np.float32))
    fd = dev(f)
    meta = dev(np.zeros((nz, ny, nx), np.uint8))
    assert lib.pyro_k_mg_meta(nx, ny, nz, ptr(fd), ptr(meta), None) == 0
    bd = dev(enc(b))
    for color, om in [(0, 1.0), (1, 1.0), (0, 1.6), (1, 1.6)]:
        e = oracle.mg_smooth((nx, ny, nz), h, b, f, p, color, om, bc_mode=bc_mode)
        pd = dev(enc(p))
        assert lib.pyro_k_mg_pass(nx, ny, nz, h, ptr(bd), ptr(meta), ptr(pd), color, om, bc_mode,
                                  storage, None) == 0, lib.pyro_last_error()
        assert np.array_equal(host(pd), enc(e)), (color, om)
    cx, cy, cz = (nx + 1) // 2, (ny + 1) // 2, (nz + 1) // 2
    bc_o, pc_o, fc_o = oracle.mg_restrict((nx, ny, nz), h, p, b, f, bc_mode=bc_mode)
    fc = dev(np.ones_like(fc_o))
    assert lib.pyro_k_mg_flags_down(nx, ny, nz, ptr(fd), cx, cy, cz, ptr(fc), None) == 0
    assert np.array_equal(host(fc), fc_o)
    bc, pc = dev(enc(np.ones_like(bc_o))), dev(enc(np.ones_like(pc_o)))
    assert lib.pyro_k_mg_restrict_m(nx, ny, nz, h, ptr(dev(enc(p))), ptr(bd), ptr(meta), cx, cy,
                                    cz, ptr(bc), ptr(pc), bc_mode, storage, None) == 0
    assert np.array_equal(host(bc), enc(bc_o))
    assert np.array_equal(host(pc), enc(pc_o))
    mc = dev(np.zeros((cz, cy, cx), np.uint8))
    assert lib.pyro_k_mg_meta(cx, cy, cz, ptr(fc), ptr(mc), None) == 0
    pcv = rng.normal(0, 1, bc_o.shape).astype(np.float32)
    if lo:
        pcv = _bf16_val(_bf16_bits(pcv))
    pf_o = oracle.mg_prolong((nx, ny, nz), pcv, f, p, fc_o)
    pd = dev(enc(p))
    assert lib.pyro_k_mg_prolong_m(nx, ny, nz, ptr(dev(enc(pcv))), ptr(meta), ptr(pd), cx, cy,
                                   cz, ptr(mc), storage, None) == 0
    assert np.array_equal(host(pd), enc(pf_o))


@pytest.mark.parametrize("nx,ny,nz,seed,h", [(32, 48, 32, 0, 0.05), (38, 40, 20, 8, 0.16),
                                             (150, 96, 24, 9, 0.02), (64, 40, 24, 3, 0.04),
                                             (19, 46, 19, 1, 0.16), (75, 64, 40, 11, 0.04)])
@pytest.mark.parametrize("bc_mode", [0, 1])
@pytest.mark.parametrize("storage", [_abi.MG_F32, _abi.MG_BF16])
def test_mg_fused_first_and_last_passes_equal_the_plain_pass(lib, nx, ny, nz, seed, h, bc_mode,
                                                             storage):
    """The preconditioner's fused level-0 passes against the oracle's pass:
    the first from phi = 0 on the FP32 right-hand side (BF16: rounded, and
    the rounded copy written out), every cell of phi written; the last on
    BF16 storage with its result widened into an FP32 array."""
    rng = np.random.default_rng(200 + seed)
    f = (rng.random((nz, ny, nx)) < 0.2).astype(np.uint32)
    r = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    lo = storage == _abi.MG_BF16
    enc = (lambda a: _bf16_bits(a)) if lo else (lambda a: np.ascontiguousarray(a, np.float32))
    meta = dev(np.zeros((nz, ny, nx), np.uint8))
    assert lib.pyro_k_mg_meta(nx, ny, nz, ptr(dev(f)), ptr(meta), None) == 0
    bq = _bf16_val(_bf16_bits(r)) if lo else r
    for color, om in [(0, 1.0), (1, 1.6)]:
        e = oracle.mg_smooth((nx, ny, nz), h, bq, f, np.zeros_like(r), color, om, bc_mode=bc_mode)
        pd = dev(enc(np.full_like(r, 7.0)))  # every cell is overwritten
        bqd = dev(np.zeros((nz, ny, nx), np.uint16)) if lo else None
        assert lib.pyro_k_mg_pass_first(nx, ny, nz, h, ptr(dev(r)), ptr(bqd) if lo else None,
                                        ptr(meta), ptr(pd), color, om, bc_mode, storage,
                                        None) == 0, lib.pyro_last_error()
        assert np.array_equal(host(pd), enc(e)), (color, om)
        if lo:
            assert np.array_equal(host(bqd), _bf16_bits(r))
    if not lo:
        return
    b = _bf16_val(_bf16_bits(r))
    p = _bf16_val(_bf16_bits(rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)))
    for color, om in [(0, 1.0), (1, 1.6)]:
        e = oracle.mg_smooth((nx, ny, nz), h, b, f, p, color, om, bc_mode=bc_mode)
        pd = dev(_bf16_bits(p))
        out = dev(np.full_like(r, 7.0))
        assert lib.pyro_k_mg_pass_last(nx, ny, nz, h, ptr(dev(_bf16_bits(b))), ptr(meta),
                                       ptr(pd), ptr(out), color, om, bc_mode,
                                       None) == 0, lib.pyro_last_error()
        assert np.array_equal(host(out), _bf16_val(_bf16_bits(e))), (color, om)
        assert np.array_equal(host(pd), _bf16_bits(p))


@pytest.mark.parametrize("nx,ny,nz,seed,h", [(32, 48, 32, 0, 0.05), (19, 46, 19, 1, 0.16),
                                             (38, 40, 20, 8, 0.16), (150, 96, 24, 9, 0.02)])
@pytest.mark.parametrize("bc_mode", [0, 1])
def test_mg_symmetric_restriction_is_the_adjoint_of_the_prolongation(lib, nx, ny, nz, seed, h,
                                                                     bc_mode):
    """The CG preconditioner's restriction R = P^T / 8 of the fluid-weighted
    prolongation P (pyro_k_mg_prolong_m, pinned to mg.wgsl above): for random
    fine r and coarse e, <R r, e> = <r, P e> / 8 (FP64 sums of the FP32
    results), and with phi = 0 the coarse guess is cleared.  BF16 storage
    gives the same restriction within its rounding."""
    rng = np.random.default_rng(300 + seed)
    f = (rng.random((nz, ny, nx)) < 0.25).astype(np.uint32)
    cx, cy, cz = (nx + 1) // 2, (ny + 1) // 2, (nz + 1) // 2
    fd = dev(f)
    fc = dev(np.zeros((cz, cy, cx), np.uint32))
    assert lib.pyro_k_mg_flags_down(nx, ny, nz, ptr(fd), cx, cy, cz, ptr(fc), None) == 0
    mf = dev(np.zeros((nz, ny, nx), np.uint8))
    mc = dev(np.zeros((cz, cy, cx), np.uint8))
    assert lib.pyro_k_mg_meta(nx, ny, nz, ptr(fd), ptr(mf), None) == 0
    assert lib.pyro_k_mg_meta(cx, cy, cz, ptr(fc), ptr(mc), None) == 0
    zero_f = dev(np.zeros((nz, ny, nx), np.float32))
    for k in range(3):
        r = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
        e = rng.normal(0, 1, (cz, cy, cx)).astype(np.float32)
        bc, pc = dev(np.ones((cz, cy, cx), np.float32)), dev(np.ones((cz, cy, cx), np.float32))
        assert lib.pyro_k_mg_restrict_sym(nx, ny, nz, h, ptr(zero_f), ptr(dev(r)), ptr(mf), cx,
                                          cy, cz, ptr(mc), ptr(bc), ptr(pc), bc_mode,
                                          _abi.MG_F32, None) == 0, lib.pyro_last_error()
        Rr = host(bc)
        assert not host(pc).any()
        pe = dev(np.zeros((nz, ny, nx), np.float32))
        assert lib.pyro_k_mg_prolong_m(nx, ny, nz, ptr(dev(e)), ptr(mf), ptr(pe), cx, cy, cz,
                                       ptr(mc), _abi.MG_F32, None) == 0
        Pe = host(pe)
        fl = f == 0
        lhs = float(np.dot(Rr.ravel().astype(np.float64), e.ravel().astype(np.float64)))
        rhs = float(np.dot(np.where(fl, r, 0).ravel().astype(np.float64),
                           Pe.ravel().astype(np.float64))) / 8.0
        scale = float(np.linalg.norm(Rr) * np.linalg.norm(e))
        assert abs(lhs - rhs) <= 1e-5 * scale, (k, lhs, rhs, scale)
        if k == 0:
            rb = _bf16_bits(r)
            bb, pb = dev(np.zeros((cz, cy, cx), np.uint16)), dev(np.ones((cz, cy, cx), np.uint16))
            assert lib.pyro_k_mg_restrict_sym(nx, ny, nz, h, ptr(dev(np.zeros_like(rb))),
                                              ptr(dev(rb)), ptr(mf), cx, cy, cz, ptr(mc),
                                              ptr(bb), ptr(pb), bc_mode, _abi.MG_BF16,
                                              None) == 0
            assert not host(pb).any()
            bf = dev(np.zeros((cz, cy, cx), np.float32))
            assert lib.pyro_k_mg_restrict_sym(nx, ny, nz, h, ptr(zero_f), ptr(dev(_bf16_val(rb))),
                                              ptr(mf), cx, cy, cz, ptr(mc), ptr(bf), ptr(pc),
                                              bc_mode, _abi.MG_F32, None) == 0
            lo, hi = _bf16_val(host(bb)), host(bf)
            assert np.abs(lo - hi).max() <= 2e-2 * np.abs(hi).max()


# slabs of one to three planes per CTA of the cluster (nz = 3: three CTAs)
COARSE_CASES = MG_CASES + [(8, 20, 8, 3, 0.32), (32, 32, 22, 4, 0.2), (20, 40, 20, 5, 0.16),
                           (16, 30, 16, 6, 0.16), (20, 40, 17, 7, 0.16), (12, 20, 3, 11, 0.3)]


@pytest.mark.parametrize("nx,ny,nz,seed,h", COARSE_CASES)
def test_mg_coarse_solve_equals_80_sor_sweeps(lib, nx, ny, nz, seed, h):
    rng = np.random.default_rng(seed)
    f = (rng.random((nz, ny, nx)) < 0.1).astype(np.uint32)
    b = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    p = rng.normal(0, 0.1, (nz, ny, nx)).astype(np.float32)
    e = p
    for _ in range(80):
        for c in (0, 1):
            e = oracle.mg_smooth((nx, ny, nz), h, b, f, e, c, 1.6)
    pd, bd, fd = dev(p), dev(b), dev(f)
    assert lib.pyro_k_mg_coarse(nx, ny, nz, h, ptr(bd), ptr(fd), ptr(pd), 80, 1.6, None) == 0
    assert np.array_equal(host(pd), e)


@pytest.mark.parametrize("nx,ny,nz,seed,h", [(20, 40, 20, 8, 0.16), (32, 32, 22, 9, 0.2),
                                             (8, 20, 8, 10, 0.32)])
@pytest.mark.parametrize("bc_mode", [0, 1])
def test_mg_coarse_symmetric_equals_alternating_sweeps(lib, nx, ny, nz, seed, h, bc_mode):
    rng = np.random.default_rng(seed)
    f = (rng.random((nz, ny, nx)) < 0.1).astype(np.uint32)
    b = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    p = rng.normal(0, 0.1, (nz, ny, nx)).astype(np.float32)
    e = p
    for it in range(40):
        for c in ((0, 1) if it % 2 == 0 else (1, 0)):
            e = oracle.mg_smooth((nx, ny, nz), h, b, f, e, c, 1.6, bc_mode=bc_mode)
    pd, bd, fd = dev(p), dev(b), dev(f)
    assert lib.pyro_k_mg_coarse_sym(nx, ny, nz, h, ptr(bd), ptr(fd), ptr(pd), 40, 1.6, bc_mode,
                                    None) == 0
    assert np.array_equal(host(pd), e)
