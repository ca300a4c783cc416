"""Pin the CPU oracle to the reference: golden vectors produced by
interpreting the reference's own WGSL kernel source (tests/golden/
make_golden.py) against the oracle on the stored inputs.

Kernels free of exp() must agree bit for bit (both evaluate the WGSL
expressions in FP32 in the source's order); kernels calling exp() agree
within 1e-5 relative plus an absolute floor of 1e-6 of each channel's
magnitude, the same bar as the GPU parity tests.  Statistics: 1e-4.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from fields import close
from pyro_b200 import _abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    p = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(p):
        pytest.fail(f"missing golden fixture {p}")
    d = np.load(p)
    return {k: d[k] for k in d.files}


def _params(d):
    P = _abi.PyroParams()
    b = bytes(d["params"])
    import ctypes
    ctypes.memmove(ctypes.byref(P), b, len(b))
    return P


def _valid(P, k):
    from fields import face_valid_mask
    return face_valid_mask(P, k)


def _stats_close(g, e, idx, rtol=1e-4):
    for i in idx:
        assert abs(g[i] - e[i]) <= rtol * abs(e[i]) + 1e-30, (i, g[i], e[i])


CASES = ["c0", "c1"]


@pytest.mark.parametrize("case", CASES)
def test_solid(case):
    d = _load(f"solid_{case}")
    P = _params(d)
    st = np.zeros(1040)
    sol, pyr, fl = oracle.solid(P, d["sol"], d["s0"], st)
    assert np.array_equal(fl, d["flags"])
    close(sol, d["sol_out"], name="sol")
    close(pyr, d["pyr"], name="pyr")
    _stats_close(st, d["stats"], [2, 7, 9])


@pytest.mark.parametrize("case", CASES)
def test_curl(case):
    d = _load(f"curl_{case}")
    P = _params(d)
    st = np.zeros(1040)
    c = oracle.curl(P, d["u"], d["v"], d["w"], st)
    assert np.array_equal(c, d["curl"])
    assert np.float32(st[5]) == d["stats"][5]


@pytest.mark.parametrize("case", CASES)
def test_adv_vel(case):
    d = _load(f"adv_vel_{case}")
    P = _params(d)
    hats, outs = oracle.adv_vel(P, d["u"], d["v"], d["w"], d["flags"])
    for k, name in enumerate(("hu", "hv", "hw")):
        m = _valid(P, k)
        assert np.array_equal(hats[k][m], d[name][m]), name
    for k, name in enumerate(("ou", "ov", "ow")):
        m = _valid(P, k)
        assert np.array_equal(outs[k][m], d[name][m]), name


@pytest.mark.parametrize("case", CASES)
def test_adv_scalars(case):
    d = _load(f"adv_scalars_{case}")
    P = _params(d)
    (h0, h1), (o0, o1) = oracle.adv_scalars(P, d["u"], d["v"], d["w"], d["s0"], d["s1"])
    for got, name in ((h0, "h0"), (h1, "h1"), (o0, "o0"), (o1, "o1")):
        assert np.array_equal(got, d[name]), name


@pytest.mark.parametrize("case", CASES)
def test_react(case):
    d = _load(f"react_{case}")
    P = _params(d)
    st = np.zeros(1040)
    o0, o1 = oracle.react(P, d["s0"], d["s1"], d["flags"], d["sol"], d["pyr"], d["curl"], st)
    close(o0, d["o0"], name="s0")
    close(o1, d["o1"], name="s1")
    _stats_close(st, d["stats"], [0, 1, 3, 6, 8])
    assert abs(st[4] - d["stats"][4]) <= 1e-5 * d["stats"][4]
    ny = int(P.ny)
    close(st[16:16 + ny].astype(np.float32), d["stats"][16:16 + ny], rtol=1e-4, name="layers")


@pytest.mark.parametrize("case", CASES)
def test_forces(case):
    d = _load(f"forces_{case}")
    P = _params(d)
    u, v, w = oracle.forces(P, d["u"], d["v"], d["w"], d["s0"], d["s1"], d["curl"], d["flags"])
    for k, (got, name) in enumerate(((u, "ou"), (v, "ov"), (w, "ow"))):
        m = _valid(P, k)
        close(got[m], d[name][m], name=name)


@pytest.mark.parametrize("case", CASES)
def test_divergence(case):
    d = _load(f"divergence_{case}")
    P = _params(d)
    b = oracle.divergence(P, d["u"], d["v"], d["w"], d["s1"], d["flags"])
    assert np.array_equal(b, d["b"])


@pytest.mark.parametrize("case", CASES)
def test_project(case):
    d = _load(f"project_{case}")
    P = _params(d)
    u, v, w = oracle.project(P, d["u"], d["v"], d["w"], d["phi"], d["flags"])
    for k, (got, name) in enumerate(((u, "ou"), (v, "ov"), (w, "ow"))):
        m = _valid(P, k)
        assert np.array_equal(got[m], d[name][m]), name


@pytest.mark.parametrize("name,color,omega", [("mg_smooth_c0_w10", 0, 1.0),
                                              ("mg_smooth_c1_w10", 1, 1.0),
                                              ("mg_smooth_c0_w16", 0, 1.6),
                                              ("mg_smooth_c1_w16", 1, 1.6)])
def test_mg_smooth(name, color, omega):
    d = _load(name)
    dims = tuple(int(v) for v in d["dims"])
    out = oracle.mg_smooth(dims, float(d["h"]), d["b"], d["f"], d["p"], color, omega)
    assert np.array_equal(out, d["out"])


def test_mg_restrict_prolong_resid():
    d = _load("mg_restrict")
    dims = tuple(int(v) for v in d["dims"])
    bc, pc, fc = oracle.mg_restrict(dims, float(d["h"]), d["p"], d["b"], d["f"])
    assert np.array_equal(fc, d["fc"])
    assert np.array_equal(bc, d["bc"])
    assert np.array_equal(pc, d["pc"])
    d = _load("mg_prolong")
    out = oracle.mg_prolong(dims, d["pc"], d["f"], d["p"], d["fc"])
    assert np.array_equal(out, d["out"])
    d = _load("mg_resid")
    r2, b2 = oracle.mg_resid(dims, float(d["h"]), d["p"], d["b"], d["f"])
    assert abs(r2 - d["stats"][10]) <= 1e-4 * r2
    assert abs(b2 - d["stats"][11]) <= 1e-4 * b2


def test_fixture_set_is_complete():
    names = {os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))}
    want = {f"{k}_{c}" for k in ("solid", "curl", "adv_vel", "adv_scalars", "react", "forces",
                                 "divergence", "project") for c in CASES}
    want |= {"mg_smooth_c0_w10", "mg_smooth_c1_w10", "mg_smooth_c0_w16", "mg_smooth_c1_w16",
             "mg_restrict", "mg_prolong", "mg_resid"}
    assert want <= names, want - names


@pytest.mark.parametrize("case", CASES)
def test_render_pack_and_bricks(case):
    """The renderer's input pack (render.wgsl:3-61): the oracle's three
    binary16 volumes and the brick maxima equal the interpreted WGSL's bit
    for bit (the texture store rounds to nearest even in both)."""
    d = _load(f"render_{case}")
    P = _params(d)
    vol, solt, vel = oracle.render_pack(P, d["s0"], d["s1"], d["sol"], d["flags"], d["u"],
                                        d["v"], d["w"])
    assert np.array_equal(vol.view(np.uint16), d["vol"].view(np.uint16))
    assert np.array_equal(solt.view(np.uint16), d["solt"].view(np.uint16))
    assert np.array_equal(vel.view(np.uint16), d["vel"].view(np.uint16))
    b = oracle.render_bricks((P.nx, P.ny, P.nz), d["vol"], d["solt"])
    assert np.array_equal(b, d["bricks"])
    assert (d["flags"] == 1).any() and (d["flags"] != 1).any()


@pytest.mark.parametrize("case", CASES)
def test_render_emission(case):
    """The fire-light emission per cell (render.wgsl:63-98; it calls exp(),
    so 1e-5 relative) and the CDF the reference forms on the CPU
    (src/render.rs:316-333)."""
    d = _load(f"render_{case}")
    P = _params(d)
    e = oracle.render_ecells(P, d["vol"], d["lut"], d["chemi"])
    close(e, d["ecell"], name="ecell")
    assert (d["ecell"] > 0).sum() > d["ecell"].size // 2
    cdf = oracle.render_cdf(d["ecell"])
    assert cdf.shape == (d["ecell"].size + 1,)
    assert np.all(np.diff(cdf[:-1]) >= 0) and cdf[-2] == 1.0
    assert abs(cdf[-1] - np.maximum(d["ecell"], 0).astype(np.float64).sum()) <= 1e-6 * cdf[-1]


def test_render_light_caches_and_blur():
    """The path tracer's light caches (render.wgsl:217-269) and their blur
    chain (render.wgsl:271-304, src/render.rs:362-396): the oracle's binary16
    caches equal the interpreted WGSL's bit for bit (8 shadow rays per cell
    instead of 96 / 128, an 8x8 ground cache instead of 256^2)."""
    d = _load("trace_cache")
    lvd = (d["lvA"].shape[2], d["lvA"].shape[1], d["lvA"].shape[0])
    a, b = oracle.render_lightvol(d["rp"], d["vol"], d["solt"], d["vel"], d["bricks"], d["lut"],
                                  d["ecdf"], lvd, lv_n=8)
    assert np.array_equal(a.view(np.uint16), d["lvA_raw"].view(np.uint16))
    assert np.array_equal(b.view(np.uint16), d["lvB_raw"].view(np.uint16))
    g = oracle.render_lightground(d["rp"], d["vol"], d["solt"], d["vel"], d["bricks"], d["lut"],
                                  d["ecdf"], d["gE_raw"].shape[1], gr_n=8)
    assert np.array_equal(g.view(np.uint16), d["gE_raw"].view(np.uint16))
    A, B, G = d["lvA_raw"], d["lvB_raw"], d["gE_raw"]
    for ax in (0, 1, 2):
        A = oracle.render_blur(A, ax, 2)
        B = oracle.render_blur(B, ax, 2)
    for ax in (0, 1):
        G = oracle.render_blur(G, ax, 3)
    for got, want in ((A, d["lvA"]), (B, d["lvB"]), (G, d["gE"])):
        assert np.array_equal(got.view(np.uint16), want.view(np.uint16))
    assert np.isfinite(d["lvA"].astype(np.float32)).all() and d["lvA"].astype(np.float32).max() > 0


@pytest.mark.parametrize("mode", ["cache", "path", "lens"])
def test_render_trace(mode):
    """Camera rays (render.wgsl:132-215 with trace_lib.wgsl): light-cache mode
    and pure path tracing (2 bounces, next-event estimation with MIS,
    Russian roulette), motion blur on; "lens" is light-cache mode through a
    thin lens (render.wgsl:148-154) at another frame and first sample.  The random numbers are the
    reference's PCG hash, so the oracle follows the interpreted WGSL's paths;
    pixels agree to the rounding of exp / sin / cos / sqrt (1e-5 relative of
    the image's largest value)."""
    d = _load(f"trace_{mode}")
    acc = oracle.render_trace(d["rp"], d["vol"], d["solt"], d["vel"], d["bricks"], d["lut"],
                              d["ecdf"], d["lvA"], d["lvB"], d["gE"])
    want = d["accum"]
    assert np.all(acc[:, 3] == want[:, 3])
    assert np.max(np.abs(acc[:, :3] - want[:, :3])) <= 1e-5 * np.abs(want[:, :3]).max()
    assert np.count_nonzero(want[:, :3]) > want[:, :3].size // 2
