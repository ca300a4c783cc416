"""The volume path tracer on the GPU, through the C ABI: the light caches
(render.wgsl:217-269), their blur chain (render.wgsl:271-304) and the camera
rays in light-cache and path-tracing modes (render.wgsl:132-215 with
trace_lib.wgsl); against the golden vectors of the reference's WGSL and the
oracle.

Both sides draw the reference's PCG random numbers, so they follow the same
paths.  The blur is bit for bit (its weights are formed on the host).  The
caches and pixels go through exp, sin and cos, which CUDA and the host's libm
round differently: caches agree to two binary16 units, pixels to 1e-4 of the
image's largest value, except where such a rounding moves a branch (a
reservoir pick, a roulette draw), which the larger cases allow in a small
fraction of texels and pixels."""
import os

import numpy as np
import pytest
import torch

import oracle
from fields import params_for, random_state
from gpu_util import dev, host, require_cuda
from pyro_b200 import _abi, color, render
from pyro_b200.scene import Scene
from pyro_b200.sim import Sim
from test_golden import _load

pytestmark = pytest.mark.gpu

SCENES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "pyro_b200", "scenes")


@pytest.fixture(scope="module")
def lib():
    return require_cuda()


def _half_empty(shape):
    return torch.full(shape, float("nan"), dtype=torch.float16, device="cuda")


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint16)


def _bind(d):
    """Device copies of a frame's volumes and tables."""
    return {k: dev(d[k]) for k in ("vol", "solt", "vel", "bricks", "lut", "ecdf")}


def _args(b):
    return b["vol"], b["solt"], b["vel"], b["bricks"], b["lut"], b["ecdf"]


def _cache_close(got, want, rtol=2e-3, max_bad=0.0):
    """binary16 caches: |got - want| <= rtol |want| + 1e-5 max|want|, in all
    but a fraction max_bad of the values."""
    g, w = got.astype(np.float64), want.astype(np.float64)
    assert np.isfinite(g).all()
    tol = rtol * np.abs(w) + 1e-5 * max(np.abs(w).max(), 1e-30)
    bad = np.abs(g - w) > tol
    assert bad.mean() <= max_bad, (bad.mean(), np.argwhere(bad)[:5])


def _pixels_close(got, want, rtol=1e-4, max_bad=0.0):
    assert np.array_equal(got[:, 3], want[:, 3])
    g, w = got[:, :3].astype(np.float64), want[:, :3].astype(np.float64)
    assert np.isfinite(g).all()
    bad = (np.abs(g - w) > rtol * np.abs(w).max()).any(axis=1)
    assert bad.mean() <= max_bad, (bad.mean(), np.argwhere(bad)[:5])


def _gpu_blur(src, axis, r):
    s = dev(src)
    d = _half_empty(s.shape)
    nz, ny, nx = src.shape[:3]
    render.blur(s, d, (nx, ny, nz), axis, r)
    return host(d)


@pytest.mark.parametrize("dims,axis,r", [((9, 7, 5), 0, 2), ((9, 7, 5), 1, 2), ((9, 7, 5), 2, 2),
                                         ((37, 19, 6), 0, 3), ((16, 16, 1), 1, 3),
                                         ((5, 4, 3), 2, 1), ((40, 3, 70), 2, 16)])
def test_blur_vs_oracle(lib, dims, axis, r):
    nx, ny, nz = dims
    rng = np.random.default_rng(nx * 7 + axis)
    src = (rng.random((nz, ny, nx, 4)) * 50.0 - 5.0).astype(np.float16)
    assert np.array_equal(_bits(_gpu_blur(src, axis, r)), _bits(oracle.render_blur(src, axis, r)))


def test_blur_chain_golden(lib):
    """The reference's chain (src/render.rs:372-381): x, y, z at radius 2 on
    both volume caches, x, y at radius 3 on the ground cache."""
    d = _load("trace_cache")
    A, B, G = d["lvA_raw"], d["lvB_raw"], d["gE_raw"]
    for ax in (0, 1, 2):
        A, B = _gpu_blur(A, ax, 2), _gpu_blur(B, ax, 2)
    for ax in (0, 1):
        G = _gpu_blur(G, ax, 3)
    for got, want in ((A, d["lvA"]), (B, d["lvB"]), (G, d["gE"])):
        assert np.array_equal(_bits(got), _bits(want))


def test_light_caches_golden(lib):
    d = _load("trace_cache")
    rp = _abi.PyroRenderParams.from_rows(d["rp"])
    b = _bind(d)
    lz, ly, lx = d["lvA_raw"].shape[:3]
    a, bb = _half_empty((lz, ly, lx, 4)), _half_empty((lz, ly, lx, 4))
    render.lightvol(rp, *_args(b), (lx, ly, lz), a, bb, rays=8)
    _cache_close(host(a), d["lvA_raw"])
    _cache_close(host(bb), d["lvB_raw"])
    gres = d["gE_raw"].shape[1]
    g = _half_empty((1, gres, gres, 4))
    render.lightground(rp, *_args(b), gres, g, rays=8)
    _cache_close(host(g), d["gE_raw"])


def _trace_gpu(d, rp, accum=None):
    b = _bind(d)
    w, h = rp.res[0], rp.res[1]
    acc = torch.zeros((w * h, 4), dtype=torch.float32, device="cuda") if accum is None else accum
    lz, ly, lx = d["lvA"].shape[:3]
    render.trace(rp, *_args(b), dev(d["lvA"]), dev(d["lvB"]), (lx, ly, lz), dev(d["gE"]),
                 d["gE"].shape[1], acc)
    return acc


@pytest.mark.parametrize("mode", ["cache", "path"])
def test_trace_golden(lib, mode):
    d = _load(f"trace_{mode}")
    rp = _abi.PyroRenderParams.from_rows(d["rp"])
    got = host(_trace_gpu(d, rp))
    _pixels_close(got, d["accum"])
    assert np.count_nonzero(got[:, :3]) > got[:, :3].size // 2


@pytest.mark.parametrize("mode", ["cache", "path"])
def test_trace_dispatches_add_up(lib, mode):
    """Samples 0..3 in one dispatch equal the same samples in four one-sample
    dispatches into the same image (the reference submits its samples in
    chunks; a chunk sums its own samples before adding them to the image,
    so only one-sample chunks keep the single dispatch's order of sums)."""
    d = _load(f"trace_{mode}")
    rp = _abi.PyroRenderParams.from_rows(d["rp"])
    rp.res[2], rp.res[3] = 0, 4
    one = host(_trace_gpu(d, rp))
    acc = None
    for first in range(4):
        rp.res[2], rp.res[3] = first, 1
        acc = _trace_gpu(d, rp, acc)
    assert np.array_equal(host(acc), one)
    assert np.all(one[:, 3] == 4.0)


def _rp_rows(P, w, h, spp, frame, cache, bounces=2.0, aperture=0.0):
    """A camera outside the domain looking at its centre (fov 45 degrees)."""
    dx = float(np.float32(P.dx))
    ext = np.array([P.nx * dx, P.ny * dx, P.nz * dx])
    target = 0.5 * ext
    pos = target + np.array([0.13, 0.07, -1.1]) * ext.max()
    fwd = (target - pos) / np.linalg.norm(target - pos)
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    se = color.soot_extinction(0.25)
    side = 3.0 * max(ext[0], ext[2])
    return [[w, h, 0, spp], [P.nx, P.ny, P.nz, frame],
            [*pos, np.tan(np.radians(22.5))], [*fwd, w / h], [*right, aperture],
            [*up, float(np.linalg.norm(target - pos))],
            [dx, 0.6, 1.0 / 60.0, 0.003], [1.0, 0.12, bounces, 0.05],
            [se[0], se[1], se[2], 0.25], [5.0, 0.92, 0.55, P.t0],
            [0.32, 0.45, 0.3, 0.05], [0.05, 0.05, 0.05, 0.05],
            [0.5 * ext[0] - 0.5 * side, 0.5 * ext[2] - 0.5 * side, side, 1.0 if cache else 0.0]]


def _glowing_state(P, seed):
    """A random burning state whose light stays within binary16's range in
    the caches: temperature <= 1000 K, soot mass fraction <= 2e-3, heat
    release <= 500 kW/m^3."""
    S = random_state(P, seed=seed)
    S["s0"][..., 0] = np.minimum(S["s0"][..., 0], 1000.0)
    S["s0"][..., 3] = np.minimum(S["s0"][..., 3], 2e-3)
    S["s1"][..., 1] = np.minimum(S["s1"][..., 1], 5e5)
    return S


def _glowing_frame(nx, ny, nz, seed):
    """A frame of the packed volumes with soot, smoke and heat release (the
    oracle's pack of a random state, clamped within binary16's range as the
    golden frames are) and its emission CDF."""
    P = params_for(nx, ny, nz, dx=0.05, dt=0.02, ign_on=1.0)
    S = random_state(P, seed=seed)
    vol, solt, vel = oracle.render_pack(P, S["s0"], S["s1"], S["sol"], S["flags"], S["u"],
                                        S["v"], S["w"])
    v32 = vol.astype(np.float32)
    v32[..., 0] = np.clip(v32[..., 0], 0.0, 2.0)
    v32[..., 3] = np.clip(v32[..., 3], 0.0, 500.0)
    v32[..., 1] = np.minimum(v32[..., 1], 1000.0)
    vol = v32.astype(np.float16)
    lut = color.build_lut()
    e = oracle.render_ecells(P, vol, lut, color.chemi_block())
    d = dict(vol=vol, solt=solt, vel=vel, bricks=oracle.render_bricks((nx, ny, nz), vol, solt),
             lut=lut, ecdf=oracle.render_cdf(e))
    return P, d


@pytest.mark.parametrize("mode", ["cache", "path"])
def test_frame_vs_oracle(lib, mode):
    """A whole frame on a 24 x 40 x 20 grid: caches (16 rays), blur chain and
    4 samples of 32 x 20 pixels, GPU against oracle, each stage on the same
    inputs."""
    nx, ny, nz = 24, 40, 20
    P, d = _glowing_frame(nx, ny, nz, seed=11)
    cache = mode == "cache"
    rows = _rp_rows(P, 32, 20, 4, 7, cache, aperture=0.02)
    rp = _abi.PyroRenderParams.from_rows(rows)
    b = _bind(d)
    lvd = ((nx + 1) // 2, (ny + 1) // 2, (nz + 1) // 2)
    gres = 16
    lz, ly, lx = lvd[2], lvd[1], lvd[0]
    if cache:
        a, bb = _half_empty((lz, ly, lx, 4)), _half_empty((lz, ly, lx, 4))
        render.lightvol(rp, *_args(b), lvd, a, bb, rays=16)
        g = _half_empty((1, gres, gres, 4))
        render.lightground(rp, *_args(b), gres, g, rays=16)
        ea, eb = oracle.render_lightvol(rows, d["vol"], d["solt"], d["vel"], d["bricks"], d["lut"],
                                        d["ecdf"], lvd, lv_n=16)
        eg = oracle.render_lightground(rows, d["vol"], d["solt"], d["vel"], d["bricks"], d["lut"],
                                       d["ecdf"], gres, gr_n=16)
        A, B, G = host(a), host(bb), host(g)
        _cache_close(A, ea, max_bad=5e-3)
        _cache_close(B, eb, max_bad=5e-3)
        _cache_close(G, eg, max_bad=5e-3)
        assert np.abs(A.astype(np.float32)).max() > 0
        # blur and trace continue from the oracle's caches, so that each
        # stage is compared on the same inputs
        for ax in (0, 1, 2):
            ea, eb = oracle.render_blur(ea, ax, 2), oracle.render_blur(eb, ax, 2)
        for ax in (0, 1):
            eg = oracle.render_blur(eg, ax, 3)
    else:
        ea = eb = np.zeros((lz, ly, lx, 4), np.float16)
        eg = np.zeros((1, gres, gres, 4), np.float16)
    d.update(lvA=ea, lvB=eb, gE=eg)
    got = host(_trace_gpu(d, rp))
    want = oracle.render_trace(rows, d["vol"], d["solt"], d["vel"], d["bricks"], d["lut"],
                               d["ecdf"], ea, eb, eg)
    _pixels_close(got, want, max_bad=0.02)
    assert abs(got[:, :3].sum() - want[:, :3].sum()) <= 2e-2 * np.abs(want[:, :3]).sum()
    assert np.count_nonzero(want[:, :3]) > want[:, :3].size // 2


def test_renderer_frame_vs_oracle_chain(lib):
    """Renderer.render on a stepped simulation holding a burning state,
    against the oracle run through the reference's frame sequence
    (src/render.rs:250-447) on the simulation's own packed volumes: light
    caches, blur chain, 12 samples in dispatches of 8, mean per pixel."""
    sc = Scene.load(os.path.join(SCENES, "pool_small_8cm.toml"))
    sc.render.width, sc.render.height = 24, 16
    sc.render.camera = [1.52, 0.8, -1.5]  # the pool is at x = z = 1.52 m
    sc.render.target = [1.52, 0.4, 1.52]
    with Sim(sc) as sim:
        for _ in range(3):
            sim.step(0.02, want_stats=False)
        S = _glowing_state(sim.p, seed=5)
        sim.write_field(_abi.F_S0, S["s0"])
        sim.write_field(_abi.F_S1, S["s1"])
        r = render.Renderer(sc, sim, lv_rays=8, gr_rays=8, ground_res=16)
        img = r.render(sim, frame=2, spp=12)
        vol, solt, vel = (sim.read_field(f) for f in (_abi.F_RVOL, _abi.F_RSOL, _abi.F_RVEL))
        bricks, ecdf = sim.read_field(_abi.F_BRICKS), sim.read_field(_abi.F_ECDF)
    lut = color.build_lut()
    rows = np.array(r.base.rows())
    rows[1, 3] = 2
    lvd = r.lv_dims
    ea, eb = oracle.render_lightvol(rows, vol, solt, vel, bricks, lut, ecdf, lvd, lv_n=8)
    eg = oracle.render_lightground(rows, vol, solt, vel, bricks, lut, ecdf, 16, gr_n=8)
    for ax in (0, 1, 2):
        ea, eb = oracle.render_blur(ea, ax, 2), oracle.render_blur(eb, ax, 2)
    for ax in (0, 1):
        eg = oracle.render_blur(eg, ax, 3)
    acc = None
    for first, n in ((0, 8), (8, 4)):
        rows[0, 2], rows[0, 3] = first, n
        acc = oracle.render_trace(rows, vol, solt, vel, bricks, lut, ecdf, ea, eb, eg, accum=acc)
    want = (acc[:, :3] / np.maximum(acc[:, 3:4], 1.0)).reshape(16, 24, 3)
    assert img.shape == (16, 24, 3) and np.isfinite(img).all()
    scale = np.abs(want).max()
    assert scale > 0
    bad = (np.abs(img - want) > 2e-3 * scale).any(axis=2)
    assert bad.mean() <= 0.05, bad.mean()
    assert abs(img.sum() - want.sum()) <= 3e-2 * np.abs(want).sum()
