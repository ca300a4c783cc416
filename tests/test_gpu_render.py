"""The renderer's per-frame prologue on the GPU, through the C ABI: the input
pack (render.wgsl:3-61) bit for bit (binary16 volumes, round to nearest
even), the fire-light emission per cell (render.wgsl:63-98, exp(): 1e-5
relative) and its CDF (src/render.rs:316-333, one unit in the last place);
against the golden vectors of the reference's WGSL, the oracle, and the
simulation's own current fields."""
import os

import numpy as np
import pytest

import oracle
from fields import close, params_for, random_state
from gpu_util import dev, host, params_dev, ptr, require_cuda
from pyro_b200 import _abi, color
from pyro_b200.scene import Scene
from pyro_b200.sim import Sim
from test_golden import CASES, _load, _params

pytestmark = pytest.mark.gpu

SCENES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "pyro_b200", "scenes")


@pytest.fixture(scope="module")
def lib():
    return require_cuda()


def _pack(lib, P, S):
    nx, ny, nz = int(P.nx), int(P.ny), int(P.nz)
    out = [dev(np.full((nz, ny, nx, 4), np.nan, np.float16)) for _ in range(3)]
    nb = ((nz + 7) // 8, (ny + 7) // 8, (nx + 7) // 8)
    br = dev(np.full(nb, -1.0, np.float32))
    assert lib.pyro_k_render_pack(ptr(params_dev(P)), nx, ny, nz, ptr(dev(S["s0"])),
                                  ptr(dev(S["s1"])), ptr(dev(S["sol"])), ptr(dev(S["flags"])),
                                  ptr(dev(S["u"])), ptr(dev(S["v"])), ptr(dev(S["w"])),
                                  ptr(out[0]), ptr(out[1]), ptr(out[2]), None) == 0
    assert lib.pyro_k_render_bricks(nx, ny, nz, ptr(out[0]), ptr(out[1]), ptr(br), None) == 0
    return [host(t) for t in out] + [host(br)]


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint16), np.asarray(b).view(np.uint16))


@pytest.mark.parametrize("case", CASES)
def test_render_pack_golden(lib, case):
    d = _load(f"render_{case}")
    vol, solt, vel, br = _pack(lib, _params(d), d)
    assert _same(vol, d["vol"]) and _same(solt, d["solt"]) and _same(vel, d["vel"])
    assert np.array_equal(br, d["bricks"])


@pytest.mark.parametrize("nx,ny,nz,seed", [(24, 32, 20, 0), (33, 17, 9, 1), (64, 40, 48, 2),
                                           (7, 70, 5, 3)])
def test_render_pack_vs_oracle(lib, nx, ny, nz, seed):
    P = params_for(nx, ny, nz, dx=0.05, dt=0.02, ign_on=1.0)
    S = random_state(P, seed=seed)
    vol, solt, vel, br = _pack(lib, P, S)
    ev, es, ew = oracle.render_pack(P, S["s0"], S["s1"], S["sol"], S["flags"], S["u"], S["v"],
                                    S["w"])
    assert _same(vol, ev) and _same(solt, es) and _same(vel, ew)
    assert np.array_equal(br, oracle.render_bricks((nx, ny, nz), ev, es))


def test_sim_render_pack_packs_the_current_fields(lib):
    sc = Scene.load(os.path.join(SCENES, "pool_small_8cm.toml"))
    with Sim(sc) as sim:
        with pytest.raises(RuntimeError):
            sim.read_field(_abi.F_RVOL)  # nothing packed yet
        for _ in range(5):
            sim.step(0.02, want_stats=False)
        vol, solt, vel, br = sim.read_render_volumes()
        P = sim.p
        f = {k: sim.read_field(w) for k, w in (("s0", _abi.F_S0), ("s1", _abi.F_S1),
                                               ("sol", _abi.F_SOL), ("flags", _abi.F_FLAGS),
                                               ("u", _abi.F_U), ("v", _abi.F_V),
                                               ("w", _abi.F_W))}
        ev, es, ew = oracle.render_pack(P, f["s0"], f["s1"], f["sol"], f["flags"], f["u"],
                                        f["v"], f["w"])
        assert _same(vol, ev) and _same(solt, es) and _same(vel, ew)
        assert np.array_equal(br, oracle.render_bricks(sim.dims, ev, es))
        assert np.isfinite(vol.astype(np.float32)).all() and br.max() > 0.0


def _emission(lib, P, vol, lut, chemi):
    nx, ny, nz = int(P.nx), int(P.ny), int(P.nz)
    e = dev(np.full((nz, ny, nx), np.nan, np.float32))
    assert lib.pyro_k_render_ecells(ptr(params_dev(P)), nx, ny, nz, ptr(dev(vol)), ptr(dev(lut)),
                                    np.ascontiguousarray(chemi, np.float32).ctypes.data_as(
                                        __import__("ctypes").c_void_p), ptr(e), None) == 0
    return host(e)


def _cdf(lib, e):
    ed = dev(np.ascontiguousarray(e, np.float32).reshape(-1))
    c = dev(np.full(e.size + 1, np.nan, np.float32))
    assert lib.pyro_k_render_cdf(e.size, ptr(ed), ptr(c), None) == 0
    return host(c)


def _cdf_close(got, exp):
    """The GPU's FP64 sums run in another order than the reference's
    sequential loop: each float of the CDF may differ by one unit in the
    last place, the total (a float) by 1e-6 relative."""
    g, x = got[:-1].astype(np.float64), exp[:-1].astype(np.float64)
    assert np.all(np.abs(g - x) <= np.spacing(np.abs(exp[:-1])).astype(np.float64))
    assert abs(float(got[-1]) - float(exp[-1])) <= 1e-6 * abs(float(exp[-1]))
    assert np.all(np.diff(got[:-1]) >= 0)


@pytest.mark.parametrize("case", CASES)
def test_render_emission_golden(lib, case):
    d = _load(f"render_{case}")
    P = _params(d)
    e = _emission(lib, P, d["vol"], d["lut"], d["chemi"])
    close(e, d["ecell"], name="ecell")
    _cdf_close(_cdf(lib, e), oracle.render_cdf(e))


@pytest.mark.parametrize("nx,ny,nz,seed", [(24, 32, 20, 0), (64, 40, 48, 2), (7, 70, 5, 3)])
def test_render_emission_vs_oracle(lib, nx, ny, nz, seed):
    P = params_for(nx, ny, nz, dx=0.05, dt=0.02, ign_on=1.0)
    S = random_state(P, seed=seed)
    vol, _, _ = oracle.render_pack(P, S["s0"], S["s1"], S["sol"], S["flags"], S["u"], S["v"],
                                   S["w"])
    lut, chemi = color.build_lut(), color.chemi_block()
    e = _emission(lib, P, vol, lut, chemi)
    close(e, oracle.render_ecells(P, vol, lut, chemi), name="ecell")
    _cdf_close(_cdf(lib, e), oracle.render_cdf(e))


def test_render_cdf_long_and_empty(lib):
    """Several scan blocks (8192 values each) and a partial last one; an
    all-zero emission gives a zero CDF and total."""
    rng = np.random.default_rng(7)
    e = rng.exponential(1.0, 8192 * 37 + 1234).astype(np.float32)
    e[rng.random(e.size) < 0.3] = 0.0
    e[:5] = -1.0  # negative emission counts as zero
    _cdf_close(_cdf(lib, e), oracle.render_cdf(e))
    z = np.zeros(1000, np.float32)
    assert np.array_equal(_cdf(lib, z), np.zeros(1001, np.float32))


def test_sim_render_emission(lib):
    sc = Scene.load(os.path.join(SCENES, "pool_small_8cm.toml"))
    with Sim(sc) as sim:
        for _ in range(3):
            sim.step(0.02, want_stats=False)
        # a burning gas state (soot, smoke, heat release) in the step's fields
        S = random_state(sim.p, seed=5)
        sim.write_field(_abi.F_S0, S["s0"])
        sim.write_field(_abi.F_S1, S["s1"])
        sim.render_pack(False)
        sim.render_emission()
        e = sim.read_field(_abi.F_ECELL)
        cdf = sim.read_field(_abi.F_ECDF)
        vol = sim.read_field(_abi.F_RVOL)
        close(e, oracle.render_ecells(sim.p, vol, color.build_lut(), color.chemi_block()),
              name="ecell")
        _cdf_close(cdf, oracle.render_cdf(e))
        assert (e > 0).any() and cdf[-1] > 0
