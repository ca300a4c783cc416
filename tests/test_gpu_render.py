"""The renderer's input pack (render.wgsl:3-61) on the GPU, through the C
ABI: the kernels against the golden vectors of the reference's WGSL and
against the oracle, and the simulation's pack of its own current fields.
Every comparison is bit for bit (binary16 volumes, round to nearest even)."""
import os

import numpy as np
import pytest

import oracle
from fields import params_for, random_state
from gpu_util import dev, host, params_dev, ptr, require_cuda
from pyro_b200 import _abi
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
