"""The CUDA kernels against the golden vectors of the reference's own WGSL
(tests/golden, see make_golden.py), through the C ABI: bit-exact where the
kernel has no exp(), 1e-5 relative otherwise."""
import numpy as np
import pytest

from fields import close, face_valid_mask
from gpu_util import dev, host, params_dev, ptr, require_cuda, stats_dev
from test_golden import CASES, _load, _params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    return require_cuda()


def _dims(P):
    return int(P.nx), int(P.ny), int(P.nz)


@pytest.mark.parametrize("case", CASES)
def test_solid_react_forces(lib, case):
    d = _load(f"solid_{case}")
    P = _params(d)
    nx, ny, nz = _dims(P)
    Pd = params_dev(P)
    so, py, fl = dev(np.zeros_like(d["sol"])), dev(np.zeros_like(d["sol"])), \
        dev(np.zeros((nz, ny, nx), np.uint32))
    sd = stats_dev()
    assert lib.pyro_k_solid(ptr(Pd), nx, ny, nz, ptr(dev(d["sol"])), ptr(so), ptr(py), ptr(fl),
                            ptr(dev(d["s0"])), ptr(sd), None) == 0
    assert np.array_equal(host(fl), d["flags"])
    close(host(so), d["sol_out"], name="sol")
    close(host(py), d["pyr"], name="pyr")
    d = _load(f"react_{case}")
    o0, o1 = dev(np.zeros_like(d["s0"])), dev(np.zeros_like(d["s1"]))
    sd = stats_dev()
    assert lib.pyro_k_react(ptr(Pd), nx, ny, nz, ptr(dev(d["s0"])), ptr(dev(d["s1"])), ptr(o0),
                            ptr(o1), ptr(dev(d["flags"])), ptr(dev(d["sol"])), ptr(dev(d["pyr"])),
                            ptr(dev(d["curl"])), ptr(sd), None) == 0
    close(host(o0), d["o0"], name="s0")
    close(host(o1), d["o1"], name="s1")
    g = host(sd)
    for i in (0, 1, 3, 6, 8):
        assert abs(g[i] - d["stats"][i]) <= 1e-4 * abs(d["stats"][i]) + 1e-30, i
    d = _load(f"forces_{case}")
    u, v, w = dev(d["u"]), dev(d["v"]), dev(d["w"])
    assert lib.pyro_k_forces(ptr(Pd), nx, ny, nz, ptr(u), ptr(v), ptr(w), ptr(dev(d["s0"])),
                             ptr(dev(d["s1"])), ptr(dev(d["curl"])), ptr(dev(d["flags"])),
                             None) == 0
    for k, (g_, name) in enumerate(((u, "ou"), (v, "ov"), (w, "ow"))):
        m = face_valid_mask(P, k)
        close(host(g_)[m], d[name][m], name=name)


@pytest.mark.parametrize("case", CASES)
def test_exact_kernels(lib, case):
    d = _load(f"curl_{case}")
    P = _params(d)
    nx, ny, nz = _dims(P)
    Pd = params_dev(P)
    c = dev(np.zeros_like(d["curl"]))
    sd = stats_dev()
    assert lib.pyro_k_curl(ptr(Pd), nx, ny, nz, ptr(dev(d["u"])), ptr(dev(d["v"])),
                           ptr(dev(d["w"])), ptr(c), ptr(sd), None) == 0
    assert np.array_equal(host(c), d["curl"])
    assert host(sd)[5] == d["stats"][5]
    d = _load(f"adv_vel_{case}")
    z = np.zeros_like(d["u"])
    bufs = [dev(z) for _ in range(6)]
    assert lib.pyro_k_adv_vel(ptr(Pd), nx, ny, nz, ptr(dev(d["u"])), ptr(dev(d["v"])),
                              ptr(dev(d["w"])), *[ptr(b) for b in bufs], ptr(dev(d["flags"])),
                              None) == 0
    for k, name in enumerate(("hu", "hv", "hw", "ou", "ov", "ow")):
        m = face_valid_mask(P, k % 3)
        assert np.array_equal(host(bufs[k])[m], d[name][m]), name
    d = _load(f"adv_scalars_{case}")
    z = np.zeros_like(d["s0"])
    bufs = [dev(z) for _ in range(4)]
    assert lib.pyro_k_adv_scalars(ptr(Pd), nx, ny, nz, ptr(dev(d["u"])), ptr(dev(d["v"])),
                                  ptr(dev(d["w"])), ptr(dev(d["s0"])), ptr(dev(d["s1"])),
                                  *[ptr(b) for b in bufs], None) == 0
    for k, name in enumerate(("h0", "h1", "o0", "o1")):
        assert np.array_equal(host(bufs[k]), d[name]), name
    d = _load(f"divergence_{case}")
    b = dev(np.zeros_like(d["b"]))
    assert lib.pyro_k_divergence(ptr(Pd), nx, ny, nz, ptr(dev(d["u"])), ptr(dev(d["v"])),
                                 ptr(dev(d["w"])), ptr(dev(d["s1"])), ptr(dev(d["flags"])), ptr(b),
                                 None) == 0
    assert np.array_equal(host(b), d["b"])
    d = _load(f"project_{case}")
    u, v, w = dev(d["u"]), dev(d["v"]), dev(d["w"])
    assert lib.pyro_k_project(ptr(Pd), nx, ny, nz, ptr(u), ptr(v), ptr(w), ptr(dev(d["phi"])),
                              ptr(dev(d["flags"])), None) == 0
    for k, (g_, name) in enumerate(((u, "ou"), (v, "ov"), (w, "ow"))):
        m = face_valid_mask(P, k)
        assert np.array_equal(host(g_)[m], d[name][m]), name


def test_mg(lib):
    for name, color, om in (("mg_smooth_c0_w10", 0, 1.0), ("mg_smooth_c1_w10", 1, 1.0),
                            ("mg_smooth_c0_w16", 0, 1.6), ("mg_smooth_c1_w16", 1, 1.6)):
        d = _load(name)
        nx, ny, nz = (int(v) for v in d["dims"])
        p = dev(d["p"])
        assert lib.pyro_k_mg_smooth(nx, ny, nz, float(d["h"]), ptr(dev(d["b"])), ptr(dev(d["f"])),
                                    ptr(p), color, om, None) == 0
        assert np.array_equal(host(p), d["out"]), name
    d = _load("mg_restrict")
    nx, ny, nz = (int(v) for v in d["dims"])
    cx, cy, cz = (nx + 1) // 2, (ny + 1) // 2, (nz + 1) // 2
    bc, pc, fc = dev(np.zeros_like(d["bc"])), dev(np.ones_like(d["pc"])), \
        dev(np.zeros_like(d["fc"]))
    assert lib.pyro_k_mg_restrict(nx, ny, nz, float(d["h"]), ptr(dev(d["p"])), ptr(dev(d["b"])),
                                  ptr(dev(d["f"])), cx, cy, cz, ptr(bc), ptr(pc), ptr(fc),
                                  None) == 0
    assert np.array_equal(host(fc), d["fc"])
    assert np.array_equal(host(bc), d["bc"])
    d = _load("mg_prolong")
    p = dev(d["p"])
    assert lib.pyro_k_mg_prolong(nx, ny, nz, ptr(dev(d["pc"])), ptr(dev(d["f"])), ptr(p), cx, cy,
                                 cz, ptr(dev(d["fc"])), None) == 0
    assert np.array_equal(host(p), d["out"])
