"""Host side of the volume renderer, without a GPU: the tracer's uniform
block (struct RP, trace_lib.wgsl:1-14) and its construction by
Renderer::new (src/render.rs:142-210), the [render] table of a scene
(src/scene.rs:141-190), and the argument checks of the tracer's C entry
points, which fail before any device work."""
import ctypes
import math

import numpy as np
import pytest

from pyro_b200 import _abi, color, render
from pyro_b200.scene import Scene
from test_golden import _load


@pytest.fixture(scope="module")
def lib():
    return _abi.load()


def test_uniform_block_layout_and_rows():
    P = _abi.PyroRenderParams
    assert ctypes.sizeof(P) == 208
    offs = {name: getattr(P, name).offset for name, _ in P._fields_}
    assert offs == {"res": 0, "dims": 16, "cam_pos": 32, "cam_fwd": 48, "cam_right": 64,
                    "cam_up": 80, "a": 96, "b": 112, "soot": 128, "c": 144, "alb": 160,
                    "gc": 192}
    for mode in ("cache", "path"):
        rows = _load(f"trace_{mode}")["rp"]
        p = P.from_rows(rows)
        assert np.array_equal(np.array(p.rows(), np.float32), rows.astype(np.float32))
    with pytest.raises(ValueError):
        P.from_rows([[0, 0, 0, 0]] * 12)


SCENE = """
[domain]
size = [1.0, 2.0, 1.0]
cell = 0.05
[sim]
fps = 30.0
ambient_temp = 290.0
[render]
width = 640
height = 360
camera = [0.5, 1.0, -3.0]
target = [0.5, 0.8, 0.5]
fov = 40.0
aperture = 0.01
bounces = 3
mode = "path"
[[object]]
kind = "box"
material = "wood"
center = [0.5, 0.1, 0.5]
size = [0.2, 0.2, 0.2]
"""


def test_scene_render_table_and_defaults():
    sc = Scene.from_toml_str(SCENE)
    assert (sc.render.width, sc.render.height, sc.render.bounces) == (640, 360, 3)
    assert sc.render.mode == "path" and sc.render.spp == 64 and sc.render.chemi == 0.05
    d = Scene.from_toml_str("[domain]\nsize = [1.0, 1.0, 1.0]\ncell = 0.1\n").render
    assert (d.width, d.height, d.fov, d.step, d.mode) == (1280, 720, 45.0, 0.6, "cache")


def test_base_params_follow_the_reference_formulas():
    sc = Scene.from_toml_str(SCENE)
    g = sc.grid()
    p = render.base_params(sc, g.dims, g.dx)
    pos, tgt = np.array(sc.render.camera), np.array(sc.render.target)
    fwd = (tgt - pos) / np.linalg.norm(tgt - pos)
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    np.testing.assert_allclose(p.cam_pos[:3], pos, rtol=1e-6)
    np.testing.assert_allclose(p.cam_fwd[:3], fwd, atol=1e-6)
    np.testing.assert_allclose(p.cam_right[:3], right, atol=1e-6)
    np.testing.assert_allclose(p.cam_up[:3], up, atol=1e-6)
    assert p.cam_pos[3] == pytest.approx(math.tan(math.radians(40.0) / 2), rel=1e-6)
    assert p.cam_fwd[3] == pytest.approx(640 / 360, rel=1e-6)
    assert p.cam_right[3] == pytest.approx(0.01)
    assert p.cam_up[3] == pytest.approx(np.linalg.norm(tgt - pos), rel=1e-6)
    assert list(p.res) == [640, 360, 0, 0] and list(p.dims) == [*g.dims, 0]
    assert list(p.a) == pytest.approx([g.dx, 0.6, 180.0 / 360.0 / 30.0, 0.003], rel=1e-6)
    assert list(p.b) == pytest.approx([1.0, 0.12, 3.0, 0.05])
    assert list(p.soot[:3]) == pytest.approx(list(color.soot_extinction(0.25)), rel=1e-6)
    assert list(p.c) == pytest.approx([5.0, 0.92, 0.55, 290.0])
    assert list(p.alb) == pytest.approx([0.05, 0.32, 0, 0, 0, 0, 0, 0])  # air, wood
    ext = [g.dims[0] * g.dx, g.dims[2] * g.dx]
    side = 3 * max(ext)
    assert list(p.gc) == pytest.approx([0.5 * ext[0] - 0.5 * side, 0.5 * ext[1] - 0.5 * side,
                                        side, 0.0], rel=1e-6)


def _rp(**kw):
    p = _abi.PyroRenderParams.from_rows(_load("trace_cache")["rp"])
    for k, v in kw.items():
        getattr(p, k[:-2])[int(k[-1])] = v  # e.g. res_3=2000
    return p


def test_tracer_entry_points_reject_bad_arguments(lib):
    bad = _abi.PYRO_E_INVALID
    buf = ctypes.c_void_p(16)  # never dereferenced: every check fails first
    b5 = [buf] * 6
    assert lib.pyro_k_render_blur(buf, buf, 4, 4, 4, 0, 2, None) == bad  # same buffer
    assert lib.pyro_k_render_blur(buf, ctypes.c_void_p(32), 4, 4, 4, 3, 2, None) == bad
    assert lib.pyro_k_render_blur(buf, ctypes.c_void_p(32), 4, 4, 4, 0, 0, None) == bad
    assert lib.pyro_k_render_blur(buf, ctypes.c_void_p(32), 4, 4, 4, 0, 17, None) == bad
    assert lib.pyro_k_render_blur(buf, ctypes.c_void_p(32), 0, 4, 4, 0, 2, None) == bad
    assert b"radius" in lib.pyro_last_error() or b"dimensions" in lib.pyro_last_error()
    assert lib.pyro_k_render_trace(None, *b5, buf, buf, 2, 2, 2, buf, 8, buf, None) == bad
    assert b"null render parameters" in lib.pyro_last_error()
    r = _rp(res_3=2000)
    assert lib.pyro_k_render_trace(ctypes.byref(r), *b5, buf, buf, 2, 2, 2, buf, 8, buf,
                                   None) == bad
    r = _rp()
    assert lib.pyro_k_render_trace(ctypes.byref(r), *b5, None, buf, 2, 2, 2, buf, 8, buf,
                                   None) == bad  # light-cache mode without lvA
    assert b"light-cache" in lib.pyro_last_error()
    r = _rp(a_0=0.0)
    assert lib.pyro_k_render_trace(ctypes.byref(r), *b5, buf, buf, 2, 2, 2, buf, 8, buf,
                                   None) == bad
    r = _rp(b_2=100.0)
    assert lib.pyro_k_render_trace(ctypes.byref(r), *b5, buf, buf, 2, 2, 2, buf, 8, buf,
                                   None) == bad
    r = _rp()
    assert lib.pyro_k_render_lightvol(ctypes.byref(r), *b5, 2, 2, 2, 0, buf,
                                      ctypes.c_void_p(32), None) == bad  # no rays
    assert lib.pyro_k_render_lightvol(ctypes.byref(r), *b5, 2, 2, 2, 8, buf, buf,
                                      None) == bad  # lvA == lvB
    assert lib.pyro_k_render_lightground(ctypes.byref(r), *b5, 0, 8, buf, None) == bad
    r = _rp(dims_0=1)
    assert lib.pyro_k_render_lightground(ctypes.byref(r), *b5, 8, 8, buf, None) == bad
    assert b"grid dimensions" in lib.pyro_last_error()


def test_frame_plan_is_the_reference_sequence():
    """src/render.rs:372-418: the blur chain and the sample chunks."""
    plan = render.frame_plan(True, 20)
    assert plan[:2] == [("lightvol",), ("lightground",)]
    assert plan[2:10] == [("blur", "lvA", "t1", 0, 2), ("blur", "t1", "t2", 1, 2),
                          ("blur", "t2", "lvA", 2, 2), ("blur", "lvB", "t1", 0, 2),
                          ("blur", "t1", "t2", 1, 2), ("blur", "t2", "lvB", 2, 2),
                          ("blur", "gE", "gtmp", 0, 3), ("blur", "gtmp", "gE", 1, 3)]
    assert plan[10:] == [("trace", 0, 8), ("trace", 8, 8), ("trace", 16, 4)]
    assert render.frame_plan(False, 5) == [("trace", 0, 2), ("trace", 2, 2), ("trace", 4, 1)]
    assert render.frame_plan(False, 0) == []
