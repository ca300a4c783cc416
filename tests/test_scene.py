"""Scene description, parameter block and voxelizer (host-input side).

The first four tests restate the reference's own unit tests
(src/scene.rs:892-931); the voxelization they check runs through the CPU
oracle here, and tests/test_gpu_sim.py checks the GPU voxelizer against it
bit for bit.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

import oracle
from pyro_b200 import _abi
from pyro_b200.scene import MATERIALS, Scene, SceneError, material, shapes_array

SCENES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "pyro_b200", "scenes")


def _scene(objects: str) -> Scene:
    return Scene.from_toml_str(
        "[domain]\nsize = [1.6, 1.6, 1.6]\ncell = 0.05\n" + objects)


def _voxelize_cpu(sc: Scene) -> np.ndarray:
    g = sc.grid()
    sh = sc.shapes()
    arr = shapes_array(sh)
    dens, kind = sc.slot_tables()
    return oracle.voxelize(arr, len(sh), g.dims[0], g.dims[1], g.dims[2], g.dx,
                           float(np.float32(sc.sim.ambient_temp)), sc.sim.seed, dens, kind)


def test_grid_dims_are_multiples_of_16():
    # src/scene.rs:893-897
    assert _scene("").grid().dims == [32, 32, 32]


def test_box_voxel_volume():
    # src/scene.rs:900-908: 0.4 m box at 5 cm -> 512..=729 cells
    sc = _scene('[[object]]\nkind = "box"\nmaterial = "wood"\ncenter = [0.8, 0.4, 0.8]\n'
                'size = [0.4, 0.4, 0.4]\n')
    sol = _voxelize_cpu(sc)
    n = int((sol[..., 1] > 0.0).sum())
    assert 512 <= n <= 729, n


def test_thin_parts_and_shallow_pools_keep_one_cell():
    # src/scene.rs:911-925
    sc = _scene('[[object]]\nkind = "box"\nmaterial = "wood"\ncenter = [0.8, 0.8, 0.8]\n'
                'size = [0.5, 0.01, 0.5]\n'
                '[[object]]\nkind = "pool"\nmaterial = "heptane"\ncenter = [0.8, 0.0, 0.8]\n'
                'radius = 0.3\ndepth = 0.001\n')
    sol = _voxelize_cpu(sc)

    def at(i, j, k):
        return sol[k, j, i]

    assert at(16, 16, 16)[1] > 0.0 or at(16, 15, 16)[1] > 0.0, "thin plate dropped"
    assert at(16, 0, 16)[1] > 0.0, "shallow pool dropped"
    assert at(16, 1, 16)[1] == 0.0


def test_unknown_material_lists_choices():
    # src/scene.rs:928-931
    with pytest.raises(SceneError) as e:
        material("lava")
    assert "heptane" in str(e.value)


def test_unknown_object_kind_and_too_many_materials():
    with pytest.raises(SceneError):
        _scene('[[object]]\nkind = "torus"\nmaterial = "wood"\n').shapes()
    objs = "".join(f'[[object]]\nkind = "box"\nmaterial = "{m.name}"\nsize=[0.1,0.1,0.1]\n'
                   for m in MATERIALS[1:9])
    with pytest.raises(SceneError):
        _scene(objs).used_materials()
    with pytest.raises(SceneError):
        _scene('[[object]]\nkind = "box"\nmaterial = "steel"\n').params()


def test_params_block_layout_and_constants():
    sc = _scene('[[object]]\nkind = "pool"\nmaterial = "heptane"\ncenter = [0.8, 0.0, 0.8]\n'
                'radius = 0.5\ndepth = 0.05\n[ignition]\npos = [0.8, 0.1, 0.8]\n')
    p = sc.params()
    assert ctypes.sizeof(p) == 576
    b = p.to_bytes()
    assert len(b) == 576
    f = np.frombuffer(b, dtype=np.float32)
    u = np.frombuffer(b, dtype=np.uint32)
    assert list(u[:3]) == [32, 32, 32]
    assert f[4] == np.float32(0.05)                          # dx
    assert f[7] == np.float32(293.0)                         # t0
    assert f[21] == np.float32(np.float32(44.6e6) / np.float32(13.1e6))  # s_o2
    assert f[24] == np.float32(np.float32(0.037) * np.float32(2.5))     # soot_form
    assert f[43] == np.float32(0.5)                          # rad_len = 0.5 * 2r
    assert f[30] == 1.0 and f[31] == np.float32(1300.0)      # ign_on, ign_temp (defaults)
    assert f[35] == np.float32(0.25) and f[36] == np.float32(40e3)  # ign_r, ign_flux
    assert f[46] == np.float32(0.33)                         # rad_frac heptane
    m = f[48:].reshape(8, 12)
    assert m[0, 3] == 2.0                                     # slot 0 air (inert)
    assert list(m[1, :4]) == [684.0, 480000.0, 371.0, 1.0]   # heptane row
    assert m[1, 9] == 1.0


def test_scene_files_parse():
    files = sorted(glob.glob(os.path.join(SCENES, "*.toml")))
    assert len(files) >= 4
    # pool_2cm_exact: the loader's rounding of 3.0 x 7.3 x 3.0 m; the bench
    # sets the exact 150 x 365 x 150 with dims_override
    expect = {"pool_small_8cm": [32, 80, 32], "pool_2cm": [160, 320, 160],
              "pallets_5cm": [128, 240, 128], "bonfire_10cm": [160, 240, 160],
              "pool_2cm_exact": [144, 368, 144]}
    for f in files:
        sc = Scene.load(f)
        name = os.path.basename(f)[:-5]
        assert sc.grid().dims == expect[name], name
        assert len(sc.shapes()) > 0
        sc.params()
    # generator sizes: pallets 12 x (6 + 7) boxes, bonfire 28 + 14 logs + 15 crib
    assert len(Scene.load(os.path.join(SCENES, "pallets_5cm.toml")).shapes()) == 156
    assert len(Scene.load(os.path.join(SCENES, "bonfire_10cm.toml")).shapes()) == 57


def test_hash_matches_reference_formula():
    # src/scene.rs:662-667 restated independently in Python integers
    def h(v):
        x = (v * 747796405 + 2891336453) & 0xFFFFFFFF
        x = (((x >> ((x >> 28) + 4)) ^ x) * 277803737) & 0xFFFFFFFF
        x = ((x >> 22) ^ x) & 0xFFFFFFFF
        return np.float32(np.float32(x) / np.float32(4294967295.0))
    for v in [0, 1, 2, 12345, 0x9E3779B9, 0xFFFFFFFF]:
        assert oracle.hash_f(v) == h(v)


def test_voxel_jitter_and_inert_mass():
    sc = _scene('[[object]]\nkind = "box"\nmaterial = "wood"\ncenter = [0.4, 0.4, 0.4]\n'
                'size = [0.3, 0.3, 0.3]\n[[object]]\nkind = "sphere"\nmaterial = "steel"\n'
                'center = [1.2, 1.2, 1.2]\nradius = 0.2\n')
    sol = _voxelize_cpu(sc)
    wood = sol[sol[..., 0] == 1]
    steel = sol[sol[..., 0] == 2]
    assert len(wood) > 0 and len(steel) > 0
    assert np.all(steel[:, 1] == 1.0)
    assert wood[:, 1].min() >= 480 * 0.85 - 1e-3 and wood[:, 1].max() <= 480 * 1.15 + 1e-3
    assert np.all(sol[..., 3] == np.float32(293.0))
