"""The simulation object through the C ABI against the CPU oracle:
voxelizer bit-exactness, one full substep (graph replay) from a developed
state, a multi-step drift budget, statistics decoding and the field API."""
import os

import numpy as np
import pytest

import oracle
from fields import close, face_valid_mask
from gpu_util import require_cuda
from pyro_b200 import _abi
from pyro_b200.scene import Scene, shapes_array
from pyro_b200.sim import Sim, Stats, voxelize

pytestmark = pytest.mark.gpu

SCENES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "pyro_b200", "scenes")


@pytest.fixture(scope="module")
def lib():
    return require_cuda()


def _scene(name, cell=None):
    sc = Scene.load(os.path.join(SCENES, name + ".toml"))
    if cell is not None:
        sc.domain.cell = cell
    return sc


def _oracle_vox(sc):
    g = sc.grid()
    sh = sc.shapes()
    dens, kind = sc.slot_tables()
    return oracle.voxelize(shapes_array(sh), len(sh), g.dims[0], g.dims[1], g.dims[2], g.dx,
                           float(np.float32(sc.sim.ambient_temp)), sc.sim.seed, dens, kind)


@pytest.mark.parametrize("name,cell", [("pool_small_8cm", None), ("pool_2cm", 0.04),
                                       ("pallets_5cm", 0.1), ("bonfire_10cm", 0.2)])
def test_voxelizer_bit_exact(lib, name, cell):
    sc = _scene(name, cell)
    g = voxelize(sc)
    e = _oracle_vox(sc)
    assert np.array_equal(g, e)
    assert (g[..., 1] > 0).sum() > 0


FIELDS = [_abi.F_S0, _abi.F_S1, _abi.F_SOL, _abi.F_PYR, _abi.F_CURL, _abi.F_U, _abi.F_V,
          _abi.F_W, _abi.F_PHI, _abi.F_B]
NAMES = {_abi.F_S0: "s0", _abi.F_S1: "s1", _abi.F_SOL: "sol", _abi.F_PYR: "pyr",
         _abi.F_CURL: "curl", _abi.F_U: "u", _abi.F_V: "v", _abi.F_W: "w", _abi.F_PHI: "phi",
         _abi.F_B: "b", _abi.F_FLAGS: "flags"}


def _developed(name="pool_small_8cm", steps=60, dt=0.01):
    """GPU simulation run until the flame develops; returns (sim, t)."""
    sc = _scene(name)
    sim = Sim(sc)
    for k in range(steps):
        sim.step(dt, False)
    sim.sync()
    return sc, sim


def _copy_to_oracle(sim):
    o = oracle.OracleSim(sim.p, sim.read_field(_abi.F_SOL), sim.cycles)
    for f in (_abi.F_S0, _abi.F_S1, _abi.F_SOL, _abi.F_U, _abi.F_V, _abi.F_W, _abi.F_PHI):
        o.write_field(f, sim.read_field(f))
    return o


def _compare(sim, o, P, rtol, floor, tag):
    assert np.array_equal(sim.read_field(_abi.F_FLAGS), o.read_field(oracle.F_FLAGS)), tag
    for f in FIELDS:
        g, e = sim.read_field(f), o.read_field(f)
        if f in (_abi.F_U, _abi.F_V, _abi.F_W):
            m = face_valid_mask(P, f - _abi.F_U)
            g, e = g[m], e[m]
        close(g, e, rtol=rtol, floor=floor, name=f"{tag}:{NAMES[f]}")


def test_one_substep_matches_oracle(lib):
    sc, sim = _developed()
    assert float(np.abs(sim.read_field(_abi.F_V)).max()) > 0.1  # the plume is moving
    o = _copy_to_oracle(sim)
    dt, t = np.float32(0.008), np.float32(sim.time)
    sim.step(dt, True)
    o.step(dt, t, 1.0, True)
    _compare(sim, o, sim.p, 1e-5, 1e-5, "step")
    g = sim.read_stats().raw
    e = o.read_stats()
    for i in (0, 1, 2, 3, 6, 7, 8, 9, 10, 11):
        assert abs(g[i] - e[i]) <= 2e-4 * abs(e[i]) + 1e-12, (i, g[i], e[i])
    for i in (4, 5):
        assert abs(g[i] - e[i]) <= 1e-5 * abs(e[i]), (i, g[i], e[i])
    sim.close()


def test_one_substep_matches_oracle_at_the_2cm_pool(lib):
    """The metric's workload: the 2 cm pool at the reference's rounding,
    160 x 320 x 160 = 8.19 M cells, 4 multigrid levels.  Developed on the GPU
    for 0.5 s of simulated time at the frame loop's CFL substep, then one
    substep (graph replay, statistics on) against the oracle from the same
    state."""
    sc = _scene("pool_2cm")
    sim = Sim(sc)
    assert tuple(sim.dims) == (160, 320, 160)
    dt = np.float32(1.0 / 180.0)
    for k in range(90):
        sim.step(dt, False)
    sim.sync()
    assert float(np.abs(sim.read_field(_abi.F_V)).max()) > 0.1  # the plume is moving
    o = _copy_to_oracle(sim)
    t = np.float32(sim.time)
    sim.step(dt, True)
    o.step(dt, t, 1.0, True)
    _compare(sim, o, sim.p, 1e-5, 1e-5, "2 cm step")
    g = sim.read_stats().raw
    e = o.read_stats()
    for i in (0, 1, 2, 3, 6, 7, 8, 9, 10, 11):
        assert abs(g[i] - e[i]) <= 2e-4 * abs(e[i]) + 1e-12, (i, g[i], e[i])
    o.close()
    sim.close()


@pytest.mark.parametrize("name,dims,dt", [("pallets_5cm", (128, 240, 128), 1.0 / 90.0),
                                          ("bonfire_10cm", (160, 240, 160), 1.0 / 60.0)])
def test_one_substep_matches_oracle_at_the_named_shapes(lib, name, dims, dt):
    """The other named workloads at full size: the 12-pallet stack at 5 cm
    (3.9 M cells, wood with char) and the log bonfire at 10 cm (6.1 M cells,
    wind), each developed on the GPU for 0.5 s and then stepped once on the
    GPU and in the oracle from the same state."""
    sc = _scene(name)
    sim = Sim(sc)
    assert tuple(sim.dims) == dims
    dt = np.float32(dt)
    for k in range(int(round(0.5 / float(dt)))):
        sim.step(dt, False)
    sim.sync()
    assert float(np.abs(sim.read_field(_abi.F_V)).max()) > 0.05
    o = _copy_to_oracle(sim)
    t = np.float32(sim.time)
    sim.step(dt, True)
    o.step(dt, t, 1.0, True)
    _compare(sim, o, sim.p, 1e-5, 1e-5, f"{name} step")
    g = sim.read_stats().raw
    e = o.read_stats()
    for i in (0, 1, 2, 3, 6, 7, 8, 9, 10, 11):
        assert abs(g[i] - e[i]) <= 2e-4 * abs(e[i]) + 1e-12, (i, g[i], e[i])
    o.close()
    sim.close()


def test_statistics_of_the_previous_substep(lib):
    """Sim.read_stats_prev returns the statistics block of the stats substep
    before the last one, the same block read_stats gave right after it."""
    sc, sim = _developed(steps=20)
    dt = np.float32(0.008)
    with pytest.raises(Exception):
        sim.read_stats_prev()  # fewer than two stats substeps
    sim.step(dt, True)
    a = sim.read_stats().raw.copy()
    sim.step(dt, False)
    sim.step(dt, True)
    p = sim.read_stats_prev().raw.copy()
    b = sim.read_stats().raw.copy()
    assert np.array_equal(p, a)
    assert not np.array_equal(b, a)
    sim.step(dt, True)
    assert np.array_equal(sim.read_stats_prev().raw, b)
    sim.close()


def test_several_substeps_stay_within_drift_budget(lib):
    sc, sim = _developed(steps=40)
    o = _copy_to_oracle(sim)
    t = np.float32(sim.time)
    for k in range(5):
        dt = np.float32(0.008)
        sim.step(dt, k == 4)
        o.step(dt, t, 1.0, k == 4)
        t = np.float32(t + dt)
    # chaotic growth of last-ulp exp() differences: 1e-3 relative of each
    # channel's magnitude after 5 substeps
    _compare(sim, o, sim.p, 1e-3, 1e-3, "5 steps")
    sim.close()


def test_stats_decode_and_flame_height(lib):
    # the pool needs ~1 s of ignition flux before it evaporates and burns
    sc, sim = _developed(steps=250)
    sim.step(0.01, True)
    st = sim.read_stats()
    assert st.max_t > 1000.0 and st.max_u > 0.0
    assert st.hrr > 0.0 and st.pyro > 0.0 and st.area > 0.0
    assert 0.0 < st.resid < 1.0
    assert len(st.layers) == sim.dims[1]
    assert abs(sum(st.layers) - st.hrr) <= 0.05 * st.hrr
    h = st.flame_height(sim.dx)
    assert 0.0 < h <= sim.dims[1] * sim.dx
    sim.close()


def test_field_roundtrip_info_and_errors(lib):
    sc = _scene("pool_small_8cm")
    sim = Sim(sc)
    info = sim.info()
    assert (info.nx, info.ny, info.nz, info.levels) == (32, 80, 32, 3)
    assert [tuple(info.level_dims[l]) for l in range(3)] == [(32, 80, 32), (16, 40, 16),
                                                              (8, 20, 8)]
    s0 = sim.read_field(_abi.F_S0)
    assert np.all(s0[..., 0] == np.float32(293.0)) and np.all(s0[..., 2] == np.float32(0.233))
    s0[..., 0] = 400.0
    sim.write_field(_abi.F_S0, s0)
    assert np.all(sim.read_field(_abi.F_S0)[..., 0] == 400.0)
    ptr_, n = sim.device_ptr(_abi.F_PHI)
    assert ptr_ != 0 and n == 32 * 80 * 32 * 4
    with pytest.raises(_abi.PyroError):
        sim.write_field(_abi.F_S0, s0[:1])
    with pytest.raises(_abi.PyroError):
        sim.read_field(99)
    sim.close()


@pytest.mark.parametrize("mode", [_abi.SOLVER_VCYCLE_TOL, _abi.SOLVER_MGPCG,
                                  _abi.SOLVER_MGPCG_BF16])
def test_tolerance_solvers_inside_the_step(lib, mode):
    sc, sim = _developed(steps=30)
    tol = 1e-4 if mode != _abi.SOLVER_VCYCLE_TOL else 2e-2
    sim.set_solver(mode, tol, 60)
    sim.step(0.01, True)
    info = sim.last_solve()
    assert info.converged == 1 and info.rel_resid <= tol, (info.iterations, info.rel_resid)
    phi, b, fl = (sim.read_field(_abi.F_PHI), sim.read_field(_abi.F_B),
                  sim.read_field(_abi.F_FLAGS))
    rel = oracle.poisson_relres(tuple(sim.dims), sim.dx, phi, b, fl)
    assert abs(rel - info.rel_resid) <= 0.02 * info.rel_resid + 1e-9
    sim.close()
