"""The simulation object: host-side mirror of the reference's `Sim`
(src/sim.rs:42-531) over the C ABI of libpyro_b200.so.

    scene = Scene.load("scenes/pool.toml")
    sim = Sim(scene)                 # Sim::new
    sim.step(dt, want_stats=True)    # Sim::step
    st = sim.read_stats()            # Sim::read_stats -> Stats
    s0, s1 = sim.read_scalars()      # Sim::read_scalars

Every substep runs on the GPU as a captured CUDA graph; this module only
passes host values (dt, time, ignition on/off) and copies results.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from . import _abi
from .scene import Scene, shapes_array

STATS_N = _abi.STATS_N


@dataclass
class Stats:
    """Per-substep statistics (src/sim.rs:73-87), decoded as read_stats
    does (src/sim.rs:510-530)."""
    hrr: float = 0.0
    rad: float = 0.0
    pyro: float = 0.0
    soot: float = 0.0
    max_t: float = 0.0
    max_u: float = 0.0
    solid: float = 0.0
    area: float = 0.0
    resid: float = 0.0
    layers: List[float] = field(default_factory=list)
    raw: Optional[np.ndarray] = None

    @staticmethod
    def decode(v: np.ndarray, ny: int) -> "Stats":
        v = np.asarray(v, dtype=np.float32)
        resid = float(np.sqrt(np.float32(v[10] / v[11]))) if v[11] > 0.0 else 0.0
        return Stats(hrr=float(v[0]), rad=float(v[1]), pyro=float(v[2]), soot=float(v[3]),
                     max_t=float(v[4]), max_u=float(v[5]), solid=float(v[7]), area=float(v[9]),
                     resid=resid, layers=[float(x) for x in v[16:16 + min(ny, 1024)]], raw=v)

    def flame_height(self, dx: float) -> float:
        """Height where the cumulative layer HRR reaches 95 % of the total
        (src/sim.rs:90-104)."""
        layers = np.asarray(self.layers, dtype=np.float32)
        tot = np.float32(layers.sum(dtype=np.float32))
        if tot <= 0.0:
            return 0.0
        acc = np.float32(0.0)
        for j, v in enumerate(layers):
            acc = np.float32(acc + v)
            if acc >= np.float32(0.95) * tot:
                return (j + 1.0) * dx
        return len(layers) * dx


def voxelize(scene: Scene) -> np.ndarray:
    """Scene::voxelize (src/scene.rs:621-667) on the GPU: returns the
    initial solid state, (nz, ny, nx, 4) float32 = (slot, mass, char, Ts)."""
    import torch  # device memory for the output only

    g = scene.grid()
    nx, ny, nz = g.dims
    shapes = scene.shapes()
    arr = shapes_array(shapes)
    dens, kind = scene.slot_tables()
    lib = _abi.load()
    out = torch.empty((nz, ny, nx, 4), dtype=torch.float32, device="cuda")
    _abi.check("pyro_voxelize", lib.pyro_voxelize(
        arr, len(shapes), nx, ny, nz, g.dx, float(np.float32(scene.sim.ambient_temp)),
        scene.sim.seed & 0xFFFFFFFF, ctypes.cast(dens, ctypes.c_void_p),
        ctypes.cast(kind, ctypes.c_void_p), ctypes.c_void_p(out.data_ptr()), None))
    return out.cpu().numpy()


class Sim:
    """GPU fire simulation with the reference `Sim`'s methods."""

    def __init__(self, scene: Scene, sol_init: Optional[np.ndarray] = None,
                 params: Optional[_abi.PyroParams] = None):
        self._lib = _abi.load()
        self.scene = scene
        self.p = params.copy() if params is not None else scene.params()
        self.dims = [self.p.nx, self.p.ny, self.p.nz]
        self.dx = float(self.p.dx)
        self.time = np.float32(0.0)
        self.cycles = int(scene.sim.pressure_cycles)
        self.ign_until = np.float32(scene.ign_until())
        if sol_init is None:
            sol_init = voxelize(scene)
        sol_init = np.ascontiguousarray(sol_init, dtype=np.float32)
        if sol_init.size != self.cells() * 4:
            raise ValueError("sol_init has the wrong size")
        h = ctypes.c_void_p()
        _abi.check("pyro_sim_create", self._lib.pyro_sim_create(
            ctypes.byref(self.p), sol_init.ctypes.data_as(ctypes.c_void_p), self.cycles,
            ctypes.byref(h)))
        self._h = h
        self._stats = np.zeros(STATS_N, dtype=np.float32)

    # ------------------------------------------------------------- lifecycle
    def close(self):
        if getattr(self, "_h", None):
            self._lib.pyro_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------ api
    def cells(self) -> int:
        return self.dims[0] * self.dims[1] * self.dims[2]

    def faces(self) -> int:
        return (self.dims[0] + 1) * (self.dims[1] + 1) * (self.dims[2] + 1)

    def step(self, dt: float, want_stats: bool) -> None:
        """One substep (src/sim.rs:246-423): dt, the current time and the
        ignition switch time < ign_until are passed to the device."""
        ign_on = 1.0 if self.time < self.ign_until else 0.0
        _abi.check("pyro_sim_step", self._lib.pyro_sim_step(
            self._h, float(np.float32(dt)), float(self.time), ign_on, 1 if want_stats else 0))
        self.time = np.float32(self.time + np.float32(dt))

    def read_stats(self) -> Stats:
        _abi.check("pyro_sim_read_stats", self._lib.pyro_sim_read_stats(
            self._h, self._stats.ctypes.data_as(ctypes.c_void_p), STATS_N))
        return Stats.decode(self._stats.copy(), self.dims[1])

    def read_stats_prev(self) -> Stats:
        """Statistics of the stats substep before the last one, waiting only
        for that substep: enqueue substep k, then read substep k - 1's while
        k runs (valid until the next stats substep is enqueued)."""
        _abi.check("pyro_sim_read_stats_prev", self._lib.pyro_sim_read_stats_prev(
            self._h, self._stats.ctypes.data_as(ctypes.c_void_p), STATS_N))
        return Stats.decode(self._stats.copy(), self.dims[1])

    def read_field(self, which: int) -> np.ndarray:
        nx, ny, nz = self.dims
        if which in (_abi.F_RVOL, _abi.F_RSOL, _abi.F_RVEL):
            out = np.empty((nz, ny, nx, 4), dtype=np.float16)
        elif which == _abi.F_ECELL:
            out = np.empty((nz, ny, nx), dtype=np.float32)
        elif which == _abi.F_ECDF:
            out = np.empty(nx * ny * nz + 1, dtype=np.float32)
        elif which == _abi.F_BRICKS:
            out = np.empty(((nz + 7) // 8, (ny + 7) // 8, (nx + 7) // 8), dtype=np.float32)
        elif which in (_abi.F_U, _abi.F_V, _abi.F_W):
            out = np.empty((nz + 1, ny + 1, nx + 1), dtype=np.float32)
        elif which == _abi.F_FLAGS:
            out = np.empty((nz, ny, nx), dtype=np.uint32)
        elif which in (_abi.F_PHI, _abi.F_B):
            out = np.empty((nz, ny, nx), dtype=np.float32)
        else:
            out = np.empty((nz, ny, nx, 4), dtype=np.float32)
        _abi.check("pyro_sim_read_field", self._lib.pyro_sim_read_field(
            self._h, which, out.ctypes.data_as(ctypes.c_void_p), out.nbytes))
        return out

    def write_field(self, which: int, arr: np.ndarray) -> None:
        arr = np.ascontiguousarray(arr)
        _abi.check("pyro_sim_write_field", self._lib.pyro_sim_write_field(
            self._h, which, arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes))

    def read_scalars(self) -> Tuple[np.ndarray, np.ndarray]:
        """(s0, s1) copies, each (nz, ny, nx, 4) (src/sim.rs:494-508)."""
        return self.read_field(_abi.F_S0), self.read_field(_abi.F_S1)

    def render_pack(self, bricks: bool = True) -> None:
        """The renderer's per-frame input pack (render.wgsl:3-61) into the
        simulation's volumes; read them with read_field(F_RVOL / F_RSOL /
        F_RVEL / F_BRICKS) or borrow them with device_ptr."""
        _abi.check("pyro_sim_render_pack",
                   self._lib.pyro_sim_render_pack(self._h, 1 if bricks else 0))

    def read_render_volumes(self, bricks: bool = True):
        """(vol, sol, vel) float16 (nz, ny, nx, 4) and the brick maxima
        (float32, one per 8^3 brick, or None) of a fresh pack."""
        self.render_pack(bricks)
        return (self.read_field(_abi.F_RVOL), self.read_field(_abi.F_RSOL),
                self.read_field(_abi.F_RVEL), self.read_field(_abi.F_BRICKS) if bricks else None)

    def render_emission(self, chemi: Optional[np.ndarray] = None, lut=None) -> None:
        """The renderer's fire-light sampling tables (render.rs:304-333) from
        the last render_pack: emission power per cell and its CDF (read with
        read_field(F_ECELL / F_ECDF)).  `lut`: a CUDA tensor of the colour
        table (color.build_lut(), its first 1024 rows are used); by default
        the table is built once and kept on the device.  `chemi`: the four
        floats of color.chemi_block()."""
        from . import color
        if lut is None:
            if getattr(self, "_lut_dev", None) is None:
                import torch  # device memory for the table only
                self._lut_dev = torch.from_numpy(color.build_lut()).cuda()
            lut = self._lut_dev
        ch = np.ascontiguousarray(color.chemi_block() if chemi is None else chemi, np.float32)
        _abi.check("pyro_sim_render_emission", self._lib.pyro_sim_render_emission(
            self._h, ctypes.c_void_p(lut.data_ptr()), ch.ctypes.data_as(ctypes.c_void_p)))

    def set_solver(self, mode: int, tol: float = 1e-3, max_iters: int = 50) -> None:
        _abi.check("pyro_sim_set_solver",
                   self._lib.pyro_sim_set_solver(self._h, mode, tol, max_iters))

    def set_net(self, net) -> None:
        """Network for mode SOLVER_MGPCG_LEARNED (None detaches); the
        caller keeps `net` alive while it is attached."""
        self._net = net
        _abi.check("pyro_sim_set_net",
                   self._lib.pyro_sim_set_net(self._h, net.handle if net else None))

    def last_solve(self) -> _abi.PyroSolveInfo:
        info = _abi.PyroSolveInfo()
        _abi.check("pyro_sim_last_solve",
                   self._lib.pyro_sim_last_solve(self._h, ctypes.byref(info)))
        return info

    def info(self) -> _abi.PyroSimInfo:
        info = _abi.PyroSimInfo()
        _abi.check("pyro_sim_info", self._lib.pyro_sim_info(self._h, ctypes.byref(info)))
        return info

    def device_ptr(self, which: int) -> Tuple[int, int]:
        p = ctypes.c_void_p()
        n = ctypes.c_size_t()
        _abi.check("pyro_sim_device_ptr", self._lib.pyro_sim_device_ptr(
            self._h, which, ctypes.byref(p), ctypes.byref(n)))
        return p.value or 0, n.value

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _abi.check("pyro_sim_stream", self._lib.pyro_sim_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def sync(self) -> None:
        _abi.check("pyro_sim_sync", self._lib.pyro_sim_sync(self._h))
