"""The CPU oracle behind the Sim interface of pyro_b200.sim (step, read_stats,
time, dx, dims), so the reference frame loop (pyro_b200.run.run_frames) can
drive it.  Test infrastructure only."""
import numpy as np

from . import OracleSim


class OracleSimAdapter:
    def __init__(self, scene, sol_init, params=None):
        from pyro_b200.sim import Stats
        self._Stats = Stats
        self.p = params if params is not None else scene.params()
        self.dims = [int(self.p.nx), int(self.p.ny), int(self.p.nz)]
        self.dx = float(self.p.dx)
        self.time = np.float32(0.0)
        self.ign_until = np.float32(scene.ign_until())
        self.o = OracleSim(self.p, sol_init, scene.sim.pressure_cycles)

    def step(self, dt, want_stats):
        ign = 1.0 if self.time < self.ign_until else 0.0
        self.o.step(float(np.float32(dt)), float(self.time), ign, want_stats)
        self.time = np.float32(self.time + np.float32(dt))

    def read_stats(self):
        return self._Stats.decode(self.o.read_stats(), self.dims[1])

    def read_field(self, which):
        return self.o.read_field(which)

    def write_field(self, which, arr):
        self.o.write_field(which, arr)

    def close(self):
        self.o.close()
