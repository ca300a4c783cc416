"""Scene description (TOML), material table, parameter block and shape list.

Host-side mirror of the reference's src/scene.rs: the TOML schema and its
defaults (src/scene.rs:8-209), the 11-material table (:240-406), grid
rounding (:485-493), the `Params` builder with every physics constant
(:523-618) and the shape generators box / cylinder / sphere / pool / crib /
pallets / bonfire (:669-879).  Arithmetic that feeds the simulation is done
in float32 (numpy scalars) as the reference does it in Rust f32.

Voxelization itself (src/scene.rs:621-667) runs on the GPU through the C ABI
(`pyro_voxelize`); `Scene.shapes()` produces its input.
"""
from __future__ import annotations

import ctypes
import math
import tomllib
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _abi

F = np.float32
PI32 = F(math.pi)
TAU32 = F(2.0 * math.pi)
FRAC_PI_2_32 = F(math.pi / 2.0)


class SceneError(ValueError):
    """Invalid scene description (unknown material or kind, too many
    materials, no combustible object)."""


# ---------------------------------------------------------------- materials
@dataclass(frozen=True)
class Material:
    """One row of the material table (src/scene.rs:218-238)."""
    name: str
    label: str
    kind: int        # 0 charring solid, 1 liquid pool, 2 inert, 3 non-charring
    density: float   # kg/m^3
    lg: float        # effective heat of gasification J/kg
    tp: float        # pyrolysis / boiling temperature K
    char_yield: float
    emissivity: float
    cp: float
    k: float
    smoke: float
    dhc: float       # heat of combustion of the volatiles J/kg
    soot: float      # soot yield


MATERIALS: List[Material] = [
    Material("air", "air", 2, 0.0, 1.0, 1e4, 0.0, 0.9, 1000.0, 0.03, 0.0, 0.0, 0.0),
    Material("wood", "wood", 0, 480.0, 1.5e6, 600.0, 0.25, 0.9, 1500.0, 0.15, 0.02, 15.0e6, 0.015),
    Material("cardboard", "cardboard", 0, 150.0, 1.8e6, 580.0, 0.2, 0.9, 1400.0, 0.08, 0.02,
             14.0e6, 0.012),
    Material("pu_foam", "polyurethane foam (sofa/mattress)", 3, 35.0, 1.4e6, 570.0, 0.0, 0.9,
             1400.0, 0.04, 0.0, 24.0e6, 0.10),
    Material("pmma", "PMMA", 3, 1190.0, 1.6e6, 630.0, 0.0, 0.9, 1500.0, 0.19, 0.0, 24.9e6, 0.022),
    Material("rubber", "rubber (tyres)", 3, 1100.0, 1.7e6, 620.0, 0.0, 0.95, 1700.0, 0.2, 0.0,
             30.0e6, 0.15),
    Material("heptane", "n-heptane pool", 1, 684.0, 0.48e6, 371.0, 0.0, 0.95, 2240.0, 0.14, 0.0,
             44.6e6, 0.037),
    Material("gasoline", "gasoline pool", 1, 740.0, 0.42e6, 345.0, 0.0, 0.95, 2200.0, 0.13, 0.0,
             43.7e6, 0.059),
    Material("diesel", "diesel pool", 1, 830.0, 0.6e6, 460.0, 0.0, 0.95, 2100.0, 0.13, 0.0,
             44.4e6, 0.07),
    Material("steel", "steel (inert)", 2, 7850.0, 1.0, 1e4, 0.0, 0.7, 500.0, 45.0, 0.0, 0.0, 0.0),
    Material("concrete", "concrete (inert)", 2, 2300.0, 1.0, 1e4, 0.0, 0.9, 900.0, 1.4, 0.0, 0.0,
             0.0),
]


def material(name: str):
    """Index and row of a material by name; the error lists the choices
    (src/scene.rs:408-421)."""
    for i, m in enumerate(MATERIALS):
        if m.name == name:
            return i, m
    choices = ", ".join(f"{m.name} ({m.label})" for m in MATERIALS[1:])
    raise SceneError(f"unknown material {name}; choices: {choices}")


# ------------------------------------------------------------------- schema
@dataclass
class Domain:
    size: List[float]
    cell: float


@dataclass
class SimCfg:
    fps: float = 24.0
    duration: float = 10.0
    cfl: float = 1.5
    vorticity: float = 3.0
    smagorinsky: float = 0.17
    pressure_cycles: int = 4
    seed: int = 1
    ambient_temp: float = 293.0


@dataclass
class Wind:
    speed: float = 0.0
    dir: float = 0.0   # degrees, 0 = +x


@dataclass
class Ignition:
    pos: List[float]
    radius: float = 0.25
    flux: float = 40e3
    temp: float = 1300.0
    until: float = 4.0
    fuel: float = 0.0


@dataclass
class FuelCfg:
    material: Optional[str] = None
    heat_of_combustion: Optional[float] = None
    soot_yield: Optional[float] = None
    soot_formation_ratio: Optional[float] = None
    soot_oxidation: Optional[float] = None
    radiative_fraction: Optional[float] = None


@dataclass
class Object:
    kind: str
    material: str
    center: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    size: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    radius: float = 0.0
    depth: float = 0.0
    a: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    b: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    yaw: float = 0.0
    count: int = 0
    sticks: int = 0
    stick: float = 0.0


@dataclass
class RenderCfg:
    """The [render] table (src/scene.rs:141-190), with its defaults."""
    width: int = 1280
    height: int = 720
    spp: int = 64
    camera: List[float] = field(default_factory=lambda: [0.0, 1.5, -6.0])
    target: List[float] = field(default_factory=lambda: [0.0, 2.0, 0.0])
    fov: float = 45.0
    exposure: float = 0.0
    auto_exposure: bool = True
    shutter: float = 180.0
    ground: bool = True
    ground_albedo: float = 0.12
    sky: float = 0.003
    bounces: int = 2
    step: float = 0.6
    glare: float = 0.04
    aperture: float = 0.0
    focus: float = 0.0
    chemi: float = 0.05
    mode: str = "cache"


@dataclass
class OutputCfg:
    dir: str = "out"
    preroll: float = 0.0
    video: bool = True


def _fill(cls, d: dict, name: str):
    """Build a table; unknown keys are ignored like serde's default."""
    known = {f for f in cls.__dataclass_fields__}
    try:
        return cls(**{k: v for k, v in d.items() if k in known})
    except TypeError as e:
        raise SceneError(f"scene file format error in [{name}]: {e}") from e


@dataclass
class Grid:
    dims: List[int]
    dx: float


@dataclass
class Scene:
    """A parsed scene (src/scene.rs:8-25)."""
    domain: Domain
    sim: SimCfg = field(default_factory=SimCfg)
    wind: Wind = field(default_factory=Wind)
    ignition: Optional[Ignition] = None
    fuel: FuelCfg = field(default_factory=FuelCfg)
    objects: List[Object] = field(default_factory=list)
    output: OutputCfg = field(default_factory=OutputCfg)
    render: RenderCfg = field(default_factory=RenderCfg)
    # Exact grid dimensions for synthetic workloads of a named shape (the
    # reference always rounds to multiples of 16; None keeps that rule).
    dims_override: Optional[List[int]] = None

    # --------------------------------------------------------------- parse
    @staticmethod
    def from_toml_str(text: str) -> "Scene":
        try:
            d = tomllib.loads(text)
        except tomllib.TOMLDecodeError as e:
            raise SceneError(f"scene file format error: {e}") from e
        if "domain" not in d:
            raise SceneError("scene file format error: missing [domain]")
        dom = _fill(Domain, d["domain"], "domain")
        sc = Scene(domain=dom)
        if "sim" in d:
            sc.sim = _fill(SimCfg, d["sim"], "sim")
        if "wind" in d:
            sc.wind = _fill(Wind, d["wind"], "wind")
        if "ignition" in d:
            sc.ignition = _fill(Ignition, d["ignition"], "ignition")
        if "fuel" in d:
            sc.fuel = _fill(FuelCfg, d["fuel"], "fuel")
        if "output" in d:
            sc.output = _fill(OutputCfg, d["output"], "output")
        if "render" in d:
            sc.render = _fill(RenderCfg, d["render"], "render")
        for o in d.get("object", []):
            sc.objects.append(_fill(Object, o, "object"))
        return sc

    @staticmethod
    def load(path: str) -> "Scene":
        """scene::load (src/scene.rs:211-215)."""
        with open(path, "rb") as fh:
            return Scene.from_toml_str(fh.read().decode("utf-8"))

    # ---------------------------------------------------------------- grid
    def grid(self) -> Grid:
        """Every dimension rounded to a multiple of 16 so multigrid can
        halve four times (src/scene.rs:485-493)."""
        dx = F(self.domain.cell)
        if self.dims_override is not None:
            return Grid(dims=[int(v) for v in self.dims_override], dx=float(dx))
        dims = []
        for s in self.domain.size:
            q = F(F(s) / dx) / F(16.0)
            r = max(math.floor(float(q) + 0.5), 1.0)   # f32::round, half away
            dims.append(int(r) * 16)
        return Grid(dims=dims, dx=float(dx))

    def used_materials(self) -> List[int]:
        """Material table indices used by the scene, slot 0 = air, at most 8
        (src/scene.rs:495-508)."""
        v = [0]
        for o in self.objects:
            i, _ = material(o.material)
            if i not in v:
                v.append(i)
        if len(v) > 8:
            raise SceneError("a scene can use at most 7 materials")
        return v

    def fuel_material(self) -> Material:
        """src/scene.rs:510-521."""
        if self.fuel.material is not None:
            return material(self.fuel.material)[1]
        for o in self.objects:
            _, m = material(o.material)
            if m.kind != 2:
                return m
        raise SceneError("the scene has no combustible object")

    # -------------------------------------------------------------- params
    def params(self) -> _abi.PyroParams:
        """The 576-byte parameter block (src/scene.rs:523-618)."""
        g = self.grid()
        fm = self.fuel_material()
        dhc = F(self.fuel.heat_of_combustion if self.fuel.heat_of_combustion is not None
                else fm.dhc)
        soot = F(self.fuel.soot_yield if self.fuel.soot_yield is not None else fm.soot)
        ratio = F(self.fuel.soot_formation_ratio
                  if self.fuel.soot_formation_ratio is not None else 2.5)
        p = _abi.PyroParams()
        for slot, mi in enumerate(self.used_materials()):
            m = MATERIALS[mi]
            row = [m.density, m.lg, m.tp, float(m.kind), m.char_yield, m.emissivity, m.cp, m.k,
                   m.smoke, 1.0, 0.0, 0.0]
            for j, v in enumerate(row):
                p.mats[slot][j] = float(F(v))
        wr = F(F(self.wind.dir) * F(math.pi / 180.0))
        ign = self.ignition
        span = F(0.5)
        for o in self.objects:
            if o.kind in ("pool", "sphere"):
                s = F(2.0) * F(o.radius)
            else:
                s = max(max(F(o.size[0]), F(o.size[2])), F(0.3))
            span = max(span, s)
        amb = F(self.sim.ambient_temp)
        p.nx, p.ny, p.nz = g.dims
        p.frame = 0
        p.dx = g.dx
        p.dt = 0.005
        p.time = 0.0
        p.t0 = float(amb)
        p.rho0 = float(F(F(1.204) * F(293.0)) / amb)
        p.g = 9.81
        p.cp = 1100.0
        p.yo2 = 0.233
        p.vort = self.sim.vorticity
        p.cs = self.sim.smagorinsky
        p.buoy = 1.0
        p.smoke_w = 0.0
        p.wind_x = float(F(self.wind.speed) * np.cos(wr))
        p.wind_z = float(F(self.wind.speed) * np.sin(wr))
        p.wind_relax = 0.3 if self.wind.speed > 0.0 else 0.0
        p.sponge = 6.0
        p.t_ign = 750.0
        p.s_o2 = float(dhc / F(13.1e6))
        p.dhc = float(dhc)
        p.tau_min = 2e-3
        p.soot_form = float(soot * ratio)
        p.soot_ox = (self.fuel.soot_oxidation if self.fuel.soot_oxidation is not None else 4.0)
        p.soot_ox_t = 1150.0
        p.smoke_conv = 0.5
        p.kap_gas = 0.1
        p.h_conv = 15.0
        p.ign_on = 1.0 if ign is not None else 0.0
        p.ign_temp = ign.temp if ign else 0.0
        p.ign_x = ign.pos[0] if ign else 0.0
        p.ign_y = ign.pos[1] if ign else 0.0
        p.ign_z = ign.pos[2] if ign else 0.0
        p.ign_r = ign.radius if ign else 0.0
        p.ign_flux = ign.flux if ign else 0.0
        p.ign_fuel = ign.fuel if ign else 0.0
        p.char_a = 465.0
        p.char_e = 68e3
        p.dh_char = 32.8e6
        p.burnout = 2.0
        p.layer = 0.005
        p.rad_len = float(F(0.5) * span)
        p.h_mass = 0.02
        p.vort_t = 500.0
        rf = {"heptane": 0.33, "gasoline": 0.35, "diesel": 0.35, "pu_foam": 0.42,
              "rubber": 0.42, "pmma": 0.31}
        p.rad_frac = (self.fuel.radiative_fraction if self.fuel.radiative_fraction is not None
                      else rf.get(fm.name, 0.30))
        p.seed = float(self.sim.seed)
        return p

    def ign_until(self) -> float:
        """Ignition end time (src/sim.rs:204)."""
        return self.ignition.until if self.ignition is not None else 0.0

    # -------------------------------------------------------------- shapes
    def shapes(self) -> List[_abi.PyroShape]:
        """Expanded primitive list in object order (src/scene.rs:628-635)."""
        g = self.grid()
        dx = F(g.dx)
        used = self.used_materials()
        out: List[_abi.PyroShape] = []
        for o in self.objects:
            mi, _ = material(o.material)
            slot = used.index(mi)
            for s in _expand(o, dx):
                s.slot = slot
                out.append(s)
        return out

    def slot_tables(self):
        """Per-slot density and kind (8 entries each) for the voxelizer."""
        dens = (ctypes.c_float * 8)()
        kind = (ctypes.c_uint32 * 8)()
        for slot, mi in enumerate(self.used_materials()):
            dens[slot] = MATERIALS[mi].density
            kind[slot] = MATERIALS[mi].kind
        for slot in range(len(self.used_materials()), 8):
            kind[slot] = 2
        return dens, kind


# ----------------------------------------------------------------- geometry
def _box(c, h, yaw) -> _abi.PyroShape:
    s = _abi.PyroShape()
    s.kind = _abi.SHAPE_BOX
    for i in range(3):
        s.c[i] = float(F(c[i]))
        s.e[i] = float(F(h[i]))
    s.sin_yaw = float(np.sin(F(yaw)))
    s.cos_yaw = float(np.cos(F(yaw)))
    return s


def _cyl(a, b, r) -> _abi.PyroShape:
    s = _abi.PyroShape()
    s.kind = _abi.SHAPE_CYL
    for i in range(3):
        s.c[i] = float(F(a[i]))
        s.e[i] = float(F(b[i]))
    s.r = float(F(r))
    return s


def _rot(p, yaw, c):
    """src/scene.rs:871-879 (inverse of the box's local transform)."""
    s, co = np.sin(F(yaw)), np.cos(F(yaw))
    return [F(F(c[0]) + co * F(p[0])) - s * F(p[2]),
            F(c[1]) + F(p[1]),
            F(F(c[2]) + s * F(p[0])) + co * F(p[2])]


def _hash(v: int) -> np.float32:
    """src/scene.rs:662-667 (the same PCG as common.wgsl:54-58)."""
    x = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    x = (((x >> ((x >> 28) + 4)) ^ x) * 277803737) & 0xFFFFFFFF
    x = ((x >> 22) ^ x) & 0xFFFFFFFF
    return F(F(x) / F(4294967295.0))


def _expand(o: Object, dx: np.float32) -> List[_abi.PyroShape]:
    """src/scene.rs:730-869."""
    yaw = F(F(o.yaw) * F(math.pi / 180.0))
    c = [F(v) for v in o.center]
    k = o.kind
    if k == "box":
        return [_box(c, [F(v) * F(0.5) for v in o.size], yaw)]
    if k == "cylinder":
        return [_cyl(o.a, o.b, o.radius)]
    if k == "sphere":
        s = _abi.PyroShape()
        s.kind = _abi.SHAPE_SPHERE
        for i in range(3):
            s.c[i] = float(c[i])
        s.r = float(F(o.radius))
        return [s]
    if k == "pool":
        s = _abi.PyroShape()
        s.kind = _abi.SHAPE_POOL
        for i in range(3):
            s.c[i] = float(c[i])
        s.r = float(F(o.radius))
        s.depth = float(F(o.depth))
        return [s]
    if k == "crib":
        n = max(o.sticks, 2)
        w = max(F(o.stick), dx)
        ln = max(F(o.size[0]), F(0.2))
        v = []
        for l in range(max(o.count, 1)):
            y = c[1] + w * F(F(l) + F(0.5))
            for s in range(n):
                off = F(F(-0.5) * ln + F(0.5) * w) + F(F((ln - w) * F(s)) / F(n - 1))
                if l % 2 == 0:
                    hx, hz, ox, oz = F(0.5) * ln, F(0.5) * w, F(0.0), off
                else:
                    hx, hz, ox, oz = F(0.5) * w, F(0.5) * ln, off, F(0.0)
                v.append(_box(_rot([ox, F(0.0), oz], yaw, [c[0], y, c[2]]),
                              [hx, F(0.5) * w, hz], yaw))
        return v
    if k == "pallets":
        v = []
        ph = F(0.144)
        for l in range(max(o.count, 1)):
            y0 = c[1] + ph * F(l)
            for z in (F(-0.45), F(0.0), F(0.45)):
                v.append(_box(_rot([F(0), F(0), z], yaw, [c[0], y0 + F(0.011), c[2]]),
                              [F(0.6), F(0.011), F(0.05)], yaw))
                v.append(_box(_rot([F(0), F(0), z], yaw, [c[0], y0 + F(0.061), c[2]]),
                              [F(0.6), F(0.039), F(0.05)], yaw))
            for s in range(7):
                x = F(-0.55) + F(F(F(1.1) * F(s)) / F(6.0))
                v.append(_box(_rot([x, F(0), F(0)], yaw, [c[0], y0 + F(0.122), c[2]]),
                              [F(0.05), F(0.011), F(0.5)], yaw))
        return v
    if k == "bonfire":
        r = max(F(o.radius), F(0.5))
        h = F(o.size[1]) if o.size[1] > 0.0 else F(1.3) * r
        n = max(o.count, 6)
        d = F(o.stick) if o.stick > 0.0 else F(0.08) * r
        v = []
        state = [0]

        def rnd():
            state[0] += 1
            return _hash(((state[0] * 2654435761) & 0xFFFFFFFF) ^ 0x5BD1E995)

        for ring, cnt, rr, hh in ((0, n, r, h), (1, n // 2, F(0.6) * r, F(0.75) * h)):
            for i in range(cnt):
                th = F(F(TAU32 * F(F(i) + F(0.5) * F(ring))) / F(cnt)) + F(0.25) * (rnd() - F(0.5))
                rb = rr * (F(0.88) + F(0.17) * rnd())
                a = [c[0] + rb * np.cos(th), c[1] + F(0.5) * d, c[2] + rb * np.sin(th)]
                tt = th + PI32 + F(0.6) * (rnd() - F(0.5))
                off = F(F(0.07) * r) * (F(0.5) + rnd())
                t0 = c[0] + off * np.cos(tt)
                t1 = c[1] + hh * (F(0.9) + F(0.15) * rnd())
                t2 = c[2] + off * np.sin(tt)
                top = [t0, t1, t2]
                ext = F(1.08) + F(0.1) * rnd()
                b = [a[j] + (top[j] - a[j]) * ext for j in range(3)]
                v.append(_cyl(a, b, F(F(0.5) * d) * (F(0.75) + F(0.5) * rnd())))
        for l in range(3):
            y = c[1] + d * F(F(l) + F(0.5))
            for s in range(5):
                off = F(F(F(-0.5) * r) + F(F(r * F(s)) / F(4.0))) + F(F(0.1) * r) * (rnd() - F(0.5))
                ln = F(0.7) * r
                ang = (F(0.0) if l % 2 == 0 else FRAC_PI_2_32) + F(0.3) * (rnd() - F(0.5))
                sa, ca = np.sin(ang), np.cos(ang)
                p0 = [c[0] - sa * off, y, c[2] + ca * off]
                a = [p0[0] - ca * ln, y, p0[2] - sa * ln]
                b = [p0[0] + ca * ln, y, p0[2] + sa * ln]
                v.append(_cyl(a, b, F(F(0.5) * d) * (F(0.7) + F(0.4) * rnd())))
        return v
    raise SceneError(f"unknown object kind {k} "
                     "(choices: box/cylinder/sphere/pool/crib/pallets/bonfire)")


def shapes_array(shapes: Sequence[_abi.PyroShape]):
    arr = (_abi.PyroShape * max(len(shapes), 1))()
    for i, s in enumerate(shapes):
        arr[i] = s
    return arr
