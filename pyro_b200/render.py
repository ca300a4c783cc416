"""The volume renderer's GPU passes on top of the simulation: host-side
mirror of the reference's `Renderer` (src/render.rs:100-447) over the C ABI.

    sc = Scene.load("pyro_b200/scenes/pool_2cm.toml")
    sim = Sim(sc)
    ...                                      # step the fire
    r = Renderer(sc, sim)                    # Renderer::new
    rgb = r.render(sim, frame=0, spp=64)     # Renderer::render -> (h, w, 3)

Per frame: the input pack and fire-light tables of the simulation
(`Sim.render_pack`, `Sim.render_emission`), then in light-cache mode the
volume and ground light caches and their blur chain, then the camera rays in
dispatches of 8 samples (2 in pure path-tracing mode), all on the
simulation's CUDA stream.  Device memory for the caches and the image comes
from torch; every pass is a kernel of libpyro_b200.so.
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional, Sequence

import numpy as np

from . import _abi, color

GROUND_RES = 256  # ground irradiance cache texels per side (src/render.rs:12)
LV_RAYS = 96      # shadow rays per volume cache cell (render.wgsl:225)
GR_RAYS = 128     # shadow rays per ground texel (render.wgsl:254)
SOOT_ALBEDO = 0.25
# surface albedo by material name (src/render.rs:155-166); others 0.05
ALBEDO = {"wood": 0.32, "cardboard": 0.45, "pu_foam": 0.55, "pmma": 0.1, "rubber": 0.05,
          "steel": 0.3, "concrete": 0.35}
# the blur chain (src/render.rs:112, 372-381): (axis, radius)
BLUR_VOL = ((0, 2), (1, 2), (2, 2))
BLUR_GROUND = ((0, 3), (1, 3))

F32 = np.float32


def _norm(a):
    l = F32(max(F32(math.sqrt(F32(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]))), F32(1e-9)))
    return [F32(v / l) for v in a]


def _cross(a, b):
    return [F32(a[1] * b[2] - a[2] * b[1]), F32(a[2] * b[0] - a[0] * b[2]),
            F32(a[0] * b[1] - a[1] * b[0])]


def base_params(scene, dims: Sequence[int], dx: float, cfg=None) -> _abi.PyroRenderParams:
    """The uniform block of Renderer::new (src/render.rs:142-210) in f32:
    camera frame, exposure-free optics, ground cache square three domain
    widths across, material albedos by slot.  res.zw and dims.w are set per
    frame and dispatch."""
    from .scene import MATERIALS
    cfg = cfg or scene.render
    w, h = int(cfg.width), int(cfg.height)
    pos = [F32(v) for v in cfg.camera]
    tgt = [F32(v) for v in cfg.target]
    sub = [F32(tgt[i] - pos[i]) for i in range(3)]
    fwd = _norm(sub)
    right = _norm(_cross(fwd, [F32(0), F32(1), F32(0)]))
    up = _cross(right, fwd)
    if cfg.focus > 0.0:
        focus = F32(cfg.focus)
    else:
        focus = F32(math.sqrt(F32(F32(sub[0] * sub[0] + sub[1] * sub[1]) + sub[2] * sub[2])))
    se = color.soot_extinction(SOOT_ALBEDO)
    alb = [0.0] * 8
    for slot, mi in enumerate(scene.used_materials()):
        alb[slot] = ALBEDO.get(MATERIALS[mi].name, 0.05)
    dxf = F32(dx)
    ext = [F32(F32(dims[0]) * dxf), F32(F32(dims[2]) * dxf)]
    side = F32(F32(3.0) * max(ext[0], ext[1]))
    half_fov = F32(np.tan(F32(F32(F32(cfg.fov) * F32(F32(math.pi) / F32(180.0))) * F32(0.5))))
    rows = [
        [w, h, 0, 0],
        [dims[0], dims[1], dims[2], 0],
        [*pos, half_fov],
        [*fwd, F32(F32(w) / F32(h))],
        [*right, cfg.aperture],
        [*up, focus],
        [dxf, cfg.step, F32(F32(F32(cfg.shutter) / F32(360.0)) / F32(scene.sim.fps)), cfg.sky],
        [1.0 if cfg.ground else 0.0, cfg.ground_albedo, float(cfg.bounces), cfg.chemi],
        [se[0], se[1], se[2], SOOT_ALBEDO],
        [5.0, 0.92, 0.55, scene.sim.ambient_temp],
        alb[:4], alb[4:],
        [F32(F32(F32(0.5) * ext[0]) - F32(F32(0.5) * side)),
         F32(F32(F32(0.5) * ext[1]) - F32(F32(0.5) * side)), side,
         1.0 if cfg.mode != "path" else 0.0],
    ]
    return _abi.PyroRenderParams.from_rows(rows)


def _ptr(x) -> Optional[int]:
    if x is None:
        return None
    return int(x.data_ptr()) if hasattr(x, "data_ptr") else int(x)


def _rp_copy(rp: _abi.PyroRenderParams) -> _abi.PyroRenderParams:
    c = _abi.PyroRenderParams()
    ctypes.memmove(ctypes.byref(c), ctypes.byref(rp), ctypes.sizeof(rp))
    return c


# ---- single passes on device buffers (torch tensors or raw pointers) -----

def lightvol(rp, vol, sol, vel, bricks, lut, ecdf, lv_dims, lvA, lvB, rays=LV_RAYS,
             stream=None) -> None:
    """render.wgsl:217-251 into lvA, lvB ((lz, ly, lx) cells of 4 binary16)."""
    _abi.call("pyro_k_render_lightvol", ctypes.byref(rp), _ptr(vol), _ptr(sol), _ptr(vel),
              _ptr(bricks), _ptr(lut), _ptr(ecdf), lv_dims[0], lv_dims[1], lv_dims[2], rays,
              _ptr(lvA), _ptr(lvB), _ptr(stream))


def lightground(rp, vol, sol, vel, bricks, lut, ecdf, gres, gE, rays=GR_RAYS,
                stream=None) -> None:
    """render.wgsl:253-269 into gE (gres x gres texels of 4 binary16)."""
    _abi.call("pyro_k_render_lightground", ctypes.byref(rp), _ptr(vol), _ptr(sol), _ptr(vel),
              _ptr(bricks), _ptr(lut), _ptr(ecdf), gres, rays, _ptr(gE), _ptr(stream))


def blur(src, dst, dims, axis: int, radius: int, stream=None) -> None:
    """render.wgsl:271-304: src -> dst along one axis."""
    _abi.call("pyro_k_render_blur", _ptr(src), _ptr(dst), dims[0], dims[1], dims[2], axis,
              radius, _ptr(stream))


def trace(rp, vol, sol, vel, bricks, lut, ecdf, lvA, lvB, lv_dims, gE, gres, accum,
          stream=None) -> None:
    """render.wgsl:132-215: accum (float4 per pixel) += samples
    rp.res[2] .. rp.res[2] + rp.res[3] - 1 of every pixel."""
    lv = lv_dims if lv_dims is not None else (0, 0, 0)
    _abi.call("pyro_k_render_trace", ctypes.byref(rp), _ptr(vol), _ptr(sol), _ptr(vel),
              _ptr(bricks), _ptr(lut), _ptr(ecdf), _ptr(lvA), _ptr(lvB), lv[0], lv[1], lv[2],
              _ptr(gE), gres, _ptr(accum), _ptr(stream))


def frame_plan(cache: bool, spp: int):
    """The passes of one frame after the input pack and the emission tables,
    in the reference's order (src/render.rs:351-418): in light-cache mode
    the volume and ground caches, then the blur chain (volume caches x -> t1,
    y -> t2, z -> back, radius 2; ground x -> gtmp, y -> back, radius 3);
    then the camera rays in dispatches of 8 samples (2 when path tracing).
    Steps: ("lightvol",), ("lightground",), ("blur", src, dst, axis,
    radius), ("trace", first sample, samples)."""
    steps = []
    if cache:
        steps += [("lightvol",), ("lightground",)]
        for c in ("lvA", "lvB"):
            chain = (c, "t1", "t2", c)
            for k, (axis, rad) in enumerate(BLUR_VOL):
                steps.append(("blur", chain[k], chain[k + 1], axis, rad))
        steps.append(("blur", "gE", "gtmp") + BLUR_GROUND[0])
        steps.append(("blur", "gtmp", "gE") + BLUR_GROUND[1])
    chunk = 8 if cache else 2
    done = 0
    while done < spp:
        n = min(chunk, spp - done)
        steps.append(("trace", done, n))
        done += n
    return steps


class Renderer:
    """Renderer::new / Renderer::render (src/render.rs:100-447) for one
    simulation: owns the light caches, their blur temporaries, the colour
    table and the accumulation image on the device.  lv_rays, gr_rays and
    ground_res default to the reference's 96, 128 and 256."""

    def __init__(self, scene, sim, cfg=None, lv_rays: int = LV_RAYS, gr_rays: int = GR_RAYS,
                 ground_res: int = GROUND_RES):
        import torch  # device memory only
        self.cfg = cfg or scene.render
        self.lv_rays, self.gr_rays, self.gres = int(lv_rays), int(gr_rays), int(ground_res)
        self.cache = self.cfg.mode != "path"
        self.w, self.h = int(self.cfg.width), int(self.cfg.height)
        self.dims = list(sim.dims)
        self.lv_dims = [(d + 1) // 2 for d in self.dims]
        self.base = base_params(scene, self.dims, sim.dx, self.cfg)
        self.chemi = color.chemi_block(self.cfg.chemi, SOOT_ALBEDO)
        dev = torch.device("cuda")
        lvn = (self.lv_dims[2], self.lv_dims[1], self.lv_dims[0], 4)
        gn = (1, self.gres, self.gres, 4)
        z = lambda shape: torch.zeros(shape, dtype=torch.float16, device=dev)
        self.lvA, self.lvB, self.t1, self.t2 = z(lvn), z(lvn), z(lvn), z(lvn)
        self.gE, self.gtmp = z(gn), z(gn)
        self.lut = torch.from_numpy(color.build_lut()).to(dev)
        self.accum = torch.zeros((self.h * self.w, 4), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()

    def render(self, sim, frame: int, spp: int) -> np.ndarray:
        """One frame: the mean radiance per pixel, (h, w, 3) float32."""
        self.render_device(sim, frame, spp)
        acc = self.accum.cpu().numpy()
        n = np.maximum(acc[:, 3:4], 1.0)
        return (acc[:, :3] / n).reshape(self.h, self.w, 3)

    def render_device(self, sim, frame: int, spp: int) -> None:
        """One frame into self.accum (h*w float4 radiance sums and sample
        counts, on the device), for pyro_b200.develop.Developer."""
        import torch
        st = sim.stream()
        sim.render_pack(True)
        sim.render_emission(chemi=self.chemi, lut=self.lut)
        cells = self.dims[0] * self.dims[1] * self.dims[2]
        nb = ((self.dims[0] + 7) // 8) * ((self.dims[1] + 7) // 8) * ((self.dims[2] + 7) // 8)
        want = {_abi.F_RVOL: 8 * cells, _abi.F_RSOL: 8 * cells, _abi.F_RVEL: 8 * cells,
                _abi.F_BRICKS: 4 * nb, _abi.F_ECDF: 4 * (cells + 1)}
        ptrs = {}
        for f, nbytes in want.items():
            p, size = sim.device_ptr(f)
            if size < nbytes:
                raise ValueError(f"render: field {f} holds {size} bytes, the grid "
                                 f"{self.dims} needs {nbytes}")
            ptrs[f] = p
        vol, sol, vel = ptrs[_abi.F_RVOL], ptrs[_abi.F_RSOL], ptrs[_abi.F_RVEL]
        bricks, ecdf = ptrs[_abi.F_BRICKS], ptrs[_abi.F_ECDF]
        rp = _rp_copy(self.base)
        rp.dims[3] = frame
        with torch.cuda.stream(torch.cuda.ExternalStream(st)):
            self.accum.zero_()
        for step in frame_plan(self.cache, spp):
            if step[0] == "lightvol":
                lightvol(rp, vol, sol, vel, bricks, self.lut, ecdf, self.lv_dims, self.lvA,
                         self.lvB, rays=self.lv_rays, stream=st)
            elif step[0] == "lightground":
                lightground(rp, vol, sol, vel, bricks, self.lut, ecdf, self.gres, self.gE,
                            rays=self.gr_rays, stream=st)
            elif step[0] == "blur":
                _, src, dst, axis, rad = step
                dims = self.lv_dims if src in ("lvA", "lvB", "t1", "t2") else (self.gres,
                                                                               self.gres, 1)
                blur(getattr(self, src), getattr(self, dst), dims, axis, rad, stream=st)
            else:
                rp.res[2], rp.res[3] = step[1], step[2]
                trace(rp, vol, sol, vel, bricks, self.lut, ecdf, self.lvA, self.lvB,
                      self.lv_dims, self.gE, self.gres, self.accum, stream=st)
        torch.cuda.ExternalStream(st).synchronize()
