"""Generate golden vectors by executing the reference's own WGSL kernels.

    python tests/golden/make_golden.py --ref <reference checkout> [--only name,...]

(or set PYRO_REFERENCE to the checkout instead of passing --ref)

For each simulation kernel (and the renderer's input pack, render.wgsl) the
script assembles the shader source exactly as
the reference's host does (src/gpu.rs:190-237: common.wgsl first unless the
kernel is a multigrid one, then the template / velocity / statistics blocks
its //@ directives name, then the kernel body), interprets it with
tests/golden/wgsl.py over the dispatch grid src/sim.rs uses (4x4x4
workgroups, g3 over cells, gv over the padded face grid, the smoother over
(ceil(nx/2), ny, nz)), and stores the seeded inputs and the outputs in
tests/golden/<kernel>.npz.  The fixtures are committed; the tests only read
them (the reference checkout is not needed to run the tests).
"""
from __future__ import annotations

import argparse
import os
import re
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
ROOT = os.path.dirname(TESTS)
sys.path.insert(0, ROOT)
sys.path.insert(0, TESTS)
sys.path.insert(0, HERE)

import wgsl  # noqa: E402
from fields import params_for, random_state  # noqa: E402

GOLDEN_DIMS = (10, 12, 9)
MG_DIMS = (11, 14, 9)


def split_kernels(text: str):
    """src/gpu.rs:190-209."""
    out, name, body = {}, None, []
    for line in text.splitlines():
        if line.startswith("//#KERNEL "):
            if name is not None:
                out[name] = "\n".join(body) + "\n"
            name, body = line[len("//#KERNEL "):].strip(), []
        elif name is not None:
            body.append(line)
    if name is not None:
        out[name] = "\n".join(body) + "\n"
    return out


class Ref:
    def __init__(self, root):
        sh = os.path.join(root, "src", "shaders")
        rd = lambda n: open(os.path.join(sh, n), encoding="utf-8").read()  # noqa: E731
        self.common = rd("common.wgsl")
        self.t_scalar = rd("tmpl_scalar.wgsl")
        self.t_comp = rd("tmpl_comp.wgsl")
        self.vel = rd("vel.wgsl")
        self.stats = rd("stats.wgsl")
        self.kernels = {}
        for f in ("advect.wgsl", "fluid.wgsl", "combust.wgsl", "mg.wgsl"):
            self.kernels.update(split_kernels(rd(f)))
        # the renderer's input pack (src/render.rs:135,229-230: with common.wgsl)
        rk = split_kernels(rd("render.wgsl"))
        for k in ("pack", "bricks", "ecells", "trace", "lightvol", "lightground", "blur"):
            self.kernels[k] = rk[k]
        self.trace_lib = rd("trace_lib.wgsl")

    def assemble(self, name):
        """src/gpu.rs:212-237 (the renderer's trace kernels and blur are
        assembled without common.wgsl, src/render.rs:229-236)."""
        body = self.kernels[name]
        no_common = name.startswith("mg_") or name in ("trace", "lightvol", "lightground", "blur")
        s = "" if no_common else self.common
        for line in body.splitlines():
            t = line.strip()
            if t.startswith("//@COMP "):
                for n in t[len("//@COMP "):].split():
                    s += self.t_comp.replace("XBUF", n)
            elif t.startswith("//@SCAL "):
                for n in t[len("//@SCAL "):].split():
                    s += self.t_scalar.replace("XBUF", n)
            elif t == "//@VEL":
                s += self.vel
            elif t.startswith("//@STATS "):
                s += self.stats.replace("STATSB", t[len("//@STATS "):].strip())
            elif t == "//@TRACE":
                s += self.trace_lib
        return s + body


# the 64-lane tree reductions become per-invocation values (see wgsl.py)
IDENT = {"wsum": lambda li, v: v, "wmax": lambda li, v: v}


def params_struct(P):
    """The uniform block as the interpreter's struct value."""
    from pyro_b200._abi import PARAM_SCALARS
    d = {}
    for name, ct in PARAM_SCALARS:
        v = getattr(P, name)
        d[name] = np.uint32(v) if ct.__name__ == "c_uint" else np.float32(v)
    mats = []
    for s in range(8):
        row = np.array(list(P.mats[s]), dtype=np.float32)
        mats.append({"a": row[0:4].copy(), "b": row[4:8].copy(), "c": row[8:12].copy()})
    d["mats"] = mats
    return d


def groups3(d):
    return tuple((v + 3) // 4 for v in d)


def flat(a):
    """(z,y,x[,4]) field -> the interpreter's flat buffer view."""
    a = np.ascontiguousarray(a)
    if a.ndim == 4:
        return a.reshape(-1, 4).copy()
    return a.reshape(-1).copy()


def run_kernel(ref, name, P, binds, grid, overrides=None):
    m = wgsl.Module(ref.assemble(name), overrides=overrides, replace=IDENT)
    if 0 in m.bindings and P is not None:
        m.bind(0, params_struct(P))
    for b, arr in binds.items():
        m.bind(b, arr)
    t = time.time()
    m.dispatch(grid)
    return time.time() - t


def stats_buf():
    return np.zeros(1040, np.uint32)


def gen_sim(ref, only):
    nx, ny, nz = GOLDEN_DIMS
    out = {}
    n = (nz, ny, nx)
    for case, (seed, dt, ign, wind) in enumerate([(11, 0.02, 1.0, 0.0), (12, 0.01, 0.0, 2.0)]):
        P = params_for(nx, ny, nz, dx=0.05, dt=dt, ign_on=ign, wind=wind, sponge=2.0)
        S = random_state(P, seed=seed)
        pb = np.frombuffer(P.to_bytes(), np.uint8).copy()
        g3 = groups3((nx, ny, nz))
        gv = groups3((nx + 1, ny + 1, nz + 1))
        tag = f"c{case}"

        def want(k):
            return only is None or k in only

        if want("solid"):
            solIn, s0 = flat(S["sol"]), flat(S["s0"])
            solOut, pyr = np.zeros_like(solIn), np.zeros_like(solIn)
            fl, st = np.zeros(nx * ny * nz, np.uint32), stats_buf()
            t = run_kernel(ref, "solid", P, {1: solIn, 2: solOut, 3: pyr, 4: fl, 5: s0, 6: st}, g3)
            out[f"solid_{tag}"] = dict(params=pb, sol=S["sol"], s0=S["s0"],
                                       sol_out=solOut.reshape(n + (4,)), pyr=pyr.reshape(n + (4,)),
                                       flags=fl.reshape(n), stats=st.view(np.float32))
            print(f"solid {tag} {t:.1f}s", flush=True)
        if want("curl"):
            u, v, w = flat(S["u"]), flat(S["v"]), flat(S["w"])
            c, st = np.zeros((nx * ny * nz, 4), np.float32), stats_buf()
            t = run_kernel(ref, "curl", P, {1: u, 2: v, 3: w, 4: c, 5: st}, g3)
            out[f"curl_{tag}"] = dict(params=pb, u=S["u"], v=S["v"], w=S["w"],
                                      curl=c.reshape(n + (4,)), stats=st.view(np.float32))
            print(f"curl {tag} {t:.1f}s", flush=True)
        if want("adv_vel"):
            u, v, w = flat(S["u"]), flat(S["v"]), flat(S["w"])
            hu, hv, hw = np.zeros_like(u), np.zeros_like(v), np.zeros_like(w)
            t1 = run_kernel(ref, "adv_vel1", P, {1: u, 2: v, 3: w, 4: hu, 5: hv, 6: hw}, gv)
            ou, ov, ow = np.zeros_like(u), np.zeros_like(v), np.zeros_like(w)
            fl = flat(S["flags"])
            t2 = run_kernel(ref, "adv_vel2", P, {1: u, 2: v, 3: w, 4: hu, 5: hv, 6: hw, 7: ou,
                                                 8: ov, 9: ow, 10: fl}, gv)
            nv = (nz + 1, ny + 1, nx + 1)
            out[f"adv_vel_{tag}"] = dict(params=pb, u=S["u"], v=S["v"], w=S["w"], flags=S["flags"],
                                         hu=hu.reshape(nv), hv=hv.reshape(nv), hw=hw.reshape(nv),
                                         ou=ou.reshape(nv), ov=ov.reshape(nv), ow=ow.reshape(nv))
            print(f"adv_vel {tag} {t1:.1f}+{t2:.1f}s", flush=True)
        if want("adv_scalars"):
            u, v, w = flat(S["u"]), flat(S["v"]), flat(S["w"])
            s0, s1 = flat(S["s0"]), flat(S["s1"])
            h0, h1 = np.zeros_like(s0), np.zeros_like(s1)
            t1 = run_kernel(ref, "adv_s1", P, {1: u, 2: v, 3: w, 4: s0, 5: s1, 6: h0, 7: h1}, g3)
            o0, o1 = np.zeros_like(s0), np.zeros_like(s1)
            t2 = run_kernel(ref, "adv_s2", P, {1: u, 2: v, 3: w, 4: s0, 5: s1, 6: h0, 7: h1,
                                               8: o0, 9: o1}, g3)
            out[f"adv_scalars_{tag}"] = dict(params=pb, u=S["u"], v=S["v"], w=S["w"], s0=S["s0"],
                                             s1=S["s1"], h0=h0.reshape(n + (4,)),
                                             h1=h1.reshape(n + (4,)), o0=o0.reshape(n + (4,)),
                                             o1=o1.reshape(n + (4,)))
            print(f"adv_scalars {tag} {t1:.1f}+{t2:.1f}s", flush=True)
        if want("react"):
            s0, s1 = flat(S["s0"]), flat(S["s1"])
            o0, o1 = np.zeros_like(s0), np.zeros_like(s1)
            st = stats_buf()
            t = run_kernel(ref, "react", P, {1: s0, 2: s1, 3: o0, 4: o1, 5: flat(S["flags"]),
                                             6: flat(S["sol"]), 7: flat(S["pyr"]),
                                             8: flat(S["curl"]), 9: st}, g3)
            out[f"react_{tag}"] = dict(params=pb, s0=S["s0"], s1=S["s1"], flags=S["flags"],
                                       sol=S["sol"], pyr=S["pyr"], curl=S["curl"],
                                       o0=o0.reshape(n + (4,)), o1=o1.reshape(n + (4,)),
                                       stats=st.view(np.float32))
            print(f"react {tag} {t:.1f}s", flush=True)
        if want("forces"):
            u, v, w = flat(S["u"]), flat(S["v"]), flat(S["w"])
            t = run_kernel(ref, "forces", P, {1: u, 2: v, 3: w, 4: flat(S["s0"]),
                                              5: flat(S["s1"]), 6: flat(S["curl"]),
                                              7: flat(S["flags"])}, gv)
            nv = (nz + 1, ny + 1, nx + 1)
            out[f"forces_{tag}"] = dict(params=pb, u=S["u"], v=S["v"], w=S["w"], s0=S["s0"],
                                        s1=S["s1"], curl=S["curl"], flags=S["flags"],
                                        ou=u.reshape(nv), ov=v.reshape(nv), ow=w.reshape(nv))
            print(f"forces {tag} {t:.1f}s", flush=True)
        if want("divergence"):
            b = np.zeros(nx * ny * nz, np.float32)
            t = run_kernel(ref, "divergence", P, {1: flat(S["u"]), 2: flat(S["v"]),
                                                  3: flat(S["w"]), 4: flat(S["s1"]),
                                                  5: flat(S["flags"]), 6: b}, g3)
            out[f"divergence_{tag}"] = dict(params=pb, u=S["u"], v=S["v"], w=S["w"], s1=S["s1"],
                                            flags=S["flags"], b=b.reshape(n))
            print(f"divergence {tag} {t:.1f}s", flush=True)
        if want("project"):
            u, v, w = flat(S["u"]), flat(S["v"]), flat(S["w"])
            t = run_kernel(ref, "project", P, {1: u, 2: v, 3: w, 4: flat(S["phi"]),
                                               5: flat(S["flags"])}, gv)
            nv = (nz + 1, ny + 1, nx + 1)
            out[f"project_{tag}"] = dict(params=pb, u=S["u"], v=S["v"], w=S["w"], phi=S["phi"],
                                         flags=S["flags"], ou=u.reshape(nv), ov=v.reshape(nv),
                                         ow=w.reshape(nv))
            print(f"project {tag} {t:.1f}s", flush=True)
    return out


def gen_render(ref, only):
    """The pack and bricks dispatches of src/render.rs:263-292 on the step's
    fields: three rgba16float textures (binary16 arrays here) and the 8^3
    brick maxima read back from two of them."""
    if only is not None and "render" not in only:
        return {}
    out = {}
    for case, (dims, seed) in enumerate([(GOLDEN_DIMS, 21), ((17, 9, 11), 22)]):
        nx, ny, nz = dims
        n = (nz, ny, nx)
        P = params_for(nx, ny, nz, dx=0.05, dt=0.02, ign_on=1.0, wind=0.0, sponge=2.0)
        S = random_state(P, seed=seed)
        pb = np.frombuffer(P.to_bytes(), np.uint8).copy()
        vol = np.zeros(n + (4,), np.float16)
        solt = np.zeros(n + (4,), np.float16)
        vel = np.zeros(n + (4,), np.float16)
        t1 = run_kernel(ref, "pack", P, {1: flat(S["s0"]), 2: flat(S["s1"]), 3: flat(S["sol"]),
                                         4: flat(S["flags"]), 5: flat(S["u"]), 6: flat(S["v"]),
                                         7: flat(S["w"]), 8: vol, 9: solt, 10: vel},
                        groups3(dims))
        nb = tuple((v + 7) // 8 for v in dims)
        bricks = np.zeros(nb[0] * nb[1] * nb[2], np.float32)
        t2 = run_kernel(ref, "bricks", P, {1: vol, 2: solt, 3: bricks}, groups3(nb))
        # the fire-light emission per cell (render.wgsl:63-98) on the packed
        # volume, with the colour table and uniform of src/render.rs:128-174
        from pyro_b200 import color
        lut = color.build_lut()
        chemi = color.chemi_block()
        ecell = np.zeros(nx * ny * nz, np.float32)
        t3 = run_kernel(ref, "ecells", P, {1: vol, 2: lut.copy(), 3: ecell, 4: chemi.copy()},
                        groups3(dims))
        out[f"render_c{case}"] = dict(params=pb, s0=S["s0"], s1=S["s1"], sol=S["sol"],
                                      flags=S["flags"], u=S["u"], v=S["v"], w=S["w"], vol=vol,
                                      solt=solt, vel=vel,
                                      bricks=bricks.reshape(nb[2], nb[1], nb[0]), lut=lut,
                                      chemi=chemi, ecell=ecell.reshape(n))
        print(f"render c{case} {t1:.1f}+{t2:.1f}+{t3:.1f}s", flush=True)
    return out


def render_rp(P, w, h, spp, frame, cache, bounces, aperture=0.0, first=0):
    """The trace kernels' uniform block (trace_lib.wgsl:1-14) for a camera
    outside the domain looking at its centre, built as src/render.rs:142-210
    does (fov 45 degrees, shutter 180 degrees at 30 fps, ground on, sky
    0.003, soot albedo 0.25); `aperture` > 0 is a thin lens focused on the
    centre, `first` the dispatch's first sample index."""
    from pyro_b200 import color
    dx = float(np.float32(P.dx))
    ext = np.array([P.nx * dx, P.ny * dx, P.nz * dx])
    target = 0.5 * ext
    pos = target + np.array([0.13, 0.07, -1.1])
    fwd = (target - pos) / np.linalg.norm(target - pos)
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right = right / np.linalg.norm(right)
    up = np.cross(right, fwd)
    focus = float(np.linalg.norm(target - pos))
    se = color.soot_extinction(0.25)
    side = 3.0 * max(ext[0], ext[2])
    f = np.float32
    return {
        "res": np.array([w, h, first, spp], np.uint32),
        "dims": np.array([P.nx, P.ny, P.nz, frame], np.uint32),
        "camPos": np.array([*pos, np.tan(np.radians(45.0) * 0.5)], f),
        "camFwd": np.array([*fwd, w / h], f),
        "camRight": np.array([*right, aperture], f),
        "camUp": np.array([*up, focus], f),
        "a": np.array([dx, 0.6, 180.0 / 360.0 / 30.0, 0.003], f),
        "b": np.array([1.0, 0.12, bounces, 0.05], f),
        "soot": np.array([se[0], se[1], se[2], 0.25], f),
        "c": np.array([5.0, 0.92, 0.55, P.t0], f),
        "alb": [np.array([0.32, 0.05, 0.05, 0.05], f), np.array([0.05, 0.05, 0.05, 0.05], f)],
        "gc": np.array([0.5 * ext[0] - 0.5 * side, 0.5 * ext[2] - 0.5 * side, side,
                        1.0 if cache else 0.0], f),
    }


RP_FIELDS = ("res", "dims", "camPos", "camFwd", "camRight", "camUp", "a", "b", "soot", "c",
             "alb0", "alb1", "gc")


def rp_array(rp):
    """The uniform block as 13 rows of 4 (u32 rows stored as their values)."""
    rows = []
    for k in RP_FIELDS:
        v = rp["alb"][int(k[-1])] if k.startswith("alb") else rp[k]
        rows.append(np.asarray(v, np.float64))
    return np.stack(rows)


def gen_trace(ref, only):
    """The renderer's light caches and camera rays (render.wgsl:100-304,
    trace_lib.wgsl) on the render golden's packed volumes, in the order of
    src/render.rs:351-418: lightvol, lightground, the blur chain, then
    trace.  Sizes are cut for the interpreter: an 8x8 ground cache (256^2 in
    the reference) and 8 shadow rays per cache cell (LV_N = 96, GR_N = 128)."""
    cases = {"cache": (6, 4, 2, 2.0, 0.0, 0, 3), "path": (4, 3, 2, 2.0, 0.0, 0, 3),
             # a thin lens, another frame and a later first sample
             "lens": (4, 3, 2, 2.0, 0.03, 5, 9)}
    if only is not None and "trace" not in only:
        cases = {k: v for k, v in cases.items() if f"trace_{k}" in only}
    if not cases:
        return {}
    from pyro_b200 import color
    d = np.load(os.path.join(HERE, "render_c0.npz"))
    P = params_from(d["params"])
    nx, ny, nz = int(P.nx), int(P.ny), int(P.nz)
    # a glowing-smoke volume: the random golden state's soot, heat release
    # and temperature clamped to 2 ppm, 500 kW/m^3 and 1000 K
    v32 = d["vol"].astype(np.float32)
    v32[..., 0] = np.clip(v32[..., 0], 0.0, 2.0)
    v32[..., 3] = np.clip(v32[..., 3], 0.0, 500.0)
    v32[..., 1] = np.minimum(v32[..., 1], 1000.0)  # cached flux stays within binary16
    vol, solt, vel = v32.astype(np.float16), d["solt"], d["vel"]
    bricks = d["bricks"].reshape(-1).astype(np.float32)
    lut = color.build_lut()
    # the emission CDF as the reference forms it: its ecells kernel on this
    # volume, then the FP64 running sum of src/render.rs:316-333
    e32 = np.zeros(nx * ny * nz, np.float32)
    run_kernel(ref, "ecells", P, {1: vol, 2: lut.copy(), 3: e32, 4: color.chemi_block()},
               groups3((nx, ny, nz)))
    e = np.maximum(e32, 0).astype(np.float64)
    acc = np.cumsum(e)
    tot = acc[-1]
    ecdf = np.append((acc / tot).astype(np.float32), np.float32(tot))
    lvd = ((nx + 1) // 2, (ny + 1) // 2, (nz + 1) // 2)
    gres = 8
    over = {"LV_N": np.uint32(8), "GR_N": np.uint32(8)}
    out = {}
    for mode, (w, h, spp, bounces, aperture, first, frame) in cases.items():
        cache = mode != "path"
        rp = render_rp(P, w, h, spp, frame, cache, bounces, aperture, first)
        lvA = np.zeros((lvd[2], lvd[1], lvd[0], 4), np.float16)
        lvB = np.zeros_like(lvA)
        gE = np.zeros((1, gres, gres, 4), np.float16)
        base = {0: rp, 1: vol, 2: solt, 3: vel, 4: None, 5: bricks, 6: lut, 8: ecdf}
        t0 = time.time()
        if cache:
            m = wgsl.Module(ref.assemble("lightvol"), overrides=over)
            for b_, v_ in {**base, 12: lvA, 13: lvB}.items():
                m.bind(b_, v_)
            m.dispatch(groups3(lvd))
            m = wgsl.Module(ref.assemble("lightground"), overrides=over)
            for b_, v_ in {**base, 14: gE}.items():
                m.bind(b_, v_)
            m.dispatch(((gres + 7) // 8, (gres + 7) // 8, 1), wg=(8, 8, 1))
            raw = dict(lvA=lvA.copy(), lvB=lvB.copy(), gE=gE.copy())
            t1 = np.zeros_like(lvA)
            t2 = np.zeros_like(lvA)
            gt = np.zeros_like(gE)
            chain = [((0, 2), lvA, t1), ((1, 2), t1, t2), ((2, 2), t2, lvA),
                     ((0, 2), lvB, t1), ((1, 2), t1, t2), ((2, 2), t2, lvB),
                     ((0, 3), gE, gt), ((1, 3), gt, gE)]
            for (axis, rad), src, dst in chain:
                m = wgsl.Module(ref.assemble("blur"))
                m.bind(0, {"axis": np.array([axis, rad, 0, 0], np.uint32)})
                m.bind(1, src)
                m.bind(2, dst)
                dd = (src.shape[2], src.shape[1], src.shape[0])
                m.dispatch(groups3(dd))
        accum = np.zeros((w * h, 4), np.float32)
        m = wgsl.Module(ref.assemble("trace"), overrides=over)
        for b_, v_ in {**base, 7: accum, 9: lvA, 10: lvB, 11: gE}.items():
            m.bind(b_, v_)
        m.dispatch(((w + 7) // 8, (h + 7) // 8, 1), wg=(8, 8, 1))
        rec = dict(params=d["params"], vol=vol, solt=solt, vel=vel, bricks=bricks, lut=lut,
                   ecdf=ecdf, rp=rp_array(rp), lvA=lvA, lvB=lvB, gE=gE, accum=accum)
        if cache:
            rec.update({k + "_raw": v for k, v in raw.items()})
        out[f"trace_{mode}"] = rec
        print(f"trace {mode} {time.time() - t0:.1f}s", flush=True)
    return out


def params_from(pb):
    from pyro_b200 import _abi
    import ctypes
    P = _abi.PyroParams()
    b = bytes(pb)
    ctypes.memmove(ctypes.byref(P), b, len(b))
    return P


def lv(d, h):
    return {"nx": np.uint32(d[0]), "ny": np.uint32(d[1]), "nz": np.uint32(d[2]), "h": np.float32(h)}


def gen_mg(ref, only):
    out = {}
    if only is not None and not ({"mg"} & set(only)):
        return out
    rng = np.random.default_rng(21)
    nx, ny, nz = MG_DIMS
    n = (nz, ny, nx)
    h = 0.1
    f = (rng.random(n) < 0.2).astype(np.uint32)
    b = rng.normal(0, 1, n).astype(np.float32)
    p = rng.normal(0, 1, n).astype(np.float32)
    # smoother: colour 0/1, omega 1 and 1.6
    for color, om in [(0, 1.0), (1, 1.0), (0, 1.6), (1, 1.6)]:
        pp = flat(p)
        m = wgsl.Module(ref.assemble("mg_smooth"), overrides={"COLOR": color, "OMEGA": om},
                        replace=IDENT)
        m.bind(0, lv((nx, ny, nz), h))
        m.bind(1, flat(b))
        m.bind(2, flat(f))
        m.bind(3, pp)
        m.dispatch(groups3(((nx + 1) // 2, ny, nz)))
        out[f"mg_smooth_c{color}_w{int(om * 10)}"] = dict(dims=np.array(MG_DIMS), h=np.float32(h),
                                                         b=b, f=f, p=p, out=pp.reshape(n))
    # restrict
    cd = tuple((v + 1) // 2 for v in MG_DIMS)
    cn = (cd[2], cd[1], cd[0])
    bc = np.zeros(cd[0] * cd[1] * cd[2], np.float32)
    pc = np.ones_like(bc)
    fc = np.zeros(cd[0] * cd[1] * cd[2], np.uint32)
    m = wgsl.Module(ref.assemble("mg_restrict"), replace=IDENT)
    m.bind(0, lv(MG_DIMS, h))
    m.bind(1, flat(p))
    m.bind(2, flat(b))
    m.bind(3, flat(f))
    m.bind(4, bc)
    m.bind(5, pc)
    m.bind(6, fc)
    m.bind(7, lv(cd, 2 * h))
    m.dispatch(groups3(cd))
    out["mg_restrict"] = dict(dims=np.array(MG_DIMS), h=np.float32(h), b=b, f=f, p=p,
                              bc=bc.reshape(cn), pc=pc.reshape(cn), fc=fc.reshape(cn))
    # prolong (coarse flags from the restriction above)
    pcv = rng.normal(0, 1, cn).astype(np.float32)
    pf = flat(p)
    m = wgsl.Module(ref.assemble("mg_prolong"), replace=IDENT)
    m.bind(0, lv(MG_DIMS, h))
    m.bind(1, flat(pcv))
    m.bind(2, flat(f))
    m.bind(3, pf)
    m.bind(4, lv(cd, 2 * h))
    m.bind(5, fc.copy())
    m.dispatch(groups3(MG_DIMS))
    out["mg_prolong"] = dict(dims=np.array(MG_DIMS), pc=pcv, f=f, fc=fc.reshape(cn), p=p,
                             out=pf.reshape(n))
    # residual sums
    st = stats_buf()
    m = wgsl.Module(ref.assemble("mg_resid"), replace=IDENT)
    m.bind(0, lv(MG_DIMS, h))
    m.bind(1, flat(p))
    m.bind(2, flat(b))
    m.bind(3, flat(f))
    m.bind(4, st)
    m.dispatch(groups3(MG_DIMS))
    out["mg_resid"] = dict(dims=np.array(MG_DIMS), h=np.float32(h), b=b, f=f, p=p,
                           stats=st.view(np.float32))
    print("mg done", flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PYRO_REFERENCE"),
                    help="the reference checkout (default: $PYRO_REFERENCE)")
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    if not a.ref:
        ap.error("give the reference checkout with --ref or PYRO_REFERENCE")
    only = set(a.only.split(",")) if a.only else None
    ref = Ref(a.ref)
    out = {}
    out.update(gen_sim(ref, only))
    out.update(gen_mg(ref, only))
    out.update(gen_render(ref, only))
    out.update(gen_trace(ref, only))
    for k, d in out.items():
        np.savez_compressed(os.path.join(HERE, k + ".npz"), **d)
    print(f"wrote {len(out)} fixtures to {HERE}")


if __name__ == "__main__":
    main()
