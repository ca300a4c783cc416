"""Python bindings of the CPU oracle (oracle/pyro_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs as the checker and the CPU baseline; the product
(pyro_b200) never imports it.

The oracle restates the reference's WGSL simulation kernels and the
src/sim.rs schedule in FP32 C++ (built with -ffp-contract=off), plus an FP64
CG solve of the pressure system.  Its kernels are pinned by golden vectors
produced by interpreting the reference's own WGSL source
(tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_D = ctypes.c_double
_U = ctypes.c_uint32

_SIGS = {
    "or_set_threads": (None, [_I]),
    "or_max_threads": (_I, []),
    "or_solid": (None, [_P] * 7),
    "or_curl": (None, [_P] * 6),
    "or_adv_vel1": (None, [_P] * 7),
    "or_adv_vel2": (None, [_P] * 11),
    "or_adv_s1": (None, [_P] * 8),
    "or_adv_s2": (None, [_P] * 10),
    "or_react": (None, [_P] * 10),
    "or_forces": (None, [_P] * 8),
    "or_divergence": (None, [_P] * 7),
    "or_project": (None, [_P] * 6),
    "or_render_pack": (None, [_P] * 11),
    "or_render_bricks": (None, [_I, _I, _I, _P, _P, _P]),
    "or_render_ecells": (None, [_P] * 5),
    "or_render_cdf": (None, [ctypes.c_size_t, _P, _P]),
    "or_render_lightvol": (None, [_P] * 7 + [_I, _I, _I, _I, _P, _P]),
    "or_render_lightground": (None, [_P] * 7 + [_I, _I, _P]),
    "or_render_blur": (None, [_P, _P, _I, _I, _I, _I, _I]),
    "or_render_trace": (None, [_P] * 7 + [_P, _P, _I, _I, _I, _P, _I, _P]),
    "or_f32_to_f16": (None, [_P, _P, ctypes.c_size_t]),
    "or_f16_to_f32": (None, [_P, _P, ctypes.c_size_t]),
    "or_mg_smooth": (None, [_I, _I, _I, _F, _P, _P, _P, _I, _F, _I]),
    "or_mg_restrict": (None, [_I, _I, _I, _F, _P, _P, _P, _I, _I, _I, _P, _P, _P, _I]),
    "or_mg_prolong": (None, [_I, _I, _I, _P, _P, _P, _I, _I, _I, _P]),
    "or_mg_resid": (None, [_I, _I, _I, _F, _P, _P, _P, _I, _P, _P]),
    "or_mg_levels": (_I, [_I, _I, _I, _P]),
    "or_vcycles": (None, [_I, _I, _I, _F, _P, _P, _P, _I, _I]),
    "or_poisson_f64": (_I, [_I, _I, _I, _D, _P, _P, _P, _D, _I, _I, _P]),
    "or_poisson_relres": (_D, [_I, _I, _I, _D, _P, _P, _P, _I]),
    "or_sim_create": (_P, [_P, _P, _U]),
    "or_sim_step": (None, [_P, _F, _F, _F, _I]),
    "or_sim_read_stats": (None, [_P, _P]),
    "or_sim_read_field": (_I, [_P, _I, _P, ctypes.c_size_t]),
    "or_sim_write_field": (_I, [_P, _I, _P, ctypes.c_size_t]),
    "or_sim_destroy": (None, [_P]),
    "or_voxelize": (None, [_P, _U, _I, _I, _I, _F, _F, _U, _P, _P, _P]),
    "or_hash_f": (_F, [_U]),
}

_lib = None


def build() -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    r = subprocess.run(["make", "-s", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def ptr(a) -> ctypes.c_void_p:
    if a is None:
        return ctypes.c_void_p(0)
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data_as(ctypes.c_void_p)
    return ctypes.cast(ctypes.byref(a), ctypes.c_void_p)


def set_threads(n: int) -> None:
    lib().or_set_threads(n)


def max_threads() -> int:
    return lib().or_max_threads()


# ----------------------------------------------------------------- kernels
def dims_of(P):
    return int(P.nx), int(P.ny), int(P.nz)


def solid(P, sol_in, s0, stats=None):
    nx, ny, nz = dims_of(P)
    sol_out = np.zeros_like(sol_in)
    pyr = np.zeros_like(sol_in)
    flags = np.zeros((nz, ny, nx), np.uint32)
    lib().or_solid(ptr(P), ptr(sol_in), ptr(sol_out), ptr(pyr), ptr(flags), ptr(s0), ptr(stats))
    return sol_out, pyr, flags


def curl(P, u, v, w, stats=None):
    nx, ny, nz = dims_of(P)
    c = np.zeros((nz, ny, nx, 4), np.float32)
    lib().or_curl(ptr(P), ptr(u), ptr(v), ptr(w), ptr(c), ptr(stats))
    return c


def adv_vel(P, u, v, w, flags):
    hu, hv, hw = np.zeros_like(u), np.zeros_like(v), np.zeros_like(w)
    ou, ov, ow = np.zeros_like(u), np.zeros_like(v), np.zeros_like(w)
    lib().or_adv_vel1(ptr(P), ptr(u), ptr(v), ptr(w), ptr(hu), ptr(hv), ptr(hw))
    lib().or_adv_vel2(ptr(P), ptr(u), ptr(v), ptr(w), ptr(hu), ptr(hv), ptr(hw), ptr(ou),
                      ptr(ov), ptr(ow), ptr(flags))
    return (hu, hv, hw), (ou, ov, ow)


def adv_scalars(P, u, v, w, s0, s1):
    h0, h1 = np.zeros_like(s0), np.zeros_like(s1)
    o0, o1 = np.zeros_like(s0), np.zeros_like(s1)
    lib().or_adv_s1(ptr(P), ptr(u), ptr(v), ptr(w), ptr(s0), ptr(s1), ptr(h0), ptr(h1))
    lib().or_adv_s2(ptr(P), ptr(u), ptr(v), ptr(w), ptr(s0), ptr(s1), ptr(h0), ptr(h1), ptr(o0),
                    ptr(o1))
    return (h0, h1), (o0, o1)


def react(P, s0in, s1in, flags, sol, pyr, curl_, stats=None):
    s0out, s1out = np.zeros_like(s0in), np.zeros_like(s1in)
    lib().or_react(ptr(P), ptr(s0in), ptr(s1in), ptr(s0out), ptr(s1out), ptr(flags), ptr(sol),
                   ptr(pyr), ptr(curl_), ptr(stats))
    return s0out, s1out


def forces(P, u, v, w, s0, s1, curl_, flags):
    u, v, w = u.copy(), v.copy(), w.copy()
    lib().or_forces(ptr(P), ptr(u), ptr(v), ptr(w), ptr(s0), ptr(s1), ptr(curl_), ptr(flags))
    return u, v, w


def divergence(P, u, v, w, s1, flags):
    nx, ny, nz = dims_of(P)
    b = np.zeros((nz, ny, nx), np.float32)
    lib().or_divergence(ptr(P), ptr(u), ptr(v), ptr(w), ptr(s1), ptr(flags), ptr(b))
    return b


def project(P, u, v, w, phi, flags):
    u, v, w = u.copy(), v.copy(), w.copy()
    lib().or_project(ptr(P), ptr(u), ptr(v), ptr(w), ptr(phi), ptr(flags))
    return u, v, w


def render_pack(P, s0, s1, sol, flags, u, v, w):
    """render.wgsl:17-35: (vol, sol, vel), float16 (nz, ny, nx, 4) each."""
    nx, ny, nz = dims_of(P)
    vol, solt, vel = (np.zeros((nz, ny, nx, 4), np.float16) for _ in range(3))
    lib().or_render_pack(ptr(P), ptr(s0), ptr(s1), ptr(sol), ptr(flags), ptr(u), ptr(v), ptr(w),
                         ptr(vol), ptr(solt), ptr(vel))
    return vol, solt, vel


def render_bricks(dims, vol, solt):
    """render.wgsl:38-61: float32 (ceil(nz/8), ceil(ny/8), ceil(nx/8))."""
    nx, ny, nz = dims
    out = np.zeros(((nz + 7) // 8, (ny + 7) // 8, (nx + 7) // 8), np.float32)
    lib().or_render_bricks(nx, ny, nz, ptr(vol), ptr(solt), ptr(out))
    return out


def render_ecells(P, vol, lut, chemi):
    """render.wgsl:63-98: float32 (nz, ny, nx) emission power per cell."""
    nx, ny, nz = dims_of(P)
    e = np.zeros((nz, ny, nx), np.float32)
    lib().or_render_ecells(ptr(P), ptr(np.ascontiguousarray(vol)),
                           ptr(np.ascontiguousarray(lut, np.float32)),
                           ptr(np.ascontiguousarray(chemi, np.float32)), ptr(e))
    return e


def render_cdf(e):
    """src/render.rs:316-333: float32 (n + 1,)."""
    e = np.ascontiguousarray(e, np.float32).reshape(-1)
    cdf = np.zeros(e.size + 1, np.float32)
    lib().or_render_cdf(ctypes.c_size_t(e.size), ptr(e), ptr(cdf))
    return cdf


def _h(a):
    return np.ascontiguousarray(a, np.float16)


def render_lightvol(rp, vol, solt, vel, bricks, lut, ecdf, lv_dims, lv_n=96):
    """render.wgsl:217-251: (lvA, lvB) float16 (lz, ly, lx, 4)."""
    lx, ly, lz = lv_dims
    a = np.zeros((lz, ly, lx, 4), np.float16)
    b = np.zeros_like(a)
    lib().or_render_lightvol(ptr(np.ascontiguousarray(rp, np.float64)), ptr(_h(vol)), ptr(_h(solt)),
                             ptr(_h(vel)), ptr(np.ascontiguousarray(bricks, np.float32)),
                             ptr(np.ascontiguousarray(lut, np.float32)),
                             ptr(np.ascontiguousarray(ecdf, np.float32)), lx, ly, lz, lv_n,
                             ptr(a), ptr(b))
    return a, b


def render_lightground(rp, vol, solt, vel, bricks, lut, ecdf, gres, gr_n=128):
    """render.wgsl:253-269: gE float16 (1, gres, gres, 4)."""
    g = np.zeros((1, gres, gres, 4), np.float16)
    lib().or_render_lightground(ptr(np.ascontiguousarray(rp, np.float64)), ptr(_h(vol)),
                                ptr(_h(solt)), ptr(_h(vel)),
                                ptr(np.ascontiguousarray(bricks, np.float32)),
                                ptr(np.ascontiguousarray(lut, np.float32)),
                                ptr(np.ascontiguousarray(ecdf, np.float32)), gres, gr_n, ptr(g))
    return g


def render_blur(src, axis, r):
    """render.wgsl:271-304: one axis of the separable Gaussian."""
    src = _h(src)
    dst = np.zeros_like(src)
    nz, ny, nx = src.shape[:3]
    lib().or_render_blur(ptr(src), ptr(dst), nx, ny, nz, axis, r)
    return dst


def render_trace(rp, vol, solt, vel, bricks, lut, ecdf, lvA, lvB, gE, accum=None):
    """render.wgsl:132-215: accum (res.y * res.x, 4) float32 += the samples."""
    rp = np.ascontiguousarray(rp, np.float64)
    w, h = int(rp[0, 0]), int(rp[0, 1])
    acc = np.zeros((w * h, 4), np.float32) if accum is None else np.ascontiguousarray(
        accum, np.float32).copy()
    lvA, lvB, gE = _h(lvA), _h(lvB), _h(gE)
    lz, ly, lx = lvA.shape[:3]
    lib().or_render_trace(ptr(rp), ptr(_h(vol)), ptr(_h(solt)), ptr(_h(vel)),
                          ptr(np.ascontiguousarray(bricks, np.float32)),
                          ptr(np.ascontiguousarray(lut, np.float32)),
                          ptr(np.ascontiguousarray(ecdf, np.float32)), ptr(lvA), ptr(lvB), lx,
                          ly, lz, ptr(gE), gE.shape[1], ptr(acc))
    return acc


def f32_to_f16(x):
    """The oracle's binary32 -> binary16 conversion (round to nearest even)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    h = np.zeros(x.shape, np.uint16)
    lib().or_f32_to_f16(ptr(x), ptr(h), ctypes.c_size_t(x.size))
    return h


def f16_to_f32(h):
    h = np.ascontiguousarray(h, dtype=np.uint16)
    x = np.zeros(h.shape, np.float32)
    lib().or_f16_to_f32(ptr(h), ptr(x), ctypes.c_size_t(h.size))
    return x


def mg_smooth(dims, h, b, f, p, color, omega, bc_mode=0):
    p = p.copy()
    lib().or_mg_smooth(dims[0], dims[1], dims[2], h, ptr(b), ptr(f), ptr(p), color, omega,
                       bc_mode)
    return p


def mg_restrict(fd, fh, pf, bf, ff, bc_mode=0):
    cd = tuple((v + 1) // 2 for v in fd)
    shape = (cd[2], cd[1], cd[0])
    bc = np.zeros(shape, np.float32)
    pc = np.ones(shape, np.float32)
    fc = np.zeros(shape, np.uint32)
    lib().or_mg_restrict(fd[0], fd[1], fd[2], fh, ptr(pf), ptr(bf), ptr(ff), cd[0], cd[1], cd[2],
                         ptr(bc), ptr(pc), ptr(fc), bc_mode)
    return bc, pc, fc


def mg_prolong(fd, pc, ff, pf, fc):
    cd = tuple((v + 1) // 2 for v in fd)
    pf = pf.copy()
    lib().or_mg_prolong(fd[0], fd[1], fd[2], ptr(pc), ptr(ff), ptr(pf), cd[0], cd[1], cd[2],
                        ptr(fc))
    return pf


def mg_resid(dims, h, p, b, f, bc_mode=0):
    r2 = ctypes.c_double()
    b2 = ctypes.c_double()
    lib().or_mg_resid(dims[0], dims[1], dims[2], h, ptr(p), ptr(b), ptr(f), bc_mode,
                      ctypes.cast(ctypes.byref(r2), ctypes.c_void_p),
                      ctypes.cast(ctypes.byref(b2), ctypes.c_void_p))
    return r2.value, b2.value


def mg_levels(nx, ny, nz):
    out = np.zeros(12, np.int32)
    n = lib().or_mg_levels(nx, ny, nz, ptr(out))
    return [tuple(int(v) for v in out[3 * i:3 * i + 3]) for i in range(n)]


def vcycles(dims, h, phi, b, f, cycles, bc_mode=0):
    phi = phi.copy()
    lib().or_vcycles(dims[0], dims[1], dims[2], h, ptr(phi), ptr(b), ptr(f), cycles, bc_mode)
    return phi


def poisson_f64(dims, h, b, f, tol=1e-12, max_iters=20000, bc_mode=0, x0=None):
    """FP64 CG solve; returns (phi64, iterations, relative residual)."""
    nx, ny, nz = dims
    x = np.zeros((nz, ny, nx), np.float64) if x0 is None else x0.astype(np.float64).copy()
    rel = ctypes.c_double()
    it = lib().or_poisson_f64(nx, ny, nz, h, ptr(b), ptr(f), ptr(x), tol, max_iters, bc_mode,
                              ctypes.cast(ctypes.byref(rel), ctypes.c_void_p))
    return x, it, rel.value


def poisson_relres(dims, h, phi, b, f, bc_mode=0) -> float:
    return lib().or_poisson_relres(dims[0], dims[1], dims[2], h, ptr(phi), ptr(b), ptr(f),
                                   bc_mode)


def voxelize(shapes, n, nx, ny, nz, dx, t0, seed, dens, kind):
    sol = np.zeros((nz, ny, nx, 4), np.float32)
    lib().or_voxelize(ctypes.cast(shapes, ctypes.c_void_p), n, nx, ny, nz, dx, t0, seed,
                      ctypes.cast(dens, ctypes.c_void_p), ctypes.cast(kind, ctypes.c_void_p),
                      ptr(sol))
    return sol


def hash_f(v: int) -> float:
    return lib().or_hash_f(v)


# ------------------------------------------------------------- whole sim
F_S0, F_S1, F_SOL, F_PYR, F_FLAGS, F_CURL, F_U, F_V, F_W, F_PHI, F_B = range(11)


class OracleSim:
    """Sim::new / Sim::step on the CPU (src/sim.rs:108-423)."""

    def __init__(self, P, sol_init, cycles):
        self.P = P
        self.dims = dims_of(P)
        sol_init = np.ascontiguousarray(sol_init, dtype=np.float32)
        self._h = lib().or_sim_create(ptr(P), ptr(sol_init), cycles)
        self.time = np.float32(0.0)

    def close(self):
        if self._h:
            lib().or_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt, time, ign_on, want_stats):
        lib().or_sim_step(self._h, dt, time, ign_on, 1 if want_stats else 0)

    def read_stats(self):
        out = np.zeros(1040, np.float32)
        lib().or_sim_read_stats(self._h, ptr(out))
        return out

    def _shape(self, which):
        nx, ny, nz = self.dims
        if which in (F_U, F_V, F_W):
            return (nz + 1, ny + 1, nx + 1), np.float32
        if which == F_FLAGS:
            return (nz, ny, nx), np.uint32
        if which in (F_PHI, F_B):
            return (nz, ny, nx), np.float32
        return (nz, ny, nx, 4), np.float32

    def read_field(self, which):
        shape, dt = self._shape(which)
        out = np.zeros(shape, dt)
        rc = lib().or_sim_read_field(self._h, which, ptr(out), out.nbytes)
        assert rc == 0
        return out

    def write_field(self, which, arr):
        shape, dt = self._shape(which)
        arr = np.ascontiguousarray(arr, dtype=dt).reshape(shape)
        rc = lib().or_sim_write_field(self._h, which, ptr(arr), arr.nbytes)
        assert rc == 0
