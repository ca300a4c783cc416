"""ctypes view of the C ABI declared in include/pyro_sim.h.

The structures here are byte-for-byte the C structs; `PyroParams` is the
reference's 576-byte uniform block (src/scene.rs:424-477,
src/shaders/common.wgsl:14-28).  `load()` opens the in-tree CUDA library
and raises when it is missing: there is no CPU fallback for the product path.
"""
from __future__ import annotations

import ctypes
import os

PYRO_OK = 0
PYRO_E_INVALID = -1
PYRO_E_CUDA = -2
PYRO_E_NOMEM = -3
PYRO_E_STATE = -4
PYRO_E_NOCONV = -5
PYRO_E_TIMEOUT = -6

STATS_N = 1040
NOALLOC_MAX_CELLS = 1 << 19
POST_SEL_WORDS = 260  # radix-select scratch of pyro_post_select
MAX_LAYERS = 1024
ABI_VERSION = 2

F_S0, F_S1, F_SOL, F_PYR, F_FLAGS, F_CURL, F_U, F_V, F_W, F_PHI, F_B = range(11)
F_RVOL, F_RSOL, F_RVEL, F_BRICKS = range(11, 15)  # renderer input pack
F_ECELL, F_ECDF = 15, 16  # renderer fire-light sampling tables

PROFILE_PHASES = ["solid", "curl", "adv_vel1", "adv_vel2", "adv_s1", "adv_s2", "react",
                  "forces", "divergence", "pressure", "project", "total"]

MG_F32, MG_BF16 = 0, 1  # storage of phi and b in the pyro_k_mg_* mask entries
# launch classes of pyro_poisson_profile_cg: those of
# pyro_sim_profile_pressure, then the CG vector kernels
CG_CLASSES = ["mg_prepare", "mg_pass_l0", "mg_restrict_l0", "mg_prolong_l0", "mg_pass_mid",
              "mg_restrict_mid", "mg_prolong_mid", "mg_coarse", "cg_vector"]
# launch classes of pyro_sim_profile_pressure
MG_CLASSES = ["mg_prepare", "mg_pass_l0", "mg_restrict_l0", "mg_prolong_l0", "mg_pass_mid",
              "mg_restrict_mid", "mg_prolong_mid", "mg_coarse"]

SOLVER_VCYCLE = 0
SOLVER_VCYCLE_TOL = 1
SOLVER_MGPCG = 2
SOLVER_MGPCG_BF16 = 3
SOLVER_MGPCG_LEARNED = 4

SHAPE_BOX, SHAPE_CYL, SHAPE_SPHERE, SHAPE_POOL = range(4)

PARAM_SCALARS = [
    ("nx", ctypes.c_uint32), ("ny", ctypes.c_uint32), ("nz", ctypes.c_uint32),
    ("frame", ctypes.c_uint32),
    ("dx", ctypes.c_float), ("dt", ctypes.c_float), ("time", ctypes.c_float),
    ("t0", ctypes.c_float),
    ("rho0", ctypes.c_float), ("g", ctypes.c_float), ("cp", ctypes.c_float),
    ("yo2", ctypes.c_float),
    ("vort", ctypes.c_float), ("cs", ctypes.c_float), ("buoy", ctypes.c_float),
    ("smoke_w", ctypes.c_float),
    ("wind_x", ctypes.c_float), ("wind_z", ctypes.c_float),
    ("wind_relax", ctypes.c_float), ("sponge", ctypes.c_float),
    ("t_ign", ctypes.c_float), ("s_o2", ctypes.c_float), ("dhc", ctypes.c_float),
    ("tau_min", ctypes.c_float),
    ("soot_form", ctypes.c_float), ("soot_ox", ctypes.c_float),
    ("soot_ox_t", ctypes.c_float), ("smoke_conv", ctypes.c_float),
    ("kap_gas", ctypes.c_float), ("h_conv", ctypes.c_float),
    ("ign_on", ctypes.c_float), ("ign_temp", ctypes.c_float),
    ("ign_x", ctypes.c_float), ("ign_y", ctypes.c_float), ("ign_z", ctypes.c_float),
    ("ign_r", ctypes.c_float),
    ("ign_flux", ctypes.c_float), ("ign_fuel", ctypes.c_float),
    ("char_a", ctypes.c_float), ("char_e", ctypes.c_float),
    ("dh_char", ctypes.c_float), ("burnout", ctypes.c_float),
    ("layer", ctypes.c_float), ("rad_len", ctypes.c_float),
    ("h_mass", ctypes.c_float), ("vort_t", ctypes.c_float),
    ("rad_frac", ctypes.c_float), ("seed", ctypes.c_float),
]


class PyroRenderParams(ctypes.Structure):
    """The path tracer's uniform block (struct RP, trace_lib.wgsl:1-14)."""
    _fields_ = [("res", ctypes.c_uint32 * 4), ("dims", ctypes.c_uint32 * 4),
                ("cam_pos", ctypes.c_float * 4), ("cam_fwd", ctypes.c_float * 4),
                ("cam_right", ctypes.c_float * 4), ("cam_up", ctypes.c_float * 4),
                ("a", ctypes.c_float * 4), ("b", ctypes.c_float * 4),
                ("soot", ctypes.c_float * 4), ("c", ctypes.c_float * 4),
                ("alb", ctypes.c_float * 8), ("gc", ctypes.c_float * 4)]
    ROWS = ("res", "dims", "cam_pos", "cam_fwd", "cam_right", "cam_up", "a", "b", "soot", "c",
            "alb", "alb", "gc")

    @classmethod
    def from_rows(cls, rows) -> "PyroRenderParams":
        """From 13 rows of 4 numbers in the block's order (u32 rows as their
        values; rows 10 and 11 the eight albedos)."""
        rows = [list(map(float, r)) for r in rows]
        if len(rows) != 13 or any(len(r) != 4 for r in rows):
            raise ValueError("render parameters: expected 13 rows of 4")
        p = cls()
        for k, name in enumerate(cls.ROWS):
            if name == "alb":
                continue
            dst = getattr(p, name)
            for j in range(4):
                dst[j] = int(rows[k][j]) if name in ("res", "dims") else rows[k][j]
        for j in range(8):
            p.alb[j] = rows[10 + j // 4][j % 4]
        return p

    def rows(self):
        """The 13 x 4 rows (inverse of from_rows)."""
        out = []
        for k, name in enumerate(self.ROWS):
            if name == "alb":
                out.append([float(self.alb[4 * (k - 10) + j]) for j in range(4)])
            else:
                out.append([float(v) for v in getattr(self, name)])
        return out


class PyroParams(ctypes.Structure):
    _fields_ = PARAM_SCALARS + [("mats", (ctypes.c_float * 12) * 8)]

    def to_bytes(self) -> bytes:
        return bytes(memoryview(self).cast("B"))

    def copy(self) -> "PyroParams":
        c = PyroParams()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(self))
        return c


assert ctypes.sizeof(PyroParams) == 576
assert ctypes.sizeof(PyroRenderParams) == 208


class PyroShape(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_uint32), ("slot", ctypes.c_uint32),
        ("c", ctypes.c_float * 3), ("e", ctypes.c_float * 3),
        ("r", ctypes.c_float), ("depth", ctypes.c_float),
        ("sin_yaw", ctypes.c_float), ("cos_yaw", ctypes.c_float),
    ]


class PyroSolveInfo(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32), ("iterations", ctypes.c_int32),
        ("rel_resid", ctypes.c_double), ("b_norm", ctypes.c_double),
        ("ms", ctypes.c_float), ("converged", ctypes.c_int32),
        ("learned", ctypes.c_int32), ("learned_ms", ctypes.c_float),
        ("rel_resid_start", ctypes.c_double), ("rel_resid_learned", ctypes.c_double),
    ]


class PyroSimInfo(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_uint32), ("ny", ctypes.c_uint32), ("nz", ctypes.c_uint32),
        ("levels", ctypes.c_uint32), ("level_dims", (ctypes.c_uint32 * 3) * 8),
        ("cells", ctypes.c_uint64), ("faces", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64),
    ]


HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpyro_b200.so")

_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_F = ctypes.c_float
_I = ctypes.c_int
_U64 = ctypes.c_uint64
_D = ctypes.c_double

# name -> argtypes; every entry point returns int.
SIGNATURES = {
    "pyro_abi_version": [],
    "pyro_sim_create": [ctypes.POINTER(PyroParams), _P, _U32, ctypes.POINTER(_P)],
    "pyro_sim_step": [_P, _F, _F, _F, _I],
    "pyro_sim_read_stats": [_P, _P, ctypes.c_size_t],
    "pyro_sim_read_stats_prev": [_P, _P, ctypes.c_size_t],
    "pyro_sim_read_field": [_P, _I, _P, ctypes.c_size_t],
    "pyro_sim_write_field": [_P, _I, _P, ctypes.c_size_t],
    "pyro_sim_device_ptr": [_P, _I, ctypes.POINTER(_P), ctypes.POINTER(ctypes.c_size_t)],
    "pyro_sim_stream": [_P, ctypes.POINTER(_P)],
    "pyro_sim_sync": [_P],
    "pyro_sim_profile_step": [_P, _F, _F, _F, _I, _P, _I],
    "pyro_sim_profile_pressure": [_P, _P, _P, _I],
    "pyro_poisson_profile_cg": [_P, _P, _P, _I, _I, _P, _P, _I],
    "pyro_post_select": [_P, _U32, _U32, _U32, _P, _P, _P, ctypes.POINTER(_F), _P],
    "pyro_post_develop": [_P, _U32, _U32, _F, _F, _P, _P, _P, _P],
    "pyro_sim_info": [_P, ctypes.POINTER(PyroSimInfo)],
    "pyro_sim_set_solver": [_P, _I, _F, _I],
    "pyro_sim_last_solve": [_P, ctypes.POINTER(PyroSolveInfo)],
    "pyro_sim_destroy": [_P],
    "pyro_sim_render_pack": [_P, _I],
    "pyro_sim_render_emission": [_P, _P, _P],
    "pyro_voxelize": [ctypes.POINTER(PyroShape), _U32, _U32, _U32, _U32, _F, _F, _U32,
                      _P, _P, _P, _P],
    "pyro_poisson_create": [_U32, _U32, _U32, _F, _I, ctypes.POINTER(_P)],
    "pyro_poisson_set_flags": [_P, _P],
    "pyro_poisson_solve": [_P, _P, _P, _I, _F, _I, ctypes.POINTER(PyroSolveInfo)],
    "pyro_poisson_stream": [_P, ctypes.POINTER(_P)],
    "pyro_poisson_destroy": [_P],
    "pyro_k_solid": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P, _P],
    "pyro_k_curl": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P],
    "pyro_k_adv_vel": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "pyro_k_adv_scalars": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "pyro_k_react": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "pyro_k_forces": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P, _P, _P],
    "pyro_k_forces_noalloc": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P, _P, _P],
    "pyro_k_divergence": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P, _P],
    "pyro_k_project": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P],
    "pyro_k_mg_smooth": [_U32, _U32, _U32, _F, _P, _P, _P, _I, _F, _P],
    "pyro_k_mg_restrict": [_U32, _U32, _U32, _F, _P, _P, _P, _U32, _U32, _U32, _P, _P, _P, _P],
    "pyro_k_mg_prolong": [_U32, _U32, _U32, _P, _P, _P, _U32, _U32, _U32, _P, _P],
    "pyro_k_mg_meta": [_U32, _U32, _U32, _P, _P, _P],
    "pyro_k_mg_flags_down": [_U32, _U32, _U32, _P, _U32, _U32, _U32, _P, _P],
    "pyro_k_mg_pass": [_U32, _U32, _U32, _F, _P, _P, _P, _I, _F, _I, _I, _P],
    "pyro_k_mg_restrict_sym": [_U32, _U32, _U32, _F, _P, _P, _P, _U32, _U32, _U32, _P, _P, _P,
                               _I, _I, _P],
    "pyro_k_mg_pass_first": [_U32, _U32, _U32, _F, _P, _P, _P, _P, _I, _F, _I, _I, _P],
    "pyro_k_mg_pass_last": [_U32, _U32, _U32, _F, _P, _P, _P, _P, _I, _F, _I, _P],
    "pyro_k_mg_restrict_m": [_U32, _U32, _U32, _F, _P, _P, _P, _U32, _U32, _U32, _P, _P, _I,
                             _I, _P],
    "pyro_k_mg_prolong_m": [_U32, _U32, _U32, _P, _P, _P, _U32, _U32, _U32, _P, _I, _P],
    "pyro_k_mg_resid": [_U32, _U32, _U32, _F, _P, _P, _P, _P, _P],
    "pyro_k_mg_coarse": [_U32, _U32, _U32, _F, _P, _P, _P, _I, _F, _P],
    "pyro_k_mg_apply": [_U32, _U32, _U32, _F, _P, _P, _P, _I, _P],
    "pyro_k_mg_coarse_sym": [_U32, _U32, _U32, _F, _P, _P, _P, _I, _F, _I, _P],
    "pyro_k_render_pack": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "pyro_k_render_bricks": [_U32, _U32, _U32, _P, _P, _P, _P],
    "pyro_k_render_ecells": [_P, _U32, _U32, _U32, _P, _P, _P, _P, _P],
    "pyro_k_render_cdf": [ctypes.c_uint64, _P, _P, _P],
    "pyro_k_render_lightvol": [_P, _P, _P, _P, _P, _P, _P, _U32, _U32, _U32, _U32, _P, _P, _P],
    "pyro_k_render_lightground": [_P, _P, _P, _P, _P, _P, _P, _U32, _U32, _P, _P],
    "pyro_k_render_blur": [_P, _P, _U32, _U32, _U32, _U32, _U32, _P],
    "pyro_k_render_trace": [_P, _P, _P, _P, _P, _P, _P, _P, _P, _U32, _U32, _U32, _P, _U32, _P,
                            _P],
    "pyro_conv3_forward": [_P, _I, _I, _I, _I, _I, _P, _I, _P, _I, _P, _I, _P],
    "pyro_conv3_backward_data": [_P, _I, _I, _I, _I, _I, _P, _I, _P, _P, _I, _P],
    "pyro_conv3_backward_weight": [_P, _I, _P, _I, _I, _I, _I, _I, _P, _P],
    "pyro_sim_set_net": [_P, _P],
    "pyro_poisson_set_net": [_P, _P],
    "pyro_learned_accept": [_D, _D, _D, _D, _D, ctypes.POINTER(_D), ctypes.POINTER(_D)],
    "pyro_net_create": [_U64, ctypes.POINTER(_P)],
    "pyro_net_destroy": [_P],
    "pyro_net_param_count": [_P, ctypes.POINTER(_U64)],
    "pyro_net_get_params": [_P, _P, _U64, ctypes.POINTER(_F)],
    "pyro_net_set_params": [_P, _P, _U64, _F],
    "pyro_net_forward": [_P, _P, _P, _U32, _U32, _U32, _U32, _F, _P, _P],
    "pyro_net_loss_grad": [_P, _P, _P, _P, _U32, _U32, _U32, _U32, _F, ctypes.POINTER(_D), _P,
                           _P],
    "pyro_net_train_step": [_P, _P, _P, _P, _U32, _U32, _U32, _U32, _F, _F, _F, _P],
    "pyro_net_last_loss": [_P, ctypes.POINTER(_D), _P],
    "pyro_net_set_loss": [_P, _F, _F],
}

_lib = None


class PyroError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, name: str, code: int, msg: str):
        super().__init__(f"{name} failed with status {code}: {msg}")
        self.code = code


def load() -> ctypes.CDLL:
    """Open libpyro_b200.so (built in-tree by pyro_b200.build).  Raises when
    the library is absent: the simulation has no CPU path."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"pyro_b200 CUDA library not found at {LIB_PATH}; build it with "
            "`python -m pyro_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    lib.pyro_last_error.restype = ctypes.c_char_p
    lib.pyro_last_error.argtypes = []
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = ctypes.c_int
        fn.argtypes = args
    if lib.pyro_abi_version() != ABI_VERSION:
        raise RuntimeError("libpyro_b200.so ABI version mismatch; rebuild it")
    _lib = lib
    return lib


def check(name: str, code: int) -> int:
    if code < 0:
        msg = _lib.pyro_last_error().decode(errors="replace") if _lib else ""
        raise PyroError(name, code, msg)
    return code


def call(name: str, *args) -> int:
    lib = load()
    return check(name, getattr(lib, name)(*args))
