"""The C-ABI library: loads without a GPU, exports every entry point that
include/pyro_sim.h declares, and rejects bad arguments before touching the
device."""
import ctypes
import os
import re
import subprocess

import pytest

from pyro_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\**(pyro_\w+)\s*\(", txt, re.M))
    return names


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_abi.LIB_PATH):
        from pyro_b200.build import build
        build()
    return _abi.load()


def test_header_declares_the_abi():
    names = _declared()
    assert {"pyro_sim_create", "pyro_sim_step", "pyro_sim_read_stats", "pyro_sim_destroy",
            "pyro_voxelize", "pyro_poisson_solve", "pyro_k_react", "pyro_last_error"} <= names


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (pyro_\w+)", out))
    missing = _declared() - exported
    assert not missing, missing
    assert set(_abi.SIGNATURES) <= exported


def test_abi_version_and_struct_sizes(lib):
    assert lib.pyro_abi_version() == _abi.ABI_VERSION
    assert ctypes.sizeof(_abi.PyroParams) == 576
    assert ctypes.sizeof(_abi.PyroShape) == 48


def test_invalid_arguments_fail_before_the_device(lib):
    h = ctypes.c_void_p()
    assert lib.pyro_sim_create(None, None, 4, ctypes.byref(h)) == _abi.PYRO_E_INVALID
    assert b"null" in lib.pyro_last_error()
    p = _abi.PyroParams()
    p.nx, p.ny, p.nz, p.dx = 1, 8, 8, 0.1
    buf = (ctypes.c_float * 4)()
    assert lib.pyro_sim_create(ctypes.byref(p), buf, 4, ctypes.byref(h)) == _abi.PYRO_E_INVALID
    assert b"dimension" in lib.pyro_last_error()
    assert lib.pyro_sim_step(None, 0.01, 0.0, 0.0, 0) == _abi.PYRO_E_INVALID
    assert lib.pyro_k_mg_smooth(1, 1, 1, 0.1, None, None, None, 0, 1.0, None) == \
        _abi.PYRO_E_INVALID
    assert lib.pyro_k_mg_restrict(16, 16, 16, 0.1, buf, buf, buf, 9, 8, 8, buf, buf, buf,
                                  None) == _abi.PYRO_E_INVALID
    assert lib.pyro_k_mg_pass(16, 16, 16, 0.1, buf, buf, buf, 0, 1.0, 0, 2, None) == \
        _abi.PYRO_E_INVALID
    assert b"storage" in lib.pyro_last_error()
    assert lib.pyro_k_mg_pass(16, 16, 16, 0.1, buf, buf, buf, 0, 1.0, 3, 0, None) == \
        _abi.PYRO_E_INVALID
    assert lib.pyro_k_mg_prolong_m(16, 16, 16, buf, buf, buf, 8, 9, 8, buf, 0, None) == \
        _abi.PYRO_E_INVALID
    # the CG preconditioner's pieces: coarse dims, null buffers, modes
    assert lib.pyro_k_mg_restrict_sym(16, 16, 16, 0.1, buf, buf, buf, 8, 8, 9, buf, buf, buf, 0,
                                      0, None) == _abi.PYRO_E_INVALID
    assert b"ceil" in lib.pyro_last_error()
    assert lib.pyro_k_mg_restrict_sym(16, 16, 16, 0.1, buf, buf, buf, 8, 8, 8, buf, buf, buf, 2,
                                      0, None) == _abi.PYRO_E_INVALID
    assert lib.pyro_k_mg_pass_first(16, 16, 16, 0.1, buf, None, buf, buf, 0, 1.0, 0,
                                    _abi.MG_BF16, None) == _abi.PYRO_E_INVALID
    assert b"null" in lib.pyro_last_error()
    assert lib.pyro_k_mg_pass_first(16, 16, 16, 0.1, buf, None, buf, buf, 2, 1.0, 0,
                                    _abi.MG_F32, None) == _abi.PYRO_E_INVALID
    assert lib.pyro_k_mg_pass_last(16, 16, 1, 0.1, buf, buf, buf, buf, 0, 1.0, 0,
                                   None) == _abi.PYRO_E_INVALID
    assert lib.pyro_poisson_create(4, 4, 4, 0.1, 7, ctypes.byref(h)) == _abi.PYRO_E_INVALID
    assert lib.pyro_sim_destroy(None) == _abi.PYRO_OK


def test_python_side_raises_with_the_message(lib):
    with pytest.raises(_abi.PyroError) as e:
        _abi.call("pyro_sim_step", None, 0.01, 0.0, 0.0, 0)
    assert e.value.code == _abi.PYRO_E_INVALID
