"""pyro_k_forces_noalloc: the forces kernels with their per-cell scratch in a
fixed device array instead of a cudaMalloc'd buffer.

It exists for callers that may not allocate device memory (a graph capture in
progress elsewhere in the process, a host pool allocator that owns all device
memory, loops that cannot take cudaMalloc's synchronisation).  The test calls
it twice in a row through the C ABI and compares each result with the
allocating entry point, pyro_k_forces, on the same inputs.  It also checks the
size limit, which is rejected before any device work.  The file sorts last so
a stopping run has executed every other test first.
"""
import numpy as np
import pytest

from fields import close, face_valid_mask, params_for, random_state
from gpu_util import dev, host, params_dev, ptr, require_cuda
from pyro_b200 import _abi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    return require_cuda()


def _forces(lib, fn, P, S):
    nx, ny, nz = int(P.nx), int(P.ny), int(P.nz)
    Pd = params_dev(P)
    u, v, w = dev(S["u"]), dev(S["v"]), dev(S["w"])
    rc = getattr(lib, fn)(ptr(Pd), nx, ny, nz, ptr(u), ptr(v), ptr(w), ptr(dev(S["s0"])),
                          ptr(dev(S["s1"])), ptr(dev(S["curl"])), ptr(dev(S["flags"])), None)
    assert rc == 0, lib.pyro_last_error()
    return host(u), host(v), host(w)


def test_noalloc_forces_matches_the_allocating_entry_point_twice(lib):
    # two different grids and states, one after the other: the second call
    # reuses the shared array left holding the first call's values
    for (nx, ny, nz, seed) in [(24, 32, 20, 5), (40, 16, 33, 6)]:
        P = params_for(nx, ny, nz, dt=0.01, wind=2.0, sponge=3.0)
        S = random_state(P, seed=seed)
        ref = _forces(lib, "pyro_k_forces", P, S)
        for _ in range(2):
            got = _forces(lib, "pyro_k_forces_noalloc", P, S)
            for k in range(3):
                m = face_valid_mask(P, k)
                close(got[k][m], ref[k][m], name=f"noalloc vel{k}")


def test_noalloc_forces_rejects_grids_above_the_fixed_scratch(lib):
    n = 128  # 128^3 = 2,097,152 cells > 524,288
    assert n ** 3 > _abi.NOALLOC_MAX_CELLS
    buf = dev(np.zeros(16, np.float32))
    rc = lib.pyro_k_forces_noalloc(ptr(buf), n, n, n, ptr(buf), ptr(buf), ptr(buf), ptr(buf),
                                   ptr(buf), ptr(buf), ptr(buf), None)
    assert rc == _abi.PYRO_E_INVALID
    assert b"exceeds the fixed scratch" in lib.pyro_last_error()
