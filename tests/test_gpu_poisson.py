"""Stand-alone pressure solver against the CPU oracle: the fixed V-cycle
schedule is bit-exact with the oracle's restatement of src/sim.rs:451-491,
and the tolerance solvers (V-cycles, FP32 MGPCG, BF16 MGPCG) reach their
tolerance with the error against the FP64 solve stated."""
import ctypes

import numpy as np
import pytest

import oracle
from gpu_util import dev, host, ptr, require_cuda
from pyro_b200 import _abi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    return require_cuda()


def _case(nx, ny, nz, seed, solid=0.05):
    """Seeded axis-aligned solid boxes (2-20 cells per edge, up to the solid
    fraction) and an N(0,1) right-hand side with zero fluid mean."""
    rng = np.random.default_rng(seed)
    f = np.zeros((nz, ny, nx), np.uint32)
    while f.mean() < solid:
        e = rng.integers(2, 21, size=3)
        o = [rng.integers(0, max(1, d - e[i])) for i, d in enumerate((nx, ny, nz))]
        f[o[2]:o[2] + e[2], o[1]:o[1] + e[1], o[0]:o[0] + e[0]] = 1
    b = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    b[f == 1] = 0
    b[f == 0] -= b[f == 0].mean()
    return f, b


def _solver(lib, dims, h, f, bc_mode=0):
    ps = ctypes.c_void_p()
    assert lib.pyro_poisson_create(*dims, h, bc_mode, ctypes.byref(ps)) == 0
    fd = dev(f)
    assert lib.pyro_poisson_set_flags(ps, ptr(fd)) == 0
    return ps


@pytest.mark.parametrize("dims,cycles", [((64, 64, 64), 4), ((38, 75, 38), 2),
                                         ((48, 96, 48), 1)])
def test_fixed_vcycles_bit_exact(lib, dims, cycles):
    nx, ny, nz = dims
    f, b = _case(nx, ny, nz, 1)
    h = 0.02
    e = oracle.vcycles(dims, h, np.zeros_like(b), b, f, cycles)
    ps = _solver(lib, dims, h, f)
    bd, pd = dev(b), dev(np.zeros_like(b))
    info = _abi.PyroSolveInfo()
    assert lib.pyro_poisson_solve(ps, ptr(bd), ptr(pd), _abi.SOLVER_VCYCLE, 1e-3, cycles,
                                  ctypes.byref(info)) == 0
    assert np.array_equal(host(pd), e)
    rel = oracle.poisson_relres(dims, h, e, b, f)
    assert abs(info.rel_resid - rel) <= 1e-6 * rel
    lib.pyro_poisson_destroy(ps)


def test_vcycle_to_tolerance_follows_the_reference_cycle(lib):
    """V-cycles until the residual target: the reference V-cycle stalls near
    1e-2 on a solid-laden grid (its README quotes 1e-3..1e-2), so the mode
    reports the cap with the same residual the oracle's cycles reach."""
    dims = (64, 64, 64)
    f, b = _case(*dims, 2)
    h = 0.02
    ps = _solver(lib, dims, h, f)
    bd, pd = dev(b), dev(np.zeros_like(b))
    info = _abi.PyroSolveInfo()
    rc = lib.pyro_poisson_solve(ps, ptr(bd), ptr(pd), _abi.SOLVER_VCYCLE_TOL, 1e-3, 12,
                                ctypes.byref(info))
    e = oracle.vcycles(dims, h, np.zeros_like(b), b, f, info.iterations)
    assert np.array_equal(host(pd), e)
    rel = oracle.poisson_relres(dims, h, e, b, f)
    assert abs(info.rel_resid - rel) <= 1e-3 * rel
    assert rc == (0 if rel <= 1e-3 else _abi.PYRO_E_NOCONV)
    rc = lib.pyro_poisson_solve(ps, ptr(bd), ptr(dev(np.zeros_like(b))), _abi.SOLVER_VCYCLE_TOL,
                                0.05, 12, ctypes.byref(info))
    assert rc == 0 and info.converged == 1 and info.rel_resid <= 0.05
    lib.pyro_poisson_destroy(ps)


@pytest.mark.parametrize("mode,tol", [(_abi.SOLVER_MGPCG, 1e-3), (_abi.SOLVER_MGPCG, 1e-6),
                                      (_abi.SOLVER_MGPCG_BF16, 1e-3),
                                      (_abi.SOLVER_MGPCG_BF16, 1e-6)])
@pytest.mark.parametrize("bc_mode", [0, 1])
def test_tolerance_solvers_vs_fp64(lib, mode, tol, bc_mode):
    dims = (64, 64, 64)
    f, b = _case(*dims, 2)
    h = 0.02
    x64, it, rel64 = oracle.poisson_f64(dims, h, b, f, tol=1e-12, bc_mode=bc_mode)
    ps = _solver(lib, dims, h, f, bc_mode)
    bd, pd = dev(b), dev(np.zeros_like(b))
    info = _abi.PyroSolveInfo()
    rc = lib.pyro_poisson_solve(ps, ptr(bd), ptr(pd), mode, tol, 200, ctypes.byref(info))
    assert rc == 0, lib.pyro_last_error()
    phi = host(pd)
    rel = oracle.poisson_relres(dims, h, phi, b, f, bc_mode)
    assert info.converged == 1 and rel <= tol * 1.05, (info.iterations, rel)
    fl = f == 0
    err = np.abs(phi[fl] - x64[fl]).max() / np.abs(x64[fl]).max()
    # error against the FP64 solve scales with the residual tolerance (the
    # Neumann-sided case is worse conditioned)
    assert err <= (200 if bc_mode == 0 else 2000) * tol, (mode, tol, err)
    lib.pyro_poisson_destroy(ps)


@pytest.mark.parametrize("bc_mode", [0, 1])
def test_coarsest_direct_solve_is_exact(lib, bc_mode):
    """A grid of at most 3072 cells is the preconditioner's coarsest level
    itself, solved by the FP64 inverse: FP32 MGPCG then converges in one or
    two iterations to the limit of FP32 vectors, and the preconditioner
    alone (first iterate) is within FP32 rounding of the FP64 oracle."""
    dims = (12, 16, 12)
    assert dims[0] * dims[1] * dims[2] <= 3072
    f, b = _case(*dims, 5, solid=0.0)
    f[3:6, 0:5, 4:9] = 1  # one solid block on the floor
    b[f == 1] = 0.0
    h = 0.1
    x64, it, rel64 = oracle.poisson_f64(dims, h, b, f, tol=1e-13, bc_mode=bc_mode)
    ps = _solver(lib, dims, h, f, bc_mode)
    bd, pd = dev(b), dev(np.zeros_like(b))
    info = _abi.PyroSolveInfo()
    rc = lib.pyro_poisson_solve(ps, ptr(bd), ptr(pd), _abi.SOLVER_MGPCG, 1e-6, 20,
                                ctypes.byref(info))
    assert rc == 0, lib.pyro_last_error()
    assert info.iterations <= 2, info.iterations
    phi = host(pd)
    fl = f == 0
    err = np.abs(phi[fl] - x64[fl]).max() / np.abs(x64[fl]).max()
    assert err <= 1e-5, err
    lib.pyro_poisson_destroy(ps)


@pytest.mark.parametrize("bc_mode", [0, 1])
def test_bf16_single_level_preconditioner_converges(lib, bc_mode):
    """A grid that is its own coarsest level: the BF16 preconditioner is the
    FP64 direct solve alone, with level 0 converted to BF16 on entry and
    back on exit (no smoothing passes), so CG converges in a few
    iterations to its tolerance, within 2e-3 of the FP64 solution."""
    dims = (12, 16, 12)
    f, b = _case(*dims, 6, solid=0.0)
    f[2:5, 0:4, 3:7] = 1
    b[f == 1] = 0.0
    h = 0.1
    x64, it, rel64 = oracle.poisson_f64(dims, h, b, f, tol=1e-13, bc_mode=bc_mode)
    ps = _solver(lib, dims, h, f, bc_mode)
    bd, pd = dev(b), dev(np.zeros_like(b))
    info = _abi.PyroSolveInfo()
    rc = lib.pyro_poisson_solve(ps, ptr(bd), ptr(pd), _abi.SOLVER_MGPCG_BF16, 1e-6, 30,
                                ctypes.byref(info))
    assert rc == 0, lib.pyro_last_error()
    assert info.converged == 1 and info.iterations <= 10, (info.iterations, info.rel_resid)
    phi = host(pd)
    rel = oracle.poisson_relres(dims, h, phi, b, f, bc_mode)
    # near 1e-7 the residual of an FP32 field is cancellation: the two FP64
    # evaluations agree to a few per cent
    assert rel <= 1.05e-6 and abs(rel - info.rel_resid) <= 0.05 * rel
    fl = f == 0
    err = np.abs(phi[fl] - x64[fl]).max() / np.abs(x64[fl]).max()
    assert err <= 2e-3, err
    lib.pyro_poisson_destroy(ps)


@pytest.mark.parametrize("mode", [_abi.SOLVER_MGPCG, _abi.SOLVER_MGPCG_BF16])
def test_cg_profile_runs_the_solve_iterations(lib, mode):
    """pyro_poisson_profile_cg runs the iterations of a solve one launch at
    a time: k iterations from phi = 0 reach the residual the solve reports
    after k iterations (the same kernels, only the scheduling differs; the
    FP64 sums are in a fixed order), and the step counts per class follow
    the hierarchy (64^3, 32^3, 16^3 smoothed, 8^3 solved directly: per
    iteration 2 x 2 x 2 level-0 passes, 4 x 2 x 2 per coarser level, one
    restriction and prolongation per smoothed level, one direct solve, 5 CG
    vector kernels)."""
    dims = (64, 64, 64)
    f, b = _case(*dims, 3)
    h = 0.02
    ps = _solver(lib, dims, h, f)
    bd = dev(b)
    info = _abi.PyroSolveInfo()
    pd = dev(np.zeros_like(b))
    rc = lib.pyro_poisson_solve(ps, ptr(bd), ptr(pd), mode, 1e-12, 4, ctypes.byref(info))
    assert rc == _abi.PYRO_E_NOCONV and info.iterations == 4
    want = host(pd)
    pp = dev(np.zeros_like(b))
    n = len(_abi.CG_CLASSES)
    ms, cnt = (ctypes.c_float * n)(), (ctypes.c_int * n)()
    assert lib.pyro_poisson_profile_cg(ps, ptr(bd), ptr(pp), mode, 4, ms, cnt, n) == 0, \
        lib.pyro_last_error()
    assert np.array_equal(host(pp), want)
    steps = dict(zip(_abi.CG_CLASSES, list(cnt)))
    nmid = 2  # 32^3 and 16^3
    assert steps["mg_pass_l0"] == 4 * 8
    assert steps["mg_pass_mid"] == 4 * 16 * nmid
    assert steps["mg_restrict_l0"] == 4 and steps["mg_prolong_l0"] == 4
    assert steps["mg_restrict_mid"] == 4 * nmid and steps["mg_prolong_mid"] == 4 * nmid
    assert steps["mg_coarse"] == 4 and steps["cg_vector"] == 4 * 5
    assert all(ms[i] >= 0.0 for i in range(n)) and sum(ms) > 0.0
    lib.pyro_poisson_destroy(ps)


@pytest.mark.parametrize("dims", [(160, 320, 160), (150, 365, 150)])
@pytest.mark.parametrize("mode", [_abi.SOLVER_MGPCG, _abi.SOLVER_MGPCG_BF16])
def test_mgpcg_at_the_2cm_pool_shapes(lib, dims, mode):
    """The preconditioner's deep hierarchy with its FP64 coarsest solve at
    the 2 cm pool's reference rounding and at the exact shape 150x365x150
    (whose levels do not halve evenly; the reference V-cycle needs the
    rounding), to 1e-4 against the float64 residual of the oracle."""
    f, b = _case(*dims, 7)
    h = 0.02
    ps = _solver(lib, dims, h, f, 0)
    bd, pd = dev(b), dev(np.zeros_like(b))
    info = _abi.PyroSolveInfo()
    rc = lib.pyro_poisson_solve(ps, ptr(bd), ptr(pd), mode, 1e-4, 100, ctypes.byref(info))
    assert rc == 0, lib.pyro_last_error()
    # the residual over the fluid connected to a Dirichlet face (sealed
    # pockets, if the boxes make any, are not solved)
    reach = _reachable(f, 0)
    flags_r = np.where(reach, 0, 1).astype(np.uint32)
    b_r = np.where(reach, b, 0.0).astype(np.float32)
    rel = oracle.poisson_relres(dims, h, host(pd), b_r, flags_r, 0)
    assert info.converged == 1 and rel <= 1.05e-4, (info.iterations, rel)
    assert abs(rel - info.rel_resid) <= 1e-3 * rel
    lib.pyro_poisson_destroy(ps)


def _reachable(f, bc_mode):
    """Fluid cells with a 6-connected fluid path to a Dirichlet face (the
    top, and with bc_mode 0 the four sides)."""
    from scipy import ndimage
    lab, n = ndimage.label(f == 0)
    faces = [lab[:, -1, :]]
    if bc_mode == 0:
        faces += [lab[0], lab[-1], lab[:, :, 0], lab[:, :, -1]]
    keep = np.unique(np.concatenate([a.ravel() for a in faces]))
    keep = keep[keep > 0]
    return np.isin(lab, keep)


@pytest.mark.parametrize("mode", [_abi.SOLVER_MGPCG, _abi.SOLVER_MGPCG_BF16])
def test_mgpcg_sealed_pockets(lib, mode):
    """Fluid sealed by solids (no path to a Dirichlet face) makes the system
    singular; the CG modes leave such cells at their initial phi and solve
    the rest (the bonfire's log pile seals a few cells like this)."""
    from pyro_b200.poisson import PoissonSolver, poisson_case
    n = 48
    f, b = poisson_case(n, n, n, seed=11)
    # a hollow solid box (walls 1 cell) enclosing a 4^3 fluid pocket, and a
    # single sealed cell
    f[10:16, 10:16, 10:16] = 1
    f[11:15, 11:15, 11:15] = 0
    f[30:33, 30:33, 30:33] = 1
    f[31, 31, 31] = 0
    b[11:15, 11:15, 11:15] = 3.0          # inconsistent source inside the pocket
    b[31, 31, 31] = -2.0
    ps = PoissonSolver((n, n, n), 0.05, bc_mode=0)
    fd = dev(f.astype(np.int32))
    ps.set_flags(fd.data_ptr())
    bd = dev(b)
    phi0 = np.zeros_like(b)
    phi0[11:15, 11:15, 11:15] = 0.25
    pd = dev(phi0)
    info = ps.solve(bd.data_ptr(), pd.data_ptr(), mode, 1e-6, 100)
    phi = host(pd)
    assert info.converged and np.isfinite(info.rel_resid)
    assert np.all(np.isfinite(phi))
    assert np.all(phi[11:15, 11:15, 11:15] == 0.25) and phi[31, 31, 31] == 0.0
    # the residual over the reachable cells agrees with the float64 oracle
    reach = f == 0
    reach[11:15, 11:15, 11:15] = False
    reach[31, 31, 31] = False
    flags_r = np.where(reach, 0, 1).astype(np.uint32)
    b_r = np.where(reach, b, 0.0).astype(np.float32)
    rel = oracle.poisson_relres((n, n, n), 0.05, phi, b_r, flags_r, bc_mode=0)
    assert rel <= 1.5e-6, rel
    assert abs(rel - info.rel_resid) <= 1e-7
    ps.close()
