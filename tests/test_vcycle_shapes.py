"""Why every workload uses the reference's grid rounding: the reference's
V-cycle (the oracle's restatement of src/sim.rs:451-491, reference
boundaries) diverges on the exact 1 m pool shape at 8 cm, 38 x 75 x 38,
whose levels do not halve evenly (75 -> 38 -> 19: the coarse grids overhang
the domain and the Dirichlet faces move between levels), and converges on
the reference's rounding of the same scene to multiples of 16, 32 x 80 x 32
(src/scene.rs:485-493).  Pure oracle, CPU only."""
import numpy as np

import oracle


def _rel_history(dims, rounds=8, cycles=4, seed=1):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    f = np.zeros((nz, ny, nx), np.uint32)
    b = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    b -= b.mean()
    phi = np.zeros_like(b)
    out = []
    for _ in range(rounds):
        phi = oracle.vcycles(dims, 0.08, phi, b, f, cycles)
        out.append(oracle.poisson_relres(dims, 0.08, phi, b, f))
    return out


def test_rounded_shape_converges():
    r = _rel_history((32, 80, 32))
    assert r[-1] < 1e-6 and r[-1] < r[0] / 1e3, r


def test_exact_shape_diverges():
    assert [l for l in oracle.mg_levels(38, 75, 38)] == [(38, 75, 38), (19, 38, 19),
                                                         (10, 19, 10)]
    r = _rel_history((38, 75, 38))
    # the residual stalls above 1e-3 and then grows cycle after cycle
    assert min(r) > 1e-3, r
    assert r[-1] > 2.0 * min(r), r
