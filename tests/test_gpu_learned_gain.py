"""What the trained learned stage (pyro_b200/weights/warmstart.pnet) does on
a pressure system it was not trained on: the 2 cm pool fire at t = 1 s (the
training pairs come from t >= 5 s of the same scene and from the pallet and
bonfire scenes).  The same system is solved to a relative residual of 1e-4
from a zero guess by BF16 MGPCG with and without the learned warm start.

The stage removes most of the initial residual (it is kept, and the
residual after it is below 0.35 of the start), but the CG iterations from
there are not fewer than from zero: the V-cycle preconditioner removes the
same high-frequency error in its first application.  So the learned mode
costs the network's forward pass and saves nothing; the solver keeps it
off by default, and this test pins the measured behaviour, not a gain."""
import json
import os

import numpy as np
import pytest
import torch

from gpu_util import require_cuda
from pyro_b200 import _abi
from pyro_b200.learned import Net
from pyro_b200.poisson import PoissonSolver

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
WEIGHTS = os.path.join(ROOT, "pyro_b200", "weights", "warmstart.pnet")


def test_learned_stage_cuts_the_initial_residual_but_not_the_iterations():
    require_cuda()
    from pyro_b200.pairs import collect
    pair = next(collect(os.path.join(ROOT, "pyro_b200", "scenes", "pool_2cm.toml"), 1, every=1,
                        preroll=1.0, refine_tol=1e-4))
    nz, ny, nx = pair["b"].shape
    b = torch.from_numpy(pair["b"]).cuda()
    f = torch.from_numpy(pair["flags"].astype(np.int32)).cuda()
    net = Net.load(WEIGHTS)
    ps = PoissonSolver((nx, ny, nz), pair["h"], bc_mode=0)
    ps.set_flags(f.data_ptr())
    ps.set_net(net)
    phi = torch.zeros_like(b)
    out = {}
    for mode, tag in ((_abi.SOLVER_MGPCG_BF16, "without"), (_abi.SOLVER_MGPCG_LEARNED, "with")):
        for _ in range(2):      # the second solve is timed warm
            phi.zero_()
            torch.cuda.synchronize()
            info = ps.solve(b.data_ptr(), phi.data_ptr(), mode, 1e-4, 100)
        out[tag] = dict(iterations=info.iterations, ms=round(info.ms, 3),
                        rel_resid=info.rel_resid, learned=info.learned,
                        learned_ms=round(info.learned_ms, 3),
                        resid_after_learned=info.rel_resid_learned)
    print(json.dumps(out))
    w, wo = out["with"], out["without"]
    assert wo["rel_resid"] <= 1e-4 and w["rel_resid"] <= 1e-4
    # the stage is kept and removes most of the initial residual
    assert w["learned"] == 1
    assert w["resid_after_learned"] <= 0.35, w
    # CG from there needs about as many iterations as from zero
    assert abs(w["iterations"] - wo["iterations"]) <= 1, (w, wo)
    ps.set_net(None)
    ps.close()
