"""The mixed-precision pressure solve in the full step: the 8 cm pool fire
run with the reference's FP32 V-cycles and with BF16-preconditioned MGPCG
to 1e-4 (pyro_b200.solver_drift) keeps the time-averaged HRR, burning rate
per area and 50 % cumulative heat-release height within 5 % of each other
(src/main.rs:240-268 summary, averaged over t >= 0.4 t_total)."""
import os

import pytest

from gpu_util import require_cuda
from pyro_b200.scene import Scene
from pyro_b200.solver_drift import compare

pytestmark = pytest.mark.gpu

SCENE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pyro_b200",
                     "scenes", "pool_small_8cm.toml")


def test_bf16_mgpcg_step_keeps_flame_statistics_within_5_percent():
    require_cuda()
    sc = Scene.load(SCENE)
    res = compare(sc, preroll=0.0, duration=6.0, tol=1e-4)
    ref, mix = res["fp32_vcycle"], res["bf16_mgpcg"]
    assert ref["frames_averaged"] == mix["frames_averaged"] > 0
    for k in ("hrr_w", "burning_rate_kg_m2s", "h50_m"):
        assert ref[k] > 0 and abs(res["drift"][k]) <= 0.05, (k, ref[k], mix[k])


def test_learned_warm_start_step_keeps_flame_statistics_within_5_percent():
    """The same with each CG solve started from the committed network's
    warm start (BASELINE's large-scene form: BF16 MGPCG + learned stage)."""
    require_cuda()
    from pyro_b200.learned import Net
    weights = os.path.join(os.path.dirname(SCENE), os.pardir, "weights", "warmstart.pnet")
    sc = Scene.load(SCENE)
    res = compare(sc, preroll=0.0, duration=6.0, tol=1e-4, net=Net.load(weights))
    assert res["learned"]
    ref, mix = res["fp32_vcycle"], res["bf16_mgpcg"]
    assert ref["frames_averaged"] == mix["frames_averaged"] > 0
    for k in ("hrr_w", "burning_rate_kg_m2s", "h50_m"):
        assert ref[k] > 0 and abs(res["drift"][k]) <= 0.05, (k, ref[k], mix[k])
