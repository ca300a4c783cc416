"""The committed roofline record is reproducible: profiles/ncu_traffic.json
(what bench.py reports as roofline.traffic) holds the DRAM bytes of the
committed per-class table in profiles/dram_traffic_pool2cm.md, and its
algorithmic bytes per launch are those of bench.py's byte model for the
2 cm pool (160 x 320 x 160, 4 levels, 4 V-cycles)."""
import json
import os
import re
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402
from pyro_b200 import slab  # noqa: E402

PROFILES = os.path.join(ROOT, "profiles")
LAUNCHES = {"mg_pass_l0": 32, "mg_restrict_l0": 4, "mg_prolong_l0": 4, "mg_pass_mid": 64,
            "mg_restrict_mid": 8, "mg_prolong_mid": 8, "mg_coarse": 4}


def _table():
    rows = {}
    with open(os.path.join(PROFILES, "dram_traffic_pool2cm.md")) as fh:
        for line in fh:
            cells = [c.strip() for c in line.strip().strip("|").split("|")]
            if len(cells) != 10 or not re.match(r"^[a-z_0-9]", cells[0]):
                continue
            try:
                vals = [float(c) for c in cells[1:]]
            except ValueError:
                continue
            rows[cells[0].split(" ")[0]] = vals
    return rows


def test_traffic_json_reproduces_the_committed_table():
    table = _table()
    with open(os.path.join(PROFILES, "ncu_traffic.json")) as fh:
        traffic = json.load(fh)
    assert set(traffic) == set(table), (sorted(traffic), sorted(table))
    for cls, rec in traffic.items():
        rd, wr, total, alg = table[cls][1], table[cls][2], table[cls][3], table[cls][4]
        assert rec["dram_read"] + rec["dram_write"] == rec["dram_bytes_per_launch"]
        assert abs(rec["dram_bytes_per_launch"] / 1e6 - total) <= 0.05 + 0.001 * total, cls
        assert abs(rec["dram_read"] / 1e6 - rd) <= 0.05 + 0.001 * rd, cls
        assert abs(rec["dram_write"] / 1e6 - wr) <= 0.05 + 0.001 * wr, cls
        assert abs(rec["alg_bytes_per_launch"] / 1e6 - alg) <= 0.05 + 0.001 * alg, cls


def test_algorithmic_bytes_are_the_bench_model_for_the_2cm_pool():
    with open(os.path.join(PROFILES, "ncu_traffic.json")) as fh:
        traffic = json.load(fh)
    dims = slab.level_dims((160, 320, 160))
    assert len(dims) == 4
    cells = 160 * 320 * 160
    mg = bench.mg_class_bytes(dims, 4)
    for cls, rec in traffic.items():
        if cls in bench.ALG_BYTES:
            want = bench.ALG_BYTES[cls] * cells
        else:
            want = mg[cls] / LAUNCHES[cls]
        assert rec["alg_bytes_per_launch"] == pytest.approx(want, rel=1e-6), cls
