"""The CUDA FP64 step reproduces the oracle's committed golden digests bit
for bit, including the 64^3 parity configuration (Roe + CT, COUR 0.4,
100 steps, one passive scalar)."""
import json
import os
import sys

import pytest

from helpers import gpu_run

HERE = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, HERE)
import make_golden  # noqa: E402

with open(os.path.join(HERE, "oracle_digests.json")) as f:
    GOLD = json.load(f)["cases"]

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", GOLD, ids=[c["name"] for c in GOLD])
def test_fp64_matches_golden_digest(case):
    ic = make_golden.make_ic(case)
    g = gpu_run(ic, tuple(case["n"]), case["riemann"], case["steps"], cour=case["cour"], npass=case["npass"])
    assert [float(x) for x in g["dts"]] == case["dts"]
    assert g["dt_next"] == case["dt_next"]
    assert make_golden.digest(g["q"], g["b"], g["p"]) == case["sha256"]
