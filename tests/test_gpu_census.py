"""Family runs of the divisor-family census on the GPU against the reference's run records.

Every survivor of the incumbent's family is run as gpu/run_mstar_family.py runs it (base check, then
each radius through the driver's bounds and the bounded GPU join); per instance, the D and I record
counts after the bounds, the residue pairs and the completions below U must equal the reference's
record lines (tests/golden/census_lambdaJ.json), radii 1..6 here.
"""
import json
import os

import pytest

from carmichael_frontier_b200 import census as C
from carmichael_frontier_b200.solve import Solver, Tuning

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "census_lambdaJ.json")


def test_family_run_matches_reference_records(cuda):
    with open(GOLD) as f:
        fam = json.load(f)
    U = int(fam["U"])
    out, completions = C.family_run(fam["survivors"], U, r_max=6,
                                    solver=Solver(cuda, tuning=Tuning(strategy="bounded")))
    assert completions == []                                # the reference found none below U either
    n = 0
    for row in fam["survivors"]:
        got, ref = out[row["D"]], fam["runs"][str(row["D"])]
        assert (got["base_carmichael"], got["base_below_U"]) == (ref["base_carmichael"], ref["base_below_U"])
        want = [x for x in ref["instances"] if x["r"] <= 6]
        assert got["skipped"] == []
        assert got["instances"] == want, row["D"]
        n += len(want)
    assert n > 500
