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


def test_family_run_on_a_modulus_above_2_64(cuda):
    # a census row of 2^64 or more (the reference marks these unsupported) runs through the driver's
    # bounds and the bounded join; each instance's D and I record counts equal the subsets within the
    # bounds, counted here with Python integers
    import itertools
    import math
    from carmichael_frontier_b200 import driver, workloads as W
    M = 36802111876251321600                       # 2^8 * an odd part of 57 bits: 65 bits
    assert M >= 1 << 64
    Q = W.eligible_pool(M, 5518)
    base, INS = Q[:64], Q[64:]
    U = math.prod(base) * 10
    out, completions = C.family_run([{"D": M, "cap": 5518, "rmax": 2}], U, r_max=2,
                                    solver=Solver(cuda, tuning=Tuning(strategy="bounded")))
    rec = out[M]
    assert completions == [] and rec["skipped"] == [] and len(rec["instances"]) >= 1
    for x in rec["instances"]:
        r, h = x["r"], x["hmax"]
        Icap, Dmin, _cap_r, aff = driver.instance_bounds(base, INS, r, U)
        nD = sum(1 for c in itertools.combinations(base, r) if math.prod(c) >= Dmin)
        nI = sum(1 for c in itertools.combinations(aff, r)
                 if math.prod(c) < Icap and sum(p > 4000 for p in c) <= h)
        assert (x["nD"], x["nI"]) == (nD, nI), r
        assert 0 < nD < math.comb(len(base), r) or 0 < nI < math.comb(len(aff), r)


def test_family_run_same_with_any_number_of_join_workers(cuda):
    # the joins run ahead on worker threads and streams; the runs and their order do not change
    with open(GOLD) as f:
        fam = json.load(f)
    U = int(fam["U"])
    rows = fam["survivors"][:12]
    s = Solver(cuda, tuning=Tuning(strategy="bounded"))
    seen = {1: [], 3: []}
    outs = {}
    for w in (1, 3):
        outs[w] = C.family_run(rows, U, r_max=8, solver=s, workers=w,
                               consider=lambda key, fac, label, w=w: seen[w].append(key) or True)
    assert outs[1] == outs[3]
    assert seen[1] == seen[3]
    assert sum(len(v["instances"]) for v in outs[1][0].values()) > 40
