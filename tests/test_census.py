"""Census producers against the reference's own census output and run records (CPU only).

The divisor-family census of the incumbent of results_k64_best_global.json must give the reference's
118 survivor rows exactly (tests/golden/census_lambdaJ.json, made by make_golden_census.py from
gpu/divisor_family_census.py and gpu/divisor_family_lambdaJ.json), and the driver bounds that the
family runs use (radii at which some h-stratum can beat U, the h bound, the affordable insertion pool)
must reproduce every instance line of the reference's records of that family.  The lambda-neighbourhood
census (new moduli one step from a seed) must give the reference's rows for the seed M0 and new primes up
to 19 (tests/golden/nbhd_M0_p19.json, from gpu/lambda_neighbourhood.py).
"""
import json
import math
import os

import pytest

from carmichael_frontier_b200 import census as C
from carmichael_frontier_b200 import driver, workloads as W

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "census_lambdaJ.json")


@pytest.fixture(scope="module")
def fam():
    with open(GOLD) as f:
        return json.load(f)


def test_divisor_family_matches_reference_census(fam):
    fm, rows = C.divisor_family(int(fam["U"]), fam["factors"])
    assert C.carmichael_lambda(fam["factors"]) == int(fam["lambda"])
    assert {str(k): v for k, v in fm.items()} == fam["lambda_factorization"]
    assert rows == fam["survivors"]


def test_pools_agree_with_eligible_pool():
    for D in (21621600, 1014485472000, 155016423578016000):
        lat = C.DivisorLattice(D)
        assert lat.pool(C._top_index(D)) == W.eligible_pool(D, cap=C.SIEVE_BOUND)
    assert C.factorize(2 ** 8 * 3 ** 4 * 263) == {2: 8, 3: 4, 263: 1}


def test_driver_bounds_reproduce_every_reference_instance_line(fam):
    U = int(fam["U"])
    n = 0
    for row in fam["survivors"]:
        D, cap = row["D"], row["cap"]
        Pc = [q for q in C.DivisorLattice(D).pool(C._top_index(D)) if q <= cap]
        assert len(Pc) == row["pool_capped"] == fam["runs"][str(D)]["pool"]
        base, INS = Pc[:64], Pc[64:]
        assert base[-1] == fam["runs"][str(D)]["base_largest"]
        lines = fam["runs"][str(D)]["instances"]
        radii = [r for r in range(1, row["rmax"] + 1) if driver.hmax_for(base, INS, r, U) >= 0]
        assert radii == [x["r"] for x in lines]
        for x in lines:
            assert driver.hmax_for(base, INS, x["r"], U) == x["hmax"]
            assert len(driver.instance_bounds(base, INS, x["r"], U)[3]) == x["ins"]
            n += 1
    assert n == 728


def test_family_instances_cover_the_survivors(fam):
    rows = fam["survivors"][:6]
    items = C.family_instances(rows, int(fam["U"]), r_max=3)
    assert {it[0]["D"] for it in items} == {r["D"] for r in rows}
    for row, r, x in items:
        assert x.M == row["D"] and len(x.B0) == 64 and len(x.B0) + len(x.INS) == row["pool_capped"]
        assert x.B == int(fam["U"]) - 1 and 0 <= r <= min(3, row["rmax"])
    with pytest.raises(ValueError):
        C.census_row(30, [7, 11, 31], 10 ** 400, [], k=64)      # too few primes and a completion below U


def test_lambda_neighbourhood_matches_reference_census(fam):
    # new moduli one step from M0 (new primes up to 19): the reference's rows, order and provenance
    with open(os.path.join(os.path.dirname(GOLD), "nbhd_M0_p19.json")) as f:
        ref = json.load(f)
    U = int(fam["U"])
    assert int(ref["U"]) == U
    rows, problems = C.lambda_neighbourhood([int(x) for x in ref["seeds"]], ref["pmax"], U, fam["factors"])
    assert problems == [] and ref["sieve_problems"] == []
    assert rows == ref["survivors"]


def test_two_witness_min_small_cases():
    # a pool of 64 primes: the cheapest product holding both witnesses, or None without them
    P = [q for q in range(3, 2000) if all(q % d for d in range(2, int(q ** 0.5) + 1))][:70]
    assert C.two_witness_min(P, 10 ** 300, M0=math.prod(q - 1 for q in P), LN=1) is None
    w = C.two_witness_min(P, 10 ** 300, M0=1, LN=1)
    assert w == math.prod(P[:64])
