"""Census producers against the reference's own census output and run records (CPU only).

The divisor-family census of the incumbent of results_k64_best_global.json must give the reference's
118 survivor rows exactly (tests/golden/census_lambdaJ.json, made by make_golden_census.py from
gpu/divisor_family_census.py and gpu/divisor_family_lambdaJ.json), and the driver bounds that the
family runs use (radii at which some h-stratum can beat U, the h bound, the affordable insertion pool)
must reproduce every instance line of the reference's records of that family.
"""
import json
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
