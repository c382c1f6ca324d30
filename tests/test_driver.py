"""Driver integration on the CPU: the instance bounds equal the reference driver's values
recorded with its own dumpers (M0 known-answer rows)."""
from carmichael_frontier_b200 import driver


def test_instance_bounds_match_the_reference_driver(golden):
    kat = golden["m0_kat"]
    for rr in kat["rows"]:
        Icap, Dmin, cap_r, INS = driver.instance_bounds(kat["B0"], kat["INS_full"], rr["r"], int(kat["U"]))
        assert (Icap, Dmin, len(INS)) == (int(rr["Icap"]), int(rr["Dmin"]), rr["n_ins"])
