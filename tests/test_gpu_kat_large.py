"""Known answers at large radii, on the GPU.

1. The M0 instances at r = 4..13 (M0 = 1768248177696000, the 64 smallest eligible primes as base, pool
   below 82178, bound U = the previous 148-digit incumbent, SPLIT = 4000, the driver's per-radius
   bounds): the reference dumpers' records (src/mitm64_idump_stream2.cpp with IDUMP_RANK=1,
   src/mitm64_ddump.cpp) were run by tests/golden/make_golden.py --m0-large and folded into record
   counts and order-independent digests (golden.json "m0_kat_large").  Here the same sides come from
   the drop-ins igen_gpu.generate_chunks and driver.build_D and must give the same counts and digests.
   r = 9 and r = 11 are also the counts INTERVAL_THEOREM.md:66-71 documents.
2. The whole M0 divisor family (gpu/mstar_divisor_family.json, 111 moduli) at every radius its run
   records hold (1..14; gpu/records/M0_U539839443357/, kept in tests/golden/census_M0.json): per
   instance the affordable pool, the D and I record counts after the bounds, the residue pairs and the
   completions below U must equal the reference's lines.
"""
import json
import os

import pytest
import torch

import oracle as O
from carmichael_frontier_b200 import census as C, driver, igen_gpu
from carmichael_frontier_b200.solve import Solver, Tuning

pytestmark = pytest.mark.gpu
GOLD_M0 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "census_M0.json")
MASK = (1 << 64) - 1


def _signed(c):
    return c - (1 << 64) if c >= 1 << 63 else c


def dev_digest_add(acc, keys, ids):
    """oracle.record_digest_add computed on the device (int64 views wrap like uint64)."""
    k = keys.view(torch.int64)
    i = ids.view(torch.int64)
    m = ((k * _signed(O.DIGEST_C1)) ^ i) * _signed(O.DIGEST_C2)
    parts = (int(k.sum()), int(i.sum()), int(m.sum()))
    return tuple((a + b) & MASK for a, b in zip(acc, parts))


@pytest.fixture(scope="module")
def kat(golden):
    return golden["m0_kat_large"]


def _row(kat, r):
    return next(x for x in kat["rows"] if x["r"] == r)


@pytest.mark.parametrize("r", range(4, 14))
def test_m0_insertion_side_matches_reference_dumper(cuda, golden, kat, r):
    rr = _row(kat, r)
    INS = kat["INS_full"][: rr["n_ins"]]
    P0 = O.product(kat["B0"])
    acc, n = (0, 0, 0), 0
    gen = igen_gpu.generate_chunks(INS, r, kat["M"], P0, int(rr["Icap"]), kat["SPLIT"], rr["hmax"],
                                   max_records=1 << 27)
    total = None
    while True:
        try:
            k, i = next(gen)
        except StopIteration as e:
            total = e.value
            break
        acc = dev_digest_add(acc, k, i)
        n += k.numel()
    assert n == total == rr["i_records"]
    assert O.record_digest_hex(acc) == rr["i_digest"]
    documented = golden["m0_kat"]["documented"]           # INTERVAL_THEOREM.md:66-71
    if str(r) in documented:
        assert n == documented[str(r)][1]


@pytest.mark.parametrize("r", range(4, 14))
def test_m0_deletion_side_matches_reference_dumper(cuda, golden, kat, r):
    rr = _row(kat, r)
    chunks, nD = driver.build_D(kat["B0"], kat["M"], r, int(rr["Dmin"]), nchunks=2)
    acc = (0, 0, 0)
    for k, i in chunks:
        acc = dev_digest_add(acc, k, i)
    assert nD == rr["d_records"]
    assert O.record_digest_hex(acc) == rr["d_digest"]
    documented = golden["m0_kat"]["documented"]
    if str(r) in documented:
        assert nD == documented[str(r)][0]


def test_m0_family_all_radii_match_reference_records(cuda):
    with open(GOLD_M0) as f:
        fam = json.load(f)
    U = int(fam["U"])
    out, completions = C.family_run(fam["survivors"], U, solver=Solver(cuda, tuning=Tuning(strategy="bounded")))
    assert completions == []                       # the reference's pass found none below U either
    n, radii = 0, set()
    for row in fam["survivors"]:
        got, ref = out[row["D"]], fam["runs"][str(row["D"])]
        assert (got["base_carmichael"], got["base_below_U"]) == (ref["base_carmichael"], ref["base_below_U"])
        assert got["skipped"] == [], row["D"]
        assert got["instances"] == ref["instances"], row["D"]
        n += len(ref["instances"])
        radii |= {x["r"] for x in ref["instances"]}
    assert n == 684 and radii == set(range(1, 15))
