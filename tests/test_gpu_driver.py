"""Driver integration on the GPU: run_instance gives the reference dumpers' record counts,
logs the line the coverage verifier reads, and hands the positive control's hit to consider."""
import re

import pytest

import oracle as O
from carmichael_frontier_b200 import driver

pytestmark = pytest.mark.gpu


def test_run_instance_counts_and_log_line(cuda, golden):
    kat = golden["m0_kat"]
    rr = kat["rows"][0]
    lines, seen = [], []
    st = {}
    ok = driver.run_instance("ksmall", kat["B0"], kat["INS_full"], rr["r"], rr["hmax"], kat["M"], int(kat["U"]),
                             kat["SPLIT"], lambda key, fac, label: seen.append(fac) or False, lines.append, st)
    assert ok and len(lines) == 1
    line = lines[0]
    m = re.search(r"D ([\d,]+) .* I ([\d,]+) rec", line)
    assert (int(m.group(1).replace(",", "")), int(m.group(2).replace(",", ""))) == (rr["d_records"], rr["i_records"])
    # what gpu/verify_family_coverage.py looks for in an instance line
    assert re.search(r" r=(\d+) ", line) and "dfilter" in line and "INCOMPLETE" not in line
    for fac in seen:                      # every completion handed over is below U and == 1 mod M
        n = O.product(fac)
        assert n < int(kat["U"]) and (n - 1) % kat["M"] == 0


def test_run_instance_recovers_positive_control(cuda, golden):
    pc = golden["positive_control"]
    N = int(pc["N"])
    got = []
    driver.run_instance("ksmall", pc["B0"], pc["INS"], pc["r"], pc["r"], pc["M"], N + 1, max(pc["INS"]),
                        lambda key, fac, label: got.append(O.product(fac)) or True, lambda s: None)
    assert N in got


def test_build_D_is_the_sorted_ddump_side(cuda, golden):
    kat = golden["m0_kat"]
    rr = kat["rows"][0]
    chunks, nD = driver.build_D(kat["B0"], kat["M"], rr["r"], int(rr["Dmin"]), nchunks=3)
    assert nD == rr["d_records"] and len(chunks) == 3
    import hashlib
    import numpy as np
    keys = np.concatenate([k.cpu().numpy().view(np.uint64) for k, _ in chunks])
    for k, _ in chunks:
        kk = k.cpu().numpy().view(np.uint64)
        assert (kk[1:] >= kk[:-1]).all()
    assert hashlib.sha256(np.sort(keys).astype("<u8").tobytes()).hexdigest()[:32] == rr["d_key_digest"]
