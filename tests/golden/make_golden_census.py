"""Golden rows of the divisor-family census and of its family runs (run here, where the reference
tree exists).

Run as: CF_REFERENCE_ROOT=<reference tree> python tests/golden/make_golden_census.py

Runs the reference's own census (gpu/divisor_family_census.py, imported from the reference tree) for
the incumbent of results_k64_best_global.json, checks that it reproduces the survivor rows the
reference committed in gpu/divisor_family_lambdaJ.json, and writes them with the incumbent's size and
primes to tests/golden/census_lambdaJ.json.  It also reads the reference's run records of that family
(gpu/records/lambdaN_U524394558743/D<D>.log, one per survivor, written by gpu/run_mstar_family.py
through gpu/mitm_gpu_mstar_driver.py) and keeps, per survivor, the base check and every instance line
(radius, affordable insertion primes, D and I record counts after the bounds, residue pairs,
completions below U).  Finally it runs the reference's lambda-neighbourhood census
(gpu/lambda_neighbourhood.py) for the seed M0 = 1768248177696000 with new primes up to 19 and writes its
rows to tests/golden/nbhd_M0_p19.json.

The second family is the one behind the reference's restricted-minimum theorem: the 111 survivor
divisors of M0 = 1768248177696000 (gpu/mstar_divisor_family.json) searched below the previous
148-digit incumbent, with run records in gpu/records/M0_U539839443357/ -- radii up to 14, among them
M0 itself at r = 7..13 with 2.2e7-3.7e7 D and 6.5e7-7.8e8 I records per radius and 2-78 residue pairs.
Those records are written, with the rows, to tests/golden/census_M0.json.
"""
import glob
import importlib.util
import subprocess
import tempfile
import json
import math
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
import build as obuild  # noqa: E402  oracle/build.py: where the reference tree is

REF = sys.argv[1] if len(sys.argv) > 1 else obuild.REF_SRC
OUT = os.path.join(HERE, "census_lambdaJ.json")
OUT_M0 = os.path.join(HERE, "census_M0.json")


def m0_family():
    """The M0 divisor family's survivor rows and the reference's run records of it."""
    rows = json.load(open(os.path.join(REF, "gpu", "mstar_divisor_family.json")))
    prev = json.load(open(os.path.join(REF, "results_k64_best_global_prev_148_539839443357.json")))
    U = int(prev["n"])
    runs = read_records(os.path.join(REF, "gpu", "records", "M0_U539839443357"), U)
    key = lambda r: r["D"]
    assert sorted(runs) == sorted(str(r["D"]) for r in rows), "records do not cover the survivors"
    json.dump({"U": str(U), "M0": 1768248177696000, "survivors": sorted(rows, key=key), "runs": runs},
              open(OUT_M0, "w"), indent=0)
    n = sum(len(v["instances"]) for v in runs.values())
    print("wrote", OUT_M0, len(rows), "rows", n, "instances")


def main():
    spec = importlib.util.spec_from_file_location("dfc", os.path.join(REF, "gpu", "divisor_family_census.py"))
    dfc = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(dfc)
    inc = json.load(open(os.path.join(REF, "results_k64_best_global.json")))
    committed = json.load(open(os.path.join(REF, "gpu", "divisor_family_lambdaJ.json")))
    U = int(inc["n"])
    F = sorted(int(p) for p in inc["factors"])
    M = math.lcm(*[p - 1 for p in F])
    fm, rows = dfc.census(U, M, F)
    key = lambda r: r["D"]
    assert sorted(rows, key=key) == sorted(committed["survivors"], key=key), "reference census != its output"
    runs = read_records(os.path.join(REF, "gpu", "records", "lambdaN_U524394558743"), U)
    assert sorted(runs) == sorted(str(r["D"]) for r in rows), "records do not cover the survivors"
    json.dump({"U": str(U), "factors": F, "lambda": str(M),
               "lambda_factorization": {str(k): v for k, v in fm.items()},
               "survivors": sorted(rows, key=key), "runs": runs}, open(OUT, "w"), indent=0)
    print("wrote", OUT, len(rows), "rows", sum(len(v["instances"]) for v in runs.values()), "instances")
    with tempfile.TemporaryDirectory() as td:
        nb = os.path.join(td, "nb.json")
        subprocess.run([sys.executable, os.path.join(REF, "gpu", "lambda_neighbourhood.py"), "--seeds",
                        "1768248177696000", "--pmax", "19", "--out", nb, "--procs", "1"], check=True)
        d = json.load(open(nb))
    out2 = os.path.join(os.path.dirname(OUT), "nbhd_M0_p19.json")
    json.dump({"U": d["U"], "seeds": d["seeds"], "pmax": d["pmax"], "sieve_problems": d["sieve_problems"],
               "survivors": d["survivors"]}, open(out2, "w"), indent=0)
    print("wrote", out2, len(d["survivors"]), "rows")


INST = re.compile(r" r=(\d+) h<=(\d+) \|INS\|=(\d+)(?:/(\d+))? (host-exact|dfilter)[^:]*: D ([\d,]+).*?\| I ([\d,]+) "
                  r"rec .*?pairs=(\d+) below_U=(\d+)")
HEAD = re.compile(r"\[runner\] family=(\w+) D=(\d+) U=(\d+) pool=(\d+) cap=(\d+) rmax=(\d+)")
BASE = re.compile(r"\[runner\] r=0 base=ksmall\((\d+) primes, largest (\d+)\) carmichael=(\w+) below_U=(\w+)")


def read_records(folder, U):
    runs = {}
    for f in sorted(glob.glob(os.path.join(folder, "D*.log"))):
        txt = open(f).read()
        assert "INCOMPLETE" not in txt, f
        h, b = HEAD.search(txt), BASE.search(txt)
        assert int(h.group(3)) == U
        inst = []
        for line in txt.splitlines():
            m = INST.search(line)
            if m:
                inst.append({"r": int(m.group(1)), "hmax": int(m.group(2)), "ins": int(m.group(3)),
                             "nD": int(m.group(6).replace(",", "")), "nI": int(m.group(7).replace(",", "")),
                             "pairs": int(m.group(8)), "below_U": int(m.group(9))})
        runs[h.group(2)] = {"pool": int(h.group(4)), "cap": int(h.group(5)), "rmax": int(h.group(6)),
                            "base_largest": int(b.group(2)), "base_carmichael": b.group(3) == "True",
                            "base_below_U": b.group(4) == "True", "instances": inst}
    return runs


if __name__ == "__main__":
    if "--m0-only" in sys.argv:
        sys.argv.remove("--m0-only")
        REF = sys.argv[1] if len(sys.argv) > 1 else obuild.REF_SRC
        m0_family()
    else:
        main()
        m0_family()
