"""Generate the golden fixtures in tests/golden/ from the REFERENCE itself.

Runs only where the reference tree is present ($CF_REFERENCE_ROOT, else
oracle/build.py's default); the fixtures it writes are committed so that tests run
without it.  Sources of truth, all the reference's own code:

  * gen_records: the CUDA kernel source string in gpu/mitm_gpu2.py:24-66,
    compiled UNCHANGED as host C++ behind a small shim (__global__ and thread
    indices defined away) and run over every thread index -> digests of the
    keys/ids arrays for small pools, radii and rank ranges.
  * src/mitm64.cpp, src/mitm.cpp, src/mitm64_idump_stream2.cpp and
    src/mitm64_ddump.cpp built from source (oracle/build.py) and run on the
    benchmark instances -> match sets, record counts, record digests.
  * The positive control of gpu/validate_mitm_gpu2_pos.py (M0, ksmall base,
    r = 7, the previous 148-digit incumbent's insertions) re-run with the
    reference dumpers and a numpy join.
  * Known-answer record counts at M0 documented in INTERVAL_THEOREM.md:66-70
    (r = 4, 5, 6 re-counted here with the reference dumpers).
  * The same M0 instances at every radius the reference's GPU driver path takes
    (r = 4..13, the counts its record log gpu/records/M0_U539839443357/
    D1768248177696000.log shows), re-run with the reference dumpers; the
    records are streamed through an order-independent digest
    (oracle.record_digest_add) because they reach 7.8e8 per side.
  * The large-radius instance (pool 160, r = 7) cut to a product-bounded
    sub-instance of 6.2e8 D and about 2e8 I records, joined from the reference
    dumpers' records in numpy (config4_bounded).

  * Whole moduli of the seeded portfolio (config3_pins): every D against every I
    subset through the reference's mitm64.

Usage: CF_REFERENCE_ROOT=<reference tree> python tests/golden/make_golden.py [--quick | --m0-large | --config4 | --config3]
(the reference tree defaults to oracle/build.py's REF_SRC).
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import math
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import build as obuild  # noqa: E402  oracle/build.py

REF = obuild.REF_SRC
from carmichael_frontier_b200 import workloads as W  # noqa: E402

OUT = os.path.join(HERE, "golden.json")


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()[:32]


# --------------------------------------------------------------------------
def build_gen_records_shim() -> C.CDLL:
    src = open(os.path.join(REF, "gpu", "mitm_gpu2.py")).read()
    m = re.search(r'_GEN_SRC = r"""(.*?)"""', src, re.S)
    kernel = m.group(1)
    shim = r"""
#include <cstdint>
struct cf_dim3 { unsigned x, y, z; };
static cf_dim3 blockIdx, blockDim, threadIdx;
#define __global__
#define __restrict__
""" + kernel + r"""
extern "C" void run_gen_records(const unsigned long long* primes, const unsigned long long* binom, int n, int R,
    int bits, unsigned long long M, unsigned long long mult, unsigned long long lo, unsigned long long count,
    unsigned long long* keys, unsigned long long* ids) {
  blockDim.x = 256; blockDim.y = blockDim.z = 1;
  unsigned long long blocks = (count + 255) / 256;
  for (unsigned long long b = 0; b < blocks; ++b)
    for (unsigned t = 0; t < 256; ++t) {
      blockIdx.x = (unsigned)b; threadIdx.x = t;
      gen_records(primes, binom, n, R, bits, M, mult, lo, count, keys, ids);
    }
}
"""
    d = tempfile.mkdtemp()
    cpp = os.path.join(d, "gen_shim.cpp")
    so = os.path.join(d, "gen_shim.so")
    open(cpp, "w").write(shim)
    subprocess.run(["g++", "-O2", "-w", "-fPIC", "-shared", cpp, "-o", so], check=True)
    L = C.CDLL(so)
    L.run_gen_records.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                  C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p]
    return L


def ref_gen_records(L, primes, r, M, mult, bits, lo=0, hi=None):
    n = len(primes)
    B = np.zeros((n + 1, r + 1), dtype=np.uint64)
    B[:, 0] = 1
    for a in range(1, n + 1):
        for b in range(1, min(a, r) + 1):
            B[a, b] = B[a - 1, b - 1] + B[a - 1, b]
    total = math.comb(n, r)
    hi = total if hi is None else hi
    cnt = hi - lo
    keys = np.zeros(cnt, dtype=np.uint64)
    ids = np.zeros(cnt, dtype=np.uint64)
    p = np.asarray(primes, dtype=np.uint64)
    Bf = np.ascontiguousarray(B.reshape(-1))
    L.run_gen_records(p.ctypes.data, Bf.ctypes.data, n, r, bits, M, mult % M, lo, cnt, keys.ctypes.data,
                      ids.ctypes.data)
    return keys, ids


def gen_cases():
    """Small gen_records cases: (name, primes, r, M, mult, bits, lo, hi)."""
    c1 = W.config1()
    w2 = W.config2(1)
    P0_1 = W.product(c1.B0)
    P0_2 = W.product(w2.B0)
    ins2 = list(w2.INS)
    cases = [
        ("cfg1_D_r2_b6", list(c1.B0), 2, c1.M, 1, 6, 0, None),
        ("cfg1_I_r2_b8", list(c1.INS), 2, c1.M, P0_1 % c1.M, 8, 0, None),
        ("cfg1_I_r3_b8_chunk", list(c1.INS), 3, c1.M, P0_1 % c1.M, 8, 1000, 250_000),
        ("cfg2s1_D_r3_b6", list(w2.B0), 3, w2.M, 1, 6, 0, None),
        ("cfg2s1_D_r5_b6_chunk", list(w2.B0), 5, w2.M, 1, 6, 3_000_000, 3_200_000),
        ("cfg2s1_I_r4_b8_chunk", ins2, 4, w2.M, P0_2 % w2.M, 8, 10_000_000, 10_150_000),
        ("cfg2s1_I_r1_b8", ins2, 1, w2.M, P0_2 % w2.M, 8, 0, None),
        ("cfg2s1_D_r8_b6_chunk", list(w2.B0), 8, w2.M, 1, 6, 4_000_000_000, 4_000_050_000),
        ("cfg2s1_D_r10_b6_chunk", list(w2.B0), 10, w2.M, 12345, 6, 10 ** 11, 10 ** 11 + 20_000),
        ("odd_modulus_r3", [3, 5, 7, 11, 13, 17, 19, 23, 29, 31], 3, 3 * 5 * 7 * 11 * 13 * 9 + 2, 7, 10, 0, None),
        ("power_of_two_r4", [3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41], 4, 1 << 40, 1, 10, 0, None),
    ]
    return cases


# --------------------------------------------------------------------------
def mitm64_case(w, threads=8, timeout=600):
    """Unpruned join (Icap = product of the r largest insertions + 1) with the reference's mitm64."""
    import oracle as O
    P0 = W.product(w.B0)
    ins = list(w.INS)
    Icap = W.product(ins[-w.r:]) + 1
    matches, err = O.run_ref_mitm64(w.M, list(w.B0), ins, w.r, P0, Icap, 1, threads, timeout=timeout)
    m = re.search(r"D_leaves=(\d+) Dres=(\d+).*I_leaves=(\d+) matches=(\d+)", err)
    d_leaves, d_res, i_leaves, nmatch = (int(x) for x in m.groups())
    hits = []
    for D, I in matches:
        S = sorted((set(w.B0) - set(D)) | set(I))
        n = W.product(S)
        if n <= w.B:
            hits.append([list(D), list(I), str(n)])
    return dict(name=w.name, M=w.M, r=w.r, B=str(w.B), Q=list(w.Q), B0=list(w.B0),
                d_leaves=d_leaves, d_res=d_res, i_leaves=i_leaves, matches=nmatch,
                pairs=sorted([list(D), list(I)] for D, I in matches), hits=sorted(hits))


def positive_control():
    """gpu/validate_mitm_gpu2_pos.py: M0, ksmall base from primes < 4000, r = 7, 30 insertions incl. N's."""
    inc = json.load(open(os.path.join(REF, "results_k64_best_global_prev_148_N.json")))
    M = int(inc["modulus"])
    N = int(inc["n"])
    Nf = sorted(int(p) for p in inc["factors"])
    P = W.eligible_pool(M, 3999)
    B0 = sorted(P)[:64]
    bset = set(B0)
    D_need = sorted(bset - set(Nf))
    I_need = sorted(set(Nf) - bset)
    R = len(D_need)
    INS = sorted(I_need + [p for p in P if p not in bset and p not in set(I_need)][:30 - R])
    P0 = W.product(B0)
    # reference dumpers: I side unpruned-by-product (Icap = N-bound as the validator), D side Dmin-filtered
    topI = W.product(sorted(INS)[-R:])
    ptb = W.product(B0[-R:])
    Icap = max(1, min(topI, (N * ptb) // P0 + 1))
    idump = os.path.join(ROOT, "oracle", "_ref", "mitm64_idump_stream2")
    ddump = os.path.join(ROOT, "oracle", "_ref", "mitm64_ddump")
    pr = subprocess.run([idump], input=f"{M} {R} {P0 % M} {Icap} 1 8 0\n64 {' '.join(map(str, B0))}\n"
                        f"{len(INS)} {' '.join(map(str, INS))}\n".encode(), capture_output=True,
                        env=dict(os.environ, IDUMP_RANK="1"), check=True)
    I = np.frombuffer(pr.stdout, dtype=np.uint64).reshape(-1, 2)
    Imin = W.product(INS[:R])
    Dmin = P0 * Imin // N
    pr = subprocess.run([ddump], input=f"{M} {R} {Dmin}\n64 {' '.join(map(str, B0))}\n".encode(),
                        capture_output=True, check=True)
    D = np.frombuffer(pr.stdout, dtype=np.uint64).reshape(-1, 2)
    Ik = np.unique(I[:, 0])
    found = []
    for dk, did in D[np.isin(D[:, 0], Ik)]:
        d = [B0[(int(did) >> (6 * q)) & 63] for q in range(R)]
        for ik, iid in I[I[:, 0] == dk]:
            # colex rank -> indices
            v = int(iid)
            idx = []
            x = len(INS) - 1
            for j in range(R - 1, -1, -1):
                while math.comb(x, j + 1) > v:
                    x -= 1
                idx.append(x)
                v -= math.comb(x, j + 1)
                x -= 1
            ii = [INS[x] for x in reversed(idx)]
            S = sorted((bset - set(d)) | set(ii))
            found.append([sorted(d), sorted(ii), str(W.product(S))])
    return dict(M=M, N=str(N), r=R, B0=B0, INS=INS, D_need=D_need, I_need=I_need, Icap=str(Icap),
                Dmin=str(Dmin), i_records=int(I.shape[0]), d_records=int(D.shape[0]), pairs=sorted(found))


def m0_kat(radii=(4, 5, 6)):
    """Known-answer record counts at M0 (INTERVAL_THEOREM.md:66-70), driver formulas
    gpu/mitm_gpu_mstar_driver.py:194-203, recounted with the reference dumpers."""
    M = 1768248177696000
    U = int(json.load(open(os.path.join(REF, "results_k64_best_global_prev_148_539839443357.json")))["n"])
    SPLIT = 4000
    P = W.eligible_pool(M, 82177)
    B0 = sorted(P)[:64]
    INSf = sorted(p for p in P if p not in set(B0))[:1024]
    P0 = W.product(B0)
    rows = []
    idump = os.path.join(ROOT, "oracle", "_ref", "mitm64_idump_stream2")
    ddump = os.path.join(ROOT, "oracle", "_ref", "mitm64_ddump")
    for r in radii:
        INS = INSf
        small = [p for p in INS if p <= SPLIT]
        large = [p for p in INS if p > SPLIT]
        Dmax = W.product(B0[-r:])
        hmax = -1
        for h in range(r + 1):
            if h > len(large) or r - h > len(small):
                continue
            if P0 * W.product(small[:r - h]) * W.product(large[:h]) < U * Dmax:
                hmax = h
        topI = W.product(INS[-r:])
        ptb = W.product(B0[-r:])
        Icap = max(1, min(topI + 1, (U * ptb) // P0 + 1))
        Imin = W.product(INS[:r])
        Dmin = (P0 * Imin) // U + 1
        cap_r = (Icap - 1) // W.product(INS[:r - 1])
        INS = [q for q in INS if q <= cap_r]
        split_idx = next((i for i, p in enumerate(INS) if p > SPLIT), len(INS))
        pi = subprocess.run([idump], input=f"{M} {r} {P0 % M} {Icap} 1 8 0\n64 {' '.join(map(str, B0))}\n"
                            f"{len(INS)} {' '.join(map(str, INS))}\n".encode(), capture_output=True,
                            env=dict(os.environ, IDUMP_RANK="1", IDUMP_SPLIT=str(SPLIT), IDUMP_HMAX=str(hmax)),
                            check=True)
        pd = subprocess.run([ddump], input=f"{M} {r} {Dmin}\n64 {' '.join(map(str, B0))}\n".encode(),
                            capture_output=True, check=True)
        tot = lambda p: int([l for l in p.stderr.decode().splitlines() if l.startswith("TOTAL")][0].split()[1])
        Iarr = np.frombuffer(pi.stdout, dtype=np.uint64).reshape(-1, 2)
        Darr = np.frombuffer(pd.stdout, dtype=np.uint64).reshape(-1, 2)
        rows.append(dict(r=r, hmax=hmax, n_ins=len(INS), split_idx=split_idx, Icap=str(Icap), Dmin=str(Dmin),
                         i_records=tot(pi), d_records=tot(pd),
                         i_id_digest=digest(np.sort(Iarr[:, 1])), i_key_digest=digest(Iarr[np.argsort(Iarr[:, 1]), 0]),
                         d_key_digest=digest(np.sort(Darr[:, 0]))))
    return dict(M=M, U=str(U), SPLIT=SPLIT, pool_cap=82177, B0=B0, INS_full=INSf, rows=rows,
                documented={"4": [333461, 8722393], "5": [2082166, 57156188], "6": [8340300, 228944388],
                            "9": [36755836, 652881611], "11": [6955830, 64758042]})


def m0_bounds(r, M, U, B0, INSf, SPLIT):
    """The driver's per-instance bounds (gpu/mitm_gpu_mstar_driver.py:84-98,188-205) at radius r:
    (hmax, Icap exclusive, Dmin, affordable INS)."""
    P0 = W.product(B0)
    small = [p for p in INSf if p <= SPLIT]
    large = [p for p in INSf if p > SPLIT]
    Dmax = W.product(B0[-r:])
    hmax = -1
    for h in range(r + 1):
        if h > len(large) or r - h > len(small):
            continue
        if P0 * W.product(small[:r - h]) * W.product(large[:h]) < U * Dmax:
            hmax = h
    topI = W.product(INSf[-r:])
    Icap = max(1, min(topI + 1, (U * Dmax) // P0 + 1))
    Dmin = (P0 * W.product(INSf[:r])) // U + 1
    cap_r = (Icap - 1) // W.product(INSf[:r - 1])
    return hmax, Icap, Dmin, [q for q in INSf if q <= cap_r]


def stream_records(cmd, stdin: bytes, env=None, block=1 << 26):
    """Run a reference dumper; fold its 16-byte stdout records into the order-independent digest.
    Returns (records read, digest hex, TOTAL from stderr, exit code)."""
    import oracle as O
    with tempfile.TemporaryFile() as err:
        p = subprocess.Popen([cmd], stdin=subprocess.PIPE, stdout=subprocess.PIPE, stderr=err, env=env)
        p.stdin.write(stdin)
        p.stdin.close()
        acc, n, tail = (0, 0, 0), 0, b""
        while True:
            buf = p.stdout.read(block)
            if not buf:
                break
            buf = tail + buf
            cut = len(buf) - len(buf) % 16
            tail = buf[cut:]
            a = np.frombuffer(buf[:cut], dtype="<u8").reshape(-1, 2)
            acc = O.record_digest_add(acc, a[:, 0], a[:, 1])
            n += a.shape[0]
        rc = p.wait()
        err.seek(0)
        lines = err.read().decode().splitlines()
    assert not tail
    tot = int([l for l in lines if l.startswith("TOTAL")][0].split()[1])
    return n, O.record_digest_hex(acc), tot, rc


def m0_kat_large(radii=range(4, 14), threads=8):
    """M0 known-answer rows at radii 4..13 through the reference dumpers: counts and digests."""
    M = 1768248177696000
    U = int(json.load(open(os.path.join(REF, "results_k64_best_global_prev_148_539839443357.json")))["n"])
    SPLIT = 4000
    P = W.eligible_pool(M, 82177)
    B0 = sorted(P)[:64]
    INSf = sorted(p for p in P if p not in set(B0))
    P0 = W.product(B0)
    idump = os.path.join(ROOT, "oracle", "_ref", "mitm64_idump_stream2")
    ddump = os.path.join(ROOT, "oracle", "_ref", "mitm64_ddump")
    rows = []
    for r in radii:
        hmax, Icap, Dmin, INS = m0_bounds(r, M, U, B0, INSf, SPLIT)
        assert Icap - 1 < 1 << 128 and hmax >= 0
        ni, di, ti, rci = stream_records(idump, f"{M} {r} {P0 % M} {Icap} 1 {threads} 0\n64 {' '.join(map(str, B0))}\n"
                                         f"{len(INS)} {' '.join(map(str, INS))}\n".encode(),
                                         env=dict(os.environ, IDUMP_RANK="1", IDUMP_SPLIT=str(SPLIT),
                                                  IDUMP_HMAX=str(hmax)))
        nd, dd, td, rcd = stream_records(ddump, f"{M} {r} {Dmin}\n64 {' '.join(map(str, B0))}\n".encode())
        assert rci == 0 and rcd == 0 and ni == ti and nd == td
        rows.append(dict(r=r, hmax=hmax, n_ins=len(INS), Icap=str(Icap), Dmin=str(Dmin), i_records=ni,
                         d_records=nd, i_digest=di, d_digest=dd,
                         d_ids="mask" if r > 10 else "6-bit"))
        print("m0 large", r, nd, ni, flush=True)
    return dict(M=M, U=str(U), SPLIT=SPLIT, pool_cap=82177, B0=B0, INS_full=INSf, rows=rows,
                digest="oracle.record_digest_add (sums mod 2^64 of key, id, ((key*C1)^id)*C2)")


def unrank_colex_py(v, r, n):
    """Colex rank -> ascending index tuple (gpu/mitm_gpu_mstar_driver.py:120-126)."""
    v, idx, x = int(v), [], n - 1
    for j in range(r - 1, -1, -1):
        while math.comb(x, j + 1) > v:
            x -= 1
        idx.append(x)
        v -= math.comb(x, j + 1)
        x -= 1
    return tuple(reversed(idx))


def config4_bounded(target_i=200_000_000, threads=8):
    """The large-radius instance (seed-0 modulus, pool of 160 primes, r = 7) cut to a product-bounded
    sub-instance the reference's dumpers and a sorted join finish in minutes: every D (Dmin = 0, all
    C(64, 7) = 6.2e8 records) against the I subsets with prod(I) < Icap, Icap chosen for about 2e8 I
    records.  Reference: src/mitm64_ddump.cpp + src/mitm64_idump_stream2.cpp (IDUMP_RANK=1) and an
    equal-key join in numpy, the method of gpu/validate_mitm_gpu2_pos.py:23-33."""
    import oracle as O
    w = W.config4(0)
    M, r, B0, INS = w.M, w.r, list(w.B0), list(w.INS)
    P0 = W.product(B0)
    # grow the cap from the smallest product by factors of 1.5 while the exact count (which costs
    # time in proportion to itself) stays below target_i, then bisect to the smallest cap, within
    # 0.1%, that admits at least target_i records
    lo = W.product(INS[:r])
    hi = lo * 3 // 2
    while O.idump_count(INS, r, M, P0, hi) < target_i:
        lo, hi = hi, hi * 3 // 2
    while hi - lo > max(1, lo // 1000):
        mid = (lo + hi) // 2
        if O.idump_count(INS, r, M, P0, mid) >= target_i:
            hi = mid
        else:
            lo = mid
    Icap = hi
    idump = os.path.join(ROOT, "oracle", "_ref", "mitm64_idump_stream2")
    ddump = os.path.join(ROOT, "oracle", "_ref", "mitm64_ddump")
    pi = subprocess.run([idump], input=f"{M} {r} {P0 % M} {Icap} 1 {threads} 0\n64 {' '.join(map(str, B0))}\n"
                        f"{len(INS)} {' '.join(map(str, INS))}\n".encode(), capture_output=True,
                        env=dict(os.environ, IDUMP_RANK="1"), check=True)
    I = np.frombuffer(pi.stdout, dtype=np.uint64).reshape(-1, 2)
    i_dig = O.record_digest_hex(O.record_digest_add((0, 0, 0), I[:, 0], I[:, 1]))
    order = np.argsort(I[:, 0], kind="stable")
    Ik, Iid = I[order, 0].copy(), I[order, 1].copy()
    del I, order, pi
    pd = subprocess.Popen([ddump], stdin=subprocess.PIPE, stdout=subprocess.PIPE)
    pd.stdin.write(f"{M} {r} 0\n64 {' '.join(map(str, B0))}\n".encode())
    pd.stdin.close()
    acc, nd, pairs = (0, 0, 0), 0, []
    while True:
        buf = pd.stdout.read(1 << 28)
        if not buf:
            break
        D = np.frombuffer(buf, dtype=np.uint64).reshape(-1, 2)
        acc = O.record_digest_add(acc, D[:, 0], D[:, 1])
        nd += D.shape[0]
        od = np.argsort(D[:, 0], kind="stable")       # sorted queries: each search starts where the last ended
        ks = D[od, 0]
        a = np.searchsorted(Ik, ks, side="left")
        hit = a < len(Ik)
        hit[hit] = Ik[a[hit]] == ks[hit]
        for jj in np.nonzero(hit)[0]:
            j = od[jj]
            b = np.searchsorted(Ik, ks[jj], side="right")
            a_j = a[jj]
            dd = sorted(B0[(int(D[j, 1]) >> (6 * q)) & 63] for q in range(r))
            for t in range(a_j, b):
                ii = [INS[x] for x in unrank_colex_py(Iid[t], r, len(INS))]
                pairs.append([dd, ii])
    assert pd.wait() == 0
    return dict(name=w.name, M=M, r=r, B0=B0, INS=INS, Icap=str(Icap), Dmin="0", i_records=int(len(Ik)),
                d_records=nd, i_digest=i_dig, d_digest=O.record_digest_hex(acc), pairs=sorted(pairs))


CONFIG3_PINS = (0, 2, 3, 5, 13, 14)      # seeded portfolio moduli whose whole join the reference finishes in seconds


def config3_pins():
    """Whole moduli of the seeded 1024-modulus portfolio (radii 4, 5 and 6, pools of 121-272 primes), every
    D against every I subset, joined by the reference's mitm64."""
    ws = W.config3(1024)
    out = []
    for k in CONFIG3_PINS:
        row = mitm64_case(ws[k], timeout=1800)
        row["index"] = k
        out.append(row)
        print("config3", k, ws[k].r, row["d_leaves"], row["i_leaves"], row["matches"], row["d_res"], flush=True)
    return out


def main():
    if "--config3" in sys.argv:
        obuild.build_oracle()
        obuild.build_reference()
        gold = json.load(open(OUT))
        gold["config3_pins"] = config3_pins()
        json.dump(gold, open(OUT, "w"), indent=0)
        print("wrote", OUT)
        return
    if "--config4" in sys.argv:
        obuild.build_oracle()
        obuild.build_reference()
        gold = json.load(open(OUT))
        gold["config4_bounded"] = config4_bounded()
        json.dump(gold, open(OUT, "w"), indent=0)
        print("wrote", OUT, gold["config4_bounded"]["i_records"], len(gold["config4_bounded"]["pairs"]))
        return
    if "--m0-large" in sys.argv:
        obuild.build_reference()
        gold = json.load(open(OUT))
        gold["m0_kat_large"] = m0_kat_large()
        json.dump(gold, open(OUT, "w"), indent=0)
        print("wrote", OUT)
        return
    quick = "--quick" in sys.argv
    obuild.build_oracle()
    obuild.build_reference()
    L = build_gen_records_shim()
    gold = {"generated_by": "tests/golden/make_golden.py", "gen_records": []}
    for name, primes, r, M, mult, bits, lo, hi in gen_cases():
        k, i = ref_gen_records(L, primes, r, M, mult, bits, lo, hi)
        gold["gen_records"].append(dict(name=name, primes=[int(p) for p in primes], r=r, M=M, mult=int(mult), bits=bits,
                                        lo=lo, hi=hi if hi is not None else math.comb(len(primes), r),
                                        key_digest=digest(k), id_digest=digest(i),
                                        head_keys=[int(x) for x in k[:4]], head_ids=[int(x) for x in i[:4]]))
        print(name, len(k))
    c1 = W.config1()
    gold["config1"] = mitm64_case(c1)
    P0 = W.product(c1.B0)
    ins = list(c1.INS)
    Icap = 10 ** 8 * c1.B0[-1] * c1.B0[-2] + 1
    pr = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "mitm")],
                        input=f"{c1.M} 2 {P0 % c1.M} {Icap} 1\n29 {' '.join(map(str, c1.B0))}\n"
                              f"{len(ins)} {' '.join(map(str, ins))}\n", capture_output=True, text=True, check=True)
    gold["config1"]["mitm_min_ratio"] = pr.stdout.split("\n")[:2]
    print("config1", gold["config1"]["matches"], gold["config1"]["hits"])
    seeds = [0, 2, 3] if quick else [0, 1, 2, 3, 4]
    gold["config2"] = []
    for s in seeds:
        w = W.config2(s)
        row = mitm64_case(w)
        gold["config2"].append(row)
        print(w.name, row["d_leaves"], row["i_leaves"], row["matches"], row["d_res"])
    gold["positive_control"] = positive_control()
    print("positive control pairs", gold["positive_control"]["pairs"])
    gold["m0_kat"] = m0_kat((4, 5) if quick else (4, 5, 6))
    if not quick:
        gold["m0_kat_large"] = m0_kat_large()
        gold["config4_bounded"] = config4_bounded()
        gold["config3_pins"] = config3_pins()
    print("m0", [(x["r"], x["d_records"], x["i_records"]) for x in gold["m0_kat"]["rows"]])
    json.dump(gold, open(OUT, "w"), indent=0)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
