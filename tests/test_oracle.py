"""The CPU checker pinned against the reference's own outputs (golden fixtures)."""
import hashlib
import math

import numpy as np
import pytest

import oracle as O
from carmichael_frontier_b200 import workloads as W


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()[:32]


def test_gen_records_restatement_matches_reference_kernel(golden):
    for c in golden["gen_records"]:
        n = c["hi"] - c["lo"]
        if n > 300_000:
            continue
        k, i = O.gen_records(c["primes"], c["r"], c["M"], c["mult"], c["bits"], c["lo"], c["hi"])
        assert digest(k) == c["key_digest"], c["name"]
        assert digest(i) == c["id_digest"], c["name"]


def test_config1_exhaustive_matches_reference_mitm64(golden):
    g = golden["config1"]
    w = W.config1()
    assert g["M"] == w.M and g["B0"] == list(w.B0) and g["Q"] == list(w.Q)
    pairs, hits = O.solve_exhaustive(w.M, w.Q, w.B0, w.r, w.B)
    # mitm64 keeps one D per residue; with Dres == D_leaves its matches are all pairs
    assert g["d_res"] == g["d_leaves"] == math.comb(29, 2)
    assert sorted([list(D), list(I)] for D, I in pairs) == g["pairs"]
    assert sorted([list(D), list(I), str(n)] for D, I, n in hits) == g["hits"]
    assert len(hits) == 2
    for D, I, n in hits:
        ok, n2 = O.verify_certificate(sorted((set(w.B0) - set(D)) | set(I)))
        assert ok and n2 == n


def test_mitm64_restatement_matches_reference_binary(golden):
    g = golden["config1"]
    w = W.config1()
    P0 = O.product(w.B0)
    Icap = O.product(list(w.INS)[-2:]) + 1
    m, st = O.mitm64_matches(w.B0, w.INS, 2, w.M, P0, Icap)
    assert sorted([list(D), list(I)] for D, I in m) == g["pairs"]
    assert st == (g["d_leaves"], g["d_res"], g["i_leaves"])


def test_join_all_restatement_config1(golden):
    w = W.config1()
    P0 = O.product(w.B0)
    d, i = O.join_all(w.B0, pow(P0, -1, w.M), w.INS, 1, 2, w.M)
    from carmichael_frontier_b200.tables import unrank_lex
    got = sorted([[list(w.B0[x] for x in unrank_lex(int(a), 29, 2)), list(w.INS[x] for x in unrank_lex(int(b), len(w.INS), 2))]
                  for a, b in zip(d, i)])
    assert got == golden["config1"]["pairs"]


def test_numpy_join_sorted_equals_pair_join():
    w = W.config1()
    P0 = O.product(w.B0)
    Dk, Did = O.gen_records(w.B0, 2, w.M, 1, 6)
    Ik, Iid = O.gen_records(w.INS, 2, w.M, P0 % w.M, 8)
    Dk, Did = O.sort_side(Dk, Did)
    Ik, Iid = O.sort_side(Ik, Iid)
    pd, pi = O.join_sorted(Dk, Did, Ik, Iid)
    assert len(pd) == 2


@pytest.mark.parametrize("row", [0, 1])
def test_idump_ddump_restatement_matches_reference_counts(golden, row):
    kat = golden["m0_kat"]
    rr = kat["rows"][row]
    r = rr["r"]
    INS = [q for q in kat["INS_full"]][: rr["n_ins"]]
    P0 = O.product(kat["B0"])
    keys, ids, cnt = O.idump(INS, r, kat["M"], P0, int(rr["Icap"]), rr["split_idx"], rr["hmax"], rank_ids=True)
    assert cnt == rr["i_records"]
    assert digest(np.sort(ids)) == rr["i_id_digest"]
    assert digest(keys[np.argsort(ids)]) == rr["i_key_digest"]
    dk, di, dcnt = O.ddump(kat["B0"], r, kat["M"], int(rr["Dmin"]))
    assert dcnt == rr["d_records"]
    assert digest(np.sort(dk)) == rr["d_key_digest"]
    assert [rr["d_records"], rr["i_records"]] == kat["documented"][str(r)]


def test_positive_control_fixture(golden):
    pc = golden["positive_control"]
    N = int(pc["N"])
    assert [pc["D_need"], pc["I_need"], pc["N"]] in pc["pairs"]
    ok, n = O.verify_certificate(sorted((set(pc["B0"]) - set(pc["D_need"])) | set(pc["I_need"])))
    assert ok and n == N


def test_config2_fixture_consistency(golden):
    for g in golden["config2"]:
        w = W.config2(int(g["name"].split("seed")[1].split("_")[0]))
        assert w.M == g["M"] and list(w.B0) == g["B0"] and list(w.Q) == g["Q"]
        assert g["d_leaves"] == math.comb(64, 5)
        assert g["i_leaves"] == math.comb(len(w.INS), 5)
        assert g["d_res"] == g["d_leaves"]        # no D-residue collision: matches == all pairs
        assert g["matches"] == len(g["pairs"])


def test_record_digest_device_form_equals_numpy_form():
    # the GPU tests fold records with int64 tensor arithmetic; it must equal the uint64 numpy form
    import torch
    from test_gpu_kat_large import dev_digest_add
    rng = np.random.default_rng(7)
    k = rng.integers(0, 1 << 64, size=100_003, dtype=np.uint64)
    i = rng.integers(0, 1 << 64, size=100_003, dtype=np.uint64)
    want = O.record_digest_add(O.record_digest_add((0, 0, 0), k[:500], i[:500]), k[500:], i[500:])
    got = dev_digest_add((0, 0, 0), torch.from_numpy(k.view(np.int64)), torch.from_numpy(i.view(np.int64)))
    assert got == want
