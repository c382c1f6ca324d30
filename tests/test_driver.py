"""Driver integration on the CPU: the instance bounds equal the reference driver's values
recorded with its own dumpers (M0 known-answer rows)."""
from carmichael_frontier_b200 import driver


def test_instance_bounds_match_the_reference_driver(golden):
    kat = golden["m0_kat"]
    for rr in kat["rows"]:
        Icap, Dmin, cap_r, INS = driver.instance_bounds(kat["B0"], kat["INS_full"], rr["r"], int(kat["U"]))
        assert (Icap, Dmin, len(INS)) == (int(rr["Icap"]), int(rr["Dmin"]), rr["n_ins"])


def test_bound_tables_match_their_definitions():
    # the exact bound tables of the bounded producers against their definitions, with Python
    # integers: G[t][x] = ceil(Dmin / (b_x ... b_{x-t})), H[t][x] = floor((Icap-1) / (a_x ... a_{x+t})),
    # and their (low, high) u64 words saturated at 2^128 - 1
    import math
    import random

    from carmichael_frontier_b200 import bounded, workloads as W
    rng = random.Random(11)
    for trial in range(12):
        Q = W.eligible_pool(W.draw_modulus(200 + trial), 5518)
        n = rng.randint(1, min(len(Q), 80))
        P = Q[:n]
        r = rng.randint(1, 10)
        for Dmin in (0, rng.randrange(1, 1 << 50), rng.randrange(1, 1 << 200)):
            G = bounded.dmin_table(P, r, Dmin)
            for t in range(r):
                for x in range(n):
                    want = (-(-Dmin // math.prod(P[x - t:x + 1])) if Dmin > 0 else 0) if t <= x and t < n \
                        else bounded.U128 - 1
                    assert G[t * n + x] == want
            words = bounded._u128_pairs(G)
            for j, v in enumerate(G):
                v = min(v, bounded.U128 - 1)
                assert int(words[2 * j]) == v & ((1 << 64) - 1) and int(words[2 * j + 1]) == v >> 64
        Icap = rng.randrange(2, 1 << 150)
        rr = min(r, n)
        H = bounded.quotient_table(P, rr, Icap)
        for t in range(rr):
            for x in range(n):
                want = (Icap - 1) // math.prod(P[x:x + t + 1]) if x + t < n else 0
                assert H[t * n + x] == want


def test_log2_screen_keeps_every_pair_at_or_below_the_bound():
    # the float screen may keep pairs above the bound (decided exactly later) but never drops one
    # at or below it, including pairs whose n equals the bound or sits one unit on either side
    import math
    import random

    from carmichael_frontier_b200 import workloads as W
    from carmichael_frontier_b200.bsolve import log2_screen
    rng = random.Random(11)
    Q = W.eligible_pool(W.draw_modulus(4242), 20000)
    B0, INS = Q[:40], Q[40:90]
    P0 = math.prod(B0)
    r = 3
    pairs = [(tuple(sorted(rng.sample(range(len(B0)), r))), tuple(sorted(rng.sample(range(len(INS)), r))))
             for _ in range(3000)]
    ns = [P0 * math.prod(INS[x] for x in i) // math.prod(B0[x] for x in d) for d, i in pairs]
    for bound in [sorted(ns)[len(ns) // 2], ns[0], ns[0] - 1, ns[0] + 1, min(ns), max(ns)]:
        keep = log2_screen(P0, B0, INS, pairs, bound)
        assert all(k for k, n in zip(keep, ns) if n <= bound)
        assert sum(keep) <= sum(1 for n in ns if n <= bound) + 5      # and drops all but a few above it
    assert len(log2_screen(P0, B0, INS, [], 10)) == 0
    assert log2_screen(P0, B0, INS, pairs[:10], 1).all()               # short lists go to the exact check
