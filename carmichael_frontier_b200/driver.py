"""Drop-in instance functions for the reference's GPU driver (gpu/mitm_gpu_mstar_driver.py).

The driver's control plane -- pool construction, bases, radius loop, h-strata
(hmax_for), checkpoints, the incumbent and its oracle -- stays the reference's.
What it calls per instance is replaced:

  build_D(B0, M, r, Dmin)        -> (sorted D chunks, nD)          (:100-118)
  run_instance(tag, B0, INS, r, hmax, ...) -> bool                  (:184-286)

``run_instance`` applies the driver's exact bounds for the current incumbent U
(Icap exclusive, Dmin, the per-radius insertion cap), joins the filtered sides
on the GPU (csrc/cf_bgen.cu producers, a record table of the D side probed by
the I leaves in registers), re-checks every pair in exact integers as the driver
does (n = P0 * prod(I) / prod(D) < U), hands each completion below U to the
driver's ``consider`` and logs the driver's instance line -- the format
gpu/verify_family_coverage.py reads (" r=<r> ", "dfilter", no "INCOMPLETE").
"""
from __future__ import annotations

import math
import time

from .bounded import generator
from .bsolve import log2_screen
from .tables import unrank_colex


def instance_bounds(B0, INS, r: int, U: int):
    """The driver's bounds for radius r below U (gpu/mitm_gpu_mstar_driver.py:188-205):
    (Icap exclusive, Dmin, cap_r, affordable INS)."""
    B0s = sorted(B0)
    P0 = math.prod(B0)
    topI = math.prod(INS[-r:])
    ptb = math.prod(B0s[-r:])
    Icap = max(1, min(topI + 1, (U * ptb) // P0 + 1))
    Imin = math.prod(INS[:r])
    Dmin = (P0 * Imin) // U + 1
    Imin1 = math.prod(INS[:r - 1])
    cap_r = (Icap - 1) // Imin1
    return Icap, Dmin, cap_r, [q for q in INS if q <= cap_r]


def hmax_for(B0, INS, r: int, U: int, split: int = 4000) -> int:
    """The driver's h-stratum bound (gpu/mitm_gpu_mstar_driver.py:84-98): the largest number h of
    insertion primes above `split` with which an r-exchange could still come in below U (the
    cheapest such product, P0 times the r-h smallest small primes and the h smallest large ones,
    below U times the largest removable D product); -1 when no stratum can."""
    small = [p for p in INS if p <= split]
    large = [p for p in INS if p > split]
    PB = math.prod(B0)
    Dmax = math.prod(sorted(B0)[-r:])
    best = -1
    for h in range(0, r + 1):
        if h > len(large) or r - h > len(small):
            continue
        if PB * math.prod(small[:r - h]) * math.prod(large[:h]) < U * Dmax:
            best = h
    return best


def build_D(B0, M: int, r: int, Dmin=None, nchunks: int = 1, device=None):
    """Sorted D-side chunks [(keys, ids), ...] and the record count: the r-subsets of the
    64-prime base with prod >= Dmin (every subset when Dmin is None), keys prod(D) mod M,
    ids 6-bit packed indices (an index mask for r > 10), as src/mitm64_ddump emits them;
    sorted with the drop-in sort_side.  The reference splits D into NCHUNKS_D pieces."""
    import torch

    from . import mitm_gpu2 as G
    g = generator(device)
    k, i, nD = g.generate_D(sorted(B0), r, M, 0 if Dmin is None else int(Dmin), bitmask=1 if r > 10 else 0)
    if nD == 0:
        return [], 0
    chunks = []
    step = -(-nD // max(1, nchunks))
    for a in range(0, nD, step):
        chunks.append(G.sort_side(k[a:a + step], i[a:a + step]))
    del k, i
    torch.cuda.empty_cache()
    return chunks, nD


def instance_join(B0, INS, r: int, hmax: int, M: int, U: int, split: int, solver=None):
    """The GPU part of run_instance: the filtered sides joined under the driver's bounds.
    Returns (pairs as (D index tuple, I index tuple), nD, nI, seconds), or None when the
    affordable pool holds fewer than r primes (nothing to search)."""
    from .solve import Solver, Tuning
    Icap, Dmin, _cap_r, INS_aff = instance_bounds(B0, INS, r, U)
    if len(INS_aff) < r:
        return None
    s = solver or Solver(tuning=Tuning(strategy="bounded"))
    if s._bounded is None:
        from .bsolve import BoundedSolve
        s._bounded = BoundedSolve(s)
    t0 = time.time()
    pairs_idx, nD, nI, _plan = s._bounded.join(sorted(B0), INS_aff, r, M, math.prod(B0), Icap, Dmin, split, hmax)
    return pairs_idx, nD, nI, time.time() - t0


def run_instance(tag, B0, INS, r: int, hmax: int, M: int, U: int, split: int, consider, log,
                 state: dict | None = None, solver=None, joined=None) -> bool:
    """One exchange instance below the bound U, as the driver's run_instance: returns True
    when the instance is complete.  consider(key, factors, label) receives every completion
    below U (the driver's incumbent update and oracle); log(str) writes the instance line
    (None: no line).  joined: instance_join's result for these arguments, when the join has
    already run (family runs join ahead on worker streams)."""
    B0s = sorted(B0)
    B0set = set(B0)
    P0 = math.prod(B0)
    Icap, Dmin, cap_r, INS_aff = instance_bounds(B0, INS, r, U)
    st = state if state is not None else {}
    if len(INS_aff) < r:
        if log is not None:
            log(f"  {tag} r={r}: affordable pool has {len(INS_aff)} < r primes (cap_r={cap_r}); nothing to search")
        st["instances"] = st.get("instances", 0) + 1
        st["last"] = dict(r=r, hmax=hmax, ins=len(INS_aff), nD=0, nI=0, pairs=0, below_U=0)
        return True
    if joined is None:
        joined = instance_join(B0, INS, r, hmax, M, U, split, solver)
    pairs_idx, nD, nI, dt = joined
    below = nb = 0
    rmin = None
    near = log2_screen(P0, B0s, INS_aff, pairs_idx, U).tolist()   # False: n certainly above U
    for (di, ii), maybe in zip(pairs_idx, near):
        if not maybe:
            continue
        D = [B0s[x] for x in di]
        I = [INS_aff[x] for x in ii]
        prodD, prodI = math.prod(D), math.prod(I)
        if prodI >= Icap or (P0 * prodI) % prodD:
            continue
        n = P0 * prodI // prodD
        if n >= U:
            continue
        below += 1
        fac = sorted((B0set - set(D)) | set(I))
        if consider((M, tag, r, hmax), fac, f"mstar_{tag}_r{r}_h<={hmax}_b200"):
            nb += 1
        if rmin is None or n < rmin:
            rmin = n
    st["instances"] = st.get("instances", 0) + 1
    st["last"] = dict(r=r, hmax=hmax, ins=len(INS_aff), nD=nD, nI=nI, pairs=len(pairs_idx), below_U=below)
    st["pairs_total"] = st.get("pairs_total", 0) + len(pairs_idx)
    st["completions_below_U"] = st.get("completions_below_U", 0) + below
    if log is None:                        # no instance line wanted (family runs): skip the allocator query
        return True
    gb = 0.0
    try:                                   # device memory held by this process's allocator (no driver query)
        import torch
        gb = torch.cuda.memory_reserved() / 2 ** 30
    except Exception:
        pass
    log(f"  {tag} r={r} h<={hmax} |INS|={len(INS_aff)} dfilter rank b200: D {nD:,} {0.0:.1f}s | I {nI:,} rec "
        f"{dt:.1f}s pairs={len(pairs_idx)} below_U={below} min_digits={len(str(rmin)) if rmin else None} "
        f"improved={nb} | GPU {gb:.1f}GB")
    return True


def join_stream(D_chunks, blocks, device=None):
    """Join sorted D chunks (build_D's) with I records arriving as host blocks -- a dumper's
    stream read by records.DumperRun -- as the reference driver does for its idump path
    (gpu/mitm_gpu_mstar_driver.py:249-262): each block is copied to the device, sorted with
    sort_side and joined against every D chunk with join_sorted.  Returns (D id array, I id
    array) of all equal-key pairs (numpy uint64) and the I records read."""
    import numpy as np
    import torch

    from . import mitm_gpu2 as G
    dev = torch.device(device if device is not None else "cuda")
    pd_all, pi_all, n = [], [], 0
    for a in blocks:
        n += a.shape[0]
        if a.shape[0] == 0 or not D_chunks:
            continue
        k = torch.from_numpy(np.ascontiguousarray(a[:, 0]).view(np.int64)).to(dev).view(torch.uint64)
        i = torch.from_numpy(np.ascontiguousarray(a[:, 1]).view(np.int64)).to(dev).view(torch.uint64)
        ks, is_ = G.sort_side(k, i)
        for Dk, Did in D_chunks:
            pd, pi = G.join_sorted(Dk, Did, ks, is_)
            if pd.numel():
                pd_all.append(pd.view(torch.int64).cpu().numpy().view(np.uint64))
                pi_all.append(pi.view(torch.int64).cpu().numpy().view(np.uint64))
    cat = lambda xs: np.concatenate(xs) if xs else np.zeros(0, np.uint64)  # noqa: E731
    return cat(pd_all), cat(pi_all), n


def decode_pair(B0, INS, r: int, d_colex: int, i_colex: int):
    """(D primes, I primes) of a pair of colex ids (the ids the bounded producers emit)."""
    B0s = sorted(B0)
    return (tuple(B0s[x] for x in unrank_colex(d_colex, r, len(B0s))),
            tuple(INS[x] for x in unrank_colex(i_colex, r, len(INS))))

