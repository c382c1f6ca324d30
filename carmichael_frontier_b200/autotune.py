"""Autotuners for the launch parameters.

``tune``: per workload class (radius and side sizes) of the partitioned join,
the partition count (through the D records per partition), the generator's
launch shape (threads per CTA x subsets per thread) and the join's CTAs per
partition, by timing complete device solves with CUDA events on a
representative instance; results cached in memory and optionally in a JSON file.

``tune_batch``: for the batched portfolio kernels, the work-queue ticket size
(records a warp takes per queue pop) and the persistent grid, by timing whole
batch runs of a prepared portfolio.

``tune_sort``: the radix digit width (8 or 9 bits) of the materialised join's
sort (sort_side) per size class, by timing whole sorts of random keys of the
class's size and key width.
"""
from __future__ import annotations

import itertools
import json
import math
import os
from dataclasses import asdict

from . import _lib
from .solve import Instance, Solver, Tuning

D_PER_PART = (3500, 7000, 14000)
ISPLIT = (0, 2, 4)


def workload_class(inst: Instance) -> str:
    nD = math.comb(len(inst.B0), inst.r)
    nI = math.comb(len(inst.INS), inst.r)
    return f"r{inst.r}_d{int(math.log2(max(nD, 1)))}_i{int(math.log2(max(nI, 1)))}"


def time_solve(solver: Solver, inst: Instance, reps: int = 3) -> float:
    """Median device milliseconds of `reps` solves (after one warm-up)."""
    solver.solve_instance(inst, verify=False)
    ts = []
    for _ in range(reps):
        res = solver.solve_instance(inst, verify=False, timed=True)
        ts.append(res.device_ms)
    ts.sort()
    return ts[len(ts) // 2]


def tune(inst: Instance, device=None, reps: int = 3, shapes=None, d_per_part=D_PER_PART, isplit=ISPLIT,
         verbose: bool = False) -> tuple[Tuning, list[dict]]:
    """Try every candidate; return the fastest Tuning and the measured table."""
    lib = _lib.load()
    shapes = range(lib.cf_gen_part_shapes()) if shapes is None else shapes
    rows = []
    best = None
    for shape, dpp, isp in itertools.product(shapes, d_per_part, isplit):
        tu = Tuning(d_per_part=dpp, gen_shape=shape, isplit=isp)
        s = Solver(device, tuning=tu)
        try:
            ms = time_solve(s, inst, reps)
        except _lib.CfError as e:        # a shape that does not fit this pool is skipped
            rows.append(dict(shape=shape, d_per_part=dpp, isplit=isp, ms=None, error=str(e)))
            continue
        rows.append(dict(shape=shape, d_per_part=dpp, isplit=isp, ms=ms))
        if verbose:
            print(f"  shape={shape} d_per_part={dpp} isplit={isp}: {ms:.3f} ms", flush=True)
        if best is None or ms < best[0]:
            best = (ms, tu)
    if best is None:
        raise RuntimeError("no launch configuration ran")
    return best[1], rows


TICKETS = (2048, 4096, 8192, 32768)
GRID_PER_SM = (0, 2, 4)                 # 0 = one resident wave (the occupancy limit)


def tune_batch(prep, device=None, reps: int = 3, tickets=TICKETS, grids=GRID_PER_SM, base=None,
               verbose: bool = False):
    """Fastest (ticket, grid) for a prepared portfolio: returns (BatchTuning, rows).  Each
    candidate re-prepares the portfolio's ticket tables and times `reps` whole runs."""
    import time

    import torch

    from .portfolio import BatchSolver, BatchTuning
    sms = torch.cuda.get_device_properties(torch.device(device if device is not None else "cuda")).multi_processor_count
    rows, best = [], None
    base = base or BatchTuning()
    for ticket, g in itertools.product(tickets, grids):
        tu = BatchTuning(ticket=ticket, grid=g * sms, mem_budget=base.mem_budget, pair_capacity=base.pair_capacity,
                         dtab=base.dtab)
        bs = BatchSolver(device, tuning=tu)
        p2 = bs.prepare(prep.instances, prep.i_limit)
        bs.run(p2, verify=False)
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            bs.run(p2, verify=False)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        ms = 1e3 * sorted(ts)[len(ts) // 2]
        rows.append(dict(ticket=ticket, grid=g * sms, ms=ms))
        if verbose:
            print(f"  ticket={ticket} grid={g * sms}: {ms:.2f} ms", flush=True)
        if best is None or ms < best[0]:
            best = (ms, tu)
        bs.release(p2)
    return best[1], rows


def sort_size_classes(sizes) -> dict[int, int]:
    """{size class: largest size in it} over the sizes above 1; a size n is in class bit_length(n),
    the key under which sort_side looks up its digit width."""
    largest: dict[int, int] = {}
    for n in sizes:
        n = int(n)
        if n > 1:
            c = n.bit_length()
            largest[c] = max(largest.get(c, 0), n)
    return dict(sorted(largest.items()))


def tune_sort(sizes, key_bits: int = 64, device=None, widths=None, reps: int = 3, seed: int = 0,
              apply: bool = True, verbose: bool = False) -> list[dict]:
    """Radix digit width of sort_side per size class (bit length of n) among `sizes`: for each
    class, the largest size in it is sorted with every candidate width on random keys below
    2^key_bits (the residue keys of a modulus M lie below 2^bit_length(M)), timed whole with CUDA
    events (median of `reps` after one warm-up).  The fastest width is recorded for the class
    (mitm_gpu2.set_sort_digit_bits) unless apply=False.  Returns one row per class and width."""
    import numpy as np
    import torch

    from . import mitm_gpu2 as G
    widths = G.SORT_DIGIT_WIDTHS if widths is None else tuple(widths)
    if not 1 <= key_bits <= 64:
        raise ValueError("key_bits must be 1..64")
    if any(w not in G.SORT_DIGIT_WIDTHS for w in widths):
        raise ValueError(f"digit widths must be among {G.SORT_DIGIT_WIDTHS}")
    dev = torch.device(device if device is not None else "cuda")
    rng = np.random.default_rng(seed)
    rows = []
    for c, n in sort_size_classes(sizes).items():
        keys = torch.from_numpy(rng.integers(0, 1 << key_bits, size=n, dtype=np.uint64)).to(dev)
        ids = torch.arange(n, device=dev, dtype=torch.int64).view(torch.uint64)
        best = None
        for db in widths:
            G.sort_side(keys, ids, digit_bits=db)
            ts = []
            for _ in range(reps):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record()
                G.sort_side(keys, ids, digit_bits=db)
                b.record()
                b.synchronize()
                ts.append(a.elapsed_time(b))
            ms = sorted(ts)[len(ts) // 2]
            rows.append(dict(size_class=c, n=n, key_bits=key_bits, digit_bits=db, ms=ms))
            if verbose:
                print(f"  n={n} key_bits={key_bits} digit_bits={db}: {ms:.3f} ms", flush=True)
            if best is None or ms < best[0]:
                best = (ms, db)
        if apply:
            G.set_sort_digit_bits(n, best[1])
        del keys, ids
    return rows


class TuningCache:
    """Tuned parameters per workload class, optionally persisted as JSON."""

    def __init__(self, path: str | None = None):
        self.path = path
        self.table: dict[str, dict] = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.table = json.load(f)

    def get(self, inst: Instance) -> Tuning | None:
        row = self.table.get(workload_class(inst))
        return Tuning(**row) if row else None

    def put(self, inst: Instance, tu: Tuning) -> None:
        self.table[workload_class(inst)] = asdict(tu)
        if self.path:
            tmp = self.path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.table, f, indent=1)
            os.replace(tmp, self.path)

    def tuned(self, inst: Instance, device=None) -> Tuning:
        tu = self.get(inst)
        if tu is None:
            tu, _ = tune(inst, device)
            self.put(inst, tu)
        return tu


if __name__ == "__main__":
    import sys

    from . import workloads as W
    seeds = [int(x) for x in sys.argv[1:]] or [0, 3]
    for sd in seeds:
        w = W.config2(sd)
        inst = Instance.build(w.M, w.Q, w.B0, w.r, w.B)
        print(f"{w.name}: n_I={w.n_I:,}", flush=True)
        tu, rows = tune(inst, verbose=True)
        print("best:", asdict(tu), flush=True)
