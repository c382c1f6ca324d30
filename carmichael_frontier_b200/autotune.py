"""Autotuner for the partitioned join's launch parameters.

Chooses, per workload class (radius and side sizes), the partition count
(through the D records per partition), the generator's launch shape (threads
per CTA x subsets per thread) and the join's CTAs per partition, by timing
complete device solves with CUDA events on a representative instance.  The
results are cached in memory and can be saved to / loaded from a JSON file.
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
