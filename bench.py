#!/usr/bin/env python3
"""Benchmark: MITM records joined/s on B200 -- single-modulus k=64 solves (r = 5).

Workload ("k64_r5_single_modulus"): each step solves one seeded modulus
M = 2^a 3^b 5^c 7^d * (4-6 primes from 11..43) in [10^15, 2^62), pool
Q(M) = primes <= 5518 with (q-1) | M (capped at 320), B0 = the 64 smallest,
r = 5, B = 10^148: D side C(64,5) = 7,624,512 records, I side C(|INS|,5)
(10^7 .. 6.8*10^8).  value = (N_D + N_I) summed over all ranks / max-over-ranks
device time.  With N GPUs each rank solves its own moduli (the portfolio
shards by modulus; no data-path collective): weak scaling.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own CPU engine (src/mitm64.cpp built
from source into oracle/_ref/, all host threads) on a bounded sample of the
same workload and prints the same JSON line with "impl": "reference".

The default line also carries the rest of the headline metric, measured in the
same run after the timed regions: "portfolio" (moduli solved/s of the batched
persistent form against the per-modulus fused form, the plain one-launch-per-
stage mitm_gpu2 form and the reference's mitm64 on all host cores, on the same
seeded moduli) and "serving" (p50/p99 solve latency, continuous batching
against serial, at one offered load).  --no-extras leaves them out.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MITM records joined/s (N_D + N_I per second, k=64 r=5 single-modulus solves)"
UNIT = "records/s"
WORKLOAD = "k64_r5_single_modulus"
SEED_POOL = 64          # candidate seeds for the step sequence
BYTES_PER_RECORD = 32   # algorithmic: one 16-B {key,id} write + one 16-B read per record entering the join
D_BUILD_SHARE = 0.05    # reference-engine samples: the serial D-side build at most ~5% of a step


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="CPU-baseline budget (seconds of work)")
    ap.add_argument("--strategy", choices=("fused", "partition"), default="fused")
    ap.add_argument("--case", type=int, default=None,
                    help="profile a single seeded modulus (every step solves config-2 seed CASE)")
    ap.add_argument("--workload", choices=("single", "portfolio", "serving", "large", "census"), default="single",
                    help="single: the headline k=64 r=5 line; portfolio / serving / large: their own lines")
    ap.add_argument("--stream-i-limit", type=int, default=1 << 29)
    ap.add_argument("--moduli", type=int, default=1024)
    ap.add_argument("--i-limit", type=int, default=1 << 24)
    ap.add_argument("--plain-moduli", type=int, default=128)
    ap.add_argument("--requests", type=int, default=120)
    ap.add_argument("--loads", default="3,5,8", help="offered requests/s of the serving runs")
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--no-extras", action="store_true", help="default line without the portfolio/serving keys")
    ap.add_argument("--extra-requests", type=int, default=60, help="serving requests in the default line")
    ap.add_argument("--extra-load", type=float, default=3.0, help="offered requests/s in the default line")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def step_seeds(steps: int, world: int, rank: int, case: int | None = None):
    """Balanced weak-scaling schedule: blocks of `world` seeds of similar I-side size per step."""
    from carmichael_frontier_b200 import workloads as W
    if case is not None:
        return [W.config2(case)] * steps
    cands = W.config2_seeds(SEED_POOL)
    need = steps * world
    pool = list(cands)
    while len(pool) < need:
        pool += cands
    pool = pool[:need]
    # sort each consecutive block of `world` by size so ranks get similar work; deterministic
    order = sorted(range(len(pool)), key=lambda i: (pool[i].n_I, i))
    blocks = [order[i:i + world] for i in range(0, need, world)]
    blocks.sort(key=lambda b: min(b))           # restore the seed sequence order across steps
    return [pool[b[rank]] for b in blocks]


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
            if self.gpu_id:
                cmd += ["-i", self.gpu_id]
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[j] for _, _, rs in rows for j, v in enumerate(rs) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def gpu_uuid(torch, dev) -> str | None:
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


# ------------------------------------------------------------------ CPU baseline (reference engine)
def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_sample(w, cores: int, seconds: float):
    """Bounded sample of one modulus for the CPU engine: the r-subsets of the nb largest base
    primes against those of the n' smallest insertion primes.  n' fills `seconds` at ~4M I leaves/s
    per core (all of the pool when it is smaller); mitm64 builds its D side on one thread before its
    I threads start (src/mitm64.cpp:50-71, 137-140), so nb is then chosen to keep that build near
    D_BUILD_SHARE of the step (~2.5M D leaves/s on one core)."""
    r = w.r
    base, ins = sorted(w.B0), list(w.INS)
    i_budget = max(1_000_000, int((1 - D_BUILD_SHARE) * seconds * 4.0e6 * cores))
    n2 = r
    while n2 < len(ins) and math.comb(n2 + 1, r) <= i_budget:
        n2 += 1
    i_seconds = math.comb(n2, r) / (4.0e6 * cores)
    d_budget = max(10_000, int(D_BUILD_SHARE / (1 - D_BUILD_SHARE) * i_seconds * 2.5e6))
    nb = r
    while nb < len(base) and math.comb(nb + 1, r) <= d_budget:
        nb += 1
    return base[-nb:], ins[:n2]


def run_cpu_engine(w, cores: int, seconds: float):
    """Time the reference's mitm64 (all host threads) on a bounded sample of modulus w.
    Returns (records, seconds, kind, cores, sample text, stage dict)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import re
    import oracle as O
    from carmichael_frontier_b200.workloads import product
    base, ins = cpu_sample(w, cores, seconds)
    P0 = product(base)
    Icap = product(ins[-w.r:]) + 1         # unpruned I side (every r-subset), as the GPU join
    n_d, n_i = math.comb(len(base), w.r), math.comb(len(ins), w.r)
    sample = (f"{w.name}: D side over the {len(base)} largest base primes (C({len(base)},{w.r}) = {n_d:,}) x I side "
              f"over the {len(ins)} smallest of {len(w.INS)} insertion primes (C({len(ins)},{w.r}) = {n_i:,})")
    if O.ref_binary("mitm64"):
        t0 = time.perf_counter()
        _m, err = O.run_ref_mitm64(w.M, base, ins, w.r, P0, Icap, 1, cores)
        dt = time.perf_counter() - t0
        m = re.search(r"D_leaves=(\d+) .*\(([\d.]+)s\)\s+I_leaves=(\d+) .*\(([\d.]+)s\)", err)
        stages = None
        if m:
            td, il, ti = float(m.group(2)), int(m.group(3)), float(m.group(4))
            stages = {"d_build_s": td, "i_leaves": il, "i_s": ti, "i_leaves_per_s": il / ti if ti > 0 else None,
                      "d_build_share": td / dt if dt > 0 else None}
        return n_d + n_i, dt, "reference", cores, sample, stages
    t0 = time.perf_counter()                # the C restatement (single thread) when the binary is absent
    O.mitm64_matches(base, ins, w.r, w.M, P0, Icap)
    dt = time.perf_counter() - t0
    return n_d + n_i, dt, "port", 1, sample + " [oracle port, 1 thread]", None


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    seeds = step_seeds(args.steps + args.warmup, 1, 0)
    per_step = max(2.0, min(8.0, 150.0 / max(1, args.steps + args.warmup)))
    recs = tsum = dsum = ileaves = isum = 0.0
    kind = ncores = sample = None
    for i, w in enumerate(seeds):
        n, dt, kind, ncores, sample, st = run_cpu_engine(w, cores, per_step)
        if i >= args.warmup:
            recs += n
            tsum += dt
            if st:
                dsum += st["d_build_s"]
                ileaves += st["i_leaves"]
                isum += st["i_s"]
    value = recs / tsum
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tsum / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded moduli)",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "engine": "src/mitm64.cpp (built from source, -O3, all host threads)",
                       "sample_per_step": "bounded: " + (sample or "")},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": kind, "sample": sample,
                             "cpu_model": cpu_model(),
                             "d_build_share": dsum / tsum if tsum else None,
                             "i_leaves_per_s": ileaves / isum if isum else None},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def run_ours(args):
    import torch
    from carmichael_frontier_b200 import Solver, _lib
    from carmichael_frontier_b200 import solve as public_solve
    from carmichael_frontier_b200 import solve_many as public_solve_many
    from carmichael_frontier_b200.solve import Instance, _default_solvers

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    def allmax(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def allsum(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    seq = step_seeds(args.steps + args.warmup, world, rank, args.case)
    warm, timed = seq[:args.warmup], seq[args.warmup:]
    from carmichael_frontier_b200 import Tuning
    solver = Solver(dev, tuning=Tuning(strategy=args.strategy))
    insts = [Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in seq]
    # inputs resident in HBM for the device-timed region: pool tables uploaded before timing
    solver.tables.max_entries = 10 ** 6
    for inst in insts:
        md = pow(inst.P0, -1, inst.M)
        pd = solver.tables.pool(inst.B0, inst.r, inst.M, md)
        pi = solver.tables.pool(inst.INS, inst.r, inst.M, 1)
        solver.tables.tail(inst.B0, inst.r, inst.M, md, pd)
        solver.tables.tail(inst.INS, inst.r, inst.M, 1, pi)
        solver.tables.screen(inst.P0, inst.B, 1e-6)
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(gpu_uuid(torch, dev))
    clocks.start()
    # warm-up through the same pipelined call (both buffer sets allocated before timing)
    solver.solve_many(insts[:args.warmup], verify=True)
    # ---- device-timed region: K solves, inputs resident
    stream = torch.cuda.current_stream(dev)
    import collections
    kt = collections.defaultdict(float)
    recs = 0
    launches = 0
    hits = 0
    barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    # one modulus after another, each its own build, probe and check; the host collects and
    # certifies each solve while the device runs the next one, and consecutive solves alternate
    # between two streams (one solve's table build runs beside the previous one's probe)
    for res in solver.solve_many(insts[args.warmup:], verify=True):
        recs += res.records
        launches += res.launches
        hits += len(res.hits)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    t_local = e0.elapsed_time(e1) / 1e3
    # per-kernel times: the same solves again on one stream (no overlap), events around each kernel
    marks_all = []
    solver.solve_many(insts[args.warmup:], verify=True, marks_list=marks_all, streams=1)
    torch.cuda.synchronize(dev)
    for marks in marks_all:
        for (t0, a), (tag, b) in zip(marks, marks[1:]):
            kt[tag] += a.elapsed_time(b) / 1e3
    t_max = allmax(t_local)
    recs_all = allsum(recs)
    value = recs_all / t_max

    # ---- end-to-end region: the public API from host inputs, every step's pool and screen tables
    # prepared on the host and copied up, every step's counters and checked rows read back
    lib = _lib.load()

    def h2d_of(w):
        return lib.cf_pool_bytes(len(w.B0), w.r) + lib.cf_pool_bytes(len(w.INS), w.r) + lib.cf_screen_bytes()

    def public_solver():
        s0 = next(iter(_default_solvers.values()))
        s0.tables.clear()
        s0.tables.max_entries = 5            # one instance's tables: no step finds its inputs cached
        s0.h2d_desc_bytes = 0
        s0.d2h_bytes = 0
        return s0

    _default_solvers.clear()
    if timed:                                # one untimed call: the public solver's device buffers
        public_solve_many(timed[:2], device=dev, strategy=args.strategy)
    s = public_solver()
    barrier()
    torch.cuda.synchronize(dev)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    t_wall0 = time.perf_counter()
    # the list call: each step joined on its own, the host preparing the next step meanwhile
    public_solve_many(timed, device=dev, strategy=args.strategy)
    f1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    t_e2e = allmax(f0.elapsed_time(f1) / 1e3)
    t_e2e_wall = allmax(time.perf_counter() - t_wall0)
    h2d = sum(h2d_of(w) for w in timed) + s.h2d_desc_bytes
    d2h = s.d2h_bytes
    e2e_value = recs_all / max(t_e2e, t_e2e_wall)
    # the one-call-per-modulus form of the same API (the reference driver's per-instance call)
    s = public_solver()
    barrier()
    torch.cuda.synchronize(dev)
    t_wall0 = time.perf_counter()
    for w in timed:
        public_solve(w.M, w.Q, w.B0, w.r, w.B, device=dev, strategy=args.strategy)
        s.tables.clear()
    torch.cuda.synchronize(dev)
    t_pc = allmax(time.perf_counter() - t_wall0)
    e2e_per_call = {"value": recs_all / t_pc, "unit": UNIT, "api": "carmichael_frontier_b200.solve",
                    "h2d_bytes_per_step": (sum(h2d_of(w) for w in timed) + s.h2d_desc_bytes) / max(len(timed), 1),
                    "d2h_bytes_per_step": s.d2h_bytes / max(len(timed), 1)}
    clk = clocks.stop()

    # ---- roofline of the join path (partitioned generation + partition join)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    t_path = kt["gen_D"] + kt["gen_I"] + kt["join"] + kt["probe"]
    achieved = BYTES_PER_RECORD * recs / t_path / 1e9 if t_path > 0 else None
    traffic = None     # DRAM bytes per step of the join-path kernels, scaled from the committed ncu capture
    tfile = os.path.join(ROOT, "profiles", "k_fused_k64_r5_seed0.md")
    if args.strategy == "fused" and os.path.exists(tfile):
        per = {}
        for line in open(tfile):
            if line.startswith("- traffic_bytes_per_"):
                k, v = line[2:].split(":")
                per[k.split()[0]] = float(v)
        if "traffic_bytes_per_I_record" in per:
            n_i_all = sum(math.comb(len(w.INS), w.r) for w in timed)
            n_d_all = sum(math.comb(len(w.B0), w.r) for w in timed)
            traffic = (per["traffic_bytes_per_I_record"] * n_i_all
                       + per.get("traffic_bytes_per_D_record", 0.0) * n_d_all) / len(timed)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            n, dt, kind, cores, sample, st = run_cpu_engine(timed[0], os.cpu_count() or 1, args.cpu_seconds)
            cpu = {"value": n / dt, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
                   "cpu_model": cpu_model(), "stages": st}
        except Exception as e:            # report, never fail the GPU line
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": None, "sample": f"failed: {e}"}

    # ceiling of the fused probe, measured in this run on this GPU: random 32-byte reads from an
    # L2-resident table the size of the k=64 r=5 fingerprint array (2^20 buckets x 32 B)
    l2_ceiling = None
    if rank == 0:
        try:
            from carmichael_frontier_b200.measure.micro import l2_random_reads
            l2_ceiling = l2_random_reads(32)
        except Exception as e:            # report, never fail the GPU line
            l2_ceiling = None
            print(f"l2 ceiling not measured: {e}", file=sys.stderr)

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras and args.case is None:
        extras["portfolio"] = measure_portfolio(dev, args, compact=True)
        extras["serving"] = measure_serving(dev, args, [args.extra_load], args.extra_requests, compact=True)

    if rank == 0:
        kern = {k: {"ms_total": 1e3 * v} for k, v in kt.items()}
        # the table is built on the smaller side and probed by the larger one
        n_build = sum(min(math.comb(len(w.B0), w.r), math.comb(len(w.INS), w.r)) for w in timed)
        n_probe = sum(max(math.comb(len(w.B0), w.r), math.comb(len(w.INS), w.r)) for w in timed)
        if kt["probe"] > 0:
            kern["probe"]["records_per_s"] = n_probe / kt["probe"]
        n_d = sum(math.comb(len(w.B0), w.r) for w in timed)
        n_i = sum(math.comb(len(w.INS), w.r) for w in timed)
        if kt["gen_I"] > 0:
            kern["gen_I"]["GB_s"] = 16 * n_i / kt["gen_I"] / 1e9
        if kt["join"] > 0:
            kern["join"]["GB_s"] = 16 * (n_i + n_d) / kt["join"] / 1e9
        if kt["gen_D"] > 0:
            kern["gen_D"]["GB_s"] = 16 * (n_build if args.strategy == "fused" else n_d) / kt["gen_D"] / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded moduli)",
            "config": {"workload": WORKLOAD, "r": 5, "k": 64, "B": "10^148", "moduli_per_step_per_gpu": 1,
                       "seeds": [w.name for w in timed][:8], "l2": "inputs larger than L2 (I side 0.17-11 GB per step)",
                       "parallelism": f"modulus-sharded x{world}", "records_per_gpu": recs},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per D and per I record "
                                            "of one capture (profiles/k_fused_k64_r5_seed0.md), scaled by this "
                                            "run's record counts" if traffic is not None else None),
                         "kernel": ("k_fused build + probe" if solver.tuning.strategy == "fused"
                                    else "k_gen_part + k_join_part") + " (join path, 32 B/record)",
                         "peak_source": peak_src},
            "strategy": solver.tuning.strategy,
            "kernels": kern,
            "kernels_source": ("CUDA events around each kernel in a second pass over the timed solves on one "
                               "stream (the timed pass overlaps consecutive solves on two streams)"),
            "l2_probe": ({"achieved_probes_per_s": n_probe / kt["probe"],
                          "ceiling_probes_per_s": l2_ceiling,
                          "frac": n_probe / kt["probe"] / l2_ceiling,
                          "note": "one 32-byte L2 sector read per probing record; ceiling = random 32-B loads/s "
                                  "from a 32 MiB table, measured in this run (measure/cf_micro.cu)"}
                         if kt["probe"] > 0 and l2_ceiling else None),
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // max(1, len(timed)),
                    "d2h_bytes_per_step": d2h // max(1, len(timed)), "api": "carmichael_frontier_b200.solve_many",
                    "per_call": e2e_per_call},
            "gpu_launches": launches,
            "hits": hits,
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                       "samples": clk["samples"]},
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ------------------------------------------------------------------ portfolio (batched vs per-modulus)
def measure_portfolio(dev, args, compact: bool = False) -> dict:
    """Seeded 1024-modulus portfolio (k=64, pools 120..400, r in {4,5,6}, B=10^148); every
    modulus joined over its full D side and the first --i-limit I ranks (a bounded sample:
    the unpruned I sides total ~1e14 records).  Forms, all on the same moduli: batched
    persistent kernels (CUDA graphs replayed), this library's per-modulus fused solve, the
    reference's per-modulus mitm_gpu2 form (generate / sort_side / join_sorted per stage), and
    the reference's mitm64 on all host cores (a bounded sample of one modulus, as records/s and
    the moduli/s it amounts to at the GPU sample's records per modulus)."""
    import torch
    from carmichael_frontier_b200 import Solver, workloads as W
    from carmichael_frontier_b200.portfolio import BatchSolver, run_per_modulus, run_plain
    from carmichael_frontier_b200.solve import Instance
    lim = args.i_limit
    ws = W.config3(args.moduli)
    insts = [Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in ws]
    bs = BatchSolver(dev)
    t0 = time.perf_counter()
    prep = bs.prepare(insts, lim)
    torch.cuda.synchronize(dev)
    t_prep = time.perf_counter() - t0
    recs = prep.records
    clocks = ClockSampler(gpu_uuid(torch, dev))
    clocks.start()
    steps = 3 if compact else args.steps
    for _ in range(1 if compact else args.warmup):
        bs.run(prep, graphs=True)
    torch.cuda.synchronize(dev)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        res = bs.run(prep, graphs=True)
        torch.cuda.synchronize(dev)
        times.append(time.perf_counter() - t0)
    t_b = statistics.median(times)
    one = Solver(dev)
    run_per_modulus(insts[:4], i_limit=lim, solver=one)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    per = run_per_modulus(insts, i_limit=lim, solver=one)
    torch.cuda.synchronize(dev)
    t_p = time.perf_counter() - t0
    npl = len(insts) if compact else min(args.plain_moduli, len(insts))
    # the plain form's sort: radix digit width per size class of its sides, by the autotuner
    from carmichael_frontier_b200 import autotune, mitm_gpu2
    sides = [n for k in range(npl) for n in (prep.nD[k], min(prep.nI[k], 1 << 27))]
    key_bits = max(x.M.bit_length() for x in insts[:npl])
    t0 = time.perf_counter()
    autotune.tune_sort(sides, key_bits=key_bits, device=dev, reps=2)
    t_tune = time.perf_counter() - t0
    digit_bits = {n.bit_length(): mitm_gpu2.sort_digit_bits(n) for n in sides if n > 1}
    run_plain(insts[:1], i_limit=1 << 16, device=dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    plain = run_plain(insts[:npl], i_limit=lim, device=dev)
    torch.cuda.synchronize(dev)
    t_pl = time.perf_counter() - t0
    clk = clocks.stop()
    bs.release(prep)
    rec_pl = sum(prep.nD[k] + prep.nI[k] for k in range(npl))
    key = lambda a: (a.residue_pairs, sorted(a.pairs), [h.n for h in a.hits])
    same = [key(a) for a in res] == [key(a) for a in per]
    same_plain = [key(a) for a in res[:npl]] == [key(a) for a in plain]
    cpu = None
    if not args.no_cpu_baseline:
        try:
            n, dt, kind, cores, sample, st = run_cpu_engine(ws[0], os.cpu_count() or 1, args.cpu_seconds / 2)
            rate = n / dt
            cpu = {"records_per_s": rate, "moduli_per_s_equiv": rate / (recs / len(insts)), "cores": cores,
                   "cpu_model": cpu_model(), "kind": kind, "sample": sample, "stages": st}
        except Exception as e:
            cpu = {"records_per_s": None, "sample": f"failed: {e}"}
    out = {
        "workload": "portfolio_1024_k64_r456", "moduli": len(insts), "i_limit": lim, "records": recs,
        "sample": f"full D sides, I ranks [0, {lim}) per modulus; every form on the same {len(insts)} moduli"
                  if npl == len(insts) else f"full D sides, I ranks [0, {lim}); plain form on the first {npl}",
        "batched": {"moduli_per_s": len(insts) / t_b, "records_per_s": recs / t_b, "s": t_b, "graphs": True},
        "per_modulus_fused": {"moduli_per_s": len(insts) / t_p, "records_per_s": recs / t_p, "s": t_p,
                              "same_results": same},
        "plain_mitm_gpu2": {"moduli": npl, "moduli_per_s": npl / t_pl, "records_per_s": rec_pl / t_pl, "s": t_pl,
                            "same_results": same_plain,
                            "sort_digit_bits": {f"2^{c - 1}..2^{c}": b for c, b in sorted(digit_bits.items())},
                            "sort_key_bits": key_bits, "sort_tune_s": t_tune},
        "batched_over_plain": (len(insts) / t_b) / (npl / t_pl),
        "mitm64_all_cores": cpu,
        "batched_over_mitm64": ((recs / t_b) / cpu["records_per_s"]) if cpu and cpu.get("records_per_s") else None,
        "targets": {"batched_over_plain": 10.0, "batched_over_mitm64": 50.0},
        "hits": sum(len(x.hits) for x in res), "residue_pairs": sum(x.residue_pairs for x in res),
        "prepare_s": t_prep, "batches": len(prep.batches),
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                   "samples": clk["samples"]},
    }
    return out


def init_dist(dev):
    """NCCL process group for torchrun launches (None for one process)."""
    import datetime
    import torch.distributed as dist
    _, world, _ = dist_env()
    if world == 1:
        return None
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    return dist


def run_portfolio_sharded(args, dev, dist):
    """The portfolio split by modulus over the ranks (carmichael_frontier_b200.shard: balanced by
    records, no data-path collective): each rank runs its share as one batch; the time is the max
    over ranks of the device-timed batch, the value the whole portfolio's moduli over it."""
    import torch
    from carmichael_frontier_b200 import shard, workloads as W
    from carmichael_frontier_b200.portfolio import BatchSolver
    from carmichael_frontier_b200.solve import Instance
    rank, world, _ = dist_env()
    lim = args.i_limit
    insts = [Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in W.config3(args.moduli)]
    weights = [math.comb(len(x.B0), x.r) + min(math.comb(len(x.INS), x.r), lim) for x in insts]
    mine = shard.assign(weights, world)[rank]
    bs = BatchSolver(dev)
    prep = bs.prepare([insts[i] for i in mine], lim)
    clocks = ClockSampler(gpu_uuid(torch, dev))
    clocks.start()
    for _ in range(args.warmup):
        bs.run(prep, graphs=True)
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    times = []
    for _ in range(args.steps):
        dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = bs.run(prep, graphs=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        t = torch.tensor([e0.elapsed_time(e1) / 1e3], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        times.append(float(t.item()))
    clk = clocks.stop()
    recs = torch.tensor([float(prep.records)], dtype=torch.float64, device=dev)
    dist.all_reduce(recs, op=dist.ReduceOp.SUM)
    g = [None] * world
    dist.all_gather_object(g, [(i, x.residue_pairs, len(x.hits)) for i, x in zip(mine, res)])
    t_b = statistics.median(times)
    if rank == 0:
        per = sorted(y for part in g for y in part)
        line = {"metric": "portfolio moduli solved/s (batched persistent kernels)", "value": len(insts) / t_b,
                "unit": "moduli/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * t_b, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "u64", "data": "synthetic (seeded moduli)",
                "config": {"workload": "portfolio_1024_k64_r456", "moduli": len(insts), "i_limit": lim,
                           "records": float(recs.item()), "parallelism": f"modulus-sharded x{world}",
                           "sample": f"full D sides, I ranks [0, {lim}) per modulus"},
                "records_per_s": float(recs.item()) / t_b, "moduli_solved": len(per),
                "residue_pairs": sum(p for _, p, _ in per), "hits": sum(h for _, _, h in per),
                "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                           "samples": clk["samples"]}}
        print(json.dumps(line), flush=True)


def run_portfolio(args):
    import torch
    rank, world, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        dist = init_dist(dev)
        try:
            run_portfolio_sharded(args, dev, dist)
        finally:
            dist.destroy_process_group()
        return
    p = measure_portfolio(dev, args)
    line = {"metric": "portfolio moduli solved/s (batched persistent kernels)", "value": p["batched"]["moduli_per_s"],
            "unit": "moduli/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * p["batched"]["s"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded moduli)",
            "config": {"workload": p["workload"], "moduli": p["moduli"], "i_limit": p["i_limit"],
                       "records": p["records"], "sample": p["sample"]},
            "portfolio": p, "clocks": p["clocks"]}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ serving (continuous batching)
def measure_serving(dev, args, loads, requests: int, compact: bool = False) -> dict:
    """The first `requests` requests of the seeded serving stream (k = 64..100, pools 80..320,
    r = 3..6, B = prod(B0) * 10^4), Poisson arrivals at each offered load, served by the
    continuous-batching loop; the serial form (one request at a time) at the same loads."""
    import torch
    from carmichael_frontier_b200 import Solver, Tuning, serve, workloads as W
    from carmichael_frontier_b200.solve import Instance
    insts = [Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in W.config5_requests(requests)]
    warm = [Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in W.config5_requests(8, seed=1)]
    alone = Solver(dev, tuning=Tuning(strategy="auto", max_nodes=1 << 22))
    for x in warm:
        alone.solve_instance(x)
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(gpu_uuid(torch, dev))
    clocks.start()
    out = {"continuous": [], "serial": []}
    same = True
    for rate in loads:
        srv = serve.Server(dev, slots=args.slots, strategy="auto").start()
        st, tickets = serve.run_poisson(srv, insts, rate=rate, seed=7)
        srv.stop()
        out["continuous"].append(st)
        torch.cuda.empty_cache()

        def one(x):
            r = alone.solve_instance(x)
            torch.cuda.synchronize(dev)
            alone._bufs.clear()
            return r
        st2, res2 = serve.run_serial(one, insts, rate=rate, seed=7)
        out["serial"].append(st2)
        pairs = lambda ts: [sorted(t.result.pairs) if t.result is not None else None for t in ts]  # noqa: E731
        same = same and pairs(tickets) == pairs(res2)
    clk = clocks.stop()
    keep = ("offered_rps", "throughput_rps", "p50_ms", "p99_ms", "mean_ms", "errors") if compact else None
    trim = (lambda d: {k: d[k] for k in keep if k in d}) if keep else (lambda d: d)
    return {"workload": "serving_k64-100_r3-6", "requests": len(insts), "slots": args.slots, "offered_rps": loads,
            "arrivals": "Poisson, seed 7", "sample": f"first {len(insts)} of the seeded 10,000-request stream",
            "continuous": [trim(x) for x in out["continuous"]], "serial": [trim(x) for x in out["serial"]],
            "same_results_alone_and_in_the_mix": same,
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                       "samples": clk["samples"]}}


def run_serving(args):
    import torch
    rank, world, local = dist_env()
    if rank != 0:
        return
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    loads = [float(x) for x in args.loads.split(",")]
    sv = measure_serving(dev, args, loads, args.requests)
    mid = sv["continuous"][len(loads) // 2]
    line = {"metric": "serving p50/p99 solve latency (ms) and requests/s", "value": mid["p99_ms"], "unit": "ms (p99)",
            "n_gpus": 1, "steps": sv["requests"], "warmup": 8, "ms_per_step": mid["mean_ms"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded request stream)",
            "config": {"workload": sv["workload"], "requests": sv["requests"], "slots": sv["slots"],
                       "offered_rps": loads, "arrivals": sv["arrivals"], "sample": sv["sample"]},
            "continuous": sv["continuous"], "serial": sv["serial"],
            "same_results_alone_and_in_the_mix": sv["same_results_alone_and_in_the_mix"], "clocks": sv["clocks"]}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ census families (bounded runs)
def run_census(args):
    """Census producers and family runs, the reference's production flow below an incumbent U:
    the divisor-family census of the incumbent of results_k64_best_global.json (its size and primes
    are in tests/golden/census_lambdaJ.json with the reference's run records of that family), every
    survivor run at radii 1..10 through the driver's bounds and the bounded GPU join, each instance
    checked against the reference's record line; then a seeded sample of 100 moduli of the
    lambda-neighbourhood census of M0 (tests/golden/nbhd_M0_p19.json) at radii 1..6, the shape of the
    reference's 50,142-modulus campaign.  Metric: family instances per second."""
    import random
    import torch
    from carmichael_frontier_b200 import census as C
    from carmichael_frontier_b200.solve import Solver, Tuning
    rank, world, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        dist = init_dist(dev)
        try:
            run_census_sharded(args, dev, dist)
        finally:
            dist.destroy_process_group()
        return
    gold = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(gold, "census_lambdaJ.json")) as f:
        fam = json.load(f)
    with open(os.path.join(gold, "nbhd_M0_p19.json")) as f:
        nb = json.load(f)
    U = int(fam["U"])
    t0 = time.perf_counter()
    _, rows = C.divisor_family(U, fam["factors"])
    t_census = time.perf_counter() - t0
    s = Solver(dev, tuning=Tuning(strategy="bounded"))
    C.family_run(rows[:3], U, r_max=3, solver=s)                 # warm-up: tables, buffers
    clocks = ClockSampler(gpu_uuid(torch, dev))
    clocks.start()

    def timed(rws, rmax):
        torch.cuda.synchronize(dev)
        a = time.perf_counter()
        o, hits = C.family_run(rws, U, r_max=rmax, solver=s)
        torch.cuda.synchronize(dev)
        return o, hits, time.perf_counter() - a

    out, hits, t_fam = timed(rows, 10)
    n_inst = sum(len(out[r["D"]]["instances"]) for r in rows)
    recs = sum(x["nD"] + x["nI"] for r in rows for x in out[r["D"]]["instances"])
    same = all(out[r["D"]]["instances"] == [x for x in fam["runs"][str(r["D"])]["instances"]
                                           if x["r"] in {y["r"] for y in out[r["D"]]["instances"]}]
               for r in rows)
    skipped = sum(len(out[r["D"]]["skipped"]) for r in rows)
    sample = random.Random(1).sample(nb["survivors"], min(100, len(nb["survivors"])))
    out2, hits2, t_nb = timed(sample, 6)
    n2 = sum(len(out2[r["D"]]["instances"]) for r in sample if "instances" in out2[r["D"]])
    recs2 = sum(x["nD"] + x["nI"] for r in sample if "instances" in out2[r["D"]] for x in out2[r["D"]]["instances"])
    clk = clocks.stop()
    print(json.dumps({
        "metric": "census family instances/s (bounded runs below the incumbent U)", "value": n_inst / t_fam,
        "unit": "instances/s", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": 1e3 * t_fam,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u128 products, u64 keys",
        "data": "the reference's incumbent U (148 digits) and its census",
        "config": {"workload": "census_lambdaJ_family_r1-10", "survivors": len(rows), "census_s": t_census},
        "family": {"instances": n_inst, "skipped_over_128_bits": skipped, "records": recs,
                   "records_per_s": recs / t_fam, "s": t_fam, "same_as_reference_records": same,
                   "completions_below_U": len(hits)},
        "neighbourhood_sample": {"moduli": len(sample), "instances": n2, "records": recs2, "s": t_nb,
                                 "instances_per_s": n2 / t_nb, "records_per_s": recs2 / t_nb,
                                 "completions_below_U": len(hits2)},
        "clocks": clk}))


def run_census_sharded(args, dev, dist):
    """The incumbent's divisor family (the census workload's first part) split by modulus over the
    ranks: each rank runs its rows' family runs; instances are checked against the reference's
    records on rank 0; the time is the max over ranks."""
    import torch
    from carmichael_frontier_b200 import census as C, shard
    from carmichael_frontier_b200.solve import Solver, Tuning
    rank, world, _ = dist_env()
    with open(os.path.join(ROOT, "tests", "golden", "census_lambdaJ.json")) as f:
        fam = json.load(f)
    U = int(fam["U"])
    rows = fam["survivors"]
    weights = [sum(x["nD"] + x["nI"] for x in fam["runs"][str(r["D"])]["instances"]) + 1000 for r in rows]
    s = Solver(dev, tuning=Tuning(strategy="bounded"))
    C.family_run(rows[:3], U, r_max=3, solver=s)                # warm-up: tables, buffers
    clocks = ClockSampler(gpu_uuid(torch, dev))
    clocks.start()
    dist.barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()

    def solve_share(rws):
        out, _hits = C.family_run(rws, U, r_max=10, solver=s)
        return [out[r["D"]] for r in rws]
    res, _mine = shard.run_sharded(rows, weights, solve_share)
    torch.cuda.synchronize(dev)
    t = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    clk = clocks.stop()
    if rank == 0:
        n_inst = sum(len(x["instances"]) for x in res)
        same = all(x["instances"] == [y for y in fam["runs"][str(r["D"])]["instances"]
                                      if y["r"] in {z["r"] for z in x["instances"]}] for r, x in zip(rows, res))
        tt = float(t.item())
        print(json.dumps({
            "metric": "census family instances/s (bounded runs below the incumbent U)", "value": n_inst / tt,
            "unit": "instances/s", "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": 1e3 * tt,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u128 products, u64 keys",
            "data": "the reference's incumbent U (148 digits) and its census",
            "config": {"workload": "census_lambdaJ_family_r1-10", "survivors": len(rows),
                       "parallelism": f"modulus-sharded x{world}"},
            "family": {"instances": n_inst, "same_as_reference_records": same, "s": tt},
            "clocks": clk}), flush=True)


# ------------------------------------------------------------------ large radius (r = 7, pool 160)
def run_large(args):
    """k=64, one seeded modulus, pool capped at 160 primes, r = 7: D = C(64,7) = 6.2e8,
    I = C(96,7) = 1.19e10 records (191 GB as 16-byte records).  Two forms:
    fused   the whole instance: table on the D side, every I record generated and probed
            in registers (nothing materialised, fits in HBM);
    streamed both sides spilled as 16-byte records to pinned host memory, partitioned by the
            top 8 bits of the residue, streamed back partition by partition and joined --
            on the I ranks [0, --stream-i-limit) (a bounded sample: the full I side is 191 GB
            of host memory)."""
    import torch
    from carmichael_frontier_b200 import Solver, Tuning, workloads as W
    from carmichael_frontier_b200.solve import Instance
    from carmichael_frontier_b200.streamed import streamed_solve
    rank, world, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    w = W.config4()
    inst = Instance.build(w.M, w.Q, w.B0, w.r, w.B)
    s = Solver(dev, tuning=Tuning(strategy="fused"))
    if world > 1:
        dist = init_dist(dev)
        try:
            run_large_split(args, dev, dist, w, inst, s)
        finally:
            dist.destroy_process_group()
        return
    clocks = ClockSampler(gpu_uuid(torch, dev))
    clocks.start()
    res = s.solve_instance(inst, timed=True)           # warm-up: tables and buffers
    times = []
    for _ in range(max(1, args.steps)):
        marks = []
        r1 = s.solve_instance(inst, timed=True, marks=marks)
        times.append(r1.device_ms / 1e3)
    t_f = statistics.median(times)
    kt = {}
    for (t0, a), (tag, b) in zip(marks, marks[1:]):
        kt[tag] = kt.get(tag, 0.0) + a.elapsed_time(b) / 1e3
    lim = args.stream_i_limit
    torch.cuda.empty_cache()
    sres, st = streamed_solve(inst, pbits=8, i_limit=lim, device=dev)
    clk = clocks.stop()
    n_sample = sres.n_D + sres.n_I
    line = {"metric": "large-radius join records/s (k=64, pool 160, r=7)", "value": r1.records / t_f,
            "unit": "records/s", "n_gpus": 1, "steps": len(times), "warmup": 1, "ms_per_step": 1e3 * t_f,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded modulus)",
            "config": {"workload": "k64_pool160_r7", "modulus": w.name, "n_D": r1.n_D, "n_I": r1.n_I,
                       "materialised_I_bytes": 16 * r1.n_I},
            "fused": {"records_per_s": r1.records / t_f, "s": t_f, "plan": {k: r1.plan.get(k) for k in
                                                                            ("bbits", "fbits", "swap")},
                      "kernel_s": kt, "residue_pairs": r1.residue_pairs, "hits": len(r1.hits)},
            "streamed": {"i_limit": lim, "records": n_sample, "records_per_s": n_sample / (st["spill_s"] + st["join_s"]),
                         "spill_s": st["spill_s"], "join_s": st["join_s"], "host_bytes": st["host_bytes"],
                         "pin_alloc_s": st["pin_alloc_s"],
                         "d2h_GB_s": st["d2h_bytes"] / st["spill_s"] / 1e9,
                         "h2d_GB_s": st["h2d_bytes"] / st["join_s"] / 1e9,
                         "residue_pairs": sres.residue_pairs, "launches": sres.launches},
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                       "samples": clk["samples"]}}
    print(json.dumps(line), flush=True)


def run_large_split(args, dev, dist, w, inst, s):
    """The large-radius instance split over the ranks by I-rank window (carmichael_frontier_b200.shard:
    every rank builds the whole D table, the small side, and probes its share of the I ranks; the
    only collectives are the gather of the window results and the max-over-ranks of the device
    time): strong scaling of one modulus."""
    import torch
    from carmichael_frontier_b200 import shard
    rank, world, _ = dist_env()
    nI = math.comb(len(inst.INS), inst.r)
    lo, hi = shard.windows(nI, world)[rank]
    s.solve_instance(inst, timed=True, i_lo=lo, i_limit=hi)          # warm-up: tables and buffers
    clocks = ClockSampler(gpu_uuid(torch, dev))
    clocks.start()
    times = []
    merged = None
    for _ in range(max(1, args.steps)):
        dist.barrier()
        got: dict = {}

        def solve_window(a, b):
            got["r"] = s.solve_instance(inst, timed=True, i_lo=a, i_limit=b)
            return got["r"]
        merged, _win = shard.run_split(solve_window, nI)
        t = torch.tensor([got["r"].device_ms / 1e3], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        times.append(float(t.item()))
    clk = clocks.stop()
    t_f = statistics.median(times)
    if rank == 0:
        recs = merged.n_D + merged.n_I
        line = {"metric": "large-radius join records/s (k=64, pool 160, r=7)", "value": recs / t_f,
                "unit": "records/s", "n_gpus": world, "steps": len(times), "warmup": 1, "ms_per_step": 1e3 * t_f,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u64",
                "data": "synthetic (seeded modulus)",
                "config": {"workload": "k64_pool160_r7", "modulus": w.name, "n_D": merged.n_D, "n_I": merged.n_I,
                           "parallelism": f"I-rank windows x{world}, D table on every rank"},
                "fused": {"records_per_s": recs / t_f, "s": t_f, "residue_pairs": merged.residue_pairs,
                          "hits": len(merged.hits)},
                "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                           "samples": clk["samples"]}}
        print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "portfolio":
        run_portfolio(args)
    elif args.workload == "serving":
        run_serving(args)
    elif args.workload == "large":
        run_large(args)
    elif args.workload == "census":
        run_census(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
