"""Measured ceilings on the running GPU (random L2 sector reads, 64-bit Montgomery products)
and the rates of the LSD radix sort (the materialised join's sort_side) and of generation.

    python -m carmichael_frontier_b200.measure.micro            # ceilings, one JSON line
    python -m carmichael_frontier_b200.measure.micro sort N [KEY_BITS [DIGIT_BITS]]
                                     # the radix sort on N random keys (default 62 bits, 8-bit digits)
    python -m carmichael_frontier_b200.measure.micro gen N      # linear generator, bounded D producer
bench.py measures the L2 figure in its own run as the fused probe's ceiling.  The ceiling kernels
live in libcfmicro.so (measure/cf_micro.cu), apart from the library's C ABI.
"""
from __future__ import annotations

import json
import math

from .. import _lib
from . import load as _load_micro


class _Micro:
    """libcfmicro.so with the library's status check."""

    def __getattr__(self, name):
        return getattr(_load_micro(), name)


def _mcheck(status: int, where: str) -> None:
    if status != 0:
        raise RuntimeError(f"{where}: status {status}")


def l2_random_reads(table_mb: int = 32, iters: int = 2048, reps: int = 3) -> float:
    """Random 32-byte reads per second from a table of `table_mb` MiB."""
    import torch
    lib = _Micro()
    nb = (table_mb << 20) // 32
    nb = 1 << (nb.bit_length() - 1)
    tab = torch.randint(0, 1 << 30, (nb * 8,), dtype=torch.int32, device="cuda")
    sink = torch.zeros(2, dtype=torch.int64, device="cuda")
    blocks = torch.cuda.get_device_properties(0).multi_processor_count * 4
    sh = torch.cuda.current_stream().cuda_stream
    _mcheck(lib.cf_micro_l2_probe(tab.data_ptr(), nb - 1, 64, blocks, sink.data_ptr(), sh), "l2 probe")
    best = 0.0
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _mcheck(lib.cf_micro_l2_probe(tab.data_ptr(), nb - 1, iters, blocks, sink.data_ptr(), sh), "l2 probe")
        e1.record()
        torch.cuda.synchronize()
        best = max(best, blocks * 512 * iters / (e0.elapsed_time(e1) * 1e-3))
    return best


def montgomery_products(iters: int = 4096, reps: int = 3) -> float:
    """64-bit Montgomery products per second."""
    import torch
    lib = _Micro()
    sink = torch.zeros(2, dtype=torch.int64, device="cuda")
    blocks = torch.cuda.get_device_properties(0).multi_processor_count * 8
    sh = torch.cuda.current_stream().cuda_stream
    _mcheck(lib.cf_micro_mulhi(16, blocks, sink.data_ptr(), sh), "mulhi")
    best = 0.0
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _mcheck(lib.cf_micro_mulhi(iters, blocks, sink.data_ptr(), sh), "mulhi")
        e1.record()
        torch.cuda.synchronize()
        best = max(best, blocks * 256 * iters * 8 / (e0.elapsed_time(e1) * 1e-3))
    return best


def sort_rate(n: int, key_bits: int = 62, digit_bits: int = 8, reps: int = 3, library: bool = True) -> dict:
    """cf_sort_pairs_digits on n random (key, id) records below 2^key_bits: records/s and the HBM
    bytes per second of its passes (each digit pass reads and writes 16 bytes per record, the
    histogram reads the keys once).  library=True adds the stable torch.sort of the same keys
    (the CUDA library's radix sort of (key, 64-bit index) pairs over all 64 key bits) for context."""
    import torch
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(7)
    k0 = torch.randint(0, 1 << key_bits, (n,), dtype=torch.int64, device="cuda", generator=g)
    keys, ids = torch.empty_like(k0), torch.arange(n, dtype=torch.int64, device="cuda")
    nb = lib.cf_sort_digits_tmp_bytes(n, key_bits, digit_bits)
    if nb == 0:
        raise ValueError(f"digit width {digit_bits} or key_bits {key_bits} not supported")
    tmp = torch.empty(nb, dtype=torch.uint8, device="cuda")
    sh = torch.cuda.current_stream().cuda_stream

    def timed(fn):
        best = None
        for _ in range(reps + 1):
            keys.copy_(k0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) * 1e-3
            best = t if best is None else min(best, t)
        return best

    best = timed(lambda: _lib.check(lib.cf_sort_pairs_digits(keys.data_ptr(), ids.data_ptr(), n, key_bits,
                                                             digit_bits, tmp.data_ptr(), nb, sh), "sort"))
    assert bool((keys[1:] >= keys[:-1]).all())
    passes = (key_bits + digit_bits - 1) // digit_bits
    out = {"n": n, "key_bits": key_bits, "digit_bits": digit_bits, "s": best, "records_per_s": n / best,
           "passes": passes, "GB_s": (32 * passes + 8) * n / best / 1e9}
    if library:
        del tmp
        t_lib = timed(lambda: torch.sort(keys, stable=True))
        out["torch_sort"] = {"s": t_lib, "records_per_s": n / t_lib}
    return out


def generation_rate(n: int, dmin_bits: int = 40, reps: int = 3) -> dict:
    """Residue generation on the k=64 r=5 instance of seed 0: the linear generator (the generate()
    drop-in, canonical residues and 10-bit packed ids, I ranks [0, n)) and the bounded D producer
    (every 5-subset of the 64-prime base with product >= 2^dmin_bits, ddump's order)."""
    import torch
    from .. import mitm_gpu2, workloads as W
    from ..bounded import BoundedGenerator
    from ..solve import Instance
    w = W.config2(0)
    inst = Instance.build(w.M, w.Q, w.B0, w.r, w.B)
    r, M = inst.r, inst.M
    n = min(n, math.comb(len(inst.INS), r))

    def timed(fn):
        best, out = None, None
        for _ in range(reps + 1):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            out = fn()
            e1.record()
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) * 1e-3
            best = t if best is None else min(best, t)
        return best, out

    t_lin, (keys, _ids) = timed(lambda: mitm_gpu2.generate(inst.INS, r, M, 1, 10, 0, n))
    gen = BoundedGenerator()
    t_bd, (_k, _i, nd) = timed(lambda: gen.generate_D(inst.B0, r, M, 1 << dmin_bits, bitmask=2))
    return {"linear": {"records": n, "s": t_lin, "records_per_s": n / t_lin, "GB_s": 16 * n / t_lin / 1e9},
            "bounded_D": {"records": nd, "dmin_bits": dmin_bits, "s": t_bd, "records_per_s": nd / t_bd,
                          "of": math.comb(len(inst.B0), r)}}


def main() -> None:
    import sys
    if len(sys.argv) > 2 and sys.argv[1] == "sort":
        kb = int(sys.argv[3]) if len(sys.argv) > 3 else 62
        db = int(sys.argv[4]) if len(sys.argv) > 4 else 8
        print(json.dumps(sort_rate(int(sys.argv[2]), kb, db)))
        return
    if len(sys.argv) > 2 and sys.argv[1] == "gen":
        print(json.dumps(generation_rate(int(sys.argv[2]))))
        return
    out = {"l2_random_32B_reads_per_s": {mb: l2_random_reads(mb) for mb in (8, 32, 64)},
           "hbm_random_32B_reads_per_s": l2_random_reads(4096, iters=256),
           "montgomery64_products_per_s": montgomery_products()}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
