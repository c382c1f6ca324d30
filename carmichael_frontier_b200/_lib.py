"""ctypes binding of the C ABI in ``include/cfmitm.h`` (``libcfmitm.so``).

The library is the only compute path: if it is missing or a call fails, an
exception is raised.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcfmitm.so")

CF_OK = 0
CF_EBADARG = -1
CF_ENOMEM = -2
CF_ECUDA = -3
CF_EOVERFLOW = -4
CF_ETIMEOUT = -5

ERR_PART_OVERFLOW = 1
ERR_PAIR_OVERFLOW = 2
ERR_TABLE_FULL = 4
ERR_SPIN_LIMIT = 8
ERR_KEY_MISMATCH = 16

HIT_KEY_EQUAL = 1
HIT_SCREEN = 2
HIT_SIZE_EXACT = 4
HIT_KORSELT = 8
HIT_DISJOINT = 16

u64 = C.c_uint64
u32 = C.c_uint32
vp = C.c_void_p
sz = C.c_size_t


class CfError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


# (name, restype, argtypes) for every symbol in include/cfmitm.h
SIGNATURES = [
    ("cf_version", C.c_int, []),
    ("cf_last_error_string", C.c_char_p, []),
    ("cf_pool_bytes", sz, [C.c_int, C.c_int]),
    ("cf_pool_prepare", C.c_int, [vp, C.c_int, C.c_int, u64, u64, vp, sz]),
    ("cf_pool_prepare_split", C.c_int, [vp, C.c_int, C.c_int, u64, C.c_int, u64, u64, vp, sz]),
    ("cf_key_of", u64, [u64, u64]),
    ("cf_canon_of", u64, [u64, u64]),
    ("cf_key_mul", u64, [u64, u64, u64]),
    ("cf_key32_mul", u64, [u64, u64, u64]),
    ("cf_screen_bytes", sz, []),
    ("cf_screen_prepare", C.c_int, [vp, C.c_int, C.c_double, C.c_double, C.c_double, vp, sz]),
    ("cf_gen_subsets", C.c_int, [vp, C.c_int, C.c_int, u64, u64, C.c_int, C.c_int, C.c_int, vp, vp, vp]),
    ("cf_tail_bytes", sz, [C.c_int, C.c_int]),
    ("cf_build_tail", C.c_int, [vp, C.c_int, C.c_int, vp, vp]),
    ("cf_gen_part_shapes", C.c_int, []),
    ("cf_gen_part_smem_bytes", sz, [C.c_int, C.c_int, C.c_int, C.c_int]),
    ("cf_gen_part", C.c_int, [vp, vp, C.c_int, C.c_int, u64, u64, C.c_int, u32, vp, vp, vp, C.c_int, vp]),
    ("cf_join_part_smem_bytes", sz, [C.c_int]),
    ("cf_join_part", C.c_int, [vp, vp, u32, vp, vp, u32, C.c_int, C.c_int, u32, u32, vp, u32, vp, vp, vp]),
    ("cf_dtab_bytes", sz, [C.c_int]),
    ("cf_dtab_fp_bytes", sz, [C.c_int]),
    ("cf_dtab_bytes2", sz, [C.c_int, C.c_int]),
    ("cf_dtab_build2", C.c_int, [vp, vp, C.c_int, C.c_int, u64, u64, vp, C.c_int, C.c_int, vp, vp]),
    ("cf_fused_probe2", C.c_int, [vp, vp, C.c_int, C.c_int, u64, u64, vp, C.c_int, C.c_int, u64, C.c_int, vp, u32,
                                  vp, vp, u32, vp]),
    ("cf_dtab_build", C.c_int, [vp, vp, C.c_int, C.c_int, u64, u64, vp, C.c_int, vp, vp]),
    ("cf_dtab_build3", C.c_int, [vp, vp, C.c_int, C.c_int, u64, u64, vp, C.c_int, C.c_int, C.c_int, vp, vp]),
    ("cf_fused_probe3", C.c_int, [vp, vp, C.c_int, C.c_int, u64, u64, vp, C.c_int, C.c_int, C.c_int, u64, C.c_int,
                                  vp, u32, vp, vp, u32, vp]),
    ("cf_fused_probe", C.c_int, [vp, vp, C.c_int, C.c_int, u64, u64, vp, C.c_int, u64, vp, u32, vp, vp, u32, vp]),
    ("cf_pair_result_bytes", sz, []),
    ("cf_check_pairs", C.c_int, [vp, vp, vp, C.c_int, vp, vp, u32, vp, vp, vp]),
    ("cf_scan_tmp_bytes", sz, [u64]),
    ("cf_scan_u64", C.c_int, [vp, u64, vp, vp, sz, vp]),
    ("cf_bgen_count", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, u64, vp, vp, vp, vp, C.c_int, C.c_int, C.c_int,
                                C.c_int, vp, vp, vp]),
    ("cf_bgen_expand", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, u64, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int,
                                 C.c_int, u64, u64, vp, vp, vp, vp, vp, vp]),
    ("cf_rec_build", C.c_int, [vp, u64, vp, C.c_int, C.c_int, vp, vp]),
    ("cf_rec_probe", C.c_int, [vp, u64, vp, C.c_int, C.c_int, C.c_int, vp, u32, vp, vp, vp]),
    ("cf_bgen_probe", C.c_int, [C.c_int, C.c_int, u64, vp, vp, vp, vp, vp, u64, u64, vp, C.c_int, C.c_int, vp, u32,
                                vp, vp, vp]),
    ("cf_rec_build_keyform", C.c_int, [vp, u64, vp, C.c_int, C.c_int, vp, vp, vp]),
    ("cf_bgen_probe_keyform", C.c_int, [C.c_int, C.c_int, u64, vp, vp, vp, vp, vp, u64, u64, vp, C.c_int, C.c_int,
                                        vp, u32, vp, vp, vp]),
    ("cf_part_hist", C.c_int, [vp, u64, u64, C.c_int, vp, vp]),
    ("cf_part_scatter", C.c_int, [vp, vp, u64, u64, C.c_int, vp, vp, vp, vp]),
    ("cf_batch_mod_bytes", sz, []),
    ("cf_batch_max_r", C.c_int, []),
    ("cf_batch_run", C.c_int, [C.c_int, vp, vp, u32, u32, vp, vp, vp, u32, vp, vp, vp, u32, vp]),
    ("cf_batch_part_buckets", u32, [C.c_int]),
    ("cf_batch_part_tile", u32, []),
    ("cf_batch_part_max_ranges", u32, []),
    ("cf_batch_ovf_bytes", sz, []),
    ("cf_batch_part", C.c_int, [C.c_int, vp, vp, u32, vp, vp, u32, vp, vp, C.c_int, C.c_int, u32, vp]),
    ("cf_sort_tmp_bytes", sz, [u64]),
    ("cf_sort_pairs", C.c_int, [vp, vp, u64, C.c_int, vp, sz, vp]),
    ("cf_sort_digits_tmp_bytes", sz, [u64, C.c_int, C.c_int]),
    ("cf_sort_pairs_digits", C.c_int, [vp, vp, u64, C.c_int, C.c_int, vp, sz, vp]),
    ("cf_sort_pairs_noalloc_max", u64, []),
    ("cf_sort_pairs_noalloc", C.c_int, [vp, vp, u64, C.c_int, vp]),
    ("cf_join_tmp_bytes", sz, [u64]),
    ("cf_join_count", C.c_int, [vp, u64, vp, u64, vp, sz, vp, vp]),
    ("cf_join_emit", C.c_int, [vp, vp, u64, vp, vp, u64, vp, vp, vp, u64, vp]),
    ("cf_igen_bounds_bytes", sz, [C.c_int, C.c_int]),
    ("cf_igen_bounds", C.c_int, [vp, C.c_int, C.c_int, u64, u64, vp, sz]),
    ("cf_igen_tmp_bytes", sz, [u64]),
    ("cf_igen_count", C.c_int, [vp, vp, u64, u64, C.c_int, C.c_int, C.c_int, C.c_int, vp, sz, vp, vp, vp, vp]),
    ("cf_igen_write", C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, vp, u64, u64, vp, vp, vp]),
    ("cf_solve_batch", C.c_int, [vp, vp]),
    ("cf_ddump_bounds_bytes", sz, [C.c_int, C.c_int]),
    ("cf_ddump_bounds", C.c_int, [vp, C.c_int, C.c_int, u64, u64, vp, sz]),
    ("cf_bounded_join", C.c_int, [vp, vp, C.c_int, vp, vp, C.c_int, C.c_int, u64, u64, C.c_int, C.c_int, C.c_int,
                                  C.c_int, vp, sz, vp, u64, vp, vp, vp, vp]),
    ("cf_merge_run_bytes", sz, []),
    ("cf_merge_join_runs", C.c_int, [vp, u64, vp, u64, vp, u64, vp, vp, vp, vp]),
]

class CfBatchQueue(C.Structure):
    """include/cfmitm.h CfBatchQueue: one prepared batch for cf_solve_batch."""
    _fields_ = [("mods", vp), ("arena", vp), ("zero_bytes", u64), ("misc", vp), ("build_tickets", vp),
                ("probe_tickets", vp), ("place_tickets", vp), ("scatter_tickets", vp), ("scatter_radius", vp),
                ("ovf", vp), ("pairs", vp), ("pair_mods", vp), ("results", vp), ("nmod", u32), ("ticket", u32),
                ("grid", u32), ("max_pairs", u32), ("ovf_cap", u32), ("n_scatter", u32), ("use_part", C.c_int),
                ("part_lb", C.c_int), ("n_probe", u32), ("pad0", u32), ("probe_tickets_r", vp), ("probe_radius", vp)]


assert C.sizeof(CfBatchQueue) == 160

_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Load libcfmitm.so (built by ``carmichael_frontier_b200._build``)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m carmichael_frontier_b200._build` "
                    "(the join has no CPU fallback)")
            lib = C.CDLL(LIB_PATH)
            for name, res, args in SIGNATURES:
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(status: int, where: str) -> None:
    if status != CF_OK:
        msg = load().cf_last_error_string().decode(errors="replace")
        raise CfError(status, where, msg)


def ptr(t) -> int | None:
    """Device (or host) address of a torch tensor / numpy array, None for None."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


def stream_handle(stream=None) -> int | None:
    """cudaStream_t of a torch stream (the current device's current stream when None, read
    without building a torch Stream object: this runs once per library call)."""
    import torch
    if stream is not None:
        return stream.cuda_stream
    torch.cuda._lazy_init()
    return torch._C._cuda_getCurrentRawStream(torch._C._cuda_getDevice())
