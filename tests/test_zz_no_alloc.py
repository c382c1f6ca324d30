"""The radix sort's no-allocation entry point against the workspace entry point.

cf_sort_pairs_noalloc serves callers that cannot hand the library device
memory (all of it belongs to another allocator, or the caller may not change
its footprint per call): it sorts in place using a fixed scratch array inside
the library.  Its result must equal cf_sort_pairs' on the same input, on two
calls in a row (the second call finds the first call's leftovers in the shared
scratch array), for an odd and an even number of digit passes, and with a
smaller call after a larger one.  This file is collected last on purpose.
"""
import numpy as np
import pytest
import torch

from carmichael_frontier_b200 import _lib

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).cuda()


@pytest.mark.parametrize("key_bits", [64, 24, 16])      # 8, 3 and 2 digit passes
def test_noalloc_sort_equals_workspace_sort_on_two_calls(cuda, key_bits):
    lib = _lib.load()
    limit = lib.cf_sort_pairs_noalloc_max()
    assert limit == 131072
    stream = torch.cuda.current_stream().cuda_stream
    for call, n in enumerate((131_072, 5_000, 100_003)):      # a smaller call after a larger one
        rng = np.random.default_rng(1234 + call + key_bits)
        keys = rng.integers(0, 1 << min(key_bits, 63), size=n, dtype=np.uint64)
        keys[::7] = keys[3]                       # ties: stability is part of the contract
        ids = rng.integers(0, 1 << 63, size=n, dtype=np.uint64)
        ka, ia = _dev(keys), _dev(ids)
        _lib.check(lib.cf_sort_pairs_noalloc(ka.data_ptr(), ia.data_ptr(), n, key_bits, stream), "noalloc")
        kb, ib = _dev(keys), _dev(ids)
        nbytes = lib.cf_sort_tmp_bytes(n)
        tmp = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        _lib.check(lib.cf_sort_pairs(kb.data_ptr(), ib.data_ptr(), n, key_bits, tmp.data_ptr(), nbytes, stream), "ws")
        torch.cuda.synchronize()
        assert torch.equal(ka, kb) and torch.equal(ia, ib)
        order = np.argsort(keys, kind="stable")
        got_k = ka.cpu().numpy().view(np.uint64)
        got_i = ia.cpu().numpy().view(np.uint64)
        assert np.array_equal(got_k, keys[order]) and np.array_equal(got_i, ids[order])


def test_noalloc_rejects_more_than_its_scratch_holds(cuda):
    lib = _lib.load()
    n = lib.cf_sort_pairs_noalloc_max() + 1
    k = torch.zeros(n, dtype=torch.int64, device="cuda")
    assert lib.cf_sort_pairs_noalloc(k.data_ptr(), k.data_ptr(), n, 64, None) == _lib.CF_EBADARG
    assert b"exceeds the fixed scratch limit" in lib.cf_last_error_string()
