"""Record streams between the GPU path and the reference's dumpers, on the GPU.

* The GPU drop-ins for the dumper processes (python -m carmichael_frontier_b200.records idump|ddump)
  read the dumpers' stdin texts and write the same 16-byte record streams, TOTAL lines and exit
  codes: checked byte for byte against the reference binaries (oracle/_ref/, one thread, so that
  their order is the depth-first order) and against the oracle, on the M0 instance at r = 4.
* The reference's idump stream piped into the GPU join (driver.join_stream: sort_side and
  join_sorted per block, as gpu/mitm_gpu_mstar_driver.py:249-262) recovers the positive control's
  pairs, and so does the GPU drop-in's stream.
"""
import math
import sys

import numpy as np
import pytest

import oracle as O
from carmichael_frontier_b200 import driver, records as R
from carmichael_frontier_b200.tables import unrank_colex

pytestmark = pytest.mark.gpu
GPU_DUMPER = [sys.executable, "-m", "carmichael_frontier_b200.records"]


def _kat_row(golden):
    kat = golden["m0_kat"]
    rr = kat["rows"][0]                              # r = 4: 8.7M I records, 333K D records
    return kat, rr, kat["INS_full"][: rr["n_ins"]]


def _stream(argv, text, env=None):
    run = R.DumperRun(argv, text, env=env)
    blocks = list(run.blocks(block_records=1 << 22))
    n = run.close()
    return (np.concatenate(blocks) if blocks else np.zeros((0, 2), np.uint64)), n, run.total


def test_gpu_idump_process_writes_the_reference_stream(cuda, golden):
    kat, rr, INS = _kat_row(golden)
    P0 = O.product(kat["B0"])
    text = R.idump_stdin(kat["M"], rr["r"], P0, int(rr["Icap"]), kat["B0"], INS, threads=1)
    env = {"IDUMP_RANK": "1", "IDUMP_SPLIT": str(kat["SPLIT"]), "IDUMP_HMAX": str(rr["hmax"])}
    got, n, total = _stream(GPU_DUMPER + ["idump"], text, env)
    assert n == total == rr["i_records"]
    k, i, cnt = O.idump(INS, rr["r"], kat["M"], P0, int(rr["Icap"]), rr["split_idx"], rr["hmax"], rank_ids=True)
    assert cnt == n and np.array_equal(got[:, 0], k) and np.array_equal(got[:, 1], i)
    exe = O.ref_binary("mitm64_idump_stream2")
    if exe:
        ref, rn, _ = _stream([exe], text, env)
        assert rn == n and ref.tobytes() == got.tobytes()


def test_gpu_ddump_process_writes_the_reference_stream(cuda, golden):
    kat, rr, _ = _kat_row(golden)
    text = R.ddump_stdin(kat["M"], rr["r"], int(rr["Dmin"]), kat["B0"])
    got, n, total = _stream(GPU_DUMPER + ["ddump"], text)
    assert n == total == rr["d_records"]
    k, i, cnt = O.ddump(kat["B0"], rr["r"], kat["M"], int(rr["Dmin"]))
    assert np.array_equal(got[:, 0], k) and np.array_equal(got[:, 1], i)
    exe = O.ref_binary("mitm64_ddump")
    if exe:
        ref, _, _ = _stream([exe], text)
        assert ref.tobytes() == got.tobytes()


def test_gpu_dumper_exit_codes(cuda, golden):
    kat, rr, INS = _kat_row(golden)
    bad = R.DumperRun(GPU_DUMPER + ["idump"], "1 2")
    list(bad.blocks())
    with pytest.raises(R.RecordStreamError, match="code 2"):
        bad.close()
    text = R.idump_stdin(kat["M"], rr["r"], 1, int(rr["Icap"]), kat["B0"], INS[::-1])
    desc = R.DumperRun(GPU_DUMPER + ["idump"], text, env={"IDUMP_RANK": "1"})
    list(desc.blocks())
    with pytest.raises(R.RecordStreamError, match="code 4"):
        desc.close()


@pytest.mark.parametrize("producer", ["reference", "gpu"])
def test_idump_stream_into_the_gpu_join_finds_the_positive_control(cuda, golden, producer):
    pc = golden["positive_control"]
    M, r, B0, INS = pc["M"], pc["r"], pc["B0"], pc["INS"]
    P0 = O.product(B0)
    argv = GPU_DUMPER + ["idump"] if producer == "gpu" else [O.ref_binary("mitm64_idump_stream2")]
    if argv[0] is None:
        pytest.skip("oracle/_ref/mitm64_idump_stream2 is not built")
    D_chunks, nD = driver.build_D(B0, M, r, int(pc["Dmin"]), nchunks=2)
    assert nD == pc["d_records"]
    run = R.DumperRun(argv, R.idump_stdin(M, r, P0, int(pc["Icap"]), B0, INS, threads=4), env={"IDUMP_RANK": "1"})
    pd, pi, nI = driver.join_stream(D_chunks, run.blocks(block_records=1 << 19))
    assert run.close() == nI == pc["i_records"]
    got = []
    for d, i in zip(pd, pi):
        D = sorted(B0[(int(d) >> (6 * q)) & 63] for q in range(r))
        I = [INS[x] for x in unrank_colex(int(i), r, len(INS))]
        S = sorted((set(B0) - set(D)) | set(I))
        got.append([D, I, str(math.prod(S))])
    assert sorted(got) == sorted(pc["pairs"])
    assert any(p[2] == pc["N"] for p in got)
