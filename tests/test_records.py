"""Record streams and stdin formats against the reference's own engines (CPU).

The reference's dumpers (built from their sources into oracle/_ref/) read the instance texts this
library writes, their 16-byte record streams are read in blocks and checked against their TOTAL
line and exit codes as the reference driver checks them (gpu/mitm_gpu_mstar_driver.py:275-282),
and the writer reproduces their stream byte for byte."""
import io
import math

import numpy as np
import pytest

import oracle as O
from carmichael_frontier_b200 import records as R, workloads as W


def _ref(name):
    p = O.ref_binary(name)
    if p is None:
        pytest.skip(f"oracle/_ref/{name} is not built here")
    return p


def _instance():
    w = W.config1()
    P0 = W.product(w.B0)
    INS = list(w.INS)[:60]
    Icap = W.product(INS[-3:]) // 50
    return w.M, 3, P0, Icap, list(w.B0), INS


def test_stdin_texts_round_trip():
    M, r, P0, Icap, B0, INS = _instance()
    a = R.parse_idump_stdin(R.idump_stdin(M, r, P0, Icap, B0, INS, threads=4))
    assert (a["M"], a["r"], a["P0modM"], a["Icap"], a["T"], a["B0"], a["INS"]) == (M, r, P0 % M, Icap, 4, B0, INS)
    b = R.parse_ddump_stdin(R.ddump_stdin(M, r, 12345, B0))
    assert (b["M"], b["r"], b["Dmin"], b["B0"]) == (M, r, 12345, B0)
    with pytest.raises(ValueError):
        R.parse_idump_stdin("1 2 3")


def test_block_reader_whole_records_and_partial_tail():
    rec = np.arange(2 * 1001, dtype="<u8").reshape(-1, 2)
    got = list(R.read_blocks(io.BytesIO(rec.tobytes()), block_records=64))
    assert [len(x) for x in got] == [64] * 15 + [41]
    assert np.array_equal(np.concatenate(got), rec)
    with pytest.raises(R.RecordStreamError):
        list(R.read_blocks(io.BytesIO(rec.tobytes() + b"abc"), block_records=64))


def test_reference_idump_stream_read_and_checked():
    exe = _ref("mitm64_idump_stream2")
    M, r, P0, Icap, B0, INS = _instance()
    run = R.DumperRun([exe], R.idump_stdin(M, r, P0, Icap, B0, INS, threads=1), env={"IDUMP_RANK": "1"})
    got = np.concatenate(list(run.blocks(block_records=1000)))
    n = run.close()
    k, i, cnt = O.idump(INS, r, M, P0, Icap, rank_ids=True)
    assert n == cnt == len(got) and run.total == cnt
    assert np.array_equal(got[:, 0], k) and np.array_equal(got[:, 1], i)     # one thread: the same order
    buf = io.BytesIO()                                                      # the writer gives back its bytes
    assert R.write_records(buf, k, i) == cnt
    assert buf.getvalue() == got.astype("<u8").tobytes()
    assert R.parse_total(R.total_line(cnt, "x")) == cnt


def test_reference_ddump_stream_and_exit_codes():
    exe = _ref("mitm64_ddump")
    w = W.config2(1)
    B = list(w.B0)
    r = 3
    Dmin = math.isqrt(W.product(B[:r]) * W.product(B[-r:]))
    run = R.DumperRun([exe], R.ddump_stdin(w.M, r, Dmin, B))
    got = np.concatenate(list(run.blocks()))
    assert run.close() == len(got)
    k, i, cnt = O.ddump(B, r, w.M, Dmin)
    assert np.array_equal(got[:, 0], k) and np.array_equal(got[:, 1], i)
    bad = R.DumperRun([exe], "12 3")                               # malformed: exit 2
    list(bad.blocks())
    with pytest.raises(R.RecordStreamError, match="code 2"):
        bad.close()
    desc = R.DumperRun([exe], R.ddump_stdin(w.M, r, 1, B[::-1]))   # not ascending: exit 4
    list(desc.blocks())
    with pytest.raises(R.RecordStreamError, match="code 4"):
        desc.close()


def test_truncated_stream_is_incomplete():
    # a producer whose stream stops short of its TOTAL line is not counted
    import sys
    prog = ("import sys; sys.stdout.buffer.write(bytes(32)); sys.stdout.flush(); "
            "sys.stderr.write('TOTAL 3 records\\n')")
    run = R.DumperRun([sys.executable, "-c", prog], "")
    assert sum(len(b) for b in run.blocks()) == 2
    with pytest.raises(R.RecordStreamError, match="read 2 records != TOTAL 3"):
        run.close()
