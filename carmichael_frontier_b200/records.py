"""Record streams and text formats shared with the reference's C++ engines.

The reference moves sides between processes as streams of 16-byte little-endian records
{u64 key, u64 id} on a dumper's stdout, closed by a "TOTAL <n> records ..." line on its stderr
and an exit code (src/mitm64_idump_stream2.cpp:55-69,84-88, src/mitm64_ddump.cpp:45-55); its
driver reads the stream in I_CHUNK blocks and counts an instance only when the records read
equal TOTAL and the exit code is 0 (gpu/mitm_gpu_mstar_driver.py:128-134,244-282).  The engines
take their instance as whitespace-separated text on stdin:

  mitm64               M r P0modM Icap prodDmin T maxmatch / nB B0... / nI INS...   (src/mitm64.cpp:18-23,126-133)
  mitm64_idump_stream2 M r P0modM Icap prodDmin T maxmatch / nB B0... / nI INS...   (:55-60; B0 read and skipped)
  mitm64_ddump         M r Dmin / 64 B0...                                            (src/mitm64_ddump.cpp:14,47-48)

This module writes and reads those formats, so the GPU path and the C++ dumpers interoperate:

  * ``idump_stdin`` / ``ddump_stdin`` / ``mitm64_stdin`` -- the stdin texts;
  * ``read_blocks`` -- a dumper's stdout in blocks of whole records, ``DumperRun`` -- a running
    dumper whose stream is checked against its TOTAL line and exit code, as the driver does;
  * ``write_records`` / ``total_line`` -- the same stream and trailer written from device or host
    records;
  * ``python -m carmichael_frontier_b200.records idump|ddump`` -- GPU processes that read a
    dumper's stdin text and environment (IDUMP_RANK, IDUMP_SPLIT, IDUMP_HMAX, DDUMP_BITMASK) and
    write its records, trailer and exit codes, with the bounded producers (csrc/cf_bgen.cu) in
    place of the CPU walk; a driver that runs the dumper binary can run this instead.
"""
from __future__ import annotations

import io
import math
import os
import subprocess
import sys

import numpy as np

RECORD_BYTES = 16
I_CHUNK = 200_000_000          # records per block, the reference driver's default block

# exit codes of the dumpers (src/mitm64_idump_stream2.cpp:55-69; src/mitm64_ddump.cpp:46-51)
EXIT_MEANING = {2: "malformed stdin", 3: "sizes out of range for the id encoding", 4: "pool not strictly ascending",
                5: "rank ids overflow u64"}


class RecordStreamError(RuntimeError):
    """A record stream that is incomplete or that its producer reported as failed."""


# -- stdin texts ---------------------------------------------------------------------------------
def _line(xs) -> str:
    return " ".join(str(int(x)) for x in xs)


def mitm64_stdin(M: int, r: int, P0: int, Icap: int, prodDmin: int, threads: int, maxmatch: int, B0, INS) -> str:
    """The instance text src/mitm64.cpp reads (and mitm64_idump_stream2, which skips B0)."""
    B0, INS = list(B0), list(INS)
    return (f"{int(M)} {int(r)} {int(P0) % int(M)} {int(Icap)} {int(prodDmin)} {int(threads)} {int(maxmatch)}\n"
            f"{len(B0)} {_line(B0)}\n{len(INS)} {_line(INS)}\n")


def idump_stdin(M: int, r: int, P0: int, Icap: int, B0, INS, threads: int = 1, prodDmin: int = 1) -> str:
    return mitm64_stdin(M, r, P0, Icap, prodDmin, threads, 0, B0, INS)


def ddump_stdin(M: int, r: int, Dmin: int, B0) -> str:
    B0 = list(B0)
    return f"{int(M)} {int(r)} {int(Dmin)}\n{len(B0)} {_line(B0)}\n"


def parse_idump_stdin(text: str) -> dict:
    """Fields of a mitm64 / mitm64_idump_stream2 instance text; ValueError when malformed."""
    t = text.split()
    try:
        M, r, p0m, Icap, pdm, T, mm = int(t[0]), int(t[1]), int(t[2]), int(t[3]), int(t[4]), int(t[5]), int(t[6])
        nB = int(t[7])
        B0 = [int(x) for x in t[8:8 + nB]]
        nI = int(t[8 + nB])
        INS = [int(x) for x in t[9 + nB:9 + nB + nI]]
    except (IndexError, ValueError) as e:
        raise ValueError(f"malformed instance text: {e}") from None
    if len(B0) != nB or len(INS) != nI:
        raise ValueError("malformed instance text: fewer primes than announced")
    return dict(M=M, r=r, P0modM=p0m, Icap=Icap, prodDmin=pdm, T=T, maxmatch=mm, B0=B0, INS=INS)


def parse_ddump_stdin(text: str) -> dict:
    t = text.split()
    try:
        M, r, Dmin, nB = int(t[0]), int(t[1]), int(t[2]), int(t[3])
        B0 = [int(x) for x in t[4:4 + nB]]
    except (IndexError, ValueError) as e:
        raise ValueError(f"malformed instance text: {e}") from None
    if len(B0) != nB:
        raise ValueError("malformed instance text: fewer primes than announced")
    return dict(M=M, r=r, Dmin=Dmin, B0=B0)


# -- reading ---------------------------------------------------------------------------------------
def read_blocks(f, block_records: int = I_CHUNK):
    """Yield (n, 2) uint64 arrays of whole records from a binary stream, block_records at a time
    (the last block may be shorter); a trailing partial record raises RecordStreamError."""
    want = max(1, int(block_records)) * RECORD_BYTES
    while True:
        buf = bytearray(want)
        mv = memoryview(buf)
        got = 0
        while got < want:
            k = f.readinto(mv[got:])
            if not k:
                break
            got += k
        if got == 0:
            return
        if got % RECORD_BYTES:
            raise RecordStreamError(f"stream ends inside a record ({got % RECORD_BYTES} stray bytes)")
        yield np.frombuffer(bytes(buf[:got]), dtype="<u8").reshape(-1, 2)
        if got < want:
            return


def parse_total(stderr_text: str) -> int | None:
    for line in stderr_text.splitlines():
        if line.startswith("TOTAL"):
            return int(line.split()[1])
    return None


class DumperRun:
    """A dumper process (a reference binary or this module's GPU drop-in) whose stdout is read
    as record blocks; ``close()`` checks the stream as the reference driver does: the exit code
    must be 0 and the records read must equal the TOTAL line (else RecordStreamError)."""

    def __init__(self, argv, stdin_text: str, env: dict | None = None):
        import tempfile
        self._err = tempfile.TemporaryFile()
        self.proc = subprocess.Popen(argv, stdin=subprocess.PIPE, stdout=subprocess.PIPE, stderr=self._err,
                                     env=None if env is None else dict(os.environ, **env))
        self.proc.stdin.write(stdin_text.encode())
        self.proc.stdin.close()
        self.read = 0
        self.total = None
        self.returncode = None

    def blocks(self, block_records: int = I_CHUNK):
        for a in read_blocks(self.proc.stdout, block_records):
            self.read += a.shape[0]
            yield a

    def close(self) -> int:
        """Wait for the producer and check the stream; returns the record count."""
        self.proc.stdout.close()
        self.returncode = self.proc.wait()
        self._err.seek(0)
        err = self._err.read().decode(errors="replace")
        self._err.close()
        self.total = parse_total(err)
        if self.returncode != 0:
            why = EXIT_MEANING.get(self.returncode, "failed")
            raise RecordStreamError(f"producer exited with code {self.returncode} ({why}): {err.strip()[:200]}")
        if self.total is None or self.total != self.read:
            raise RecordStreamError(f"read {self.read:,} records != TOTAL {self.total}")
        return self.read


# -- writing ---------------------------------------------------------------------------------------
def write_records(f, keys, ids) -> int:
    """Write records {keys[j], ids[j]} as 16-byte little-endian pairs (device tensors are copied to
    the host first); returns the number written."""
    def host(a):
        if hasattr(a, "detach"):
            import torch
            return a.detach().view(torch.int64).cpu().numpy().view(np.uint64)
        return np.asarray(a, dtype=np.uint64)
    k, i = host(keys), host(ids)
    if k.shape != i.shape:
        raise ValueError("keys and ids differ in length")
    out = np.empty((k.shape[0], 2), dtype="<u8")
    out[:, 0] = k
    out[:, 1] = i
    f.write(out.tobytes())
    return int(k.shape[0])


def total_line(n: int, what: str) -> str:
    return f"TOTAL {int(n)} records ({what})\n"


# -- GPU drop-ins for the dumper processes -----------------------------------------------------------
def _idump_main(stdin_text: str, out, err, env) -> int:
    from .bounded import generator
    try:
        a = parse_idump_stdin(stdin_text)
    except ValueError:
        return 2
    M, r, INS = a["M"], a["r"], a["INS"]
    rank = env.get("IDUMP_RANK", "0") not in ("", "0")
    nI = len(INS)
    if nI > 1024 or r > 16 or (not rank and (nI > 256 or r > 8)):
        err.write("8-bit packing needs nI<=256, r<=8; IDUMP_RANK=1 allows nI<=1024, r<=16\n")
        return 3
    if rank and math.comb(nI, r) >= 1 << 64:
        err.write(f"rank ids overflow u64: C({nI},{r}) >= 2^64\n")
        return 5
    if any(INS[j] <= INS[j - 1] for j in range(1, nI)):
        err.write("INS must be strictly ascending\n")
        return 4
    if not rank:
        err.write("this GPU drop-in writes colex-rank ids only (IDUMP_RANK=1)\n")
        return 3
    split = int(env["IDUMP_SPLIT"]) if "IDUMP_SPLIT" in env else None
    hmax = int(env["IDUMP_HMAX"]) if "IDUMP_HMAX" in env else None
    split_idx = nI if split is None else next((j for j, p in enumerate(INS) if p > split), nI)
    # keys P0 * prod(I) mod M with P0 mod M given: the producer takes any multiplier mod M
    total = 0
    for k, i in generator().generate_I(INS, r, M, a["P0modM"], a["Icap"], split, hmax):
        total += write_records(out, k, i)
    out.flush()
    err.write(total_line(total, f"r={r}, |INS|={nI}, split_idx={split_idx}, "
                                f"hmax={hmax if hmax is not None else 1 << 30}, ids=colex-rank"))
    return 0


def _ddump_main(stdin_text: str, out, err, env) -> int:
    from .bounded import generator
    try:
        a = parse_ddump_stdin(stdin_text)
    except ValueError:
        return 2
    M, r, B0 = a["M"], a["r"], a["B0"]
    bitmask = env.get("DDUMP_BITMASK", "0") not in ("", "0") or r > 10
    if len(B0) != 64 or r < 1 or r > 16:
        err.write("need 64 base primes and 1<=r<=16\n")
        return 3
    if any(B0[j] <= B0[j - 1] for j in range(1, len(B0))):
        err.write("base must be strictly ascending\n")
        return 4
    k, i, n = generator().generate_D(B0, r, M, a["Dmin"], bitmask=1 if bitmask else 0)
    if n:
        write_records(out, k, i)
    out.flush()
    err.write(total_line(n, f"r={r}, filtered by prodD >= Dmin, ids={'bitmask' if bitmask else '6-bit'}"))
    return 0


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv or argv[0] not in ("idump", "ddump"):
        sys.stderr.write("usage: python -m carmichael_frontier_b200.records idump|ddump < instance text\n")
        return 2
    text = sys.stdin.read()
    out = sys.stdout.buffer if hasattr(sys.stdout, "buffer") else io.BytesIO()
    fn = _idump_main if argv[0] == "idump" else _ddump_main
    return fn(text, out, sys.stderr, os.environ)


if __name__ == "__main__":
    sys.exit(main())
