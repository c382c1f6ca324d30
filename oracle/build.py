"""Build the CPU checker: oracle/_build/libcforacle.so from cf_oracle.c, and --
when the reference tree is present (it is not on GPU hosts) -- the reference's
own CPU engines into oracle/_ref/ straight from their source files with g++
(no build system of the reference is run):

  oracle/_ref/mitm64              src/mitm64.cpp
  oracle/_ref/mitm                src/mitm.cpp
  oracle/_ref/mitm64_idump_stream2 src/mitm64_idump_stream2.cpp
  oracle/_ref/mitm64_ddump        src/mitm64_ddump.cpp

TEST INFRASTRUCTURE ONLY: the product never links or runs anything built here.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
REF_SRC = os.environ.get("CF_REFERENCE_ROOT", "/root/reference")
LIB = os.path.join(BUILD, "libcforacle.so")
REF_PROGRAMS = ("mitm64", "mitm", "mitm64_idump_stream2", "mitm64_ddump")


def build_oracle(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "cf_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", src, "-o", LIB + ".tmp"], check=True)
        os.replace(LIB + ".tmp", LIB)
    return LIB


def build_reference(force: bool = False) -> list[str]:
    """Compile the reference's CPU engines if the reference tree is here; returns built paths."""
    src_dir = os.path.join(REF_SRC, "src")
    if not os.path.isdir(src_dir):
        return [os.path.join(REF_OUT, p) for p in REF_PROGRAMS if os.path.exists(os.path.join(REF_OUT, p))]
    os.makedirs(REF_OUT, exist_ok=True)
    out = []
    for prog in REF_PROGRAMS:
        src = os.path.join(src_dir, prog + ".cpp")
        dst = os.path.join(REF_OUT, prog)
        if force or not os.path.exists(dst) or os.path.getmtime(dst) < os.path.getmtime(src):
            subprocess.run(["g++", "-O3", "-w", "-std=c++17", "-pthread", src, "-o", dst + ".tmp"], check=True)
            os.replace(dst + ".tmp", dst)
        out.append(dst)
    return out


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    for p in build_reference(force="--force" in sys.argv):
        print(p)
