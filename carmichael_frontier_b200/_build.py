"""Build the CUDA C-ABI library ``libcfmitm.so`` in-tree for sm_100a.

Run ``python -m carmichael_frontier_b200._build`` (or ``__graft_entry__.build()``).
The shared library lands next to this file so that it travels with the source
tree; intermediate objects go to ``_build/`` at the repository root.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libcfmitm.so")
MICRO_SRC = os.path.join(PKG, "measure", "cf_micro.cu")
MICRO_LIB = os.path.join(PKG, "libcfmicro.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "-Xptxas", "-O3", "--expt-relaxed-constexpr", "-I", CSRC, "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libcfmitm.so")
    return cand


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose_ptxas:
        cmd[1:1] = ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
    if verbose_ptxas and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def headers_mtime() -> float:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def build_micro(force: bool = False) -> str:
    """Compile the measurement kernels (measure/cf_micro.cu) into libcfmicro.so."""
    if not force and os.path.exists(MICRO_LIB) and os.path.getmtime(MICRO_LIB) >= max(
            os.path.getmtime(MICRO_SRC), headers_mtime(), os.path.getmtime(__file__)):
        return MICRO_LIB
    cmd = [nvcc(), *ARCH, *FLAGS, "-shared", MICRO_SRC, "-o", MICRO_LIB + ".tmp", "-lcudart_static", "-lrt",
           "-lpthread", "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {MICRO_SRC}:\n{r.stderr}")
    os.replace(MICRO_LIB + ".tmp", MICRO_LIB)
    return MICRO_LIB


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    """Compile every csrc/*.cu and link libcfmitm.so, then the measurement library; returns
    the path of libcfmitm.so."""
    os.makedirs(OBJ, exist_ok=True)
    srcs = sources()
    newest = max([os.path.getmtime(s) for s in srcs] + [headers_mtime(), os.path.getmtime(__file__)])
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        build_micro(force)
        return LIB
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    build_micro(force)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
