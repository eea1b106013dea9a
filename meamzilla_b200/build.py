"""Build the evaluator library in-tree: meamzilla_b200/libmz_b200.so.

    python -m meamzilla_b200.build

compiles the CUDA kernels for sm_100a only and the host C++ (potential and
configuration parsers, neighbour-list builder) with -ffp-contract=off, so
neighbour distances and knot shifts round exactly as the reference's do.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libmz_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

SOURCES = ["mz_host.cpp", "mz_device.cu", "mz_nbr.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _source_hash() -> str:
    """Content hash of every source and header (mtimes do not survive copies)."""
    import hashlib
    h = hashlib.sha256()
    for d in (CSRC, INCLUDE):
        for f in sorted(os.listdir(d)):
            p = os.path.join(d, f)
            if os.path.isfile(p):
                h.update(f.encode())
                with open(p, "rb") as fh:
                    h.update(fh.read())
    h.update(" ".join(ARCH).encode())
    return h.hexdigest()


def up_to_date() -> bool:
    stamp = LIB + ".stamp"
    if not (os.path.exists(LIB) and os.path.exists(stamp)):
        return False
    with open(stamp) as fh:
        return fh.read().strip() == _source_hash()


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-I", INCLUDE, "-I", CSRC, "-Xcompiler", "-fPIC,-ffp-contract=off"]
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc()] + common + ARCH + ["-lineinfo"]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        cmd += ["-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.run([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"], check=True)
    os.replace(tmp, LIB)
    with open(LIB + ".stamp", "w") as fh:
        fh.write(_source_hash())
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
